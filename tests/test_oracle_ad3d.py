"""The 3D autograd oracle (oracle/fdtd3d_ad.py) on the CPU.

* Its forward run equals the numpy oracle (oracle/fdtd3d_np.py, pinned to
  the reference's own simulate_3d by tests/test_golden_oracle.py) to 1e-12:
  a Jz source, an RVS port with the port overwrite, CPML, a region-limited
  DFT at two frequencies.
* Its reverse sweep (torch autograd with segment recomputation, the
  sqrt(N) checkpointing of fdtd3d.py:735-749) equals central finite
  differences of its own forward run: the exact gradient the GPU adjoint is
  checked against (the reference's exact_design_gradient_3d,
  freq_adjoint.py:724-771).
"""

import numpy as np
import torch

from oracle import fdtd2d_np as o2
from oracle import fdtd3d_ad as ad
from oracle import fdtd3d_np as o3


def _case():
    g = o3.Grid3D(14, 13, 12, 1e-3, 1.1e-3, 0.9e-3)
    n = 120
    t = (np.arange(n) + 0.5) * g.dt
    src = o2.gaussian_derivative(t, 20 * g.dt, 6 * g.dt)
    rng = np.random.default_rng(2)
    eps = 1.0 + rng.uniform(0, 2, (g.nx, g.ny, g.nz))
    sig = rng.uniform(0, 3, (g.nx, g.ny, g.nz))
    kw = dict(source_ijk=(7, 6, 5), source_current=src, port_ijk=(5, 8, 6),
              port_voltage=0.3 * src, port_resistance=50.0, dft_freqs=(30e9, 45e9),
              cpml=o2.CPMLSpec(3))
    regions = {"ez": ((4, 4, 3), (10, 9, 8)), "hx": ((5, 3, 4), (9, 10, 7))}
    return g, eps, sig, kw, regions


def test_forward_matches_numpy_oracle():
    g, eps, sig, kw, regions = _case()
    o = o3.simulate_3d(g, eps_r=eps, sigma=sig, dft_regions=regions, **kw)
    dft, pv, pi = ad.simulate_3d_ad(g, eps_r=torch.tensor(eps), sigma=torch.tensor(sig),
                                    dft_regions=regions, segment=37, **kw)
    rel = lambda a, b: float(np.abs(a - b).max() / np.abs(b).max())  # noqa: E731
    assert rel(pv.numpy(), o.port_v) <= 1e-12
    assert rel(pi.numpy(), o.port_i) <= 1e-12
    for k in regions:
        assert rel(dft[k].numpy(), o.dft[k]) <= 1e-12, k


def test_reverse_sweep_matches_central_differences():
    g, eps, sig, kw, regions = _case()
    region = (slice(6, 9), slice(5, 7), slice(4, 6))

    def objective(dft, pv, pi):
        return (dft["ez"].abs() ** 2).sum() * 1e20 + (pv ** 2).sum() * 1e3

    base = sig[region].copy()
    grad, val = ad.exact_design_gradient_3d(
        g, objective, design_sigma=base, design_region=region, eps_r_background=eps,
        sigma_background=sig, dft_regions=regions, segment=40, **kw)
    rng = np.random.default_rng(0)
    d = rng.normal(size=base.shape)
    h = 1e-3

    def f(s):
        s_full = sig.copy()
        s_full[region] = s
        dft, pv, pi = ad.simulate_3d_ad(g, eps_r=torch.tensor(eps), sigma=torch.tensor(s_full),
                                        dft_regions=regions, segment=1000, **kw)
        return float(objective(dft, pv, pi))

    fd = (f(base + h * d) - f(base - h * d)) / (2 * h)
    an = float(np.sum(grad["sigma"] * d))
    assert abs(fd - an) <= 1e-6 * abs(an), (fd, an)
