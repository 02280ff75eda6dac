"""The 3D time-domain gradient on the CUDA solver (gdn_yee_run_*).

* Resumable runs: a run split in two at step 40, the second resumed from the
  first's state blob (GdnYeeBuffers.state_in / state_out), reproduces the
  single run bit for bit (final fields, Ex / Ey / Ez probe records, port V
  and I); the two runs' DFT partial sums (phases of the absolute steps) add
  up to the single run's phasors within rounding.
* time_domain_gradient_3d against torch autograd through the oracle's 3D
  loop (oracle/fdtd3d_ad.py, the stand-in for the reference's
  exact_design_gradient_3d, freq_adjoint.py:724-771) in float64, <= 1e-9
  peak-normalised, for sigma and eps_r designs, a pulse-driven Jz source and
  a driven port inside the design region, whole histories (S = 1) and
  checkpointed segments (S = 4), full-grid and port-limited DFTs.
* float32 fields: the same gradients within 1e-3 of the float64 autograd
  result (printed).
* A patch-sized pulse run (64 x 64 x 32, 400 steps) with S = 20 = sqrt(N)
  checkpoints equals the whole-history gradient to rounding.
"""

import numpy as np
import pytest
import torch

from gradenna_b200.cpml import CPMLSpec
from gradenna_b200.fdtd3d import simulate_3d
from gradenna_b200.freq_adjoint3d import _port_v_i_3d
from gradenna_b200.grid import Grid3D
from gradenna_b200.time_adjoint3d import time_domain_gradient_3d
from oracle import fdtd2d_np as o2
from oracle import fdtd3d_np as o3
from oracle.fdtd3d_ad import exact_design_gradient_3d

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / (np.max(np.abs(b)) + 1e-300))


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_resumed_runs_equal_one_run(dtype):
    g = Grid3D(22, 20, 18, 1e-3, 1e-3, 1e-3)
    n, cut = 80, 40
    dt = g.dt
    t = (np.arange(n) + 0.5) * dt
    src = o2.gaussian_derivative(t, 15 * dt, 4 * dt)
    rng = np.random.default_rng(2)
    eps = torch.as_tensor(1 + rng.uniform(size=g.shape), dtype=dtype, device="cuda")
    sig = torch.as_tensor(rng.uniform(0, 5, size=g.shape), dtype=dtype, device="cuda")
    probes = np.array([[5, 6, 7], [9, 9, 9], [12, 4, 10], [3, 15, 2]])
    pcomp = np.array([0, 1, 2, 2])
    freqs = (5e9, 8e9)
    kw = dict(eps_r=eps, sigma=sig, probe_ijk=probes, probe_comp=pcomp, cpml=CPMLSpec(4),
              dtype=dtype, device="cuda", dft_freqs=freqs, dft_dtype=np.complex128,
              source_ijk=[(8, 8, 8)], port_ijk=(12, 11, 9), port_resistance=50.0)
    whole = simulate_3d(g, source_current=src[:, None], port_voltage=0.2 * src, **kw)
    a = simulate_3d(g, source_current=src[:cut, None], port_voltage=0.2 * src[:cut],
                    return_state=True, **kw)
    b = simulate_3d(g, source_current=src[cut:, None], port_voltage=0.2 * src[cut:],
                    state_in=a.state, dft_step0=cut, **kw)
    torch.cuda.synchronize()
    for nm in ("ex", "ey", "ez", "hx", "hy", "hz"):
        assert torch.equal(getattr(b, nm), getattr(whole, nm)), nm
        both = getattr(a.dft, nm) + getattr(b.dft, nm)
        assert _rel(both.cpu(), getattr(whole.dft, nm).cpu()) <= 1e-12, nm
    assert torch.equal(torch.cat([a.probe_ez, b.probe_ez]), whole.probe_ez)
    assert torch.equal(torch.cat([a.port_v, b.port_v]), whole.port_v)
    assert torch.equal(torch.cat([a.port_i, b.port_i]), whole.port_i)
    # The Ex / Ey / Ez probes record those components.
    for q, (c, (i, j, k)) in enumerate(zip(pcomp, probes)):
        fld = (b.ex, b.ey, b.ez)[c]
        assert float(b.probe_ez[-1, q]) == float(fld[i, j, k])


def _case():
    g = Grid3D(20, 18, 16, 1e-3, 1e-3, 1e-3)
    n = 120
    dt = g.dt
    rng = np.random.default_rng(7)
    t = (np.arange(n) + 0.5) * dt
    src = o2.gaussian_derivative(t, 20 * dt, 6 * dt)
    dreg = (slice(8, 12), slice(7, 11), slice(6, 9))
    return dict(grid=g, n=n, src=src, dreg=dreg, ds=rng.uniform(0, 40, (4, 4, 3)),
                de=rng.uniform(1, 3, (4, 4, 3)), freqs=(6e9, 9e9), port=(9, 8, 7))


def _objectives(g, port, freqs):
    def point(ez, hx, ey):
        return ((ez[:, 13, 9, 10].abs() ** 2).sum() + 0.3 * (hx[:, 6, 11, 6].abs() ** 2).sum()
                + 0.2 * (ey[:, 12, 12, 5].abs() ** 2).sum())

    def port_obj(ez, hx, hy):
        v, i = _port_v_i_3d(ez, hx, hy, g, port, freqs)
        return (v.abs() ** 2).sum() + 50.0 ** 2 * (i.abs() ** 2).sum() - 0.5 * (v * i.conj()).real.sum()

    return {
        None: (lambda ph: point(ph.dft_ez, ph.dft_hx, ph.dft_ey),
               lambda d, pv, pc: point(d["ez"], d["hx"], d["ey"])),
        "port": (lambda ph: port_obj(ph.dft_ez, ph.dft_hx, ph.dft_hy),
                 lambda d, pv, pc: port_obj(d["ez"], d["hx"], d["hy"])),
    }


_EXACT = {}


def _exact(kind):
    if kind not in _EXACT:
        c = _case()
        g = c["grid"]
        og = o3.Grid3D(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz)
        _, obj_ad = _objectives(g, c["port"], c["freqs"])[kind]
        _EXACT[kind] = exact_design_gradient_3d(
            og, obj_ad, design_sigma=c["ds"], design_eps_r=c["de"], design_region=c["dreg"],
            dft_freqs=c["freqs"], cpml=o2.CPMLSpec(4), segment=30, device="cuda",
            source_ijk=[(6, 9, 8)], source_current=c["src"][:, None], port_ijk=c["port"],
            port_voltage=0.3 * c["src"], port_resistance=50.0)
    return _EXACT[kind]


def _ours(kind, segments, dtype):
    c = _case()
    g = c["grid"]
    obj, _ = _objectives(g, c["port"], c["freqs"])[kind]
    return time_domain_gradient_3d(
        g, obj, design_sigma=c["ds"], design_eps_r=c["de"], design_region=c["dreg"],
        dft_freqs=c["freqs"], cpml=CPMLSpec(4), checkpoint_segments=segments, dtype=dtype,
        device="cuda", return_value=True, objective_kind=kind, source_ijk=[(6, 9, 8)],
        source_current=c["src"][:, None], port_ijk=c["port"], port_voltage=0.3 * c["src"],
        port_resistance=50.0)


@pytest.mark.parametrize("kind", [None, "port"])
@pytest.mark.parametrize("segments", [None, 4])
def test_gradient_matches_autograd_float64(kind, segments):
    want, wval = _exact(kind)
    got, val = _ours(kind, segments, torch.float64)
    assert abs(val / wval - 1) <= 1e-10
    for k in want:
        e = _rel(got[k].cpu(), want[k])
        assert e <= 1e-9, (k, e)


@pytest.mark.parametrize("kind", [None, "port"])
def test_gradient_float32_fields(kind):
    want, wval = _exact(kind)
    got, val = _ours(kind, 4, torch.float32)
    errs = {k: _rel(got[k].cpu(), want[k]) for k in want}
    print(f"\nfloat32 fields vs float64 autograd ({kind}): value {abs(val / wval - 1):.1e}, "
          + ", ".join(f"{k} {e:.1e}" for k, e in errs.items()))
    assert abs(val / wval - 1) <= 1e-4
    assert max(errs.values()) <= 1e-3, errs


def test_sqrt_n_checkpoints_on_a_patch_sized_run():
    g = Grid3D(64, 64, 32, 5e-4, 5e-4, 5e-4)
    n = 400
    dt = g.dt
    t = (np.arange(n) + 0.5) * dt
    src = o2.gaussian_derivative(t, 60 * dt, 18 * dt)
    rng = np.random.default_rng(11)
    eps_bg = np.ones(g.shape)
    eps_bg[:, :, 8:12] = 4.4
    dreg = (slice(20, 44), slice(20, 44), slice(12, 13))
    ds = rng.uniform(0, 1e3, (24, 24, 1))
    freqs = (6e9, 8e9, 1e10)

    def obj(ph):
        return (ph.dft_ez[:, 32, 32, 20].abs() ** 2).sum() + (ph.dft_ex[:, 40, 24, 16].abs() ** 2).sum()

    kw = dict(design_sigma=ds, design_region=dreg, dft_freqs=freqs, cpml=CPMLSpec(8),
              eps_r_background=eps_bg, source_ijk=[(30, 30, 10)], source_current=src[:, None],
              port_ijk=(34, 28, 10), port_voltage=0.1 * src, dtype=torch.float64, device="cuda",
              return_value=True)
    whole, v1 = time_domain_gradient_3d(g, obj, checkpoint_segments=None, **kw)
    ckpt, v2 = time_domain_gradient_3d(g, obj, checkpoint_segments=20, **kw)
    assert abs(v2 / v1 - 1) <= 1e-12
    assert _rel(ckpt["sigma"].cpu(), whole["sigma"].cpu()) <= 1e-10
    assert float(whole["sigma"].abs().max()) > 0
