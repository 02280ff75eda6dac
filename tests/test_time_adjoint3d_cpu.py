"""Host logic of the checkpointed 3D time-domain gradient, on the CPU.

``gradenna_b200.time_adjoint3d`` drives the CUDA solver through
``simulate_3d`` (resumable runs, E-component probes, monitor boxes). Here
the numpy oracle, which has the same resumable interface, stands in for the
solver, so the segment bookkeeping (checkpoints, recomputed segments, the
pairing of adjoint and forward rows, the H-force delay, the port's
conductance) is checked against torch autograd through the oracle's 3D loop
(oracle/fdtd3d_ad.py, the stand-in for the reference's
exact_design_gradient_3d) without a GPU. The objective reads fields outside
the CPML slabs, where the adjoint is exact. The same function on the CUDA
solver is tests/test_time_adjoint3d_gpu.py.
"""

import types
import warnings

import numpy as np
import pytest
import torch

from gradenna_b200 import time_adjoint3d as ta
from gradenna_b200.cpml import CPMLSpec
from gradenna_b200.fdtd3d import DFTMonitor
from gradenna_b200.grid import Grid3D
from oracle import fdtd2d_np as o2
from oracle import fdtd3d_np as o3
from oracle.fdtd3d_ad import exact_design_gradient_3d

COMPS = ("ex", "ey", "ez", "hx", "hy", "hz")


def _oracle_solver(grid, *, eps_r, sigma, cpml, dtype, device, probe_ijk, probe_comp,
                   state_in=None, return_state=False, dft_freqs=None, dft_dtype=None,
                   dft_monitors=None, dft_step0=0, port_ijk=None, port_voltage=None,
                   port_resistance=50.0, **src):
    """simulate_3d's resumable interface over the numpy oracle."""
    def np_(a):
        return a.cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)

    kw = {k: np_(v) for k, v in src.items() if v is not None}
    if port_ijk is not None:
        kw.update(port_ijk=port_ijk, port_voltage=np_(port_voltage),
                  port_resistance=port_resistance)
    g = o3.Grid3D(grid.nx, grid.ny, grid.nz, grid.dx, grid.dy, grid.dz)
    r = o3.simulate_3d(g, eps_r=np_(eps_r), sigma=np_(sigma), cpml=o2.CPMLSpec(cpml.thickness),
                       probe_ijk=probe_ijk, probe_comp=probe_comp, state_in=state_in,
                       return_state=return_state, step0=dft_step0, dft_freqs=dft_freqs, **kw)
    dft = mons = None
    if dft_freqs is not None:
        full = {k: torch.as_tensor(r.dft[k]) for k in COMPS}
        if dft_monitors is None:
            dft = DFTMonitor(torch.as_tensor(dft_freqs), *(full[k] for k in COMPS))
        else:
            mons = [full[COMPS[c]][:, lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]].clone()
                    for c, lo, hi in dft_monitors]

    def t(a):
        return None if a is None else torch.as_tensor(a)

    return types.SimpleNamespace(probe_ez=torch.as_tensor(r.probe_ez), port_v=t(r.port_v),
                                 port_i=t(r.port_i), dft=dft, monitors=mons, state=r.state)


def _case():
    g = Grid3D(14, 13, 12, 1e-3, 1e-3, 1e-3)
    n = 60
    dt = g.dt
    rng = np.random.default_rng(5)
    t = (np.arange(n) + 0.5) * dt
    src = o2.gaussian_derivative(t, 15 * dt, 4 * dt)
    dreg = (slice(5, 8), slice(4, 7), slice(5, 7))
    return dict(grid=g, n=n, src=src, dreg=dreg, ds=rng.uniform(0, 40, (3, 3, 2)),
                de=rng.uniform(1, 3, (3, 3, 2)), freqs=(7e9, 1.0e10), port=(6, 5, 5))


def test_segment_bounds_and_design_probes():
    assert ta.segment_bounds(12, None) == [(0, 12)]
    assert ta.segment_bounds(12, 3) == [(0, 4), (4, 8), (8, 12)]
    for bad in (0, 5, -2):
        with pytest.raises(ValueError):
            ta.segment_bounds(12, bad)
    g = Grid3D(10, 10, 10, 1e-3, 1e-3, 1e-3)
    ijk, comp, node = ta.design_probes_3d(g, ((0, 3), (4, 6), (8, 10)))
    # Ex: i 0..2, Ey / Ez: i 1..2 (i = 0 is PEC); k = 9 is PEC for Ex and Ey
    # and the last Ez row (k <= nz - 2 = 8) keeps only k = 8.
    assert np.bincount(comp).tolist() == [6, 4, 4]
    assert ijk.shape == (14, 3) and node.max() < 3 * 2 * 2


@pytest.mark.parametrize("segments", [None, 3])
def test_checkpointed_gradient_equals_autograd(monkeypatch, segments):
    c = _case()
    g, n = c["grid"], c["n"]
    monkeypatch.setattr(ta, "simulate_3d", _oracle_solver)
    monkeypatch.setattr(ta._native, "require_cuda", lambda device=None: torch.device("cpu"))
    kw = dict(source_ijk=[(4, 6, 6)], source_current=c["src"][:, None], port_ijk=c["port"],
              port_voltage=0.3 * c["src"], port_resistance=50.0)

    def obj_ad(dft, pv, pcur):
        return ((dft["ez"][:, 8, 5, 6].abs() ** 2).sum()
                + 0.3 * (dft["hx"][:, 4, 8, 5].abs() ** 2).sum()
                + 0.2 * (dft["ey"][:, 9, 8, 4].abs() ** 2).sum())

    def obj(ph):
        return obj_ad({"ez": ph.dft_ez, "hx": ph.dft_hx, "ey": ph.dft_ey}, None, None)

    og = o3.Grid3D(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz)
    want, wval = exact_design_gradient_3d(og, obj_ad, design_sigma=c["ds"], design_eps_r=c["de"],
                                          design_region=c["dreg"], dft_freqs=c["freqs"],
                                          cpml=o2.CPMLSpec(3), segment=20, **kw)
    got, val = ta.time_domain_gradient_3d(g, obj, design_sigma=c["ds"], design_eps_r=c["de"],
                                          design_region=c["dreg"], dft_freqs=c["freqs"],
                                          cpml=CPMLSpec(3), checkpoint_segments=segments,
                                          device="cpu", return_value=True, **kw)
    assert abs(val / wval - 1) <= 1e-12
    for k in want:
        e = float(np.max(np.abs(got[k].numpy() - want[k])) / np.max(np.abs(want[k])))
        assert e <= 1e-9, (k, e)


def test_objective_inside_cpml_warns():
    g = Grid3D(14, 13, 12, 1e-3, 1e-3, 1e-3)
    cot = [None, None, torch.zeros((1, 14, 13, 11), dtype=torch.complex128), None, None, None]
    cot[2][0, 10, 5, 8] = 1.0  # k = 8 > nz - 2 - 3
    with pytest.warns(UserWarning, match="CPML"):
        ta._adjoint_channels(g, cot, 3)
    cot[2][0, 10, 5, 8] = 0.0
    cot[2][0, 8, 5, 6] = 1.0
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        assert list(ta._adjoint_channels(g, cot, 3)) == [2]
