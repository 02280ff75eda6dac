"""The fused 2D objective (gdn_tm_objective_prad_s11) against the generic path.

The generic path scatters the forward run's monitor phasors onto full grids,
evaluates poynting_flux_box_2d and the port S11 with torch and takes the
cotangents by autograd (freq_adjoint.py:317-352 of the reference for the
adjoint weights). The fused kernel must give the same value, P_k, S11_k and
adjoint weights (<= 1e-12 of their peak, float64 phasors), and
freq_adjoint_gradient must give the same gradient either way (<= 1e-10).
"""

import numpy as np
import pytest
import torch

import gradenna_b200 as gb
from gradenna_b200 import freq_adjoint as fa
from gradenna_b200.monitors import port_monitors
from gradenna_b200.objectives import RadiatedPowerS11

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = torch.as_tensor(a).cpu()
    b = torch.as_tensor(b).cpu()
    return float((a - b).abs().max() / (b.abs().max() + 1e-300))


def _case(dtype=torch.float64):
    g = gb.Grid2D(120, 110, 1e-3, 1e-3)
    n = 1500
    freqs = (5.0e9, 6.5e9, 8.0e9)
    t = (np.arange(n) + 0.5) * g.dt
    env = np.clip(np.arange(n) / 300.0, 0, 1)
    vs = env * sum(np.sin(2 * np.pi * f * t + 0.3 * q) for q, f in enumerate(freqs))
    rng = np.random.default_rng(4)
    dreg = (slice(40, 80), slice(35, 75))
    ds = rng.uniform(0, 30, (40, 40))
    box = (22, 97, 20, 90)
    ports = (gb.Port((30, 55), 50.0, vs), gb.Port((88, 60), 50.0, None))
    obj = RadiatedPowerS11(g, box, ports[0].ij, freqs, resistance=50.0, w_prad=1.0, w_s11=-0.7)
    mons = obj.monitors() + port_monitors(ports[1].ij)
    return g, freqs, env, dreg, ds, ports, obj, mons


def test_fused_objective_matches_torch_path():
    g, freqs, env, dreg, ds, ports, obj, mons = _case()
    plan = fa._make_plan(g, dreg, freqs, env, None, None, ports, gb.CPMLSpec(10), torch.float64,
                         "cuda", mons)
    eps_r, sigma = fa._full_eps_sigma(g, torch.as_tensor(ds), None, dreg, plan.device)
    fwd = fa._forward(plan, eps_r, sigma)
    val, p_rad, s11, lists = obj.fused_tm(mons, list(fwd.monitors[1:]), plan.device)
    full = fa._scatter_full(plan, fwd)
    want_val, cot = fa._cotangents(plan, obj, full, fwd)
    want_srcs = fa._adjoint_sources(plan, cot)
    torch.cuda.synchronize()
    assert abs(float(val) / float(want_val) - 1) <= 1e-12
    from gradenna_b200.monitors import poynting_flux_box_2d
    p_want = poynting_flux_box_2d(full[0], full[1], full[2], g, obj.box)
    assert _rel(p_rad, p_want) <= 1e-12
    v, i = fa.ports_from_fields(full[0], full[1], full[2], g, [ports[0].ij], freqs)
    assert _rel(s11, (v[:, 0] - 50.0 * i[:, 0]) / (v[:, 0] + 50.0 * i[:, 0])) <= 1e-12
    for (idx, w), (widx, ww) in zip(lists, want_srcs):
        got = {tuple(c): w[m].cpu() for m, c in enumerate(idx.tolist())}
        assert widx is not None
        peak = float(ww.abs().max())
        for m, c in enumerate(widx.tolist()):
            assert float((got.pop(tuple(c)) - ww[m].cpu()).abs().max()) <= 1e-12 * peak
        # cells the generic path dropped carry zero weight
        for rest in got.values():
            assert float(rest.abs().max()) <= 1e-12 * peak


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_gradient_through_fused_objective(dtype):
    g, freqs, env, dreg, ds, ports, obj, mons = _case()
    kw = dict(design_sigma=torch.as_tensor(ds, device="cuda"), design_region=dreg,
              dft_freqs=freqs, env=env, ports=ports, cpml=gb.CPMLSpec(10), dtype=dtype,
              device="cuda", objective_monitors=mons)
    fused = fa.freq_adjoint_gradient(g, obj, **kw)["sigma"]
    generic = fa.freq_adjoint_gradient(g, lambda ph: obj(ph), **kw)["sigma"]
    torch.cuda.synchronize()
    assert _rel(fused, generic) <= 1e-10
    assert float(generic.abs().max()) > 0


def test_fused_objective_launches_one_kernel():
    g, freqs, env, dreg, ds, ports, obj, mons = _case()
    from gradenna_b200 import _native

    plan = fa._make_plan(g, dreg, freqs, env, None, None, ports, gb.CPMLSpec(10), torch.float64,
                         "cuda", mons)
    eps_r, sigma = fa._full_eps_sigma(g, torch.as_tensor(ds), None, dreg, plan.device)
    fwd = fa._forward(plan, eps_r, sigma)
    torch.cuda.synchronize()
    n0 = _native.kernel_launches()
    obj.fused_tm(mons, list(fwd.monitors[1:]), plan.device)
    torch.cuda.synchronize()
    assert _native.kernel_launches() - n0 == 1
