"""The GPU frequency-domain adjoint against the EXACT time-domain gradient.

The reference accepts its frequency-domain adjoint by comparing it with
jax.grad of the whole simulation (tests/test_freq_adjoint.py:37-230):
cosine >= 0.999 and a random-direction relative error <= 1e-2. Here the
exact gradient comes from oracle/fdtd2d_ad.py (the same time loop restated
in torch float64, reverse sweep by autograd with segment recomputation; run
with torch operations on the GPU only to make the checker fast) on the
reference's cases: 44 x 44 grid, CPML 8, CW 3 GHz with a 300-step ramp,
10000 steps, 8 x 8 design.
"""

import numpy as np
import pytest
import torch

from oracle import fdtd2d_ad as ad
from oracle import fdtd2d_np as onp

pytestmark = pytest.mark.gpu

N_STEPS = 10000
F0 = 3e9
BOX = (12, 31, 12, 31)


def _cw(dt):
    n = np.arange(N_STEPS)
    env = np.clip(n / 300.0, 0.0, 1.0)
    return env * np.sin(2 * np.pi * F0 * (n + 0.5) * dt), env


def _compare(g_ex, g_fa, seed=0):
    a, b = np.asarray(g_ex).ravel(), np.asarray(g_fa).ravel()
    cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))
    v = np.random.default_rng(seed).normal(size=a.shape)
    return cos, abs(b @ v - a @ v) / abs(a @ v)


def _flux_case(key, theta):
    import gradenna_b200 as gb
    from gradenna_b200.freq_adjoint import freq_adjoint_gradient
    from gradenna_b200.monitors import poynting_flux_box_2d

    grid = gb.Grid2D(44, 44, 2e-3, 2e-3)
    cur, env = _cw(grid.dt)
    region = (slice(18, 26), slice(18, 26))

    def obj(ph):
        return poynting_flux_box_2d(ph.dft_ez, ph.dft_hx, ph.dft_hy, grid, BOX).sum()

    g_fa = freq_adjoint_gradient(grid, obj, **{f"design_{key}": theta}, design_region=region,
                                 dft_freqs=(F0,), env=env, source_ij=(14, 22),
                                 source_current=cur, cpml=gb.CPMLSpec(8))[key].cpu().numpy()
    og = onp.Grid2D(44, 44, 2e-3, 2e-3)
    g_ex, _ = ad.exact_design_gradient(
        og, lambda ez, hx, hy, pv, pi: ad.poynting_flux_box_2d_t(ez, hx, hy, og, BOX).sum(),
        **{f"design_{key}": theta}, design_region=region, dft_freqs=(F0,), source_ij=(14, 22),
        source_current=cur, cpml=onp.CPMLSpec(8), segment=500, device="cuda")
    return g_ex[key], g_fa


def test_flux_sigma_against_exact_gradient():
    g_ex, g_fa = _flux_case("sigma", 0.01 * np.ones((8, 8)))
    cos, rel = _compare(g_ex, g_fa)
    assert cos >= 0.999 and rel <= 1e-2, (cos, rel)


def test_flux_eps_r_against_exact_gradient():
    g_ex, g_fa = _flux_case("eps_r", 1.0 + 1.5 * np.random.default_rng(3).random((8, 8)))
    cos, rel = _compare(g_ex, g_fa)
    assert cos >= 0.999 and rel <= 1e-2, (cos, rel)


def test_s11_sigma_against_exact_gradient():
    import gradenna_b200 as gb
    from gradenna_b200.freq_adjoint import freq_adjoint_gradient
    from gradenna_b200.sparams import s11_power_wave

    grid = gb.Grid2D(44, 44, 2e-3, 2e-3)
    cur, env = _cw(grid.dt)
    region = (slice(20, 28), slice(18, 26))
    theta = 0.02 * np.ones((8, 8))

    def obj(ph):
        s = s11_power_wave(ph.port_v[0, 0], ph.port_i[0, 0], 50.0)
        return s.real**2 + s.imag**2

    g_fa = freq_adjoint_gradient(grid, obj, design_sigma=theta, design_region=region,
                                 dft_freqs=(F0,), env=env, ports=(gb.Port((14, 22), 50.0, cur),),
                                 cpml=gb.CPMLSpec(8))["sigma"].cpu().numpy()
    og = onp.Grid2D(44, 44, 2e-3, 2e-3)

    def obj_t(ez, hx, hy, pv, pi):
        v = ad.half_step_dft_t(pv[:, 0], og.dt, (F0,))
        i = ad.half_step_dft_t(pi[:, 0], og.dt, (F0,))
        s = (v - 50.0 * i) / (v + 50.0 * i)
        return (s.real**2 + s.imag**2).sum()

    g_ex, _ = ad.exact_design_gradient(og, obj_t, design_sigma=theta, design_region=region,
                                       dft_freqs=(F0,), ports=(onp.Port((14, 22), 50.0, cur),),
                                       cpml=onp.CPMLSpec(8), segment=500, device="cuda")
    cos, rel = _compare(g_ex["sigma"], g_fa)
    assert cos >= 0.999 and rel <= 1e-2, (cos, rel)
