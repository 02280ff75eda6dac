"""GPU checks of the exact time-domain adjoint (gradenna_b200.time_adjoint)
against torch autograd through the oracle's time loop
(oracle/fdtd2d_ad.py, the stand-in for the reference's jax.grad of
simulate_tm): pulse drives, lossy and permittivity designs, metal designs
under a port drive at two frequencies, an S11 objective, a float32 run and
the autograd wrapper. In float64 the two gradients agree to rounding (for
S11, built here from the field phasors, the time-series S11 of the oracle
differs by the final port field's boundary term, 5e-6 relative).
"""

import numpy as np
import pytest
import torch

from oracle import fdtd2d_ad as ad
from oracle import fdtd2d_np as onp

pytestmark = pytest.mark.gpu

N = 1200
BOX = (12, 29, 12, 29)
REG = (slice(18, 26), slice(18, 26))


def _pulse(dt, f0=3e9):
    t = (np.arange(N) + 0.5) * dt
    return np.sin(2 * np.pi * f0 * t) * np.exp(-((t - 120 * dt) / (40 * dt)) ** 2)


def _rel(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _flux(grid):
    from gradenna_b200.monitors import poynting_flux_box_2d

    return lambda ph: poynting_flux_box_2d(ph.dft_ez, ph.dft_hx, ph.dft_hy, grid, BOX).sum()


def _flux_t(og):
    return lambda ez, hx, hy, pv, pi: ad.poynting_flux_box_2d_t(ez, hx, hy, og, BOX).sum()


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-9), (torch.float32, 3e-3)])
def test_pulse_source_lossy_and_permittivity_design(dtype, tol):
    import gradenna_b200 as gb
    from gradenna_b200.time_adjoint import time_domain_gradient

    grid = gb.Grid2D(40, 40, 2e-3, 2e-3)
    og = onp.Grid2D(40, 40, 2e-3, 2e-3)
    rng = np.random.default_rng(1)
    sig, er = rng.uniform(0, 30, (8, 8)), 1 + 2 * rng.uniform(0, 1, (8, 8))
    src = _pulse(grid.dt)
    g = time_domain_gradient(grid, _flux(grid), design_sigma=sig, design_eps_r=er,
                             design_region=REG, dft_freqs=(3e9,), source_ij=(14, 22),
                             source_current=src, cpml=gb.CPMLSpec(8), dtype=dtype)
    ex, _ = ad.exact_design_gradient(og, _flux_t(og), design_sigma=sig, design_eps_r=er,
                                     design_region=REG, dft_freqs=(3e9,), source_ij=(14, 22),
                                     source_current=src, cpml=onp.CPMLSpec(8), segment=300,
                                     device="cuda")
    assert _rel(g["sigma"].cpu().numpy(), ex["sigma"]) <= tol
    assert _rel(g["eps_r"].cpu().numpy(), ex["eps_r"]) <= tol


def test_port_drive_metal_design_two_frequencies():
    import gradenna_b200 as gb
    from gradenna_b200.time_adjoint import time_domain_gradient

    grid = gb.Grid2D(40, 40, 2e-3, 2e-3)
    og = onp.Grid2D(40, 40, 2e-3, 2e-3)
    sig = 10.0 ** (-4 + 9 * np.random.default_rng(2).uniform(0, 1, (8, 8)))
    v = _pulse(grid.dt)
    F = (2.5e9, 3.5e9)
    g = time_domain_gradient(grid, _flux(grid), design_sigma=sig, design_region=REG,
                             dft_freqs=F, ports=(gb.Port((15, 22), 50.0, v),),
                             cpml=gb.CPMLSpec(8), dtype=torch.float64)
    ex, _ = ad.exact_design_gradient(og, _flux_t(og), design_sigma=sig, design_region=REG,
                                     dft_freqs=F, ports=(onp.Port((15, 22), 50.0, v),),
                                     cpml=onp.CPMLSpec(8), segment=300, device="cuda")
    assert _rel(g["sigma"].cpu().numpy(), ex["sigma"]) <= 1e-9


def test_s11_objective_and_autograd_wrapper():
    import gradenna_b200 as gb
    from gradenna_b200.sparams import s11_power_wave
    from gradenna_b200.time_adjoint import time_domain_gradient, time_domain_objective

    grid = gb.Grid2D(40, 40, 2e-3, 2e-3)
    og = onp.Grid2D(40, 40, 2e-3, 2e-3)
    sig = np.random.default_rng(3).uniform(0, 5, (8, 8))
    v = _pulse(grid.dt)
    reg = (slice(20, 28), slice(18, 26))

    def obj(ph):
        s = s11_power_wave(ph.port_v[0, 0], ph.port_i[0, 0], 50.0)
        return s.real ** 2 + s.imag ** 2

    def obj_fields(ez, hx, hy, pv, pi):
        # the same objective on the oracle's phasors: port V, I rebuilt from
        # the field phasors exactly as FreqPhasors.port_v / port_i are
        from gradenna_b200.freq_adjoint import ports_from_fields

        v_, i_ = ports_from_fields(ez, hx, hy, grid, [(14, 22)], (3e9,))
        s = (v_[0, 0] - 50.0 * i_[0, 0]) / (v_[0, 0] + 50.0 * i_[0, 0])
        return s.real ** 2 + s.imag ** 2

    def obj_t(ez, hx, hy, pv, pi):
        # S11 from the DFT of the port's V / I time series: differs from the
        # field-phasor form by the final port field's boundary term
        vv = ad.half_step_dft_t(pv[:, 0], og.dt, (3e9,))
        ii = ad.half_step_dft_t(pi[:, 0], og.dt, (3e9,))
        s = (vv - 50.0 * ii) / (vv + 50.0 * ii)
        return (s.real ** 2 + s.imag ** 2).sum()

    kw = dict(design_region=reg, dft_freqs=(3e9,), ports=(gb.Port((14, 22), 50.0, v),),
              cpml=gb.CPMLSpec(8), dtype=torch.float64)
    g = time_domain_gradient(grid, obj, design_sigma=sig, **kw)
    common = dict(design_sigma=sig, design_region=reg, dft_freqs=(3e9,),
                  ports=(onp.Port((14, 22), 50.0, v),), cpml=onp.CPMLSpec(8), segment=300,
                  device="cuda")
    ex, _ = ad.exact_design_gradient(og, obj_fields, **common)
    assert _rel(g["sigma"].cpu().numpy(), ex["sigma"]) <= 1e-9
    ex_t, _ = ad.exact_design_gradient(og, obj_t, **common)
    assert _rel(g["sigma"].cpu().numpy(), ex_t["sigma"]) <= 1e-4
    s = torch.as_tensor(sig, device="cuda").requires_grad_(True)
    val = time_domain_objective(s, grid, obj, **kw)
    val.backward()
    torch.testing.assert_close(s.grad, g["sigma"], rtol=1e-12, atol=0)
