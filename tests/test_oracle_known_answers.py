"""Pin the CPU oracle against the reference test-suite's known answers.

The reference's JAX/Rust paths cannot run here and it ships no golden
vectors for simulate_tm, so the oracle is pinned by reproducing the
reference's own analytic acceptance tests through it:

* CPML reflection below -60 dB, edge and corner (tests/test_cpml.py:46-57);
* late-time energy decay to 1e-10 of the peak (tests/test_cpml.py:60-65);
* CPML table identities: thickness 0 is plain Yee, kappa_max=1 & alpha=0
  gives c = b - 1, no NaNs (tests/test_cpml.py:68-93);
* Courant stability on both sides of the limit (tests/test_stability.py:20-35);
* RVS port: Re Zin = w mu0 / 4 within 5 %, power wave = Vs/2 within 1e-3,
  port power = Poynting flux within 3 % (tests/test_ports.py:169-237);
* PEC-enclosed port |S11| = 1 within 2 % (tests/test_ports.py:240-260).

The large runs use the C oracle (itself checked against the numpy oracle in
test_oracle_c.py); the table identities use the numpy oracle directly.
"""

import numpy as np
import pytest

from oracle import fdtd2d_np as onp
from oracle.tm2d_c import simulate_tm_c

DX = 2e-3
TAU = 1.0 / (2 * np.pi * 2.5e9)


def _record(n, n_steps, cpml, probe_offset):
    g = onp.Grid2D(n, n, DX, DX)
    c = n // 2
    t = (np.arange(n_steps) + 0.5) * g.dt
    cur = onp.gaussian_derivative(t, 6 * TAU, TAU)
    res, _ = simulate_tm_c(g, source_ij=(c, c), source_current=cur,
                           probe_ij=((c + probe_offset[0], c + probe_offset[1]),), cpml=cpml,
                           record_energy=True)
    return res.probe_ez[:, 0], res


@pytest.mark.parametrize("probe_offset", [(0, 41), (32, 32)], ids=["edge", "corner"])
def test_cpml_reflection_below_minus_60db(probe_offset):
    cpml = onp.CPMLSpec(thickness=10, alpha_max=onp.alpha_max_for_fmin(0.5e9))
    e_test, _ = _record(110, 600, cpml, probe_offset)
    e_ref, _ = _record(560, 600, onp.CPMLSpec(thickness=0), probe_offset)
    r_db = 20.0 * np.log10(np.max(np.abs(e_test - e_ref)) / np.max(np.abs(e_ref)))
    assert r_db <= -60.0, f"CPML reflection {r_db:.1f} dB"


def test_late_time_energy_decay():
    cpml = onp.CPMLSpec(thickness=10, alpha_max=onp.alpha_max_for_fmin(0.5e9))
    _, res = _record(110, 1500, cpml, (0, 41))
    assert res.energy[-1] <= 1e-10 * res.energy.max()


def test_cpml_table_identities():
    co = onp.axis_coefficients(64, DX, 1e-12, onp.CPMLSpec(thickness=0), half=False, dtype=np.float64)
    assert np.abs(co.c).max() == 0.0 and np.abs(co.inv_kappa - 1.0).max() == 0.0
    for half in (False, True):
        spec = onp.CPMLSpec(thickness=8, kappa_max=1.0, alpha_max=0.0)
        co = onp.axis_coefficients(40, DX, 3e-12, spec, half=half, dtype=np.float64)
        inside = co.c != 0.0
        assert np.allclose(co.c[inside], co.b[inside] - 1.0)
        assert np.abs(co.inv_kappa - 1.0).max() == 0.0
        for spec in (onp.CPMLSpec(), onp.CPMLSpec(alpha_max=0.05), onp.CPMLSpec(thickness=0)):
            co = onp.axis_coefficients(50, DX, 3e-12, spec, half=half, dtype=np.float64)
            assert all(np.all(np.isfinite(a)) for a in co)


def _courant_run(courant, n_steps):
    g = onp.Grid2D(60, 60, DX, DX, courant=courant)
    tau = 20 * g.dt
    t = (np.arange(n_steps) + 0.5) * g.dt
    res, _ = simulate_tm_c(g, source_ij=(30, 30), source_current=onp.gaussian_derivative(t, 6 * tau, tau),
                           cpml=onp.CPMLSpec(0), record_energy=True)
    return res.energy


def test_courant_stability_both_sides():
    after = _courant_run(0.99, 2000)[400:]
    assert after.max() <= 1.02 * after[:100].max() and np.all(np.isfinite(after))
    with np.errstate(all="ignore"):
        e = _courant_run(1.01, 600)
    assert (not np.isfinite(e[-1])) or e[-1] > 1e6 * e[100]


F_MIN, F_MAX = 1.5e9, 4.5e9
EVAL = (2.5e9, 2.75e9, 3.0e9, 3.25e9, 3.5e9)
RS = 50.0


@pytest.fixture(scope="module")
def radiation_run():
    n = 120
    g = onp.Grid2D(n, n, DX, DX)
    pulse = onp.gaussian_pulse_for_band(F_MIN, F_MAX)
    t = (np.arange(1400) + 0.5) * g.dt
    vs = pulse(t)
    cpml = onp.CPMLSpec(thickness=10, alpha_max=onp.alpha_max_for_fmin(F_MIN))
    res, _ = simulate_tm_c(g, ports=(onp.Port((n // 2, n // 2), RS, vs),), dft_freqs=EVAL, cpml=cpml)
    return g, res, vs


def test_radiation_resistance_matches_line_current_theory(radiation_run):
    g, res, _ = radiation_run
    v, i = onp.port_dft(res.port_v[:, 0], res.port_i[:, 0], g.dt, EVAL)
    zin = v / i
    expected = 2.0 * np.pi * np.asarray(EVAL) * onp.MU0 / 4.0
    assert (np.abs(zin.real - expected) / expected).max() < 0.05
    assert np.all(zin.imag > 0.0)


def test_power_wave_matches_incident_wave(radiation_run):
    g, res, vs = radiation_run
    v, i = onp.port_dft(res.port_v[:, 0], res.port_i[:, 0], g.dt, EVAL)
    vs_hat = onp.half_step_dft(vs, g.dt, EVAL)
    assert (np.abs(0.5 * (v + RS * i) - vs_hat / 2) / np.abs(vs_hat / 2)).max() < 1e-3


def test_port_power_equals_poynting_flux(radiation_run):
    g, res, _ = radiation_run
    v, i = onp.port_dft(res.port_v[:, 0], res.port_i[:, 0], g.dt, EVAL)
    p_port = 0.5 * np.real(v * np.conj(i))
    c, k = g.nx // 2, 20
    p_flux = onp.poynting_flux_box_2d(res.dft_ez, res.dft_hx, res.dft_hy, g, (c - k, c + k - 1, c - k, c + k - 1))
    assert np.all(p_port > 0.0)
    assert (np.abs(p_flux - p_port) / p_port).max() < 0.03
    f = np.asarray(EVAL)
    assert abs(np.trapezoid(p_flux, f) - np.trapezoid(p_port, f)) / np.trapezoid(p_port, f) < 0.03


def test_pec_enclosed_port_is_totally_reflecting():
    n = 17
    g = onp.Grid2D(n, n, DX, DX)
    pulse = onp.gaussian_pulse_for_band(2e9, 8e9)
    t = (np.arange(30000) + 0.5) * g.dt
    res, _ = simulate_tm_c(g, ports=(onp.Port((n // 2, n // 2), RS, pulse(t)),), cpml=onp.CPMLSpec(0))
    freqs = (3e9, 5e9, 6.6e9, 7.5e9)
    v, i = onp.port_dft(res.port_v[:, 0], res.port_i[:, 0], g.dt, freqs)
    s11 = np.abs(onp.s11_power_wave(v, i, RS))
    assert np.abs(s11 - 1.0).max() < 0.02
