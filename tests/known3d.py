"""The reference's 3D known-answer checks (tests/test_fdtd3d.py:37-140),
written once against a `simulate_3d`-like callable so they pin both the CPU
oracle (test_oracle3d_known_answers.py) and the GPU path (test_known3d_gpu.py).
"""

import math

import numpy as np

DX = 4e-3
C0 = 299792458.0


def _np(x):
    return x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)


def openems_gauss(t, f0, fc):
    sigma = 3.0 / (2.0 * math.sqrt(2.0) * math.pi * fc)
    t0 = 9.0 / (2.0 * math.pi * fc)
    return np.cos(2.0 * math.pi * f0 * (t - t0)) * np.exp(-0.5 * ((t - t0) / sigma) ** 2)


def gaussian_derivative(t, t0, tau):
    u = (np.asarray(t) - t0) / tau
    return -u * np.exp(0.5 * (1.0 - u**2))


def dipole(mod, n=48, n_steps=800, **kw):
    """Free-space z-directed 1-cell RVS port at the centre (test_fdtd3d.py:37-52)."""
    grid = mod.Grid3D(n, n, n, DX, DX, DX)
    vs = openems_gauss((np.arange(n_steps) + 0.5) * grid.dt, 2.5e9, 1.0e9)
    c = n // 2
    res = mod.simulate_3d(grid, port_ijk=(c, c, c), port_voltage=vs, port_resistance=50.0,
                          cpml=mod.CPMLSpec(10, alpha_max=mod.alpha_max_for_fmin(1.5e9)), **kw)
    return grid, res


def check_dipole(mod, grid, res):
    """R_r = 80 pi^2 (dz/lambda)^2 within 15 %, capacitive, and the raw
    (not de-embedded) resistance biased upward by the gap shunt."""
    freqs = np.linspace(1.8e9, 3.2e9, 8)
    zin = _np(mod.port_impedance(res, grid, freqs))
    r_theory = 80.0 * math.pi**2 * (grid.dz * freqs / C0) ** 2
    assert (np.abs(zin.real - r_theory) / r_theory).max() <= 0.15
    assert np.all(zin.imag < 0.0)
    f3 = np.linspace(2.0e9, 3.0e9, 3)
    z_raw = _np(mod.port_impedance(res, grid, f3, deembed_gap=False))
    z_cor = _np(mod.port_impedance(res, grid, f3, deembed_gap=True))
    assert np.all(z_raw.real > z_cor.real)


def check_energy_decay(mod, **kw):
    n = 36
    grid = mod.Grid3D(n, n, n, DX, DX, DX)
    tau = 1.0 / (2.0 * math.pi * 2.5e9)
    cur = gaussian_derivative((np.arange(1400) + 0.5) * grid.dt, 6 * tau, tau)
    c = n // 2
    res = mod.simulate_3d(grid, source_ijk=(c, c, c), source_current=cur, record_energy=True,
                          cpml=mod.CPMLSpec(10, alpha_max=mod.alpha_max_for_fmin(0.5e9)), **kw)
    e = _np(res.energy)
    assert np.all(np.isfinite(e)) and e[-1] / e.max() <= 1e-15


def check_mirror_symmetry(mod, **kw):
    n = 31
    grid = mod.Grid3D(n, n, n, DX, DX, DX)
    c = n // 2
    cur = gaussian_derivative((np.arange(300) + 0.5) * grid.dt, 60 * grid.dt, 12 * grid.dt)
    probes = ((c + 4, c, c), (c - 4, c, c), (c, c + 4, c), (c, c - 4, c))
    res = mod.simulate_3d(grid, source_ijk=(c, c, c), source_current=cur, probe_ijk=probes,
                          cpml=mod.CPMLSpec(8), **kw)
    p = _np(res.probe_ez)
    assert np.abs(p - p[:, :1]).max() / np.abs(p).max() <= 1e-12
