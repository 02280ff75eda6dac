"""The reference's NTFF acceptance checks (tests/test_ntff.py:37-238), written
once against a namespace of solver + transform callables so they pin both the
CPU oracle (test_oracle_ntff_known_answers.py) and the GPU path
(test_ntff_gpu.py).

2D: dx = 2 mm, 40 cells per wavelength, 150 x 150 grid, 1100 steps, CPML 10,
contour 25 cells in. 3D: dx = 4 mm, 25 cells per wavelength, 48^3 grid, 600
steps, CPML 10, box 14 cells in. ``mod`` provides Grid2D, Grid3D, CPMLSpec,
alpha_max_for_fmin, simulate_tm, simulate_3d, and numpy-returning
ntff2(res, grid, margin, freqs, angles), ntff3(res, grid, margin, freqs,
thetas, phis), power2(e_far, angles), power3(e_th, e_ph, thetas, phis),
directivity3(e_th, e_ph, thetas, phis).
"""

import math

import numpy as np

C0 = 299792458.0
MU0 = 1.25663706212e-06

DX2 = 2e-3
N2 = 150
F2 = C0 / (40.0 * DX2)
MARGIN2 = 25
STEPS2 = 1100
ANGLES2 = np.linspace(0.0, 2.0 * np.pi, 360, endpoint=False)

DX3 = 4e-3
N3 = 48
F3 = C0 / (25.0 * DX3)
MARGIN3 = 14
STEPS3 = 600
THETAS3 = np.linspace(0.0, np.pi, 37)
PHIS3 = np.linspace(0.0, 2.0 * np.pi, 24, endpoint=False)


def modulated_gaussian(t, f0, t0, tau):
    """sources.py:27-30."""
    u = (t - t0) / tau
    return np.sin(2.0 * np.pi * f0 * (t - t0)) * np.exp(-0.5 * u**2)


def time_series_dft(x, dt, freqs, t0=0.0):
    t = t0 + dt * np.arange(len(x))
    f = np.atleast_1d(freqs)
    return dt * np.exp(-2j * np.pi * f[:, None] * t[None, :]) @ np.asarray(x, np.float64)


def run_2d(mod, kind):
    """kind 'single' | 'pair' | 'endfire' (test_ntff.py:48-71, 131-150)."""
    grid = mod.Grid2D(N2, N2, DX2, DX2)
    c = N2 // 2
    tau = 8.0 / (2.0 * np.pi * F2)
    t = (np.arange(STEPS2) + 0.5) * grid.dt
    cur = modulated_gaussian(t, F2, 6.0 * tau, tau)
    if kind == "single":
        ij, src = (c, c), cur
    elif kind == "pair":
        ij, src = ((c - 10, c), (c + 10, c)), np.stack([cur, cur], axis=1)
    else:
        lag = modulated_gaussian(t, F2, 6.0 * tau + 0.25 / F2, tau)
        ij, src = ((c - 5, c), (c + 5, c)), np.stack([cur, lag], axis=1)
    res = mod.simulate_tm(grid, source_ij=ij, source_current=src, dft_freqs=(F2,),
                          cpml=mod.CPMLSpec(thickness=10,
                                            alpha_max=mod.alpha_max_for_fmin(F2 / 2.0)))
    return grid, cur, mod.ntff2(res, grid, MARGIN2, (F2,), ANGLES2)


def check_isotropy(e_far):
    mag = np.abs(e_far[0])
    spread = (mag.max() - mag.min()) / mag.mean()
    assert spread <= 0.02, f"isotropy spread {spread:.4f} > 2%"


def check_line_power(mod, grid, cur, e_far):
    p_ntff = float(mod.power2(e_far, ANGLES2)[0])
    i_hat = time_series_dft(cur, grid.dt, (F2,), t0=0.5 * grid.dt)[0]
    p_exact = 2.0 * np.pi * F2 * MU0 * abs(i_hat) ** 2 / 8.0
    ratio = p_ntff / p_exact
    assert abs(ratio - 1.0) <= 0.03, f"P_ntff/P_exact = {ratio:.4f}"


def check_pair(e_far):
    pattern = np.abs(e_far[0]) ** 2
    pattern = pattern / pattern.max()
    analytic = np.cos(0.5 * np.pi * np.cos(ANGLES2)) ** 2
    assert np.corrcoef(pattern, analytic)[0, 1] >= 0.99
    peak = ANGLES2[int(np.argmax(pattern))]
    assert min(abs(peak - np.pi / 2), abs(peak - 3 * np.pi / 2)) <= 2.0 * np.pi / 360 + 1e-12
    assert pattern[0] <= 0.02 and pattern[180] <= 0.02


def check_endfire(e_far):
    pattern = np.abs(e_far[0]) ** 2
    pattern = pattern / pattern.max()
    analytic = np.cos(0.25 * np.pi * (np.cos(ANGLES2) - 1.0)) ** 2
    assert np.corrcoef(pattern, analytic)[0, 1] >= 0.99
    peak = ANGLES2[int(np.argmax(pattern))]
    assert min(peak, 2.0 * np.pi - peak) <= np.radians(15.0) + 1e-12
    assert pattern[180] <= 0.02
    assert pattern[0] >= 0.9


def run_3d(mod):
    """z current element at the centre (test_ntff.py:186-199)."""
    grid = mod.Grid3D(N3, N3, N3, DX3, DX3, DX3)
    c = N3 // 2
    tau = 6.0 / (2.0 * np.pi * F3)
    t = (np.arange(STEPS3) + 0.5) * grid.dt
    cur = modulated_gaussian(t, F3, 5.0 * tau, tau)
    res = mod.simulate_3d(grid, source_ijk=(c, c, c), source_current=cur,
                          dft_freqs=np.array([F3]),
                          cpml=mod.CPMLSpec(thickness=10,
                                            alpha_max=mod.alpha_max_for_fmin(F3 / 2.0)))
    return grid, cur, mod.ntff3(res, grid, MARGIN3, (F3,), THETAS3, PHIS3)


def check_dipole_3d(mod, grid, cur, e_far):
    d = mod.directivity3(e_far[..., 0], e_far[..., 1], THETAS3, PHIS3)
    d90 = float(np.mean(d[0, 18, :]))
    assert abs(d90 - 1.5) <= 0.075, f"D(90 deg) = {d90:.4f}"
    spread = float((d[0, 18, :].max() - d[0, 18, :].min()) / d[0, 18, :].mean())
    assert spread <= 0.05
    u = (np.abs(e_far[0, :, :, 0]) ** 2 + np.abs(e_far[0, :, :, 1]) ** 2).mean(axis=1)
    assert np.corrcoef(u / u.max(), np.sin(THETAS3) ** 2)[0, 1] >= 0.99
    p = float(mod.power3(e_far[..., 0], e_far[..., 1], THETAS3, PHIS3)[0])
    i_hat = time_series_dft(cur, grid.dt, (F3,), t0=0.5 * grid.dt)[0]
    r_r = 80.0 * math.pi**2 * (grid.dz * F3 / C0) ** 2
    ratio = p / (0.5 * r_r * abs(i_hat) ** 2)
    assert abs(ratio - 1.0) <= 0.05, f"P_ntff/P_exact = {ratio:.4f}"
    return d90, ratio
