"""Pin the NTFF oracle (oracle/ntff_np.py over the numpy 2D/3D steppers)
against the reference's NTFF acceptance tests (tests/test_ntff.py):
line-current isotropy and power, broadside and endfire array patterns, and
the z-dipole's directivity, pattern and radiation resistance."""

import functools
import types

import numpy as np
import pytest

from oracle import fdtd2d_np as o2
from oracle import fdtd3d_np as o3
from oracle import ntff_np as on
from tests import known_ntff as kn


def _ntff2(res, grid, margin, freqs, angles):
    return on.ntff_2d(res.dft_ez, res.dft_hx, res.dft_hy, grid.nx, grid.ny, grid.dx, grid.dy,
                      margin, freqs, angles)


def _ntff3(res, grid, margin, freqs, thetas, phis):
    return on.ntff_3d(res.dft, grid.nx, grid.ny, grid.nz, grid.dx, grid.dy, grid.dz, margin,
                      freqs, thetas, phis)


MOD = types.SimpleNamespace(
    Grid2D=o2.Grid2D, Grid3D=o3.Grid3D, CPMLSpec=o2.CPMLSpec,
    alpha_max_for_fmin=o2.alpha_max_for_fmin, simulate_tm=o2.simulate_tm,
    simulate_3d=o3.simulate_3d, ntff2=_ntff2, ntff3=_ntff3, power2=on.radiated_power_2d,
    power3=on.radiated_power_3d, directivity3=on.directivity_3d)


@functools.lru_cache(maxsize=3)
def _run2(kind):
    return kn.run_2d(MOD, kind)


def test_line_current_isotropic_pattern():
    kn.check_isotropy(_run2("single")[2])


def test_line_current_radiated_power():
    grid, cur, e_far = _run2("single")
    kn.check_line_power(MOD, grid, cur, e_far)


def test_two_element_array_pattern():
    kn.check_pair(_run2("pair")[2])


def test_endfire_pair_propagation_phase_sign():
    kn.check_endfire(_run2("endfire")[2])


def test_dipole_3d_directivity_pattern_power():
    grid, cur, e_far = kn.run_3d(MOD)
    kn.check_dipole_3d(MOD, grid, cur, e_far)


def test_trapezoid_weights_match_rules():
    """Uniform circle -> 2 pi / n each; duplicated endpoint -> half weights."""
    a = np.linspace(0.0, 2 * np.pi, 8, endpoint=False)
    assert np.allclose(on.periodic_trapezoid_weights(a, 2 * np.pi), 2 * np.pi / 8)
    b = np.linspace(0.0, 2 * np.pi, 9)
    w = on.periodic_trapezoid_weights(b, 2 * np.pi)
    assert np.isclose(w.sum(), 2 * np.pi)
    with pytest.raises(ValueError):
        on.periodic_trapezoid_weights([0.0], 2 * np.pi)
    t = np.linspace(0.0, np.pi, 5)
    assert np.allclose(on.trapezoid_weights(t), np.pi / 4 * np.array([0.5, 1, 1, 1, 0.5]))
