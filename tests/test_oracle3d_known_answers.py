"""Pin the 3D numpy oracle against the reference's 3D known answers
(tests/test_fdtd3d.py:37-141): small-dipole radiation resistance within
15 %, the gap-shunt bias of the raw port impedance, CPML energy decay to
1e-15 of the peak and x/y mirror symmetry to 1e-12."""

import types

from oracle import fdtd2d_np as o2
from oracle import fdtd3d_np as o3
from tests import known3d

MOD = types.SimpleNamespace(Grid3D=o3.Grid3D, CPMLSpec=o2.CPMLSpec,
                            alpha_max_for_fmin=o2.alpha_max_for_fmin,
                            simulate_3d=o3.simulate_3d, port_impedance=o3.port_impedance)


def test_small_dipole_radiation_resistance():
    grid, res = known3d.dipole(MOD)
    known3d.check_dipole(MOD, grid, res)


def test_cpml_energy_decay():
    known3d.check_energy_decay(MOD)


def test_mirror_symmetry_x_and_y():
    known3d.check_mirror_symmetry(MOD)
