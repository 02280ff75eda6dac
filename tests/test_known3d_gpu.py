"""The reference's 3D known answers (tests/test_fdtd3d.py:37-141) through the
CUDA path, in float64 and float32 (the dipole check in both; energy decay
needs float64's range for its 1e-15 floor)."""

import numpy as np
import pytest

from tests import known3d

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_small_dipole_radiation_resistance(dtype):
    import gradenna_b200 as gb

    grid, res = known3d.dipole(gb, dtype=dtype)
    known3d.check_dipole(gb, grid, res)


def test_cpml_energy_decay():
    import gradenna_b200 as gb

    known3d.check_energy_decay(gb, dtype=np.float64)


def test_mirror_symmetry_x_and_y():
    import gradenna_b200 as gb

    known3d.check_mirror_symmetry(gb, dtype=np.float64)
