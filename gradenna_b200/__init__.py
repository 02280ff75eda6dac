"""gradenna_b200: B200-native (sm_100a) FDTD time-stepping for gradenna's hot path.

Same Python surface as the reference's time-stepping core (Grid2D, CPMLSpec,
Port, simulate_tm, ...), with the time loop running in hand-written CUDA
kernels behind a C ABI (include/gradenna_b200.h) and torch tensors as the
array type.
"""

from gradenna_b200.constants import C0, EPS0, ETA0, MU0
from gradenna_b200.cpml import CPMLSpec, alpha_max_for_fmin, axis_coefficients
from gradenna_b200.fdtd2d import DZ, Port, SimResult, simulate_tm
from gradenna_b200.fdtd3d import DFTMonitor, SimResult3D, port_impedance, simulate_3d, time_series_dft
from gradenna_b200.grid import Grid2D, Grid3D
from gradenna_b200.sources import gaussian, gaussian_derivative, modulated_gaussian

__all__ = [
    "C0", "EPS0", "ETA0", "MU0",
    "CPMLSpec", "alpha_max_for_fmin", "axis_coefficients",
    "DZ", "Port", "SimResult", "simulate_tm",
    "DFTMonitor", "SimResult3D", "simulate_3d", "time_series_dft", "port_impedance",
    "Grid2D", "Grid3D",
    "gaussian", "gaussian_derivative", "modulated_gaussian",
]
