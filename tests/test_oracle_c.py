"""The C oracle (multi-threaded CPU restatement used for the CPU baseline)
agrees with the numpy oracle: float64 to 1e-12 and float32 to 1e-5,
peak-normalised, on a case with CPML, two sources, two ports (one active),
magnetic currents, probes, energy and a DFT (full grid and monitors)."""

import numpy as np
import pytest

from oracle import fdtd2d_np as onp
from oracle.tm2d_c import simulate_tm_c


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / (np.max(np.abs(b)) + 1e-300))


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
def test_c_oracle_matches_numpy_oracle(dtype, tol):
    g = onp.Grid2D(41, 37, 2e-3, 2e-3)
    n = 260
    t = (np.arange(n) + 0.5) * g.dt
    base = onp.gaussian_derivative(t, 20 * g.dt, 6 * g.dt).astype(dtype)
    kw = dict(source_ij=((15, 18), (25, 22)), source_current=np.stack([base, 0.3 * base], 1),
              probe_ij=((10, 12), (30, 30)), dft_freqs=(3e9, 5e9), cpml=onp.CPMLSpec(7),
              record_energy=True, mx_ij=((18, 20),), mx_current=0.2 * base[:, None],
              my_ij=((20, 12),), my_current=-0.1 * base[:, None],
              ports=[onp.Port((20, 20), 50.0, 0.5 * base), onp.Port((22, 24), 75.0, None)])
    r_np = onp.simulate_tm(g, dtype=dtype, dft_dtype=np.complex128, **kw)
    r_c, _ = simulate_tm_c(g, dtype=dtype, **kw)
    for name in ("probe_ez", "port_v", "port_i", "energy", "dft_ez", "dft_hx", "dft_hy", "ez", "hx", "hy"):
        e = rel(getattr(r_c, name), getattr(r_np, name))
        assert e <= (tol if name not in ("ez", "hx", "hy") else 10 * tol), f"{name}: {e:.2e}"
    _, mons = simulate_tm_c(g, dtype=dtype, dft_monitors=[(0, 5, 6, 20, 30), (2, 1, 2, 3, 30)], **kw)
    assert rel(mons[0], r_np.dft_ez[:, 5:20, 6:30]) <= tol
    assert rel(mons[1], r_np.dft_hy[:, 1:3, 2:30]) <= tol
