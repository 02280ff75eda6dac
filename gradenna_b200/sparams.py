"""S-parameter extraction for lumped RVS ports (src/gradenna/sparams.py:1-134).

Exact-phase DFT of the (n+1/2) dt port samples, the Kurokawa power-wave S11,
the analytic incident wave of a matched port and the openEMS-compatible band
pulse. Works on torch tensors (any device) and numpy arrays alike; results
are complex128 torch tensors.
"""

from __future__ import annotations

import math
from typing import NamedTuple

import numpy as np
import torch


def _as_t(x, device=None):
    if isinstance(x, torch.Tensor):
        return x.to(torch.float64) if not x.is_complex() else x.to(torch.complex128)
    return torch.as_tensor(np.asarray(x), device=device).to(torch.float64)


def half_step_dft(x_t, dt: float, freqs):
    """X(f) = dt sum_n x[n] exp(-i 2 pi f (n + 1/2) dt)   (sparams.py:24-46).

    x_t: (n_steps,) or (n_steps, k); returns (n_freq,) or (n_freq, k).
    """
    x = _as_t(x_t)
    f = torch.as_tensor(np.atleast_1d(np.asarray(freqs, np.float64)), device=x.device)
    t = (torch.arange(x.shape[0], device=x.device, dtype=torch.float64) + 0.5) * dt
    kern = torch.exp(-2j * math.pi * f[:, None] * t[None, :]) * dt
    return torch.tensordot(kern, x.to(torch.complex128), dims=([1], [0]))


def port_dft(v_t, i_t, dt: float, freqs):
    """(V_hat, I_hat) of the port series, both sampled at (n+1/2) dt (sparams.py:49-65)."""
    return half_step_dft(v_t, dt, freqs), half_step_dft(i_t, dt, freqs)


def s11_power_wave(v_hat, i_hat, z0=50.0):
    """Kurokawa power-wave reflection S11 = (V - Z0 I)/(V + Z0 I) (sparams.py:68-79)."""
    return (v_hat - z0 * i_hat) / (v_hat + z0 * i_hat)


def incident_voltage(vs_hat):
    """Incident wave of a matched RVS port, V_inc = Vs/2 (sparams.py:82-91)."""
    return vs_hat / 2.0


class BandPulse(NamedTuple):
    """Modulated Gaussian cos(2 pi f0 (t-t0)) exp(-(t-t0)^2/(2 sigma^2)) (sparams.py:94-118)."""

    f0: float
    fc: float
    sigma: float
    t0: float

    @property
    def duration(self) -> float:
        return 2.0 * self.t0

    def __call__(self, t):
        u = np.asarray(t) - self.t0
        return np.cos(2.0 * np.pi * self.f0 * u) * np.exp(-(u**2) / (2.0 * self.sigma**2))


def gaussian_pulse_for_band(f_min: float, f_max: float) -> BandPulse:
    """Band pulse with -20 dB edges at f_min, f_max (sparams.py:121-134)."""
    if not 0.0 < f_min < f_max:
        raise ValueError(f"need 0 < f_min < f_max, got [{f_min}, {f_max}]")
    f0 = 0.5 * (f_min + f_max)
    fc = 0.5 * (f_max - f_min)
    sigma = 3.0 / (2.0 * math.sqrt(2.0) * math.pi * fc)
    t0 = 9.0 / (2.0 * math.pi * fc)
    return BandPulse(f0=f0, fc=fc, sigma=sigma, t0=t0)
