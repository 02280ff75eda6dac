"""Excitation waveforms (src/gradenna/sources.py:1-30), numpy versions.

All take a time array [s] and return order-one amplitudes.
"""

from __future__ import annotations

import numpy as np


def gaussian(t, t0: float, tau: float):
    """Gaussian pulse exp(-(t-t0)^2 / (2 tau^2)). Contains DC."""
    u = (np.asarray(t) - t0) / tau
    return np.exp(-0.5 * u**2)


def gaussian_derivative(t, t0: float, tau: float):
    """Differentiated Gaussian (no DC), peak amplitude ~1; spectrum peaks at 1/(2 pi tau)."""
    u = (np.asarray(t) - t0) / tau
    return -u * np.exp(0.5 * (1.0 - u**2))


def modulated_gaussian(t, f0: float, t0: float, tau: float):
    """Sine carrier at f0 under a Gaussian envelope."""
    t = np.asarray(t)
    u = (t - t0) / tau
    return np.sin(2.0 * np.pi * f0 * (t - t0)) * np.exp(-0.5 * u**2)
