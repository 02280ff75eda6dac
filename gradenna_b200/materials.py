"""Metal interpolations for density-based design (src/gradenna/materials.py:28-73)."""

from __future__ import annotations

import math

import numpy as np
import torch


def sigma_from_density(rho, sigma_min: float = 1e-4, sigma_max: float = 1e5):
    """sigma(rho) = 10 ** (log10 sigma_min + rho (log10 sigma_max - log10 sigma_min))."""
    if not 0.0 < sigma_min < sigma_max:
        raise ValueError(f"need 0 < sigma_min < sigma_max, got [{sigma_min}, {sigma_max}]")
    lo, hi = math.log10(sigma_min), math.log10(sigma_max)
    if isinstance(rho, torch.Tensor):
        return torch.pow(10.0, (hi - lo) * rho + lo)
    return 10.0 ** ((hi - lo) * np.asarray(rho) + lo)


def sheet_conductivity(sigma_bulk: float, thickness: float, dz: float) -> float:
    """Equivalent conductivity of a thin sheet smeared over one cell: sigma t / dz."""
    if thickness <= 0.0 or dz <= 0.0:
        raise ValueError("thickness and dz must be positive")
    return sigma_bulk * thickness / dz
