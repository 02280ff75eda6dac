"""CPML (CFS, Roden & Gedney 2000) coefficient tables, built on the host.

Same parameterisation and formulas as the reference (src/gradenna/cpml.py):

    psi^n = b psi^{n-1} + c (spatial difference)^n
    b = exp(-(sigma/kappa + alpha) dt/eps0)
    c = sigma (b - 1) / (kappa (sigma + kappa alpha))      (0 where undefined)
    sigma(rho) = sigma_max rho^m,  kappa(rho) = 1 + (kappa_max - 1) rho^m,
    alpha(rho) = alpha_max (1 - rho)^ma,
    sigma_max = sigma_factor 0.8 (m+1) / (eta0 dx sqrt(eps_r_bg)).

The tables are tiny 1D arrays computed once per run in the field dtype (the
reference evaluates them in the field dtype too, cpml.py:183-208) and uploaded
to the device; psi itself is stored only on the two PML slabs of each
stretched axis and updated by the CUDA kernels.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import NamedTuple

import numpy as np

from gradenna_b200.constants import EPS0, ETA0


@dataclass(frozen=True)
class CPMLSpec:
    """CPML parameters (cpml.py:35-44; Taflove & Hagness defaults)."""

    thickness: int = 10  # cells per side; 0 disables the PML (PEC box)
    m: float = 3.0  # polynomial grading order for sigma and kappa
    ma: float = 1.0  # grading order for alpha
    kappa_max: float = 5.0
    alpha_max: float = 0.0  # CFS term [S/m]; see alpha_max_for_fmin
    sigma_factor: float = 0.75  # sigma_max as a fraction of sigma_opt


def alpha_max_for_fmin(f_min: float) -> float:
    """CFS alpha_max so the transition frequency sits at the band lower edge."""
    return 2.0 * math.pi * f_min * EPS0


class AxisCoefficients(NamedTuple):
    """Per-position CPML tables along one axis: b, c and 1/kappa."""

    b: np.ndarray
    c: np.ndarray
    inv_kappa: np.ndarray


def slab_slices(n: int, thickness: int) -> tuple[slice, slice]:
    """Low/high PML slab slices along an axis of `n` samples (cpml.py:85-96)."""
    if not 0 <= 2 * thickness <= n:
        raise ValueError(f"PML slab thickness {thickness} too large for axis length {n}")
    return slice(0, thickness), slice(n - thickness, n)


def axis_coefficients(
    n: int,
    delta: float,
    dt: float,
    spec: CPMLSpec,
    *,
    half: bool,
    eps_r_bg: float = 1.0,
    dtype=np.float64,
) -> AxisCoefficients:
    """CPML tables for one axis of `n` integer (Ez) points (cpml.py:161-208).

    ``half=False`` samples the integer positions (length n, E-type psi);
    ``half=True`` samples i+1/2 (length n-1, H-type psi). Outside the layer
    c = 0 and 1/kappa = 1, so the update reduces exactly to plain Yee.
    """
    dtype = np.dtype(dtype)
    npml = spec.thickness
    if half:
        pos = np.arange(n - 1, dtype=dtype) + dtype.type(0.5)
    else:
        pos = np.arange(n, dtype=dtype)
    if npml == 0:
        zeros = np.zeros_like(pos)
        return AxisCoefficients(zeros, zeros.copy(), np.ones_like(pos))
    depth_left = (dtype.type(npml) - pos) / dtype.type(npml)
    depth_right = (pos - dtype.type(n - 1 - npml)) / dtype.type(npml)
    rho = np.clip(np.maximum(depth_left, depth_right), 0.0, 1.0).astype(dtype)
    sigma_max = spec.sigma_factor * 0.8 * (spec.m + 1.0) / (ETA0 * delta * math.sqrt(eps_r_bg))
    sigma = (sigma_max * rho**spec.m).astype(dtype)
    kappa = (1.0 + (spec.kappa_max - 1.0) * rho**spec.m).astype(dtype)
    alpha = np.where(rho > 0.0, spec.alpha_max * (1.0 - rho) ** spec.ma, 0.0).astype(dtype)
    b = np.exp(-(sigma / kappa + alpha) * dt / EPS0).astype(dtype)
    denom = sigma + kappa * alpha
    safe = np.where(denom > 0.0, denom, 1.0).astype(dtype)
    c = np.where(denom > 0.0, sigma * (b - 1.0) / (kappa * safe), 0.0).astype(dtype)
    return AxisCoefficients(b, c, (1.0 / kappa).astype(dtype))


def slab_tables(b: np.ndarray, c: np.ndarray, thickness: int):
    """(b_lo, c_lo, b_hi, c_hi): the tables restricted to the two slabs."""
    lo, hi = slab_slices(b.shape[0], thickness)
    return (
        np.ascontiguousarray(b[lo]),
        np.ascontiguousarray(c[lo]),
        np.ascontiguousarray(b[hi]),
        np.ascontiguousarray(c[hi]),
    )
