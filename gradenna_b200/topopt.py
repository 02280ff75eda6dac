"""Design-parameterisation pieces used to build design densities
(src/gradenna/topopt.py:55-150): conic filter, tanh projection, the
sigmoid -> filter -> projection transform and the beta continuation.

torch implementations (differentiable, any device). The conic filter is a
direct "same" convolution with the renormalised boundary of the reference
(fftconvolve(rho, K) / fftconvolve(1, K)); the kernel is symmetric, so
correlation and convolution coincide.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch
import torch.nn.functional as F


def conic_kernel(radius_cells: float, ndim: int = 2) -> np.ndarray:
    """Normalised hat kernel w = max(0, 1 - d/R) on offsets |o| <= ceil(R)-1 (topopt.py:55-62)."""
    radius = float(radius_cells)
    n = int(np.ceil(radius)) - 1
    offsets = np.meshgrid(*([np.arange(-n, n + 1)] * ndim), indexing="ij")
    d2 = sum(o.astype(np.float64) ** 2 for o in offsets)
    w = np.maximum(0.0, 1.0 - np.sqrt(d2) / radius)
    return w / w.sum()


def conic_filter(rho: torch.Tensor, radius_cells: float) -> torch.Tensor:
    """(K * rho) / (K * 1) with a conic kernel of radius R cells (topopt.py:65-90)."""
    radius = float(radius_cells)
    if radius <= 1.0:
        return rho
    if rho.ndim != 2:
        raise ValueError("conic_filter here supports 2D densities")
    k = torch.as_tensor(conic_kernel(radius, 2), dtype=rho.dtype, device=rho.device)
    pad = k.shape[0] // 2
    num = F.conv2d(rho[None, None], k[None, None], padding=pad)[0, 0]
    den = F.conv2d(torch.ones_like(rho)[None, None], k[None, None], padding=pad)[0, 0]
    return num / den


def tanh_projection(rho: torch.Tensor, beta, eta: float = 0.5) -> torch.Tensor:
    """Smoothed Heaviside of Wang, Lazarov & Sigmund (topopt.py:93-105)."""
    beta = torch.as_tensor(beta, dtype=rho.dtype, device=rho.device)
    num = torch.tanh(beta * eta) + torch.tanh(beta * (rho - eta))
    den = torch.tanh(beta * eta) + torch.tanh(beta * (1.0 - eta))
    return num / den


@dataclass(frozen=True)
class DesignTransform:
    """theta -> sigmoid -> conic filter -> tanh projection (topopt.py:109-127)."""

    radius_cells: float
    eta: float = 0.5

    def __call__(self, theta: torch.Tensor, beta) -> torch.Tensor:
        rho = torch.sigmoid(theta)
        rho = conic_filter(rho, self.radius_cells)
        return tanh_projection(rho, beta, self.eta)


def beta_schedule(betas=(8.0, 16.0, 32.0, 64.0), steps_per_beta: int = 100):
    """beta continuation: iteration -> beta, one stage per ``steps_per_beta``
    iterations, holding the last stage afterwards (topopt.py:130-150)."""
    if steps_per_beta < 1:
        raise ValueError("steps_per_beta must be >= 1")
    stages = tuple(float(b) for b in betas)
    if not stages:
        raise ValueError("betas must be non-empty")

    def schedule(step: int) -> float:
        return stages[min(step // steps_per_beta, len(stages) - 1)]

    return schedule


def seeded_density(shape, seed: int = 0, radius_cells: float = 3.0, beta: float = 8.0,
                   eta: float = 0.5, device=None, dtype=torch.float64) -> torch.Tensor:
    """tanh_projection(conic_filter(U(0,1) noise, R), beta, eta) from numpy default_rng(seed)."""
    noise = np.random.default_rng(seed).uniform(0.0, 1.0, size=shape)
    rho = torch.as_tensor(noise, dtype=dtype, device=device)
    return tanh_projection(conic_filter(rho, radius_cells), beta, eta)
