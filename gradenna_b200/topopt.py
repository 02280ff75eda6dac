"""Topology-optimisation pieces (src/gradenna/topopt.py): conic filter,
tanh projection, the sigmoid -> filter -> projection transform, beta
continuation, the gray indicator, the fabrication checks and the Adam
driver ``optimize``.

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
    """(K * rho) / (K * 1) with a conic kernel of radius R cells, for 1D, 2D
    or 3D densities (topopt.py:65-90)."""
    radius = float(radius_cells)
    if radius <= 1.0:
        return rho
    if rho.ndim not in (1, 2, 3):
        raise ValueError("conic_filter supports 1D, 2D and 3D densities")
    conv = {1: F.conv1d, 2: F.conv2d, 3: F.conv3d}[rho.ndim]
    k = torch.as_tensor(conic_kernel(radius, rho.ndim), dtype=rho.dtype, device=rho.device)
    pad = k.shape[0] // 2
    num = conv(rho[None, None], k[None, None], padding=pad)[0, 0]
    den = conv(torch.ones_like(rho)[None, None], k[None, None], padding=pad)[0, 0]
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


def _register_design_entry_points():
    import ctypes

    from gradenna_b200 import _native

    v, i, d = ctypes.c_void_p, ctypes.c_int32, ctypes.c_double
    _native.register("gdn_design_forward", ctypes.c_int, [v, i, i, i, v, i, d, d, v, v, v, v])
    _native.register("gdn_design_backward", ctypes.c_int,
                     [v, v, v, v, i, i, i, v, i, d, d, v, v])


_register_design_entry_points()


class _DesignTransformCUDA(torch.autograd.Function):
    """sigmoid -> conic filter -> tanh projection of a batch of float64
    designs on the GPU (gdn_design_forward / gdn_design_backward)."""

    @staticmethod
    def forward(ctx, theta, beta, radius, eta):
        import ctypes

        from gradenna_b200 import _native

        lib = _native.load()
        th = theta.detach().contiguous()
        B, H, W = th.shape
        if radius > 1.0:
            kern = torch.as_tensor(conic_kernel(radius, 2), dtype=torch.float64, device=th.device)
        else:
            kern = torch.ones((1, 1), dtype=torch.float64, device=th.device)
        n = (kern.shape[0] - 1) // 2
        filt, norm, rho = (torch.empty_like(th) for _ in range(3))
        s = ctypes.c_void_p(torch.cuda.current_stream(th.device).cuda_stream)
        with torch.cuda.device(th.device):
            _native.check(lib.gdn_design_forward(th.data_ptr(), B, H, W, kern.data_ptr(), n,
                                                 float(beta), float(eta), filt.data_ptr(),
                                                 norm.data_ptr(), rho.data_ptr(), s))
        ctx.save_for_backward(th, filt, norm, kern)
        ctx.args = (float(beta), float(eta), n)
        return rho

    @staticmethod
    def backward(ctx, g):
        import ctypes

        from gradenna_b200 import _native

        th, filt, norm, kern = ctx.saved_tensors
        beta, eta, n = ctx.args
        g = g.contiguous().to(torch.float64)
        out = torch.empty_like(th)
        B, H, W = th.shape
        s = ctypes.c_void_p(torch.cuda.current_stream(th.device).cuda_stream)
        with torch.cuda.device(th.device):
            _native.check(_native.load().gdn_design_backward(
                th.data_ptr(), filt.data_ptr(), norm.data_ptr(), g.data_ptr(), B, H, W,
                kern.data_ptr(), n, beta, eta, out.data_ptr(), s))
        return out, None, None, None


def design_transform_batch(theta: torch.Tensor, beta, radius: float,
                           eta: float = 0.5) -> torch.Tensor:
    """DesignTransform of a batch theta (B, H, W), differentiable. float64
    CUDA tensors run the library's fused kernels (one launch forward, one
    backward); other tensors run the torch form."""
    if theta.is_cuda and theta.dtype == torch.float64 and theta.ndim == 3:
        return _DesignTransformCUDA.apply(theta, float(beta), float(radius), float(eta))
    rho = torch.sigmoid(theta)
    if radius > 1.0:
        k = torch.as_tensor(conic_kernel(radius, 2), dtype=rho.dtype, device=rho.device)
        pad = k.shape[0] // 2
        num = F.conv2d(rho[:, None], k[None, None], padding=pad)[:, 0]
        den = F.conv2d(torch.ones_like(rho[:1, None]), k[None, None], padding=pad)[:, 0]
        rho = num / den
    return tanh_projection(rho, beta, eta)


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


def gray_indicator(rho: torch.Tensor) -> torch.Tensor:
    """Mean of 4 rho (1 - rho): 0 for a binary field, 1 at rho = 0.5 (topopt.py:153-155)."""
    return torch.mean(4.0 * rho * (1.0 - rho))


# ---------------------------------------------------------------------------
# Post-processing checks (host, non-differentiable; topopt.py:158-237)
# ---------------------------------------------------------------------------


def _np(x):
    return x.detach().cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)


def connected_to_seed(rho_binary, seed_ij) -> np.ndarray:
    """Solid (> 0.5) 4-connected component containing the seed pixel; all
    False when the seed is not solid (topopt.py:163-184)."""
    from scipy import ndimage

    solid = _np(rho_binary) > 0.5
    labels, _ = ndimage.label(solid)
    lab = labels[tuple(int(v) for v in seed_ij)]
    if lab == 0:
        return np.zeros_like(solid, dtype=bool)
    return labels == lab


def _disk_footprint(width_cells: int) -> np.ndarray:
    """Disk of radius (w - 1) / 2 cells (topopt.py:187-199)."""
    radius = (width_cells - 1) / 2.0
    n = int(np.floor(radius))
    y, x = np.mgrid[-n:n + 1, -n:n + 1]
    return (x * x + y * y) <= radius * radius + 1e-9


def minimum_feature_size(rho_binary, width_cells: int) -> np.ndarray:
    """Solid pixels removed by a binary opening with the disk footprint: the
    features thinner than the minimum width (topopt.py:202-237). Erosion
    treats the domain edge as solid, so clipped features are not flagged."""
    from scipy import ndimage

    solid = _np(rho_binary) > 0.5
    if width_cells <= 1:
        return np.zeros_like(solid, dtype=bool)
    fp = _disk_footprint(int(width_cells))
    eroded = ndimage.binary_erosion(solid, structure=fp, border_value=1)
    opened = ndimage.binary_dilation(eroded, structure=fp, border_value=0)
    return solid & ~opened


# ---------------------------------------------------------------------------
# Optimisation driver (topopt.py:245-319)
# ---------------------------------------------------------------------------


def optimize(loss_fn, theta0, n_steps: int = 400, betas=(8.0, 16.0, 32.0, 64.0),
             learning_rate: float = 0.02, transform: DesignTransform | None = None,
             n_snapshots: int = 4) -> dict:
    """Adam with beta continuation over the three-field parameterisation.

    ``loss_fn(rho, beta)`` returns a scalar tensor differentiable in rho by
    torch autograd (for FDTD objectives: freq_adjoint_objective, whose
    backward is the two-run adjoint on the GPU). ``theta0`` is the latent
    design; it stays on its device, where the transform and the Adam update
    (torch.optim.Adam: beta1 0.9, beta2 0.999, eps 1e-8, the optax.adam
    defaults of the reference) run. ``n_steps`` are split evenly over
    ``betas``. Returns the reference's dict: "theta", "rho" (the final theta
    projected at the final beta), per-step "loss", "gray" and "beta" arrays,
    and "snapshots" [(step, rho numpy)].
    """
    if transform is None:
        transform = DesignTransform(radius_cells=2.0)
    betas = tuple(betas)
    schedule = beta_schedule(betas, max(1, n_steps // len(betas)))
    theta = torch.as_tensor(theta0).detach().clone().requires_grad_(True)
    opt = torch.optim.Adam([theta], lr=learning_rate, betas=(0.9, 0.999), eps=1e-8)
    snap_at = set(int(round(v)) for v in np.linspace(0, n_steps - 1, max(1, n_snapshots)))
    losses, grays, beta_hist, snaps = [], [], [], []
    for i in range(n_steps):
        beta = schedule(i)
        opt.zero_grad(set_to_none=True)
        rho = transform(theta, beta)
        loss = loss_fn(rho, beta)
        loss.backward()
        opt.step()
        losses.append(float(loss.detach()))
        grays.append(float(gray_indicator(rho.detach())))
        beta_hist.append(beta)
        if i in snap_at:
            snaps.append((i, rho.detach().cpu().numpy()))
    with torch.no_grad():
        rho = transform(theta, schedule(max(0, n_steps - 1)))
    return {"theta": theta.detach(), "rho": rho, "loss": np.asarray(losses),
            "gray": np.asarray(grays), "beta": np.asarray(beta_hist), "snapshots": snaps}
