"""Frequency-domain power monitors (src/gradenna/monitors.py:20-103).

``poynting_flux_box_2d`` is the closed-contour spectral Poynting flux of the
2D TM solver. Its forward reduction and its cotangent are CUDA kernels
(``gdn_poynting_box_2d`` / ``gdn_poynting_box_2d_grad``) behind a
``torch.autograd.Function``, so objectives built from it differentiate with
torch autograd on the device.
"""

from __future__ import annotations

import ctypes

import torch

from gradenna_b200 import _native
from gradenna_b200.grid import Grid2D

__all__ = ["poynting_flux_box_2d", "log_radiated_fraction", "poynting_box_monitors",
           "port_monitors"]

_I32x4 = ctypes.c_int32 * 4
_native.register("gdn_poynting_box_2d", ctypes.c_int, [
    ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
    ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p])
_native.register("gdn_poynting_box_2d_grad", ctypes.c_int, [
    ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
    ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
    ctypes.c_void_p])


def _check_box(box, grid):
    il, ir, jb, jt = (int(v) for v in box)
    if not (0 <= il < ir < grid.nx - 1 and 0 <= jb < jt < grid.ny - 1):
        raise ValueError(f"box {box!r} is not a valid contour on a {grid.nx}x{grid.ny} grid")
    return il, ir, jb, jt


class _PoyntingBox(torch.autograd.Function):
    @staticmethod
    def forward(ctx, ez, hx, hy, nx, ny, box, dx, dy):
        lib = _native.load()
        c128 = ez.dtype == torch.complex128
        ez, hx, hy = (t.contiguous() for t in (ez, hx, hy))
        out = torch.empty(ez.shape[0], dtype=torch.float64, device=ez.device)
        bx = _I32x4(*box)
        stream = torch.cuda.current_stream(ez.device).cuda_stream
        with torch.cuda.device(ez.device):
            _native.check(lib.gdn_poynting_box_2d(nx, ny, ez.shape[0], bx, dx, dy, int(c128),
                                                  ez.data_ptr(), hx.data_ptr(), hy.data_ptr(),
                                                  out.data_ptr(), stream))
        ctx.save_for_backward(ez, hx, hy)
        ctx.geom = (nx, ny, box, dx, dy, c128)
        return out

    @staticmethod
    def backward(ctx, g):
        ez, hx, hy = ctx.saved_tensors
        nx, ny, box, dx, dy, c128 = ctx.geom
        lib = _native.load()
        g = g.to(torch.float64).contiguous()
        gez, ghx, ghy = (torch.zeros_like(t) for t in (ez, hx, hy))
        stream = torch.cuda.current_stream(ez.device).cuda_stream
        with torch.cuda.device(ez.device):
            _native.check(lib.gdn_poynting_box_2d_grad(
                nx, ny, ez.shape[0], _I32x4(*box), dx, dy, int(c128), ez.data_ptr(),
                hx.data_ptr(), hy.data_ptr(), g.data_ptr(), gez.data_ptr(), ghx.data_ptr(),
                ghy.data_ptr(), stream))
        return gez, ghx, ghy, None, None, None, None, None


def poynting_flux_box_2d(dft_ez, dft_hx, dft_hy, grid: Grid2D, box):
    """Outward spectral Poynting flux through the dual-grid rectangle ``box``.

    box = (il, ir, jb, jt): the contour runs through the H sample points half
    a cell outside the Ez nodes il/ir/jb/jt. S = 1/2 Re(E x H*), Ez averaged
    onto the H positions of each face (monitors.py:20-70). Phasors are full
    grid complex tensors (n_freq, ...) on a CUDA device; returns (n_freq,)
    float64. Differentiable (torch autograd) in the phasors.
    """
    il, ir, jb, jt = _check_box(box, grid)
    for t, shp in ((dft_ez, (grid.nx, grid.ny)), (dft_hx, (grid.nx, grid.ny - 1)),
                   (dft_hy, (grid.nx - 1, grid.ny))):
        if tuple(t.shape[1:]) != shp:
            raise ValueError(f"phasor shape {tuple(t.shape)} does not match the grid {shp}")
    cd = torch.promote_types(torch.promote_types(dft_ez.dtype, dft_hx.dtype), dft_hy.dtype)
    ez, hx, hy = (t.to(cd) for t in (dft_ez, dft_hx, dft_hy))
    return _PoyntingBox.apply(ez, hx, hy, grid.nx, grid.ny, (il, ir, jb, jt), grid.dx, grid.dy)


def log_radiated_fraction(p_rad, p_avail):
    """Scale-invariant objective log P_rad - log P_avail (monitors.py:73-103)."""
    return torch.log(torch.as_tensor(p_rad)) - torch.log(torch.as_tensor(p_avail))


def poynting_box_monitors(box):
    """DFT monitor boxes (comp, lo_i, lo_j, hi_i, hi_j) covering exactly the
    phasors poynting_flux_box_2d reads: four Ez strips two cells wide, the
    two Hy rows and the two Hx columns of the contour. Recording only these
    (instead of full grids) is the 2D analogue of the reference's
    ntff_box_regions (src/gradenna/dft_region.py:187-227)."""
    il, ir, jb, jt = (int(v) for v in box)
    return [
        (0, il, jb + 1, il + 2, jt + 1), (0, ir, jb + 1, ir + 2, jt + 1),
        (0, il + 1, jb, ir + 1, jb + 2), (0, il + 1, jt, ir + 1, jt + 2),
        (2, il, jb + 1, il + 1, jt + 1), (2, ir, jb + 1, ir + 1, jt + 1),
        (1, il + 1, jb, ir + 1, jb + 1), (1, il + 1, jt, ir + 1, jt + 1),
    ]


def port_monitors(ij):
    """Monitor boxes covering what the port phasor rebuild reads at Ez cell
    (i, j): Ez(i, j), Hy(i-1..i, j), Hx(i, j-1..j) (freq_adjoint.py:536-558)."""
    i, j = (int(v) for v in ij)
    return [(0, i, j, i + 1, j + 1), (2, i - 1, j, i + 1, j + 1), (1, i, j - 1, i + 1, j + 1)]
