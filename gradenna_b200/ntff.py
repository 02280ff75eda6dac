"""Near-to-far-field (NTFF) transforms for the 2D TM and 3D solvers
(src/gradenna/ntff.py:1-520).

The running-DFT phasors of the tangential fields on a closed contour (2D) or
box (3D) become equivalent surface currents Js = n x H, Ms = -n x E, whose
free-space radiation is the far-field pattern. Conventions follow the
reference exactly (ntff.py:1-45): engineering e^{+j omega t} time convention,
dt-scaled DFT phasors, pattern amplitudes with the radial spreading and the
propagation phase removed, phase referenced to the grid centre, and the Yee
samples averaged spatially onto the surface points.

Split of the work on B200: gathering the staggered samples onto the surface
points is a handful of strided slices (torch, differentiable by autograd);
the projection itself, n_freq x n_dir x n_pts complex exponentials, is a
CUDA kernel (``gdn_ntff3d_project`` / ``gdn_ntff2d_project``) behind a
``torch.autograd.Function`` whose backward is the adjoint kernel, so a
directivity or gain objective differentiates back onto the DFT phasors on
the device.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from gradenna_b200 import _native
from gradenna_b200.constants import C0, ETA0
from gradenna_b200.grid import Grid2D, Grid3D

__all__ = [
    "directivity_2d",
    "directivity_3d",
    "gain",
    "ntff_2d",
    "ntff_3d",
    "radiated_power_2d",
    "radiated_power_3d",
]

_V = ctypes.c_void_p
_I = ctypes.c_int32
_D = ctypes.c_double
_native.register("gdn_ntff3d_project", ctypes.c_int,
                 [_I, _I, _I, _I, _V, _V, _V, _V, _V, _V, _D, _V, _V])
_native.register("gdn_ntff3d_project_grad", ctypes.c_int,
                 [_I, _I, _I, _I, _V, _V, _V, _V, _D, _V, _V, _V, _V])
_native.register("gdn_ntff2d_project", ctypes.c_int,
                 [_I, _I, _I, _I, _V, _V, _V, _V, _V, _V, _D, _V, _V])
_native.register("gdn_ntff2d_project_grad", ctypes.c_int,
                 [_I, _I, _I, _I, _V, _V, _V, _V, _D, _V, _V, _V, _V])


# ---------------------------------------------------------------------------
# Quadrature weights (ntff.py:64-92)
# ---------------------------------------------------------------------------


def _as_f64(a, device=None) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a.detach().to(dtype=torch.float64, device=device)
    return torch.as_tensor(np.asarray(a, np.float64), device=device)


def _periodic_trapezoid_weights(angles, period: float, device=None) -> torch.Tensor:
    """Half the cyclic distance to both neighbours per sample (ntff.py:64-84)."""
    a = _as_f64(angles, device)
    if a.ndim != 1 or a.shape[0] < 2:
        raise ValueError("need a 1D array of at least 2 angles")
    d_next = torch.remainder(torch.roll(a, -1) - a, period)
    d_prev = torch.remainder(a - torch.roll(a, 1), period)
    return 0.5 * (d_next + d_prev)


def _trapezoid_weights(x, device=None) -> torch.Tensor:
    """Plain trapezoid weights for sorted samples (ntff.py:87-92)."""
    x = _as_f64(x, device)
    if x.ndim != 1 or x.shape[0] < 2:
        raise ValueError("need a 1D array of at least 2 samples")
    d = torch.diff(x)
    return 0.5 * torch.cat([d[:1], d[:-1] + d[1:], d[-1:]])


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


def _wavenumbers(freqs, n_freq, dev):
    freqs = np.atleast_1d(np.asarray(freqs, np.float64))
    if freqs.shape[0] != n_freq:
        raise ValueError(f"freqs has {freqs.shape[0]} entries but the phasors have {n_freq} rows")
    return torch.as_tensor(2.0 * np.pi * freqs / C0, device=dev)


# ---------------------------------------------------------------------------
# Projection kernels behind autograd
# ---------------------------------------------------------------------------


class _Project2D(torch.autograd.Function):
    @staticmethod
    def forward(ctx, jz, ez, pos, w, k, angles):
        lib = _native.load()
        c128 = jz.dtype == torch.complex128
        jz, ez = jz.contiguous(), ez.contiguous()
        n_freq, n_pts = jz.shape
        out = torch.empty((n_freq, angles.shape[0]), dtype=jz.dtype, device=jz.device)
        with torch.cuda.device(jz.device):
            _native.check(lib.gdn_ntff2d_project(
                n_freq, n_pts, angles.shape[0], int(c128), pos.data_ptr(), w.data_ptr(),
                jz.data_ptr(), ez.data_ptr(), k.data_ptr(), angles.data_ptr(), ETA0,
                out.data_ptr(), _stream(jz.device)))
        ctx.save_for_backward(pos, w, k, angles)
        ctx.meta = (n_freq, n_pts, c128, jz.dtype)
        return out

    @staticmethod
    def backward(ctx, g):
        pos, w, k, angles = ctx.saved_tensors
        n_freq, n_pts, c128, cdt = ctx.meta
        lib = _native.load()
        g = g.to(cdt).contiguous()
        gj = torch.empty((n_freq, n_pts), dtype=cdt, device=g.device)
        ge = torch.empty_like(gj)
        with torch.cuda.device(g.device):
            _native.check(lib.gdn_ntff2d_project_grad(
                n_freq, n_pts, angles.shape[0], int(c128), pos.data_ptr(), w.data_ptr(),
                k.data_ptr(), angles.data_ptr(), ETA0, g.data_ptr(), gj.data_ptr(),
                ge.data_ptr(), _stream(g.device)))
        return gj, ge, None, None, None, None


class _Project3D(torch.autograd.Function):
    @staticmethod
    def forward(ctx, j, m, pos, w, k, dirs):
        lib = _native.load()
        c128 = j.dtype == torch.complex128
        j, m = j.contiguous(), m.contiguous()
        n_freq, n_pts = j.shape[0], j.shape[1]
        n_dir = dirs.shape[0]
        out = torch.empty((n_freq, n_dir, 2), dtype=j.dtype, device=j.device)
        with torch.cuda.device(j.device):
            _native.check(lib.gdn_ntff3d_project(
                n_freq, n_pts, n_dir, int(c128), pos.data_ptr(), w.data_ptr(), j.data_ptr(),
                m.data_ptr(), k.data_ptr(), dirs.data_ptr(), ETA0, out.data_ptr(),
                _stream(j.device)))
        ctx.save_for_backward(pos, w, k, dirs)
        ctx.meta = (n_freq, n_pts, c128, j.dtype)
        return out

    @staticmethod
    def backward(ctx, g):
        pos, w, k, dirs = ctx.saved_tensors
        n_freq, n_pts, c128, cdt = ctx.meta
        lib = _native.load()
        g = g.to(cdt).contiguous()
        gj = torch.empty((n_freq, n_pts, 3), dtype=cdt, device=g.device)
        gm = torch.empty_like(gj)
        with torch.cuda.device(g.device):
            _native.check(lib.gdn_ntff3d_project_grad(
                n_freq, n_pts, dirs.shape[0], int(c128), pos.data_ptr(), w.data_ptr(),
                k.data_ptr(), dirs.data_ptr(), ETA0, g.data_ptr(), gj.data_ptr(),
                gm.data_ptr(), _stream(g.device)))
        return gj, gm, None, None, None, None


def _complex_dtype(*ts):
    return torch.complex128 if any(t.dtype == torch.complex128 for t in ts) else torch.complex64


# ---------------------------------------------------------------------------
# 2D TM
# ---------------------------------------------------------------------------


def contour_points_2d(grid: Grid2D, contour_margin: int):
    """Geometry of the ntff_2d contour (ntff.py:152-213).

    Returns (pos, w, sides): pos (n_pts, 4) = (x, y, n_x, n_y) relative to
    the grid centre, w (n_pts,) trapezoid weights per side (corner nodes
    appear once per side at half weight), and the (i0, i1, j0, j1) node
    indices of the rectangle. Sides are ordered right, left, top, bottom.
    """
    nx, ny = grid.nx, grid.ny
    m = int(contour_margin)
    if m < 1:
        raise ValueError("contour_margin must be >= 1 (H averaging needs one cell)")
    i0, i1 = m, nx - 1 - m
    j0, j1 = m, ny - 1 - m
    if i1 - i0 < 2 or j1 - j0 < 2:
        raise ValueError(f"contour_margin {m} leaves no contour on a {nx}x{ny} grid")
    xn = (np.arange(nx) - 0.5 * (nx - 1)) * grid.dx
    yn = (np.arange(ny) - 0.5 * (ny - 1)) * grid.dy

    def weights(n, dl):
        w = np.full(n, dl)
        w[0] *= 0.5
        w[-1] *= 0.5
        return w

    ys, xs = yn[j0:j1 + 1], xn[i0:i1 + 1]
    nj, ni = ys.shape[0], xs.shape[0]
    pos, ws = [], []
    for x, y, n_x, n_y, w in (
        (np.full(nj, xn[i1]), ys, 1.0, 0.0, weights(nj, grid.dy)),
        (np.full(nj, xn[i0]), ys, -1.0, 0.0, weights(nj, grid.dy)),
        (xs, np.full(ni, yn[j1]), 0.0, 1.0, weights(ni, grid.dx)),
        (xs, np.full(ni, yn[j0]), 0.0, -1.0, weights(ni, grid.dx)),
    ):
        pos.append(np.stack([x, y, np.full(x.shape, n_x), np.full(x.shape, n_y)], axis=-1))
        ws.append(w)
    return np.concatenate(pos), np.concatenate(ws), (i0, i1, j0, j1)


def _contour_currents_2d(dft_ez, dft_hx, dft_hy, sides):
    """Jz = n x H (z part) with H averaged onto the Ez nodes, and Ez (ntff.py:178-211)."""
    i0, i1, j0, j1 = sides
    jr, ir = slice(j0, j1 + 1), slice(i0, i1 + 1)
    jz = torch.cat([
        0.5 * (dft_hy[:, i1 - 1, jr] + dft_hy[:, i1, jr]),
        -0.5 * (dft_hy[:, i0 - 1, jr] + dft_hy[:, i0, jr]),
        -0.5 * (dft_hx[:, ir, j1 - 1] + dft_hx[:, ir, j1]),
        0.5 * (dft_hx[:, ir, j0 - 1] + dft_hx[:, ir, j0]),
    ], dim=1)
    ez = torch.cat([dft_ez[:, i1, jr], dft_ez[:, i0, jr], dft_ez[:, ir, j1], dft_ez[:, ir, j0]],
                   dim=1)
    return jz, ez


def ntff_2d(dft_ez, dft_hx, dft_hy, grid: Grid2D, contour_margin: int, freqs, angles):
    """2D TM near-to-far-field transform on a rectangular contour (ntff.py:100-232).

    E_far(f, phi) = -sqrt(j k / 8 pi) * closed-integral (eta0 Jz - M_phi)
    e^{+jk(x' cos phi + y' sin phi)} dl' over the Ez-node rectangle
    ``contour_margin`` cells inside the grid boundary, with Jz = n'_x Hy -
    n'_y Hx and M_phi = (n' . u_phi) Ez.

    Args:
        dft_ez, dft_hx, dft_hy: (n_freq, nx, ny) / (n_freq, nx, ny-1) /
            (n_freq, nx-1, ny) complex phasors on a CUDA device
            (``SimResult.dft_ez`` etc.).
        grid: the 2D Yee grid.
        contour_margin: contour distance from the boundary in cells (>= 1).
        freqs: (n_freq,) frequencies [Hz] of the phasor axis.
        angles: (n_angles,) observation angles phi [rad] from +x.

    Returns:
        Complex (n_freq, n_angles) pattern amplitude, differentiable w.r.t.
        the three phasor tensors.
    """
    dev = dft_ez.device
    if dev.type != "cuda":
        raise RuntimeError("ntff_2d runs on a CUDA device; phasors are on " + str(dev))
    pos, w, sides = contour_points_2d(grid, contour_margin)
    k = _wavenumbers(freqs, dft_ez.shape[0], dev)
    cdt = _complex_dtype(dft_ez, dft_hx, dft_hy)
    jz, ez = _contour_currents_2d(dft_ez.to(cdt), dft_hx.to(cdt), dft_hy.to(cdt), sides)
    ang = _as_f64(angles, dev).reshape(-1).contiguous()
    return _Project2D.apply(jz, ez, torch.as_tensor(pos, device=dev).contiguous(),
                            torch.as_tensor(w, device=dev), k, ang)


def radiated_power_2d(e_far, angles):
    """P' = closed-integral |E_far|^2 / (2 eta0) dphi (ntff.py:235-244); (n_freq,)."""
    w = _periodic_trapezoid_weights(angles, 2.0 * math.pi, e_far.device)
    return torch.sum(w * torch.abs(e_far) ** 2, dim=-1) / (2.0 * ETA0)


def directivity_2d(e_far, angles):
    """D(phi) = 2 pi |E_far|^2 / closed-integral |E_far|^2 dphi (ntff.py:247-256)."""
    e2 = torch.abs(e_far) ** 2
    w = _periodic_trapezoid_weights(angles, 2.0 * math.pi, e_far.device)
    total = torch.sum(w * e2, dim=-1, keepdim=True)
    return 2.0 * math.pi * e2 / total


# ---------------------------------------------------------------------------
# 3D
# ---------------------------------------------------------------------------


class _Comp:
    """One monitor component in full-grid coordinates, full or slab-limited."""

    def __init__(self, arr, lo):
        self.arr, self.lo = arr, lo

    def __getitem__(self, idx):
        sl = [slice(None)]
        for d, ix in enumerate(idx):
            o = self.lo[d]
            if isinstance(ix, slice):
                a, b = ix.start - o, ix.stop - o
                if a < 0 or b > self.arr.shape[d + 1]:
                    raise ValueError("the DFT monitor region does not cover the NTFF box")
                sl.append(slice(a, b))
            else:
                if not 0 <= ix - o < self.arr.shape[d + 1]:
                    raise ValueError("the DFT monitor region does not cover the NTFF box")
                sl.append(ix - o)
        return self.arr[tuple(sl)]


def _monitor_components(mon):
    names = ("ex", "ey", "ez", "hx", "hy", "hz")
    regions = getattr(mon, "regions", None)
    comps = []
    for c, name in enumerate(names):
        arr = getattr(mon, name)
        if arr is None:
            raise ValueError(f"the DFT monitor has no {name} component; ntff_3d needs all six")
        lo = (0, 0, 0) if regions is None or regions[c] is None else tuple(regions[c].lo)
        comps.append(_Comp(arr, lo))
    return comps


def box_points_3d(grid3d: Grid3D, box_margin: int):
    """Geometry of the ntff_3d box (ntff.py:322-372).

    Returns (pos, w, bounds): pos (n_pts, 3) face-patch centres relative to
    the grid centre, w (n_pts,) patch areas, bounds = (i0, i1, j0, j1, k0,
    k1). Faces are ordered +x, -x, +y, -y, +z, -z; each face is flattened in
    C order over its two in-plane cell indices.
    """
    nx, ny, nz = grid3d.nx, grid3d.ny, grid3d.nz
    dx, dy, dz = grid3d.dx, grid3d.dy, grid3d.dz
    m = int(box_margin)
    if m < 1:
        raise ValueError("box_margin must be >= 1 (H averaging needs one cell)")
    i0, i1, j0, j1, k0, k1 = m, nx - 1 - m, m, ny - 1 - m, m, nz - 1 - m
    if i1 - i0 < 1 or j1 - j0 < 1 or k1 - k0 < 1:
        raise ValueError(f"box_margin {m} leaves no box on a {nx}x{ny}x{nz} grid")
    xn = (np.arange(nx) - 0.5 * (nx - 1)) * dx
    yn = (np.arange(ny) - 0.5 * (ny - 1)) * dy
    zn = (np.arange(nz) - 0.5 * (nz - 1)) * dz
    xc, yc, zc = xn[i0:i1] + 0.5 * dx, yn[j0:j1] + 0.5 * dy, zn[k0:k1] + 0.5 * dz
    pos, ws = [], []
    for i in (i1, i0):
        yy, zz = np.meshgrid(yc, zc, indexing="ij")
        pos.append(np.stack([np.full(yy.size, xn[i]), yy.ravel(), zz.ravel()], -1))
        ws.append(np.full(yy.size, dy * dz))
    for j in (j1, j0):
        xx, zz = np.meshgrid(xc, zc, indexing="ij")
        pos.append(np.stack([xx.ravel(), np.full(xx.size, yn[j]), zz.ravel()], -1))
        ws.append(np.full(xx.size, dx * dz))
    for kk in (k1, k0):
        xx, yy = np.meshgrid(xc, yc, indexing="ij")
        pos.append(np.stack([xx.ravel(), yy.ravel(), np.full(xx.size, zn[kk])], -1))
        ws.append(np.full(xx.size, dx * dy))
    return np.concatenate(pos), np.concatenate(ws), (i0, i1, j0, j1, k0, k1)


def _box_currents_3d(comps, bounds, cdt):
    """Js = n x H, Ms = -n x E on the face-patch centres (ntff.py:345-395).

    Tangential E is the 2-point and tangential H the 4-point average onto
    each patch centre. Returns J, M of shape (n_freq, n_pts, 3).
    """
    ex, ey, ez, hx, hy, hz = comps
    i0, i1, j0, j1, k0, k1 = bounds
    ic, icp = slice(i0, i1), slice(i0 + 1, i1 + 1)
    jc, jcp = slice(j0, j1), slice(j0 + 1, j1 + 1)
    kc, kcp = slice(k0, k1), slice(k0 + 1, k1 + 1)

    def flat(c):
        return c.reshape(c.shape[0], -1).to(cdt)

    js, ms = [], []

    def face(jc3, mc3):
        z = torch.zeros_like(next(flat(c) for c in jc3 if c is not None))
        js.append(torch.stack([z if c is None else flat(c) for c in jc3], -1))
        ms.append(torch.stack([z if c is None else flat(c) for c in mc3], -1))

    for i, s in ((i1, 1.0), (i0, -1.0)):
        ey_f = 0.5 * (ey[i, jc, kc] + ey[i, jc, kcp])
        ez_f = 0.5 * (ez[i, jc, kc] + ez[i, jcp, kc])
        hy_f = 0.25 * (hy[i - 1, jc, kc] + hy[i, jc, kc] + hy[i - 1, jcp, kc] + hy[i, jcp, kc])
        hz_f = 0.25 * (hz[i - 1, jc, kc] + hz[i, jc, kc] + hz[i - 1, jc, kcp] + hz[i, jc, kcp])
        face((None, -s * hz_f, s * hy_f), (None, s * ez_f, -s * ey_f))
    for j, s in ((j1, 1.0), (j0, -1.0)):
        ex_f = 0.5 * (ex[ic, j, kc] + ex[ic, j, kcp])
        ez_f = 0.5 * (ez[ic, j, kc] + ez[icp, j, kc])
        hx_f = 0.25 * (hx[ic, j - 1, kc] + hx[ic, j, kc] + hx[icp, j - 1, kc] + hx[icp, j, kc])
        hz_f = 0.25 * (hz[ic, j - 1, kc] + hz[ic, j, kc] + hz[ic, j - 1, kcp] + hz[ic, j, kcp])
        face((s * hz_f, None, -s * hx_f), (-s * ez_f, None, s * ex_f))
    for kk, s in ((k1, 1.0), (k0, -1.0)):
        ex_f = 0.5 * (ex[ic, jc, kk] + ex[ic, jcp, kk])
        ey_f = 0.5 * (ey[ic, jc, kk] + ey[icp, jc, kk])
        hx_f = 0.25 * (hx[ic, jc, kk - 1] + hx[ic, jc, kk] + hx[icp, jc, kk - 1] + hx[icp, jc, kk])
        hy_f = 0.25 * (hy[ic, jc, kk - 1] + hy[ic, jc, kk] + hy[ic, jcp, kk - 1] + hy[ic, jcp, kk])
        face((-s * hy_f, s * hx_f, None), (s * ey_f, -s * ex_f, None))
    return torch.cat(js, dim=1), torch.cat(ms, dim=1)


def _directions(thetas, phis):
    th = np.atleast_1d(np.asarray(_as_f64(thetas).cpu(), np.float64))
    ph = np.atleast_1d(np.asarray(_as_f64(phis).cpu(), np.float64))
    tt, pp = np.meshgrid(th, ph, indexing="ij")
    dirs = np.stack([np.cos(tt), np.sin(tt), np.cos(pp), np.sin(pp)], -1).reshape(-1, 4)
    return dirs, th.shape[0], ph.shape[0]


def ntff_3d(dft_monitor, grid3d: Grid3D, box_margin: int, freqs, thetas, phis):
    """3D near-to-far-field transform on a closed box (ntff.py:262-431).

    With Js = n x H and Ms = -n x E on the six faces ``box_margin`` cells
    inside the boundary, N = sum Js e^{+jk rhat.r'} dA, L likewise with Ms,

        E_theta = -jk/(4 pi) (L_phi + eta0 N_theta),
        E_phi   = +jk/(4 pi) (L_theta - eta0 N_phi).

    Args:
        dft_monitor: ``SimResult3D.dft`` with all six components, either the
            full-grid ``DFTMonitor`` or a slab ``RegionDFTMonitor`` covering
            the box (``ntff_box_regions``).
        grid3d: the 3D Yee grid.
        box_margin: box distance from the boundary in cells (>= 1).
        freqs: (n_freq,) frequencies [Hz] of the monitor's first axis.
        thetas: (n_theta,) polar angles [rad]; phis: (n_phi,) azimuths [rad].

    Returns:
        Complex (n_freq, n_theta, n_phi, 2): [..., 0] = E_theta, [..., 1] =
        E_phi, differentiable w.r.t. the monitor phasors.
    """
    comps = _monitor_components(dft_monitor)
    dev = comps[0].arr.device
    if dev.type != "cuda":
        raise RuntimeError("ntff_3d runs on a CUDA device; phasors are on " + str(dev))
    n_freq = comps[0].arr.shape[0]
    k = _wavenumbers(freqs, n_freq, dev)
    pos, w, bounds = box_points_3d(grid3d, box_margin)
    cdt = _complex_dtype(*(c.arr for c in comps))
    j, m = _box_currents_3d(comps, bounds, cdt)
    dirs, n_th, n_ph = _directions(thetas, phis)
    out = _Project3D.apply(j, m, torch.as_tensor(pos, device=dev).contiguous(),
                           torch.as_tensor(w, device=dev), k,
                           torch.as_tensor(dirs, device=dev).contiguous())
    return out.reshape(n_freq, n_th, n_ph, 2)


def _intensity(e_theta, e_phi):
    return (torch.abs(e_theta) ** 2 + torch.abs(e_phi) ** 2) / (2.0 * ETA0)


def radiated_power_3d(e_theta, e_phi, thetas, phis):
    """P = closed-integral U sin(theta) dtheta dphi (ntff.py:441-455); (n_freq,)."""
    dev = e_theta.device
    u = _intensity(e_theta, e_phi)
    u_phi = torch.sum(u * _periodic_trapezoid_weights(phis, 2.0 * math.pi, dev), dim=-1)
    th = _as_f64(thetas, dev)
    w_th = _trapezoid_weights(th, dev) * torch.sin(th)
    return torch.sum(u_phi * w_th, dim=-1)


def directivity_3d(e_theta, e_phi, thetas, phis):
    """D(theta, phi) = 4 pi U / P_rad (ntff.py:458-466)."""
    u = _intensity(e_theta, e_phi)
    p_rad = radiated_power_3d(e_theta, e_phi, thetas, phis)
    return 4.0 * math.pi * u / p_rad[:, None, None]


def gain(directivity, p_rad, p_in):
    """G = (P_rad / P_in) D, broadcast over the trailing angle axes (ntff.py:469-484)."""
    d = torch.as_tensor(directivity)
    eff = torch.as_tensor(p_rad, device=d.device) / torch.as_tensor(p_in, device=d.device)
    eff = eff.reshape(tuple(eff.shape) + (1,) * (d.ndim - eff.ndim))
    return d * eff
