"""numpy restatement of the reference 2D TM stepper (test oracle only).

Follows, in the same update order:

* ``src/gradenna/constants.py:3-6``          physical constants
* ``src/gradenna/grid.py:33-36``              dt at the Courant fraction
* ``src/gradenna/cpml.py:161-208``            axis_coefficients (b, c, 1/kappa)
* ``src/gradenna/cpml.py:85-96``              slab_slices
* ``src/gradenna/cpml.py:120-158``            psi_step on slab storage
* ``src/gradenna/fdtd2d.py:248-500``          simulate_tm setup + step + DFT scale

Every array is computed in ``dtype`` (float32 or float64); the DFT phase
tables are built in float64 and cast to the accumulator type, exactly as the
reference does (``fdtd2d.py:393-398``). Only tests and CPU-baseline code may
import this module.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import NamedTuple

import numpy as np

# constants.py:3-6
C0 = 299792458.0
MU0 = 1.25663706212e-06
EPS0 = 1.0 / (MU0 * C0**2)
ETA0 = MU0 * C0
DZ = 1.0  # fdtd2d.py:78


@dataclass(frozen=True)
class Grid2D:
    """grid.py:12-39."""

    nx: int
    ny: int
    dx: float
    dy: float
    courant: float = 0.99

    @property
    def dt(self) -> float:
        return self.courant / (C0 * math.sqrt(1.0 / self.dx**2 + 1.0 / self.dy**2))

    @property
    def shape(self):
        return (self.nx, self.ny)


@dataclass(frozen=True)
class CPMLSpec:
    """cpml.py:35-44."""

    thickness: int = 10
    m: float = 3.0
    ma: float = 1.0
    kappa_max: float = 5.0
    alpha_max: float = 0.0
    sigma_factor: float = 0.75


def alpha_max_for_fmin(f_min: float) -> float:
    """cpml.py:47-49."""
    return 2.0 * math.pi * f_min * EPS0


class Axis(NamedTuple):
    b: np.ndarray
    c: np.ndarray
    inv_kappa: np.ndarray


def axis_coefficients(n, delta, dt, spec: CPMLSpec, *, half, dtype, eps_r_bg=1.0) -> Axis:
    """cpml.py:161-208, evaluated in ``dtype`` like the jnp original."""
    dtype = np.dtype(dtype)
    npml = spec.thickness
    if half:
        pos = np.arange(n - 1, dtype=dtype) + dtype.type(0.5)
    else:
        pos = np.arange(n, dtype=dtype)
    if npml == 0:
        z = np.zeros_like(pos)
        return Axis(z, z.copy(), np.ones_like(pos))
    depth_left = (dtype.type(npml) - pos) / dtype.type(npml)
    depth_right = (pos - dtype.type(n - 1 - npml)) / dtype.type(npml)
    rho = np.clip(np.maximum(depth_left, depth_right), 0.0, 1.0).astype(dtype)
    sigma_max = spec.sigma_factor * 0.8 * (spec.m + 1.0) / (ETA0 * delta * math.sqrt(eps_r_bg))
    sigma = (sigma_max * rho ** spec.m).astype(dtype)
    kappa = (1.0 + (spec.kappa_max - 1.0) * rho ** spec.m).astype(dtype)
    alpha = np.where(rho > 0.0, spec.alpha_max * (1.0 - rho) ** spec.ma, 0.0).astype(dtype)
    b = np.exp(-(sigma / kappa + alpha) * dt / EPS0).astype(dtype)
    denom = sigma + kappa * alpha
    safe = np.where(denom > 0.0, denom, 1.0).astype(dtype)
    c = np.where(denom > 0.0, sigma * (b - 1.0) / (kappa * safe), 0.0).astype(dtype)
    return Axis(b, c, (1.0 / kappa).astype(dtype))


def slab_slices(n: int, thickness: int):
    """cpml.py:85-96."""
    if not 0 <= 2 * thickness <= n:
        raise ValueError(f"PML slab thickness {thickness} too large for axis length {n}")
    return slice(0, thickness), slice(n - thickness, n)


def _expand(a, axis, ndim):
    shape = [1] * ndim
    shape[axis] = a.shape[0]
    return a.reshape(shape)


def psi_step(psi, diff, b, c, slabs, axis, inv_kappa):
    """cpml.py:120-158: psi = b psi + c diff on both slabs, term = diff/kappa + psi.

    ``b``/``c`` are the 1D tables already sampled at the psi positions along
    ``axis``; ``inv_kappa`` broadcasts against ``diff``.
    """
    lo, hi = slabs
    if lo.stop == lo.start:
        return psi, diff
    ndim = diff.ndim
    idx = lambda s: (slice(None),) * axis + (s,)  # noqa: E731
    mid = slice(lo.stop, hi.start)
    p_lo = _expand(b[lo], axis, ndim) * psi[0] + _expand(c[lo], axis, ndim) * diff[idx(lo)]
    p_hi = _expand(b[hi], axis, ndim) * psi[1] + _expand(c[hi], axis, ndim) * diff[idx(hi)]
    term = np.concatenate(
        [
            diff[idx(lo)] * inv_kappa[idx(lo)] + p_lo,
            diff[idx(mid)],
            diff[idx(hi)] * inv_kappa[idx(hi)] + p_hi,
        ],
        axis=axis,
    )
    return (p_lo, p_hi), term


class Port(NamedTuple):
    """fdtd2d.py:81-98."""

    ij: tuple
    resistance: float = 50.0
    voltage: np.ndarray | None = None


class SimResult(NamedTuple):
    """fdtd2d.py:101-126."""

    probe_ez: np.ndarray
    energy: np.ndarray | None
    ez: np.ndarray
    hx: np.ndarray
    hy: np.ndarray
    port_v: np.ndarray | None = None
    port_i: np.ndarray | None = None
    dft_ez: np.ndarray | None = None
    dft_hx: np.ndarray | None = None
    dft_hy: np.ndarray | None = None


def _idx(ij, name, grid, margin):
    """fdtd2d.py:172-178."""
    idx = np.asarray(ij, dtype=np.int64).reshape(-1, 2)
    lo = np.array([margin, margin])
    hi = np.array([grid.nx - 1 - margin, grid.ny - 1 - margin])
    if idx.size and (np.any(idx < lo) or np.any(idx > hi)):
        raise ValueError(f"{name} {idx.tolist()} outside the interior (PML margin {margin})")
    return idx


def simulate_tm(
    grid: Grid2D,
    *,
    source_ij=None,
    source_current=None,
    eps_r=1.0,
    sigma=0.0,
    probe_ij=(),
    ports=(),
    dft_freqs=(),
    dft_dtype=None,
    cpml: CPMLSpec = CPMLSpec(),
    record_energy=False,
    mx_ij=None,
    mx_current=None,
    my_ij=None,
    my_current=None,
    dtype=np.float64,
) -> SimResult:
    """fdtd2d.py:181-500 restated in numpy; ``dtype`` is the field dtype."""
    dtype = np.dtype(dtype)
    f = dtype.type
    nx, ny = grid.nx, grid.ny
    if min(nx, ny) <= 2 * cpml.thickness + 2:
        raise ValueError("grid too small for CPML")
    dt = grid.dt
    ports = tuple(p if isinstance(p, Port) else Port(*p) for p in ports)
    n_ports = len(ports)
    vs_list = [None if p.voltage is None else np.asarray(p.voltage, dtype) for p in ports]
    n_steps = None
    if source_current is not None:
        source_current = np.asarray(source_current, dtype)
        n_steps = source_current.shape[0]
    for v in vs_list:
        if v is not None:
            if n_steps is None:
                n_steps = v.shape[0]
            elif v.shape[0] != n_steps:
                raise ValueError("port voltage length mismatch")
    if n_steps is None:
        for cur in (mx_current, my_current):
            if cur is not None:
                n_steps = np.asarray(cur).shape[0]
    if n_steps is None:
        raise ValueError("need a source or port waveform")

    probe_idx = _idx(probe_ij, "probe_ij", grid, 0)
    if source_current is None:
        src_idx = np.zeros((0, 2), np.int64)
        src_cur = np.zeros((n_steps, 0), dtype)
    else:
        src_idx = _idx(source_ij, "source_ij", grid, 1)
        src_cur = source_current[:, None] if source_current.ndim == 1 else source_current
    if n_ports:
        port_idx = _idx([p.ij for p in ports], "port ij", grid, 1)
        port_rs = np.asarray([float(p.resistance) for p in ports])
        port_vs = np.stack([np.zeros(n_steps, dtype) if v is None else v for v in vs_list], 1)
        pi, pj = port_idx[:, 0], port_idx[:, 1]

    def mag(m_ij, m_cur):
        if m_cur is None:
            return np.zeros((0, 2), np.int64), np.zeros((n_steps, 0), dtype)
        idx = np.asarray(m_ij, np.int64).reshape(-1, 2)
        mc = np.asarray(m_cur, dtype)
        return idx, (mc[:, None] if mc.ndim == 1 else mc)

    mx_idx, mx_cur = mag(mx_ij, mx_current)
    my_idx, my_cur = mag(my_ij, my_current)

    # fdtd2d.py:343-352 (materials, port conductivity, ca/cb) in dtype.
    eps = (EPS0 * np.broadcast_to(np.asarray(eps_r, dtype), (nx, ny))).astype(dtype)
    sig = np.array(np.broadcast_to(np.asarray(sigma, dtype), (nx, ny)), dtype)
    if n_ports:
        np.add.at(sig, (pi, pj), (DZ / (port_rs * grid.dx * grid.dy)).astype(dtype))
    half_loss = (sig * f(dt) / (f(2.0) * eps)).astype(dtype)
    ca = ((f(1.0) - half_loss) / (f(1.0) + half_loss)).astype(dtype)
    cb = ((f(dt) / eps) / (f(1.0) + half_loss)).astype(dtype)

    # fdtd2d.py:354-374 (CPML tables, slab slices).
    cx_e = axis_coefficients(nx, grid.dx, dt, cpml, half=False, dtype=dtype)
    cx_h = axis_coefficients(nx, grid.dx, dt, cpml, half=True, dtype=dtype)
    cy_e = axis_coefficients(ny, grid.dy, dt, cpml, half=False, dtype=dtype)
    cy_h = axis_coefficients(ny, grid.dy, dt, cpml, half=True, dtype=dtype)
    npml = cpml.thickness
    sx_e, sy_e = slab_slices(nx - 2, npml), slab_slices(ny - 2, npml)
    sx_h, sy_h = slab_slices(nx - 1, npml), slab_slices(ny - 1, npml)
    kx_e = cx_e.inv_kappa[1:-1, None]
    ky_e = cy_e.inv_kappa[None, 1:-1]
    kx_h = cx_h.inv_kappa[:, None]
    ky_h = cy_h.inv_kappa[None, :]

    inv_dx, inv_dy = f(1.0 / grid.dx), f(1.0 / grid.dy)
    cb_src = (cb[src_idx[:, 0], src_idx[:, 1]] * (inv_dx * inv_dy)).astype(dtype)
    if n_ports:
        cb_vs = (cb[pi, pj] / (port_rs * grid.dx * grid.dy)).astype(dtype)

    dft_freqs = tuple(float(v) for v in dft_freqs)
    n_freq = len(dft_freqs)
    if n_freq:
        cdtype = np.result_type(dtype, np.complex64) if dft_dtype is None else np.dtype(dft_dtype)
        fr = np.asarray(dft_freqs, np.float64)
        nn = np.arange(n_steps, dtype=np.float64)
        ph_e = np.exp(-2j * np.pi * np.outer(nn + 1.0, fr) * dt).astype(cdtype)
        ph_h = np.exp(-2j * np.pi * np.outer(nn + 0.5, fr) * dt).astype(cdtype)
        acc_e = np.zeros((n_freq, nx, ny), cdtype)
        acc_hx = np.zeros((n_freq, nx, ny - 1), cdtype)
        acc_hy = np.zeros((n_freq, nx - 1, ny), cdtype)

    dt_mu = f(dt / MU0)
    z = lambda s: np.zeros(s, dtype)  # noqa: E731
    ez, hx, hy = z((nx, ny)), z((nx, ny - 1)), z((nx - 1, ny))
    psi = {
        "ezx": (z((npml, ny - 2)), z((npml, ny - 2))),
        "ezy": (z((nx - 2, npml)), z((nx - 2, npml))),
        "hyx": (z((npml, ny)), z((npml, ny))),
        "hxy": (z((nx, npml)), z((nx, npml))),
    }
    probe_out = np.zeros((n_steps, probe_idx.shape[0]), dtype)
    v_out = np.zeros((n_steps, n_ports), dtype)
    i_out = np.zeros((n_steps, n_ports), dtype)
    energy = np.zeros(n_steps, dtype) if record_energy else None
    cell = f(grid.dx * grid.dy)

    for n in range(n_steps):
        # fdtd2d.py:416-421
        dez_dy = (ez[:, 1:] - ez[:, :-1]) * inv_dy
        psi["hxy"], term_hx = psi_step(psi["hxy"], dez_dy, cy_h.b, cy_h.c, sy_h, 1, ky_h)
        hx = hx - dt_mu * term_hx
        if mx_idx.shape[0]:
            np.add.at(hx, (mx_idx[:, 0], mx_idx[:, 1]), -dt_mu * mx_cur[n])
        # fdtd2d.py:423-428
        dez_dx = (ez[1:, :] - ez[:-1, :]) * inv_dx
        psi["hyx"], term_hy = psi_step(psi["hyx"], dez_dx, cx_h.b, cx_h.c, sx_h, 0, kx_h)
        hy = hy + dt_mu * term_hy
        if my_idx.shape[0]:
            np.add.at(hy, (my_idx[:, 0], my_idx[:, 1]), -dt_mu * my_cur[n])
        # fdtd2d.py:430-436
        if n_ports:
            i_port = (hy[pi, pj] - hy[pi - 1, pj]) * f(grid.dy) - (
                hx[pi, pj] - hx[pi, pj - 1]
            ) * f(grid.dx)
            ez_before = ez[pi, pj].copy()
        # fdtd2d.py:438-444
        dhy_dx = (hy[1:, 1:-1] - hy[:-1, 1:-1]) * inv_dx
        dhx_dy = (hx[1:-1, 1:] - hx[1:-1, :-1]) * inv_dy
        psi["ezx"], term_x = psi_step(psi["ezx"], dhy_dx, cx_e.b[1:-1], cx_e.c[1:-1], sx_e, 0, kx_e)
        psi["ezy"], term_y = psi_step(psi["ezy"], dhx_dy, cy_e.b[1:-1], cy_e.c[1:-1], sy_e, 1, ky_e)
        curl = term_x - term_y
        ez = ez.copy()
        ez[1:-1, 1:-1] = ca[1:-1, 1:-1] * ez[1:-1, 1:-1] + cb[1:-1, 1:-1] * curl
        if src_idx.shape[0]:
            np.add.at(ez, (src_idx[:, 0], src_idx[:, 1]), -cb_src * src_cur[n])
        # fdtd2d.py:446-451
        if n_ports:
            np.add.at(ez, (pi, pj), -cb_vs * port_vs[n])
            v_out[n] = f(-0.5 * DZ) * (ez_before + ez[pi, pj])
            i_out[n] = i_port
        # fdtd2d.py:453-458
        if n_freq:
            acc_e += ph_e[n][:, None, None] * ez
            acc_hx += ph_h[n][:, None, None] * hx
            acc_hy += ph_h[n][:, None, None] * hy
        # fdtd2d.py:461-463, field_energy fdtd2d.py:160-169
        probe_out[n] = ez[probe_idx[:, 0], probe_idx[:, 1]]
        if record_energy:
            ue = f(0.5) * np.sum(eps * ez**2) * cell
            uh = f(0.5) * f(MU0) * (np.sum(hx**2) + np.sum(hy**2)) * cell
            energy[n] = ue + uh

    dft_ez = dft_hx = dft_hy = None
    if n_freq:
        dft_ez, dft_hx, dft_hy = acc_e * dt, acc_hx * dt, acc_hy * dt
    return SimResult(
        probe_out, energy, ez, hx, hy,
        v_out if n_ports else None, i_out if n_ports else None,
        dft_ez, dft_hx, dft_hy,
    )


# ---------------------------------------------------------------------------
# sources.py / sparams.py / monitors.py / materials.py restatements
# ---------------------------------------------------------------------------


def gaussian_derivative(t, t0, tau):
    """sources.py:18-24."""
    u = (np.asarray(t) - t0) / tau
    return -u * np.exp(0.5 * (1.0 - u**2))


class BandPulse(NamedTuple):
    """sparams.py:94-118."""

    f0: float
    fc: float
    sigma: float
    t0: float

    def __call__(self, t):
        u = np.asarray(t) - self.t0
        return np.cos(2.0 * np.pi * self.f0 * u) * np.exp(-(u**2) / (2.0 * self.sigma**2))


def gaussian_pulse_for_band(f_min, f_max) -> BandPulse:
    """sparams.py:121-134."""
    f0 = 0.5 * (f_min + f_max)
    fc = 0.5 * (f_max - f_min)
    sigma = 3.0 / (2.0 * math.sqrt(2.0) * math.pi * fc)
    t0 = 9.0 / (2.0 * math.pi * fc)
    return BandPulse(f0, fc, sigma, t0)


def half_step_dft(x_t, dt, freqs):
    """sparams.py:24-46."""
    x_t = np.asarray(x_t, np.float64)
    fr = np.atleast_1d(np.asarray(freqs, np.float64))
    t = (np.arange(x_t.shape[0]) + 0.5) * dt
    kern = np.exp(-2j * np.pi * fr[:, None] * t[None, :]) * dt
    return np.tensordot(kern, x_t, axes=(1, 0))


def port_dft(v_t, i_t, dt, freqs):
    """sparams.py:49-65."""
    return half_step_dft(v_t, dt, freqs), half_step_dft(i_t, dt, freqs)


def s11_power_wave(v_hat, i_hat, z0=50.0):
    """sparams.py:68-79."""
    return (v_hat - z0 * i_hat) / (v_hat + z0 * i_hat)


def poynting_flux_box_2d(dft_ez, dft_hx, dft_hy, grid, box):
    """monitors.py:20-70."""
    il, ir, jb, jt = (int(v) for v in box)
    dx, dy = grid.dx, grid.dy
    js = slice(jb + 1, jt + 1)
    isl = slice(il + 1, ir + 1)
    ez_r = 0.5 * (dft_ez[:, ir, js] + dft_ez[:, ir + 1, js])
    p = -0.5 * np.real(ez_r * np.conj(dft_hy[:, ir, js])).sum(-1) * dy
    ez_l = 0.5 * (dft_ez[:, il, js] + dft_ez[:, il + 1, js])
    p += 0.5 * np.real(ez_l * np.conj(dft_hy[:, il, js])).sum(-1) * dy
    ez_t = 0.5 * (dft_ez[:, isl, jt] + dft_ez[:, isl, jt + 1])
    p += 0.5 * np.real(ez_t * np.conj(dft_hx[:, isl, jt])).sum(-1) * dx
    ez_b = 0.5 * (dft_ez[:, isl, jb] + dft_ez[:, isl, jb + 1])
    p -= 0.5 * np.real(ez_b * np.conj(dft_hx[:, isl, jb])).sum(-1) * dx
    return p


def sigma_from_density(rho, sigma_min=1e-4, sigma_max=1e5):
    """materials.py:28-51."""
    lo, hi = math.log10(sigma_min), math.log10(sigma_max)
    return 10.0 ** ((hi - lo) * np.asarray(rho) + lo)
