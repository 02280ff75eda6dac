"""numpy restatement of the reference 3D Yee stepper (test oracle only).

Follows src/gradenna/fdtd3d.py:258-770 in the same update order:
H (Hx, Hy, Hz with 6 slab psi) -> Mx/My/Mz -> port Ampere current ->
Ex, Ey, Ez (6 slab psi) with Jx/Jy injection after their component and Jz
after Ez -> semi-implicit RVS port overwrite of the port Ez edge -> running
DFT (full grid or region slabs; phases pre-scaled by dt) -> probes / port V /
energy. Field shapes (fdtd3d.py:1-13):

    Ex (nx-1, ny, nz)   Ey (nx, ny-1, nz)   Ez (nx, ny, nz-1)
    Hx (nx, ny-1, nz-1) Hy (nx-1, ny, nz-1) Hz (nx-1, ny-1, nz)

Test conveniences beyond the reference's interface (the algorithm is
unchanged): ``probe_comp`` records Ex / Ey / Ez probes, and ``state_in`` /
``return_state`` / ``step0`` resume a run from an earlier run's state (six
fields and twelve psi pairs) with the DFT phases of the absolute steps, so
that checkpointed gradient logic can be checked on the CPU.

Only tests and CPU-baseline code may import this module.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import NamedTuple

import numpy as np

from oracle.fdtd2d_np import EPS0, MU0, C0, CPMLSpec, axis_coefficients, psi_step, slab_slices


@dataclass(frozen=True)
class Grid3D:
    """grid.py:43-72."""

    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    courant: float = 0.99

    @property
    def dt(self) -> float:
        return self.courant / (C0 * math.sqrt(1 / self.dx**2 + 1 / self.dy**2 + 1 / self.dz**2))

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)


class SimResult3D(NamedTuple):
    """fdtd3d.py:87-109 (dft: dict comp -> (K, ...) or None)."""

    probe_ez: np.ndarray
    port_v: np.ndarray | None
    port_i: np.ndarray | None
    energy: np.ndarray | None
    dft: dict | None
    ex: np.ndarray
    ey: np.ndarray
    ez: np.ndarray
    hx: np.ndarray
    hy: np.ndarray
    hz: np.ndarray
    state: tuple | None = None


def full_shapes(nx, ny, nz):
    """dft_region.py:95-104."""
    return {"ex": (nx - 1, ny, nz), "ey": (nx, ny - 1, nz), "ez": (nx, ny, nz - 1),
            "hx": (nx, ny - 1, nz - 1), "hy": (nx - 1, ny, nz - 1), "hz": (nx - 1, ny - 1, nz)}


def simulate_3d(grid: Grid3D, *, eps_r=1.0, sigma=0.0, source_ijk=None, source_current=None,
                source_x_ijk=None, source_x_current=None, source_y_ijk=None,
                source_y_current=None, mx_ijk=None, mx_current=None, my_ijk=None,
                my_current=None, mz_ijk=None, mz_current=None, port_ijk=None,
                port_voltage=None, port_resistance=50.0, probe_ijk=(), cpml=CPMLSpec(),
                dft_freqs=None, dft_regions=None, record_energy=False, dtype=np.float64,
                probe_comp=None, state_in=None, return_state=False, step0=0):
    """fdtd3d.py:258-770 restated; dft_regions: dict comp -> (lo, hi) boxes."""
    dtype = np.dtype(dtype)
    f = dtype.type
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    dt = grid.dt
    dx, dy, dz = grid.dx, grid.dy, grid.dz

    def chan(idx, cur):
        if idx is None:
            return np.zeros((0, 3), np.int64), None
        c = np.asarray(cur, dtype)
        return np.asarray(idx, np.int64).reshape(-1, 3), (c[:, None] if c.ndim == 1 else c)

    src_idx, src_cur = chan(source_ijk, source_current)
    jx_idx, jx_cur = chan(source_x_ijk, source_x_current)
    jy_idx, jy_cur = chan(source_y_ijk, source_y_current)
    mx_idx, mx_cur = chan(mx_ijk, mx_current)
    my_idx, my_cur = chan(my_ijk, my_current)
    mz_idx, mz_cur = chan(mz_ijk, mz_current)
    has_port = port_ijk is not None
    n_steps = None
    for c in (src_cur, jx_cur, jy_cur, mx_cur, my_cur, mz_cur):
        if c is not None:
            n_steps = c.shape[0]
    if has_port:
        port_voltage = np.asarray(port_voltage, dtype).reshape(-1)
        n_steps = port_voltage.shape[0]
        pi, pj, pk = (int(v) for v in np.asarray(port_ijk).reshape(3))
    probe_idx = np.asarray(probe_ijk, np.int64).reshape(-1, 3)

    eps = (EPS0 * np.broadcast_to(np.asarray(eps_r, dtype), (nx, ny, nz))).astype(dtype)
    sig = np.broadcast_to(np.asarray(sigma, dtype), (nx, ny, nz)).astype(dtype)
    half_loss = (sig * f(dt) / (f(2.0) * eps)).astype(dtype)
    ca = ((f(1.0) - half_loss) / (f(1.0) + half_loss)).astype(dtype)
    cb = ((f(dt) / eps) / (f(1.0) + half_loss)).astype(dtype)
    ca_ex, cb_ex = ca[:-1, 1:-1, 1:-1], cb[:-1, 1:-1, 1:-1]
    ca_ey, cb_ey = ca[1:-1, :-1, 1:-1], cb[1:-1, :-1, 1:-1]
    ca_ez, cb_ez = ca[1:-1, 1:-1, :-1], cb[1:-1, 1:-1, :-1]

    ax = {}
    for name, (n, d, h) in {"xe": (nx, dx, False), "ye": (ny, dy, False), "ze": (nz, dz, False),
                            "xh": (nx, dx, True), "yh": (ny, dy, True), "zh": (nz, dz, True)}.items():
        ax[name] = axis_coefficients(n, d, dt, cpml, half=h, dtype=dtype)
    kx_e = ax["xe"].inv_kappa[1:-1, None, None]
    ky_e = ax["ye"].inv_kappa[None, 1:-1, None]
    kz_e = ax["ze"].inv_kappa[None, None, 1:-1]
    kx_h = ax["xh"].inv_kappa[:, None, None]
    ky_h = ax["yh"].inv_kappa[None, :, None]
    kz_h = ax["zh"].inv_kappa[None, None, :]
    npml = cpml.thickness
    sx_e, sy_e, sz_e = slab_slices(nx - 2, npml), slab_slices(ny - 2, npml), slab_slices(nz - 2, npml)
    sx_h, sy_h, sz_h = slab_slices(nx - 1, npml), slab_slices(ny - 1, npml), slab_slices(nz - 1, npml)
    bx_e, cx_e = ax["xe"].b[1:-1], ax["xe"].c[1:-1]
    by_e, cy_e = ax["ye"].b[1:-1], ax["ye"].c[1:-1]
    bz_e, cz_e = ax["ze"].b[1:-1], ax["ze"].c[1:-1]
    bx_h, cx_h = ax["xh"].b, ax["xh"].c
    by_h, cy_h = ax["yh"].b, ax["yh"].c
    bz_h, cz_h = ax["zh"].b, ax["zh"].c

    inv_dx, inv_dy, inv_dz = f(1 / dx), f(1 / dy), f(1 / dz)
    dt_mu = f(dt / MU0)
    cb_src = (cb[src_idx[:, 0], src_idx[:, 1], src_idx[:, 2]] * (inv_dx * inv_dy)).astype(dtype)
    cb_jx = (cb[jx_idx[:, 0], jx_idx[:, 1], jx_idx[:, 2]] * (inv_dy * inv_dz)).astype(dtype)
    cb_jy = (cb[jy_idx[:, 0], jy_idx[:, 1], jy_idx[:, 2]] * (inv_dx * inv_dz)).astype(dtype)
    if has_port:
        eps_p = eps[pi, pj, pk]
        h_p = sig[pi, pj, pk] * f(dt) / (f(2.0) * eps_p)
        beta = f(dt) * f(dz) / (f(2.0) * f(port_resistance) * eps_p * f(dx) * f(dy))
        denom = f(1.0) + h_p + beta
        a_port = (f(1.0) - h_p - beta) / denom
        b_port = (f(dt) / eps_p) / denom
        c_port = -f(dt) / (f(port_resistance) * eps_p * f(dx) * f(dy) * denom)

    has_dft = dft_freqs is not None
    if has_dft:
        fr = np.atleast_1d(np.asarray(dft_freqs, np.float64))
        cdtype = np.result_type(dtype, np.complex64)
        nn = np.arange(step0, step0 + n_steps, dtype=np.float64)
        e_phase = (dt * np.exp(-2j * np.pi * np.outer(nn + 1.0, fr) * dt)).astype(cdtype)
        h_phase = (dt * np.exp(-2j * np.pi * np.outer(nn + 0.5, fr) * dt)).astype(cdtype)
        shapes = full_shapes(nx, ny, nz)
        regions = dft_regions if dft_regions is not None else {k: ((0, 0, 0), s) for k, s in shapes.items()}
        acc = {}
        for k, reg in regions.items():
            if reg is None:
                continue
            lo, hi = reg
            acc[k] = np.zeros((len(fr),) + tuple(h - l for l, h in zip(lo, hi)), cdtype)

    z = lambda s: np.zeros(s, dtype)  # noqa: E731
    ex, ey, ez = z((nx - 1, ny, nz)), z((nx, ny - 1, nz)), z((nx, ny, nz - 1))
    hx, hy, hz = z((nx, ny - 1, nz - 1)), z((nx - 1, ny, nz - 1)), z((nx - 1, ny - 1, nz))
    pair = lambda s: (z(s), z(s))  # noqa: E731
    psi = dict(
        exy=pair((nx - 1, npml, nz - 2)), exz=pair((nx - 1, ny - 2, npml)),
        eyx=pair((npml, ny - 1, nz - 2)), eyz=pair((nx - 2, ny - 1, npml)),
        ezx=pair((npml, ny - 2, nz - 1)), ezy=pair((nx - 2, npml, nz - 1)),
        hxy=pair((nx, npml, nz - 1)), hxz=pair((nx, ny - 1, npml)),
        hyx=pair((npml, ny, nz - 1)), hyz=pair((nx - 1, ny, npml)),
        hzx=pair((npml, ny - 1, nz)), hzy=pair((nx - 1, npml, nz)),
    )
    if state_in is not None:
        ex, ey, ez, hx, hy, hz = (a.copy() for a in state_in[:6])
        psi = {k: tuple(a.copy() for a in v) for k, v in state_in[6].items()}
    probe_out = np.zeros((n_steps, probe_idx.shape[0]), dtype)
    v_out = np.zeros(n_steps, dtype)
    i_out = np.zeros(n_steps, dtype)
    energy = np.zeros(n_steps, dtype) if record_energy else None

    def add(arr, idx, val):
        if idx.shape[0]:
            np.add.at(arr, (idx[:, 0], idx[:, 1], idx[:, 2]), val)

    for n in range(n_steps):
        # H update (fdtd3d.py:564-588)
        dey_dz = (ey[:, :, 1:] - ey[:, :, :-1]) * inv_dz
        dez_dy = (ez[:, 1:, :] - ez[:, :-1, :]) * inv_dy
        psi["hxz"], t_hxz = psi_step(psi["hxz"], dey_dz, bz_h, cz_h, sz_h, 2, kz_h)
        psi["hxy"], t_hxy = psi_step(psi["hxy"], dez_dy, by_h, cy_h, sy_h, 1, ky_h)
        hx = hx + dt_mu * (t_hxz - t_hxy)
        if mx_cur is not None:
            add(hx, mx_idx, -dt_mu * mx_cur[n])
        dez_dx = (ez[1:, :, :] - ez[:-1, :, :]) * inv_dx
        dex_dz = (ex[:, :, 1:] - ex[:, :, :-1]) * inv_dz
        psi["hyx"], t_hyx = psi_step(psi["hyx"], dez_dx, bx_h, cx_h, sx_h, 0, kx_h)
        psi["hyz"], t_hyz = psi_step(psi["hyz"], dex_dz, bz_h, cz_h, sz_h, 2, kz_h)
        hy = hy + dt_mu * (t_hyx - t_hyz)
        if my_cur is not None:
            add(hy, my_idx, -dt_mu * my_cur[n])
        dex_dy = (ex[:, 1:, :] - ex[:, :-1, :]) * inv_dy
        dey_dx = (ey[1:, :, :] - ey[:-1, :, :]) * inv_dx
        psi["hzy"], t_hzy = psi_step(psi["hzy"], dex_dy, by_h, cy_h, sy_h, 1, ky_h)
        psi["hzx"], t_hzx = psi_step(psi["hzx"], dey_dx, bx_h, cx_h, sx_h, 0, kx_h)
        hz = hz + dt_mu * (t_hzy - t_hzx)
        if mz_cur is not None:
            add(hz, mz_idx, -dt_mu * mz_cur[n])
        if has_port:  # fdtd3d.py:590-594
            i_loop = (hy[pi, pj, pk] - hy[pi - 1, pj, pk]) * f(dy) + (
                hx[pi, pj - 1, pk] - hx[pi, pj, pk]) * f(dx)
        # E update (fdtd3d.py:596-626)
        dhz_dy = (hz[:, 1:, :] - hz[:, :-1, :])[:, :, 1:-1] * inv_dy
        dhy_dz = (hy[:, :, 1:] - hy[:, :, :-1])[:, 1:-1, :] * inv_dz
        psi["exy"], t_exy = psi_step(psi["exy"], dhz_dy, by_e, cy_e, sy_e, 1, ky_e)
        psi["exz"], t_exz = psi_step(psi["exz"], dhy_dz, bz_e, cz_e, sz_e, 2, kz_e)
        ex = ex.copy()
        ex[:, 1:-1, 1:-1] = ca_ex * ex[:, 1:-1, 1:-1] + cb_ex * (t_exy - t_exz)
        if jx_cur is not None:
            add(ex, jx_idx, -cb_jx * jx_cur[n])
        dhx_dz = (hx[:, :, 1:] - hx[:, :, :-1])[1:-1, :, :] * inv_dz
        dhz_dx = (hz[1:, :, :] - hz[:-1, :, :])[:, :, 1:-1] * inv_dx
        psi["eyz"], t_eyz = psi_step(psi["eyz"], dhx_dz, bz_e, cz_e, sz_e, 2, kz_e)
        psi["eyx"], t_eyx = psi_step(psi["eyx"], dhz_dx, bx_e, cx_e, sx_e, 0, kx_e)
        ey = ey.copy()
        ey[1:-1, :, 1:-1] = ca_ey * ey[1:-1, :, 1:-1] + cb_ey * (t_eyz - t_eyx)
        if jy_cur is not None:
            add(ey, jy_idx, -cb_jy * jy_cur[n])
        dhy_dx = (hy[1:, :, :] - hy[:-1, :, :])[:, 1:-1, :] * inv_dx
        dhx_dy = (hx[:, 1:, :] - hx[:, :-1, :])[1:-1, :, :] * inv_dy
        psi["ezx"], t_ezx = psi_step(psi["ezx"], dhy_dx, bx_e, cx_e, sx_e, 0, kx_e)
        psi["ezy"], t_ezy = psi_step(psi["ezy"], dhx_dy, by_e, cy_e, sy_e, 1, ky_e)
        curl_z = t_ezx - t_ezy
        ez_prev = ez
        ez = ez.copy()
        ez[1:-1, 1:-1, :] = ca_ez * ez[1:-1, 1:-1, :] + cb_ez * curl_z
        if src_cur is not None:
            add(ez, src_idx, -cb_src * src_cur[n])
        if has_port:  # fdtd3d.py:627-633
            ez[pi, pj, pk] = (a_port * ez_prev[pi, pj, pk] + b_port * curl_z[pi - 1, pj - 1, pk]
                              + c_port * port_voltage[n])
        if has_dft:  # fdtd3d.py:635-662
            fields = dict(ex=ex, ey=ey, ez=ez, hx=hx, hy=hy, hz=hz)
            for k, a in acc.items():
                lo, hi = regions[k]
                ph = e_phase[n] if k[0] == "e" else h_phase[n]
                patch = fields[k][lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
                a += ph[:, None, None, None] * patch[None]
        if probe_comp is None:
            probe_out[n] = ez[probe_idx[:, 0], probe_idx[:, 1], probe_idx[:, 2]]
        else:
            for q, (pc, (a, b, c)) in enumerate(zip(probe_comp, probe_idx)):
                probe_out[n, q] = (ex, ey, ez)[pc][a, b, c]
        if has_port:
            v_out[n] = f(-0.5) * f(dz) * (ez_prev[pi, pj, pk] + ez[pi, pj, pk])
            i_out[n] = i_loop
        if record_energy:  # fdtd3d.py:171-183
            cell = dx * dy * dz
            ue = 0.5 * cell * (np.sum(eps[:-1] * ex**2) + np.sum(eps[:, :-1] * ey**2)
                               + np.sum(eps[:, :, :-1] * ez**2))
            uh = 0.5 * MU0 * cell * (np.sum(hx**2) + np.sum(hy**2) + np.sum(hz**2))
            energy[n] = ue + uh

    return SimResult3D(probe_out, v_out if has_port else None, i_out if has_port else None,
                       energy, acc if has_dft else None, ex, ey, ez, hx, hy, hz,
                       (ex, ey, ez, hx, hy, hz, psi) if return_state else None)


def time_series_dft(x, dt, freqs, t0=0.0):
    """fdtd3d.py:186-197."""
    x = np.asarray(x, np.float64)
    f = np.atleast_1d(np.asarray(freqs, np.float64))
    t = t0 + dt * np.arange(x.shape[0])
    return dt * np.tensordot(np.exp(-2j * np.pi * f[:, None] * t[None, :]), x, axes=1)


def port_impedance(res, grid, freqs, deembed_gap=True, eps_r_port=1.0):
    """fdtd3d.py:200-243."""
    dt = grid.dt
    v = time_series_dft(res.port_v, dt, freqs, 0.5 * dt)
    i = time_series_dft(res.port_i, dt, freqs, 0.5 * dt)
    if not deembed_gap:
        return v / i
    f = np.atleast_1d(np.asarray(freqs, np.float64))
    omega_d = 2.0 * np.tan(np.pi * f * dt) / dt
    c_gap = EPS0 * eps_r_port * grid.dx * grid.dy / grid.dz
    return 1.0 / (i / v + 1j * omega_d * c_gap)
