"""3D Yee FDTD on B200: the ``simulate_3d`` surface over the CUDA C ABI.

Yee staggering on a uniform grid with a PEC outer shell
(src/gradenna/fdtd3d.py:1-13):

    Ex (nx-1, ny, nz)   Ey (nx, ny-1, nz)   Ez (nx, ny, nz-1)
    Hx (nx, ny-1, nz-1) Hy (nx-1, ny, nz-1) Hz (nx-1, ny-1, nz)

Materials are per node; node (i, j, k) supplies the three E edges leaving
it. One z-directed lumped RVS port uses the semi-implicit update
(fdtd3d.py:25-46, 517-525, 627-633). This module builds the coefficient
tables on the host in the field dtype (fdtd3d.py:462-557) and calls
``gdn_yee_run_f32`` / ``_f64`` once; the whole time loop runs on the GPU.
"""

from __future__ import annotations

import ctypes
import math
from typing import NamedTuple

import numpy as np
import torch

from gradenna_b200 import _native
from gradenna_b200.constants import EPS0, MU0
from gradenna_b200.cpml import CPMLSpec, axis_coefficients, slab_tables
from gradenna_b200.dft_region import DFTRegions, RegionDFTMonitor, full_field_shapes
from gradenna_b200.fdtd2d import _to_dev, infer_dtype, phase_tables
from gradenna_b200.grid import Grid3D

__all__ = ["DFTMonitor", "SimResult3D", "simulate_3d", "time_series_dft", "port_impedance",
           "field_energy_3d"]


class DFTMonitor(NamedTuple):
    """Full-grid spectra of all six components (fdtd3d.py:69-84)."""

    freqs: torch.Tensor
    ex: torch.Tensor
    ey: torch.Tensor
    ez: torch.Tensor
    hx: torch.Tensor
    hy: torch.Tensor
    hz: torch.Tensor


class SimResult3D(NamedTuple):
    """Time series, monitors and final fields (fdtd3d.py:87-109)."""

    probe_ez: torch.Tensor
    port_v: torch.Tensor | None
    port_i: torch.Tensor | None
    energy: torch.Tensor | None
    dft: object
    ex: torch.Tensor
    ey: torch.Tensor
    ez: torch.Tensor
    hx: torch.Tensor
    hy: torch.Tensor
    hz: torch.Tensor
    monitors: list | None = None
    state: torch.Tensor | None = None


def field_energy_3d(ex, ey, ez, hx, hy, hz, eps, grid: Grid3D):
    """1/2 (eps E^2 + mu H^2) dV (fdtd3d.py:171-183)."""
    cell = grid.dx * grid.dy * grid.dz
    ue = 0.5 * cell * (torch.sum(eps[:-1] * ex**2) + torch.sum(eps[:, :-1] * ey**2)
                       + torch.sum(eps[:, :, :-1] * ez**2))
    uh = 0.5 * MU0 * cell * (torch.sum(hx**2) + torch.sum(hy**2) + torch.sum(hz**2))
    return ue + uh


def time_series_dft(x, dt: float, freqs, *, t0: float = 0.0):
    """X(f) = dt sum_n x_n exp(-i 2 pi f (t0 + n dt)) (fdtd3d.py:186-197)."""
    x = x if isinstance(x, torch.Tensor) else torch.as_tensor(np.asarray(x))
    x = x.to(torch.complex128)
    f = torch.as_tensor(np.atleast_1d(np.asarray(freqs, np.float64)), device=x.device)
    t = t0 + dt * torch.arange(x.shape[0], device=x.device, dtype=torch.float64)
    phase = torch.exp(-2j * math.pi * f[:, None] * t[None, :])
    return dt * torch.tensordot(phase, x, dims=1)


def port_impedance(result: SimResult3D, grid: Grid3D, freqs, *, deembed_gap: bool = True,
                   eps_r_port: float = 1.0):
    """Z(f) from the port V/I records, optionally removing the gap shunt
    j w_d C_gap with w_d = 2 tan(w dt/2)/dt (fdtd3d.py:200-243)."""
    if result.port_v is None or result.port_i is None:
        raise ValueError("result has no port records")
    dt = grid.dt
    v = time_series_dft(result.port_v, dt, freqs, t0=0.5 * dt)
    i = time_series_dft(result.port_i, dt, freqs, t0=0.5 * dt)
    if not deembed_gap:
        return v / i
    f = torch.as_tensor(np.atleast_1d(np.asarray(freqs, np.float64)), device=v.device)
    omega_d = 2.0 * torch.tan(math.pi * f * dt) / dt
    c_gap = EPS0 * eps_r_port * grid.dx * grid.dy / grid.dz
    return 1.0 / (i / v + 1j * omega_d * c_gap)


class YeeParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in (
        "nx", "ny", "nz", "npml", "n_steps", "n_src", "n_jx", "n_jy", "n_mx", "n_my", "n_mz",
        "n_probes", "has_port", "n_freq", "dft_f64", "n_monitors", "record_energy",
        "cw_sources")] + [(n, ctypes.c_double) for n in ("dt", "dx", "dy", "dz", "mu0")]


class YeePoints(ctypes.Structure):
    _fields_ = [(n, _native.P_i32) for n in ("src", "jx", "jy", "mx", "my", "mz", "probe")] + [
        ("port", ctypes.c_int32 * 3), ("monitors", ctypes.POINTER(_native.DftMonitor)),
        ("probe_comp", _native.P_i32)]


V = ctypes.c_void_p


class YeeBuffers(ctypes.Structure):
    _fields_ = ([("ca", V), ("cb", V), ("eps", V), ("ik_e", V * 3), ("ik_h", V * 3)]
                + [(n, V * 3) for n in ("b_e_lo", "c_e_lo", "b_e_hi", "c_e_hi", "b_h_lo",
                                         "c_h_lo", "b_h_hi", "c_h_hi")]
                + [(n, ctypes.c_double) for n in ("dt_mu", "inv_dx", "inv_dy", "inv_dz",
                                                   "a_port", "b_port", "c_port")]
                + [(n, V) for n in ("cb_src", "cb_jx", "cb_jy", "src_cur", "jx_cur", "jy_cur",
                                    "mx_cur", "my_cur", "mz_cur", "port_vs", "cw_env", "src_w",
                                    "jx_w", "jy_w", "mx_w", "my_w", "mz_w", "ph_e", "ph_h",
                                    "ex", "ey", "ez", "hx", "hy", "hz", "out_probe", "out_v",
                                    "out_i", "out_energy")]
                + [("dft", V * 6), ("workspace", V), ("workspace_bytes", ctypes.c_size_t),
                   ("state_in", V), ("state_out", V)])


_native.register("gdn_yee_workspace_size", ctypes.c_int, [
    ctypes.POINTER(YeeParams), ctypes.POINTER(YeePoints), ctypes.c_int,
    ctypes.POINTER(ctypes.c_size_t)])
_native.register("gdn_yee_state_size", ctypes.c_int, [
    ctypes.POINTER(YeeParams), ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)])
for _name in ("gdn_yee_run_f32", "gdn_yee_run_f64"):
    _native.register(_name, ctypes.c_int, [ctypes.POINTER(YeeParams), ctypes.POINTER(YeePoints),
                                           ctypes.POINTER(YeeBuffers), ctypes.c_void_p])


def _idx3(ijk, name, shape, margin_ij=0):
    idx = np.asarray(ijk if ijk is not None else np.zeros((0, 3)), np.int64).reshape(-1, 3)
    lo = np.array([margin_ij, margin_ij, 0])
    hi = np.array([shape[0] - 1 - margin_ij, shape[1] - 1 - margin_ij, shape[2] - 1])
    if idx.size and (np.any(idx < lo) or np.any(idx > hi)):
        raise ValueError(f"{name} {idx.tolist()} outside the valid range of its grid {shape}")
    return np.ascontiguousarray(idx, np.int32)


def simulate_3d(
    grid: Grid3D,
    *,
    eps_r=1.0,
    sigma=0.0,
    source_ijk=None,
    source_current=None,
    source_x_ijk=None,
    source_x_current=None,
    source_y_ijk=None,
    source_y_current=None,
    mx_ijk=None,
    mx_current=None,
    my_ijk=None,
    my_current=None,
    mz_ijk=None,
    mz_current=None,
    port_ijk=None,
    port_voltage=None,
    port_resistance: float = 50.0,
    probe_ijk=(),
    cpml: CPMLSpec = CPMLSpec(),
    dft_freqs=None,
    dft_dtype=None,
    dft_regions=None,
    dft_monitors=None,
    record_energy: bool = False,
    checkpoint_segments: int | None = None,
    dtype=None,
    device=None,
    cw_sources=None,
    probe_comp=None,
    state_in=None,
    return_state: bool = False,
    dft_step0: int = 0,
) -> SimResult3D:
    """Run a 3D FDTD simulation on the GPU (drop-in for fdtd3d.simulate_3d).

    Arguments follow the reference (fdtd3d.py:258-330). ``checkpoint_segments``
    only shapes the reference's reverse-mode tape; it must divide n_steps as
    there (fdtd3d.py:738-741) and does not change the forward results.
    Additions: ``dtype``, ``device``, ``cw_sources`` = dict(env, src_w, jx_w,
    jy_w, mx_w, my_w, mz_w) for device-synthesised CW waveforms (the 3D
    frequency-domain adjoint's drive), and ``dft_monitors`` = [(comp, lo,
    hi), ...] boxes (several per component allowed) whose spectra come back
    as ``SimResult3D.monitors`` in the same order (``dft`` is then None).

    Resumable runs (additions): ``probe_comp`` (one of 0, 1, 2 per probe)
    records Ex / Ey / Ez instead of Ez only; ``state_in`` (a uint8 device
    tensor returned as ``SimResult3D.state`` by an earlier run with
    ``return_state=True``) starts the run from that state instead of rest;
    ``dft_step0`` is the absolute index of the run's first step, so that the
    DFT phases of a resumed run continue the whole run's (its phasors are
    the partial sums over its own steps). Waveforms are this run's rows.
    """
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    if min(nx, ny, nz) <= 2 * cpml.thickness + 2:
        raise ValueError(f"grid {nx}x{ny}x{nz} is too small for CPML thickness {cpml.thickness}")
    dt = grid.dt
    dx, dy, dz = grid.dx, grid.dy, grid.dz
    dev = _native.require_cuda(device)
    lib = _native.load()
    shapes = full_field_shapes(nx, ny, nz)
    cw = cw_sources is not None

    chans = {}
    for key, ijk, cur, comp, margin in (
        ("src", source_ijk, source_current, 2, 1), ("jx", source_x_ijk, source_x_current, 0, 0),
        ("jy", source_y_ijk, source_y_current, 1, 0), ("mx", mx_ijk, mx_current, 3, 0),
        ("my", my_ijk, my_current, 4, 0), ("mz", mz_ijk, mz_current, 5, 0),
    ):
        if (ijk is None) != (cur is None) and not cw:
            raise ValueError(f"{key} indices and current must be given together")
        chans[key] = (_idx3(ijk, key, shapes[comp], margin), cur)
    has_port = port_ijk is not None
    if has_port != (port_voltage is not None):
        raise ValueError("port_ijk and port_voltage must be given together")
    if not (has_port or any(c[0].shape[0] for c in chans.values())):
        raise ValueError("at least one current/voltage source is required")
    if has_port:
        pidx = _idx3(port_ijk, "port_ijk", shapes[2], 1)[0]
        if port_resistance <= 0.0:
            raise ValueError("port_resistance must be positive")

    n_steps = None
    for key, (idx, cur) in chans.items():
        if cur is not None and not cw:
            n = int(np.shape(cur)[0])
            if n_steps is not None and n != n_steps:
                raise ValueError(f"{key} waveform length {n} does not match n_steps {n_steps}")
            n_steps = n
    if has_port:
        n = int(port_voltage.numel() if isinstance(port_voltage, torch.Tensor)
                else np.size(port_voltage))
        if n_steps is not None and n != n_steps:
            raise ValueError("source_current and port_voltage lengths differ")
        n_steps = n
    if n_steps is None and cw:
        n_steps = int(np.shape(cw_sources["env"])[0])
    if checkpoint_segments is not None:
        kseg = int(checkpoint_segments)
        if kseg <= 0 or n_steps % kseg != 0:
            raise ValueError(f"checkpoint_segments={checkpoint_segments} must divide n_steps={n_steps}")

    operands = [eps_r, sigma, port_voltage] + [c[1] for c in chans.values()]
    fdt = infer_dtype(operands, dtype)
    npdt = np.float32 if fdt == torch.float32 else np.float64

    eps = (EPS0 * torch.broadcast_to(_to_dev(eps_r, fdt, dev), (nx, ny, nz))).contiguous()
    sig = torch.broadcast_to(_to_dev(sigma, fdt, dev), (nx, ny, nz)).contiguous()
    half_loss = sig * dt / (2.0 * eps)
    ca = ((1.0 - half_loss) / (1.0 + half_loss)).contiguous()
    cb = ((dt / eps) / (1.0 + half_loss)).contiguous()

    def pick(t, idx):
        ii = torch.as_tensor(idx.astype(np.int64), device=dev)
        return t[ii[:, 0], ii[:, 1], ii[:, 2]] if idx.shape[0] else torch.zeros(0, dtype=fdt, device=dev)

    inv = (1.0 / dx, 1.0 / dy, 1.0 / dz)
    cb_src = (pick(cb, chans["src"][0]) * (inv[0] * inv[1])).contiguous()
    cb_jx = (pick(cb, chans["jx"][0]) * (inv[1] * inv[2])).contiguous()
    cb_jy = (pick(cb, chans["jy"][0]) * (inv[0] * inv[2])).contiguous()
    a_port = b_port = c_port = 0.0
    if has_port:
        # fdtd3d.py:517-525, in the field dtype.
        f = npdt
        eps_p = f(float(eps[tuple(pidx)]))
        sig_p = f(float(sig[tuple(pidx)]))
        h_p = sig_p * f(dt) / (f(2.0) * eps_p)
        beta = f(dt) * f(dz) / (f(2.0) * f(port_resistance) * eps_p * f(dx) * f(dy))
        den = f(1.0) + h_p + beta
        a_port = float((f(1.0) - h_p - beta) / den)
        b_port = float((f(dt) / eps_p) / den)
        c_port = float(-f(dt) / (f(port_resistance) * eps_p * f(dx) * f(dy) * den))

    # CPML tables (fdtd3d.py:478-503).
    npml = cpml.thickness
    keep = []

    def dv(a):
        t = torch.as_tensor(np.ascontiguousarray(a if a.size else np.zeros(1, npdt)), device=dev)
        keep.append(t)
        return t.data_ptr()

    bufs = YeeBuffers()
    for a, (n, d) in enumerate(((nx, dx), (ny, dy), (nz, dz))):
        ae = axis_coefficients(n, d, dt, cpml, half=False, dtype=npdt)
        ah = axis_coefficients(n, d, dt, cpml, half=True, dtype=npdt)
        bufs.ik_e[a] = dv(ae.inv_kappa[1:-1])
        bufs.ik_h[a] = dv(ah.inv_kappa)
        be_lo, ce_lo, be_hi, ce_hi = slab_tables(ae.b[1:-1], ae.c[1:-1], npml)
        bh_lo, ch_lo, bh_hi, ch_hi = slab_tables(ah.b, ah.c, npml)
        bufs.b_e_lo[a], bufs.c_e_lo[a], bufs.b_e_hi[a], bufs.c_e_hi[a] = (
            dv(be_lo), dv(ce_lo), dv(be_hi), dv(ce_hi))
        bufs.b_h_lo[a], bufs.c_h_lo[a], bufs.b_h_hi[a], bufs.c_h_hi[a] = (
            dv(bh_lo), dv(ch_lo), dv(bh_hi), dv(ch_hi))

    # Waveforms.
    def wav(key):
        idx, cur = chans[key]
        if idx.shape[0] == 0 or cw:
            return None
        c = _to_dev(cur, fdt, dev)
        if c.ndim == 1:
            c = c[:, None]
        if c.shape != (n_steps, idx.shape[0]):
            raise ValueError(f"{key} waveform has shape {tuple(c.shape)}, want {(n_steps, idx.shape[0])}")
        c = c.contiguous()
        keep.append(c)
        return c.data_ptr()

    for key in ("src", "jx", "jy", "mx", "my", "mz"):
        setattr(bufs, f"{key}_cur", wav(key))
    port_vs = None
    if has_port:
        port_vs = _to_dev(port_voltage, fdt, dev).reshape(-1).contiguous()
        bufs.port_vs = port_vs.data_ptr()

    freqs = None
    n_freq = 0
    if dft_freqs is not None:
        freqs = np.atleast_1d(np.asarray(dft_freqs, np.float64))
        n_freq = len(freqs)
    if dft_dtype is None:
        cdt = torch.complex64 if fdt == torch.float32 else torch.complex128
    else:
        cdt = dft_dtype if isinstance(dft_dtype, torch.dtype) else {
            np.dtype(np.complex64): torch.complex64,
            np.dtype(np.complex128): torch.complex128}[np.dtype(dft_dtype)]
    ph_e = ph_h = None
    if n_freq:
        pe, phh = phase_tables(freqs, n_steps, dt, int(dft_step0))
        ph_e = torch.as_tensor(pe, device=dev)
        ph_h = torch.as_tensor(phh, device=dev)
        bufs.ph_e, bufs.ph_h = ph_e.data_ptr(), ph_h.data_ptr()
    if cw:
        if not n_freq:
            raise ValueError("cw_sources needs dft_freqs")
        env = torch.as_tensor(np.asarray(cw_sources["env"], np.float64), device=dev)
        keep.append(env)
        bufs.cw_env = env.data_ptr()
        for key in ("src", "jx", "jy", "mx", "my", "mz"):
            w = cw_sources.get(f"{key}_w")
            if w is None or chans[key][0].shape[0] == 0:
                continue
            wt = (w.detach().to(device=dev, dtype=torch.complex128) if isinstance(w, torch.Tensor)
                  else torch.as_tensor(np.asarray(w), dtype=torch.complex128, device=dev))
            wt = wt.reshape(chans[key][0].shape[0], n_freq).contiguous()
            keep.append(wt)
            setattr(bufs, f"{key}_w", wt.data_ptr())

    # Outputs.
    fields = [torch.empty(s, dtype=fdt, device=dev) for s in shapes]
    if probe_comp is None:
        probe_idx = _idx3(probe_ijk, "probe_ijk", shapes[2], 0)
        pcomp = None
    else:
        raw = np.asarray(probe_ijk, np.int64).reshape(-1, 3)
        pcomp = np.ascontiguousarray(np.asarray(probe_comp, np.int64).reshape(-1), np.int32)
        if pcomp.shape[0] != raw.shape[0] or np.any((pcomp < 0) | (pcomp > 2)):
            raise ValueError("probe_comp needs one E component (0, 1 or 2) per probe")
        hi = np.array([shapes[c] for c in range(3)])[pcomp] - 1
        if raw.size and (np.any(raw < 0) or np.any(raw > hi)):
            raise ValueError("a probe lies outside its component's grid")
        probe_idx = np.ascontiguousarray(raw, np.int32)
    out_probe = torch.empty((n_steps, probe_idx.shape[0]), dtype=fdt, device=dev)
    out_v = torch.empty(n_steps, dtype=fdt, device=dev) if has_port else None
    out_i = torch.empty(n_steps, dtype=fdt, device=dev) if has_port else None
    out_e = torch.empty(n_steps, dtype=fdt, device=dev) if record_energy else None
    regions = None
    mon_out = [None] * 6
    mons = []
    if dft_regions is not None and dft_monitors is not None:
        raise ValueError("give dft_regions or dft_monitors, not both")
    if n_freq and dft_monitors is not None:
        for c, lo, hi in dft_monitors:
            lo, hi = tuple(int(v) for v in lo), tuple(int(v) for v in hi)
            if not 0 <= c < 6 or any(l < 0 or h > s or h <= l
                                     for l, h, s in zip(lo, hi, shapes[c])):
                raise ValueError(f"dft monitor {(c, lo, hi)} outside component {c}")
            t = torch.empty((n_freq,) + tuple(h - l for l, h in zip(lo, hi)), dtype=cdt,
                            device=dev)
            mons.append((c, lo, hi, t))
    elif n_freq:
        if dft_regions is None:
            mon_out = [torch.empty((n_freq,) + s, dtype=cdt, device=dev) for s in shapes]
        else:
            regions = DFTRegions(*dft_regions)
            for c, slab in enumerate(regions):
                if slab is None:
                    continue
                lo, hi = tuple(slab.lo), tuple(slab.hi)
                if any(l < 0 or h > s or h <= l for l, h, s in zip(lo, hi, shapes[c])):
                    raise ValueError(f"dft region {slab} outside component {c} {shapes[c]}")
                mon_out[c] = torch.empty((n_freq,) + tuple(h - l for l, h in zip(lo, hi)),
                                         dtype=cdt, device=dev)
                mons.append((c, lo, hi, mon_out[c]))

    prm = YeeParams()
    prm.nx, prm.ny, prm.nz, prm.npml, prm.n_steps = nx, ny, nz, npml, n_steps
    prm.n_src, prm.n_jx, prm.n_jy = (chans[k][0].shape[0] for k in ("src", "jx", "jy"))
    prm.n_mx, prm.n_my, prm.n_mz = (chans[k][0].shape[0] for k in ("mx", "my", "mz"))
    prm.n_probes, prm.has_port = probe_idx.shape[0], int(has_port)
    limited = dft_regions is not None or dft_monitors is not None
    prm.n_freq = n_freq if (not limited or mons or cw) else 0
    prm.dft_f64 = int(cdt == torch.complex128)
    prm.n_monitors = len(mons) if limited else 0
    prm.record_energy, prm.cw_sources = int(bool(record_energy)), int(cw)
    prm.dt, prm.dx, prm.dy, prm.dz, prm.mu0 = dt, dx, dy, dz, MU0

    pts = YeePoints()
    for key in ("src", "jx", "jy", "mx", "my", "mz"):
        arr = chans[key][0]
        setattr(pts, key, arr.ctypes.data_as(_native.P_i32) if arr.shape[0] else None)
    pts.probe = probe_idx.ctypes.data_as(_native.P_i32) if probe_idx.shape[0] else None
    pts.probe_comp = (pcomp.ctypes.data_as(_native.P_i32)
                      if pcomp is not None and pcomp.shape[0] else None)
    if has_port:
        pts.port[0], pts.port[1], pts.port[2] = (int(v) for v in pidx)
    mon_arr = (_native.DftMonitor * max(len(mons), 1))()
    for k, (c, lo, hi, t) in enumerate(mons):
        mon_arr[k].comp = c
        for a in range(3):
            mon_arr[k].lo[a], mon_arr[k].hi[a] = lo[a], hi[a]
        mon_arr[k].out = t.data_ptr()
    pts.monitors = mon_arr

    bufs.ca, bufs.cb, bufs.eps = ca.data_ptr(), cb.data_ptr(), eps.data_ptr()
    bufs.dt_mu, bufs.inv_dx, bufs.inv_dy, bufs.inv_dz = dt / MU0, inv[0], inv[1], inv[2]
    bufs.a_port, bufs.b_port, bufs.c_port = a_port, b_port, c_port
    bufs.cb_src = cb_src.data_ptr() if cb_src.numel() else None
    bufs.cb_jx = cb_jx.data_ptr() if cb_jx.numel() else None
    bufs.cb_jy = cb_jy.data_ptr() if cb_jy.numel() else None
    bufs.ex, bufs.ey, bufs.ez, bufs.hx, bufs.hy, bufs.hz = (t.data_ptr() for t in fields)
    bufs.out_probe = out_probe.data_ptr() if out_probe.numel() else None
    bufs.out_v = _native.ptr(out_v)
    bufs.out_i = _native.ptr(out_i)
    bufs.out_energy = _native.ptr(out_e)
    if n_freq and not limited:
        for c in range(6):
            bufs.dft[c] = mon_out[c].data_ptr()

    f64 = fdt == torch.float64
    nbytes = ctypes.c_size_t(0)
    _native.check(lib.gdn_yee_workspace_size(ctypes.byref(prm), ctypes.byref(pts), int(f64),
                                             ctypes.byref(nbytes)))
    ws = torch.empty(max(int(nbytes.value), 1), dtype=torch.uint8, device=dev)
    bufs.workspace, bufs.workspace_bytes = ws.data_ptr(), int(nbytes.value)
    state_out = None
    if state_in is not None or return_state:
        sbytes = ctypes.c_size_t(0)
        _native.check(lib.gdn_yee_state_size(ctypes.byref(prm), int(f64), ctypes.byref(sbytes)))
        if state_in is not None:
            if (not isinstance(state_in, torch.Tensor) or state_in.dtype != torch.uint8
                    or state_in.numel() != int(sbytes.value) or state_in.device != ws.device
                    or not state_in.is_contiguous()):
                raise ValueError("state_in must be the contiguous uint8 device state of a run "
                                 f"on this grid and dtype ({int(sbytes.value)} bytes)")
            bufs.state_in = state_in.data_ptr()
        if return_state:
            state_out = torch.empty(int(sbytes.value), dtype=torch.uint8, device=dev)
            bufs.state_out = state_out.data_ptr()
    stream = torch.cuda.current_stream(dev)
    run = lib.gdn_yee_run_f64 if f64 else lib.gdn_yee_run_f32
    with torch.cuda.device(dev):
        _native.check(run(ctypes.byref(prm), ctypes.byref(pts), ctypes.byref(bufs),
                          ctypes.c_void_p(stream.cuda_stream)))
    del keep

    dft = None
    monitors = None
    if n_freq:
        ft = torch.as_tensor(freqs, device=dev)
        if dft_monitors is not None:
            monitors = [t for (_, _, _, t) in mons]
        elif dft_regions is None:
            dft = DFTMonitor(ft, *mon_out)
        else:
            dft = RegionDFTMonitor(ft, regions, *mon_out)
    return SimResult3D(out_probe, out_v, out_i, out_e, dft, *fields, monitors, state_out)
