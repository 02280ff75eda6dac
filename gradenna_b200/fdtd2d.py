"""2D TM FDTD on B200: the ``simulate_tm`` surface over the CUDA C ABI.

Non-zero components Ez(i, j), Hx(i, j+1/2), Hy(i+1/2, j); the outermost Ez
ring is PEC. The update, port and DFT conventions are those of the reference
``simulate_tm`` (src/gradenna/fdtd2d.py:1-56):

    Hx^{n+1/2} = Hx - dt/mu [ dEz/dy / kappa_y + psi_Hx,y ]
    Hy^{n+1/2} = Hy + dt/mu [ dEz/dx / kappa_x + psi_Hy,x ]
    Ez^{n+1}   = Ca Ez + Cb [ dHy/dx / kappa_x + psi_Ez,x - dHx/dy / kappa_y - psi_Ez,y ]
    Ez[src]   -= Cb_src J,   Ez[port] -= Cb_vs Vs,
    V^{n+1/2}  = -DZ (Ez^n + Ez^{n+1}) / 2,  I^{n+1/2} = Ampere loop of H^{n+1/2}
    X(f)       = dt sum_n x^n exp(-i 2 pi f t_n), t_n = (n+1) dt (E), (n+1/2) dt (H)

This module does the host-side work only: argument validation, the
coefficient tables (built in the field dtype exactly as the reference builds
them, fdtd2d.py:343-398, so the device loop does no coefficient math), and
one call into ``gdn_tm_run_f32`` / ``gdn_tm_run_f64``, which runs the whole
time loop on the GPU. Arrays are torch tensors on a CUDA device; there is no
CPU fallback.
"""

from __future__ import annotations

import ctypes
import functools
from typing import NamedTuple

import numpy as np
import torch

from gradenna_b200 import _native
from gradenna_b200.constants import EPS0, MU0
from gradenna_b200.cpml import CPMLSpec, axis_coefficients, slab_tables
from gradenna_b200.grid import Grid2D

#: Unit length [m] of the 2D TM slice; port voltage is V = -Ez * DZ.
DZ = 1.0

__all__ = ["DZ", "Port", "SimResult", "simulate_tm", "field_energy"]


class Port(NamedTuple):
    """Lumped resistive voltage source (RVS) port on one Ez cell (fdtd2d.py:81-98).

    ij: (i, j) of the Ez cell; resistance: Rs > 0 [ohm m]; voltage: Vs(t)
    sampled at (n+1/2) dt, shape (n_steps,), or None for a passive load.
    """

    ij: tuple
    resistance: float = 50.0
    voltage: object = None


class SimResult(NamedTuple):
    """Time series, DFT monitors and final fields (fdtd2d.py:101-126).

    probe_ez (n_steps, n_probes); energy (n_steps,) or None; ez/hx/hy final
    fields; port_v/port_i (n_steps, n_ports) or None; dft_ez/hx/hy complex
    (n_freq, ...) phasors already scaled by dt, or None. With ``dft_region``
    the DFT arrays cover only the requested rectangles.
    """

    probe_ez: torch.Tensor
    energy: torch.Tensor | None
    ez: torch.Tensor
    hx: torch.Tensor
    hy: torch.Tensor
    port_v: torch.Tensor | None = None
    port_i: torch.Tensor | None = None
    dft_ez: torch.Tensor | None = None
    dft_hx: torch.Tensor | None = None
    dft_hy: torch.Tensor | None = None
    monitors: list | None = None


def field_energy(ez, hx, hy, eps, grid: Grid2D):
    """Total energy per unit length 1/2 (eps E^2 + mu H^2) dA (fdtd2d.py:160-169)."""
    cell = grid.dx * grid.dy
    ue = 0.5 * torch.sum(eps * ez**2) * cell
    uh = 0.5 * MU0 * (torch.sum(hx**2) + torch.sum(hy**2)) * cell
    return ue + uh


def _as_index_array(ij, name: str, grid: Grid2D, margin: int) -> np.ndarray:
    """(n, 2) int32 indices inside the interior with `margin` (fdtd2d.py:172-178)."""
    idx = np.asarray(ij, dtype=np.int64).reshape(-1, 2)
    lo = np.array([margin, margin])
    hi = np.array([grid.nx - 1 - margin, grid.ny - 1 - margin])
    if idx.size and (np.any(idx < lo) or np.any(idx > hi)):
        raise ValueError(f"{name} {idx.tolist()} outside the interior (PML margin {margin})")
    return idx.astype(np.int32)


def _torch_dtype(dt) -> torch.dtype:
    if isinstance(dt, torch.dtype):
        return dt
    return {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64}[np.dtype(dt)]


def _operand_dtype(x):
    if isinstance(x, torch.Tensor):
        return x.dtype
    if isinstance(x, np.ndarray):
        return _torch_dtype(x.dtype) if x.dtype in (np.float32, np.float64) else None
    return None  # python scalars / lists are weakly typed


def infer_dtype(operands, dtype=None) -> torch.dtype:
    """Field dtype: explicit ``dtype`` or the widest float among array operands.

    Python scalars do not promote (as in the reference's weak typing);
    float32 is the default when no operand carries a dtype.
    """
    if dtype is not None:
        dt = dtype if isinstance(dtype, torch.dtype) else _torch_dtype(np.dtype(dtype))
    else:
        dt = torch.float32
        for x in operands:
            d = _operand_dtype(x)
            if d == torch.float64:
                dt = torch.float64
    if dt not in (torch.float32, torch.float64):
        raise ValueError(f"field dtype must be float32 or float64, got {dt}")
    return dt


def _to_dev(x, dtype, device):
    if isinstance(x, torch.Tensor):
        return x.detach().to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.asarray(x), dtype=dtype, device=device).contiguous()


def _waveforms(cur, n_steps, n_pts, dtype, device, name):
    if cur is None:
        return torch.zeros((n_steps, 0), dtype=dtype, device=device)
    c = _to_dev(cur, dtype, device)
    if c.ndim == 1:
        c = c[:, None]
    if c.shape[0] != n_steps:
        raise ValueError(f"{name} length {c.shape[0]} != n_steps {n_steps}")
    if c.shape[1] != n_pts:
        raise ValueError(f"{name} has {c.shape[1]} columns for {n_pts} sources")
    return c.contiguous()


def phase_tables(freqs, n_steps: int, dt: float, step0: int = 0):
    """Exact-phase tables exp(-2 pi i f t_n) in float64 (fdtd2d.py:393-398).

    Returns (ph_e, ph_h), each complex128 numpy (n_steps, n_freq), with
    t_n = (n+1) dt and (n+1/2) dt for the absolute steps n = step0 ..
    step0 + n_steps - 1 (step0 > 0: the rows of a resumed run).
    """
    f = np.asarray(freqs, np.float64)
    nn = np.arange(step0, step0 + n_steps, dtype=np.float64)
    ph_e = np.exp(-2j * np.pi * np.outer(nn + 1.0, f) * dt)
    ph_h = np.exp(-2j * np.pi * np.outer(nn + 0.5, f) * dt)
    return ph_e, ph_h


@functools.lru_cache(maxsize=256)
def _phase_tables_dev(freqs: tuple, n_steps: int, dt: float, device: torch.device):
    """phase_tables on the device, cached: the forward and adjoint runs of a
    problem, and every iteration of an optimisation, read the same tables.
    The kernels only read them."""
    ph_e, ph_h = phase_tables(freqs, n_steps, dt)
    return torch.as_tensor(ph_e, device=device), torch.as_tensor(ph_h, device=device)


@functools.lru_cache(maxsize=256)
def _cpml_tables_dev(nx: int, ny: int, dx: float, dy: float, dt: float, cpml: CPMLSpec,
                     npdt, device: torch.device):
    """The 2D CPML slab tables and 1/kappa tables on the device
    (fdtd2d.py:354-374), cached per grid, CPML and dtype; read-only."""
    npml = cpml.thickness
    cx_e = axis_coefficients(nx, dx, dt, cpml, half=False, dtype=npdt)
    cx_h = axis_coefficients(nx, dx, dt, cpml, half=True, dtype=npdt)
    cy_e = axis_coefficients(ny, dy, dt, cpml, half=False, dtype=npdt)
    cy_h = axis_coefficients(ny, dy, dt, cpml, half=True, dtype=npdt)
    tabs = {}
    for key, (b, c) in {
        "ezx": (cx_e.b[1:-1], cx_e.c[1:-1]), "ezy": (cy_e.b[1:-1], cy_e.c[1:-1]),
        "hyx": (cx_h.b, cx_h.c), "hxy": (cy_h.b, cy_h.c),
    }.items():
        b_lo, c_lo, b_hi, c_hi = slab_tables(b, c, npml)
        for nm, arr in (("b_lo", b_lo), ("c_lo", c_lo), ("b_hi", b_hi), ("c_hi", c_hi)):
            tabs[f"{nm[0]}_{key}_{nm[2:]}"] = torch.as_tensor(
                np.ascontiguousarray(arr) if arr.size else np.zeros(1, npdt), device=device)
    ik = {
        "inv_kx_e": cx_e.inv_kappa[1:-1], "inv_ky_e": cy_e.inv_kappa[1:-1],
        "inv_kx_h": cx_h.inv_kappa, "inv_ky_h": cy_h.inv_kappa,
    }
    ik = {k: torch.as_tensor(np.ascontiguousarray(v), device=device) for k, v in ik.items()}
    return tabs, ik


def _i32(a) -> ctypes.POINTER(ctypes.c_int32):
    return a.ctypes.data_as(_native.P_i32)


def _region_rect(r, shape):
    if r is None:
        return None
    lo0, lo1, hi0, hi1 = (int(v) for v in r)
    if not (0 <= lo0 < hi0 <= shape[0] and 0 <= lo1 < hi1 <= shape[1]):
        raise ValueError(f"dft region {r} outside the component shape {shape}")
    return (lo0, lo1, hi0, hi1)


def _prepare_tm(
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
    record_energy: bool = False,
    mx_ij=None,
    mx_current=None,
    my_ij=None,
    my_current=None,
    dtype=None,
    device=None,
    dft_region=None,
    dft_monitors=None,
    cw_sources=None,
) -> "_Prep":
    """Validate the arguments of simulate_tm and build its C-ABI structs,
    device inputs and output tensors (everything but the workspace and the
    call)."""
    nx, ny = grid.nx, grid.ny
    if min(nx, ny) <= 2 * cpml.thickness + 2:
        raise ValueError(f"grid {nx}x{ny} is too small for CPML thickness {cpml.thickness}")
    dt = grid.dt
    dev = _native.require_cuda(device)
    lib = _native.load()

    if (source_ij is None) != (source_current is None) and cw_sources is None:
        raise ValueError("source_ij and source_current must be given together")
    ports = tuple(p if isinstance(p, Port) else Port(*p) for p in ports)
    n_ports = len(ports)

    # n_steps from the source and/or port waveforms (fdtd2d.py:260-279).
    n_steps = None
    if source_current is not None:
        n_steps = int(np.shape(source_current)[0])
    for p in ports:
        if p.voltage is None:
            continue
        shp = tuple(np.shape(p.voltage))
        if len(shp) != 1:
            raise ValueError(f"port voltage waveform must be 1D, got shape {shp}")
        if n_steps is None:
            n_steps = shp[0]
        elif shp[0] != n_steps:
            raise ValueError(f"port voltage length {shp[0]} does not match n_steps {n_steps}")
    if n_steps is None:
        for cur in (mx_current, my_current):
            if cur is not None:
                n_steps = int(np.shape(cur)[0])
                break
    if n_steps is None and cw_sources is not None:
        n_steps = int(np.shape(cw_sources["env"])[0])
    if n_steps is None:
        raise ValueError("need source_current and/or at least one port with a voltage waveform")

    operands = [eps_r, sigma, source_current, mx_current, my_current]
    operands += [p.voltage for p in ports]
    fdt = infer_dtype(operands, dtype)
    npdt = np.float32 if fdt == torch.float32 else np.float64

    probe_idx = _as_index_array(probe_ij, "probe_ij", grid, margin=0)
    if cw_sources is not None:
        src_idx = (np.zeros((0, 2), np.int32) if source_ij is None
                   else _as_index_array(source_ij, "source_ij", grid, margin=1))
        src_cur = None
    elif source_current is None:
        src_idx = np.zeros((0, 2), np.int32)
        src_cur = torch.zeros((n_steps, 0), dtype=fdt, device=dev)
    else:
        src_idx = _as_index_array(source_ij, "source_ij", grid, margin=1)
        src_cur = _waveforms(source_current, n_steps, src_idx.shape[0], fdt, dev, "source_current")

    def setup_mag(m_ij, m_cur, shape, name):
        if (m_ij is None) != (m_cur is None) and cw_sources is None:
            raise ValueError(f"{name}_ij and {name}_current must be given together")
        if m_ij is None:
            return np.zeros((0, 2), np.int32), None
        idx = np.asarray(m_ij, np.int64).reshape(-1, 2)
        hi = np.array([shape[0] - 1, shape[1] - 1])
        if idx.size and (np.any(idx < 0) or np.any(idx > hi)):
            raise ValueError(f"{name}_ij {idx.tolist()} outside the {name} grid {tuple(shape)}")
        if cw_sources is not None:
            return idx.astype(np.int32), None
        return idx.astype(np.int32), _waveforms(m_cur, n_steps, idx.shape[0], fdt, dev,
                                                f"{name}_current")

    mx_idx, mx_cur = setup_mag(mx_ij, mx_current, (nx, ny - 1), "mx")
    my_idx, my_cur = setup_mag(my_ij, my_current, (nx - 1, ny), "my")

    # Materials, port conductivity and ca/cb in the field dtype (fdtd2d.py:343-352).
    eps = (EPS0 * torch.broadcast_to(_to_dev(eps_r, fdt, dev), (nx, ny))).contiguous()
    sig = torch.broadcast_to(_to_dev(sigma, fdt, dev), (nx, ny)).clone()
    if n_ports:
        port_idx = _as_index_array([p.ij for p in ports], "port ij", grid, margin=1)
        rs = np.asarray([float(p.resistance) for p in ports])
        if np.any(rs <= 0.0):
            raise ValueError("port resistance must be positive")
        port_rs = torch.as_tensor(rs, dtype=fdt, device=dev)
        pi = torch.as_tensor(port_idx[:, 0].astype(np.int64), device=dev)
        pj = torch.as_tensor(port_idx[:, 1].astype(np.int64), device=dev)
        sig.index_put_((pi, pj), DZ / (port_rs * grid.dx * grid.dy), accumulate=True)
        vs = [torch.zeros(n_steps, dtype=fdt, device=dev) if p.voltage is None
              else _to_dev(p.voltage, fdt, dev).reshape(-1) for p in ports]
        port_vs = torch.stack(vs, dim=1).contiguous()
    else:
        port_idx = np.zeros((0, 2), np.int32)
        port_vs = torch.zeros((n_steps, 0), dtype=fdt, device=dev)
    half_loss = sig * dt / (2.0 * eps)
    ca = ((1.0 - half_loss) / (1.0 + half_loss)).contiguous()
    cb = ((dt / eps) / (1.0 + half_loss)).contiguous()

    inv_dx, inv_dy = 1.0 / grid.dx, 1.0 / grid.dy
    si = torch.as_tensor(src_idx[:, 0].astype(np.int64), device=dev)
    sj = torch.as_tensor(src_idx[:, 1].astype(np.int64), device=dev)
    cb_src = (cb[si, sj] * (inv_dx * inv_dy)).contiguous()
    if n_ports:
        cb_vs = (cb[pi, pj] / (port_rs * grid.dx * grid.dy)).contiguous()
    else:
        cb_vs = torch.zeros(0, dtype=fdt, device=dev)

    # CPML tables (fdtd2d.py:354-374), built once per grid, CPML and dtype.
    npml = cpml.thickness
    tabs, ik = _cpml_tables_dev(nx, ny, float(grid.dx), float(grid.dy), float(dt), cpml, npdt,
                                torch.device(dev))

    # DFT (fdtd2d.py:384-398).
    dft_freqs = tuple(float(f) for f in dft_freqs)
    n_freq = len(dft_freqs)
    if dft_dtype is None:
        cdt = torch.complex64 if fdt == torch.float32 else torch.complex128
    else:
        cdt = {np.dtype(np.complex64): torch.complex64, np.dtype(np.complex128): torch.complex128}.get(
            np.dtype(dft_dtype) if not isinstance(dft_dtype, torch.dtype) else None, dft_dtype)
        if cdt not in (torch.complex64, torch.complex128):
            raise ValueError(f"dft_dtype must be a complex dtype, got {dft_dtype}")
    ph_e_t = ph_h_t = None
    if n_freq:
        ph_e_t, ph_h_t = _phase_tables_dev(dft_freqs, int(n_steps), float(dt), torch.device(dev))
    if cw_sources is not None and not n_freq:
        raise ValueError("cw_sources needs dft_freqs")

    full_shapes = ((nx, ny), (nx, ny - 1), (nx - 1, ny))
    # Monitor list: (comp, rect) pairs; full grid when nothing is requested.
    mon_specs = []
    if n_freq:
        if dft_monitors is not None:
            for m in dft_monitors:
                comp = int(m[0])
                if comp not in (0, 1, 2):
                    raise ValueError(f"monitor component {comp} not in 0..2")
                mon_specs.append((comp, _region_rect(m[1:5], full_shapes[comp])))
        elif dft_region is not None:
            for comp, (r, shp) in enumerate(zip(dft_region, full_shapes)):
                rr = _region_rect(r, shp)
                if rr is not None:
                    mon_specs.append((comp, rr))
    mon_out = [torch.empty((n_freq, r[2] - r[0], r[3] - r[1]), dtype=cdt, device=dev)
               for _, r in mon_specs]
    dft_out = [None, None, None]
    if n_freq and dft_monitors is None:
        if dft_region is None:
            dft_out = [torch.empty((n_freq,) + s_, dtype=cdt, device=dev) for s_ in full_shapes]
        else:
            for (comp, _), t in zip(mon_specs, mon_out):
                dft_out[comp] = t

    # Outputs.
    ez = torch.empty((nx, ny), dtype=fdt, device=dev)
    hx = torch.empty((nx, ny - 1), dtype=fdt, device=dev)
    hy = torch.empty((nx - 1, ny), dtype=fdt, device=dev)
    out_probe = torch.empty((n_steps, probe_idx.shape[0]), dtype=fdt, device=dev)
    out_v = torch.empty((n_steps, n_ports), dtype=fdt, device=dev)
    out_i = torch.empty((n_steps, n_ports), dtype=fdt, device=dev)
    out_energy = torch.empty(n_steps, dtype=fdt, device=dev) if record_energy else None

    cw = None
    if cw_sources is not None:
        env = torch.as_tensor(np.asarray(cw_sources["env"], np.float64), device=dev).contiguous()
        if env.shape[0] != n_steps:
            raise ValueError("cw env length must equal n_steps")

        def wts(key, n):
            w = cw_sources.get(key)
            if n == 0:
                return None
            if isinstance(w, torch.Tensor):
                w = w.detach().to(device=dev, dtype=torch.complex128)
            else:
                w = torch.as_tensor(np.asarray(w), dtype=torch.complex128, device=dev)
            return w.reshape(n, n_freq).contiguous()

        cw = dict(env=env, src_w=wts("src_w", src_idx.shape[0]), mx_w=wts("mx_w", mx_idx.shape[0]),
                  my_w=wts("my_w", my_idx.shape[0]))

    params = _native.TmParams()
    params.nx, params.ny, params.npml, params.n_steps = nx, ny, npml, n_steps
    params.n_sources, params.n_ports = src_idx.shape[0], n_ports
    params.n_mx, params.n_my, params.n_probes = mx_idx.shape[0], my_idx.shape[0], probe_idx.shape[0]
    params.n_freq = n_freq
    params.record_energy = int(bool(record_energy))
    params.dft_f64 = int(cdt == torch.complex128)
    params.cw_sources = int(cw is not None)
    use_mons = bool(n_freq) and (dft_monitors is not None or dft_region is not None)
    params.n_monitors = len(mon_specs) if use_mons else 0
    mon_arr = (_native.DftMonitor * max(len(mon_specs), 1))()
    for k, ((comp, r), t) in enumerate(zip(mon_specs, mon_out)):
        mon_arr[k].comp = comp
        mon_arr[k].lo[0], mon_arr[k].lo[1], mon_arr[k].lo[2] = r[0], r[1], 0
        mon_arr[k].hi[0], mon_arr[k].hi[1], mon_arr[k].hi[2] = r[2], r[3], 1
        mon_arr[k].out = t.data_ptr()
    if use_mons and not mon_specs and cw_sources is None:
        params.n_freq = 0  # every requested box is empty: no DFT work at all
    params.dt, params.dx, params.dy, params.dz, params.mu0 = dt, grid.dx, grid.dy, DZ, MU0

    idx_arrays = {
        "src": np.ascontiguousarray(src_idx, np.int32),
        "port": np.ascontiguousarray(port_idx, np.int32),
        "mx": np.ascontiguousarray(mx_idx, np.int32),
        "my": np.ascontiguousarray(my_idx, np.int32),
        "probe": np.ascontiguousarray(probe_idx, np.int32),
    }
    cols = {k: (np.ascontiguousarray(v[:, 0]), np.ascontiguousarray(v[:, 1]))
            for k, v in idx_arrays.items()}
    pts = _native.TmPoints()
    for k, (a, b) in cols.items():
        setattr(pts, f"{k}_i", _i32(a))
        setattr(pts, f"{k}_j", _i32(b))
    pts.monitors = mon_arr

    bufs = _native.TmBuffers()
    bufs.ca, bufs.cb, bufs.eps = ca.data_ptr(), cb.data_ptr(), eps.data_ptr()
    for k, v in ik.items():
        setattr(bufs, k, v.data_ptr())
    for k, v in tabs.items():
        setattr(bufs, k, v.data_ptr())
    bufs.dt_mu, bufs.inv_dx, bufs.inv_dy = dt / MU0, inv_dx, inv_dy
    bufs.cb_src = cb_src.data_ptr() if cb_src.numel() else None
    bufs.src_cur = _native.ptr(src_cur) if src_cur is not None and src_cur.numel() else None
    bufs.cb_vs = cb_vs.data_ptr() if n_ports else None
    bufs.port_vs = port_vs.data_ptr() if n_ports else None
    bufs.mx_cur = _native.ptr(mx_cur) if mx_cur is not None else None
    bufs.my_cur = _native.ptr(my_cur) if my_cur is not None else None
    if cw is not None:
        bufs.cw_env = cw["env"].data_ptr()
        bufs.src_w = _native.ptr(cw["src_w"])
        bufs.mx_w = _native.ptr(cw["mx_w"])
        bufs.my_w = _native.ptr(cw["my_w"])
    bufs.ph_e = _native.ptr(ph_e_t)
    bufs.ph_h = _native.ptr(ph_h_t)
    bufs.ez, bufs.hx, bufs.hy = ez.data_ptr(), hx.data_ptr(), hy.data_ptr()
    bufs.out_probe = out_probe.data_ptr() if out_probe.numel() else None
    bufs.out_v = out_v.data_ptr() if out_v.numel() else None
    bufs.out_i = out_i.data_ptr() if out_i.numel() else None
    bufs.out_energy = _native.ptr(out_energy)
    bufs.dft_ez, bufs.dft_hx, bufs.dft_hy = (_native.ptr(t) for t in dft_out)

    keep = (ca, cb, eps, tabs, ik, src_cur, mx_cur, my_cur, port_vs, cb_src, cb_vs, ph_e_t,
            ph_h_t, cw)
    host = (idx_arrays, cols, mon_arr)
    result = SimResult(
        probe_ez=out_probe,
        energy=out_energy,
        ez=ez,
        hx=hx,
        hy=hy,
        port_v=out_v if n_ports else None,
        port_i=out_i if n_ports else None,
        dft_ez=dft_out[0],
        dft_hx=dft_out[1],
        dft_hy=dft_out[2],
        monitors=mon_out if dft_monitors is not None else None,
    )
    return _Prep(params, pts, bufs, keep, host, result, fdt == torch.float64, dev)


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
    record_energy: bool = False,
    mx_ij=None,
    mx_current=None,
    my_ij=None,
    my_current=None,
    dtype=None,
    device=None,
    dft_region=None,
    dft_monitors=None,
    cw_sources=None,
) -> SimResult:
    """Run a 2D TM FDTD simulation on the GPU (drop-in for fdtd2d.simulate_tm).

    Arguments and semantics follow the reference (fdtd2d.py:181-247):
    ``source_ij``/``source_current`` Jz line currents sampled at (n+1/2) dt;
    ``eps_r``/``sigma`` scalars or (nx, ny); ``probe_ij`` Ez probes;
    ``ports`` lumped RVS ports; ``dft_freqs`` running-DFT frequencies with
    ``dft_dtype`` accumulators (default complex64 for float32 fields);
    ``cpml``; ``record_energy``; ``mx_*``/``my_*`` magnetic currents on the
    Hx/Hy grids injected as H -= (dt/mu) M.

    Additions: ``dtype`` forces the field dtype; ``device`` selects the CUDA
    device; ``dft_region`` = (ez_rect, hx_rect, hy_rect), each
    (lo_i, lo_j, hi_i, hi_j) or None, limits the DFT to those rectangles;
    ``dft_monitors`` = [(comp, lo_i, lo_j, hi_i, hi_j), ...] with comp 0/1/2 =
    ez/hx/hy records only those boxes (returned in ``SimResult.monitors``,
    dft_ez/hx/hy are then None); ``cw_sources`` = dict(env, src_w, mx_w, my_w) synthesises the Jz/Mx/My
    waveforms on the device as env[n] Re(sum_k W_k exp(+i w_k t_n)) (the
    frequency-domain adjoint's CW drive) instead of reading tabulated ones.
    """
    p = _prepare_tm(grid, source_ij=source_ij, source_current=source_current, eps_r=eps_r, sigma=sigma, probe_ij=probe_ij, ports=ports, dft_freqs=dft_freqs, dft_dtype=dft_dtype, cpml=cpml, record_energy=record_energy, mx_ij=mx_ij, mx_current=mx_current, my_ij=my_ij, my_current=my_current, dtype=dtype, device=device, dft_region=dft_region, dft_monitors=dft_monitors, cw_sources=cw_sources)
    lib = _native.load()
    nbytes = ctypes.c_size_t(0)
    _native.check(lib.gdn_tm_workspace_size(ctypes.byref(p.params), ctypes.byref(p.pts),
                                            int(p.f64), ctypes.byref(nbytes)))
    ws = torch.empty(max(int(nbytes.value), 1), dtype=torch.uint8, device=p.dev)
    p.bufs.workspace, p.bufs.workspace_bytes = ws.data_ptr(), int(nbytes.value)
    stream = torch.cuda.current_stream(p.dev)
    run = lib.gdn_tm_run_f64 if p.f64 else lib.gdn_tm_run_f32
    with torch.cuda.device(p.dev):
        _native.check(run(ctypes.byref(p.params), ctypes.byref(p.pts), ctypes.byref(p.bufs),
                          ctypes.c_void_p(stream.cuda_stream)))
    # Keep device inputs alive until the stream has consumed them.
    for t in _flatten((ws, p.keep)):
        t.record_stream(stream)
    return p.result


class _Prep(NamedTuple):
    params: object
    pts: object
    bufs: object
    keep: tuple
    host: tuple
    result: SimResult
    f64: bool
    dev: object


def _flatten(x):
    if isinstance(x, torch.Tensor):
        yield x
    elif isinstance(x, dict):
        for v in x.values():
            yield from _flatten(v)
    elif isinstance(x, (list, tuple)):
        for v in x:
            yield from _flatten(v)
