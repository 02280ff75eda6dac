"""Python driver of the C oracle (oracle/tm2d_ref.c): test/baseline use only.

``simulate_tm_c`` has the argument set of the numpy oracle's simulate_tm and
returns the same SimResult, but runs the multi-threaded C time loop. The
coefficient tables are built here with the oracle's own restatement of the
reference set-up (fdtd2d.py:343-398), not with the product's code. Only the
ctypes mirrors of the C structs are shared with the product (their layout is
checked against include/gradenna_b200.h by the ABI tests).
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from oracle import fdtd2d_np as onp

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "build", "liboracle_tm2d.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        from gradenna_b200 import _native as nt

        lib = ctypes.CDLL(LIB)
        for name in ("oracle_tm_run_f32", "oracle_tm_run_f64"):
            fn = getattr(lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.POINTER(nt.TmParams), ctypes.POINTER(nt.TmPoints),
                           ctypes.POINTER(nt.TmBuffers)]
        _lib = lib
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def simulate_tm_c(grid, *, source_ij=None, source_current=None, eps_r=1.0, sigma=0.0,
                  probe_ij=(), ports=(), dft_freqs=(), cpml=onp.CPMLSpec(),
                  record_energy=False, mx_ij=None, mx_current=None, my_ij=None,
                  my_current=None, dtype=np.float64, dft_monitors=None, cw=None):
    """C-oracle run; DFT accumulators are double (returned complex128)."""
    from gradenna_b200 import _native as nt

    lib = load()
    dtype = np.dtype(dtype)
    f = dtype.type
    nx, ny = grid.nx, grid.ny
    dt = grid.dt
    ports = tuple(p if isinstance(p, onp.Port) else onp.Port(*p) for p in ports)
    n_steps = None
    if source_current is not None:
        n_steps = np.shape(source_current)[0]
    for p in ports:
        if p.voltage is not None:
            n_steps = np.shape(p.voltage)[0]
    for c in (mx_current, my_current):
        if n_steps is None and c is not None:
            n_steps = np.shape(c)[0]
    if n_steps is None and cw is not None:
        n_steps = len(cw["env"])

    def idx(ij, margin):
        return onp._idx(ij if ij is not None else np.zeros((0, 2)), "idx", grid, margin).astype(np.int32)

    src = idx(source_ij, 1)
    prb = idx(probe_ij, 0)
    mxi = np.asarray(mx_ij if mx_ij is not None else np.zeros((0, 2)), np.int32).reshape(-1, 2)
    myi = np.asarray(my_ij if my_ij is not None else np.zeros((0, 2)), np.int32).reshape(-1, 2)
    prt = idx([p.ij for p in ports], 1) if ports else np.zeros((0, 2), np.int32)

    def wav(cur, n):
        if cur is None or cw is not None:
            return np.zeros((n_steps, max(n, 1)), dtype)
        c = np.asarray(cur, dtype)
        return np.ascontiguousarray(c[:, None] if c.ndim == 1 else c)

    eps = (onp.EPS0 * np.broadcast_to(np.asarray(eps_r, dtype), (nx, ny))).astype(dtype)
    sig = np.array(np.broadcast_to(np.asarray(sigma, dtype), (nx, ny)), dtype)
    rs = np.asarray([float(p.resistance) for p in ports])
    if ports:
        np.add.at(sig, (prt[:, 0], prt[:, 1]), (onp.DZ / (rs * grid.dx * grid.dy)).astype(dtype))
    hl = (sig * f(dt) / (f(2.0) * eps)).astype(dtype)
    ca = np.ascontiguousarray((f(1.0) - hl) / (f(1.0) + hl), dtype)
    cb = np.ascontiguousarray((f(dt) / eps) / (f(1.0) + hl), dtype)
    cb_src = np.ascontiguousarray(cb[src[:, 0], src[:, 1]] * f(1.0 / (grid.dx * grid.dy)), dtype)
    cb_vs = np.ascontiguousarray(cb[prt[:, 0], prt[:, 1]] / (rs * grid.dx * grid.dy), dtype) if ports else np.zeros(1, dtype)
    vs = (np.stack([np.zeros(n_steps, dtype) if p.voltage is None else np.asarray(p.voltage, dtype)
                    for p in ports], 1) if ports else np.zeros((n_steps, 1), dtype))
    vs = np.ascontiguousarray(vs, dtype)

    ax = {k: onp.axis_coefficients(n, d, dt, cpml, half=h, dtype=dtype)
          for k, (n, d, h) in {"xe": (nx, grid.dx, False), "xh": (nx, grid.dx, True),
                               "ye": (ny, grid.dy, False), "yh": (ny, grid.dy, True)}.items()}
    npml = cpml.thickness
    tabs = {}
    for key, (b, c) in {"ezx": (ax["xe"].b[1:-1], ax["xe"].c[1:-1]),
                        "ezy": (ax["ye"].b[1:-1], ax["ye"].c[1:-1]),
                        "hyx": (ax["xh"].b, ax["xh"].c), "hxy": (ax["yh"].b, ax["yh"].c)}.items():
        lo, hi = onp.slab_slices(b.shape[0], npml)
        for nm, arr in (("b_%s_lo", b[lo]), ("c_%s_lo", c[lo]), ("b_%s_hi", b[hi]), ("c_%s_hi", c[hi])):
            tabs[nm % key] = np.ascontiguousarray(arr if arr.size else np.zeros(1, dtype), dtype)
    ik = {"inv_kx_e": ax["xe"].inv_kappa[1:-1], "inv_ky_e": ax["ye"].inv_kappa[1:-1],
          "inv_kx_h": ax["xh"].inv_kappa, "inv_ky_h": ax["yh"].inv_kappa}
    ik = {k: np.ascontiguousarray(v, dtype) for k, v in ik.items()}

    K = len(tuple(dft_freqs))
    ph_e = ph_h = None
    if K:
        fr = np.asarray(dft_freqs, np.float64)
        nn = np.arange(n_steps, dtype=np.float64)
        ph_e = np.ascontiguousarray(np.exp(-2j * np.pi * np.outer(nn + 1.0, fr) * dt))
        ph_h = np.ascontiguousarray(np.exp(-2j * np.pi * np.outer(nn + 0.5, fr) * dt))

    ez = np.zeros((nx, ny), dtype)
    hx = np.zeros((nx, ny - 1), dtype)
    hy = np.zeros((nx - 1, ny), dtype)
    out_probe = np.zeros((n_steps, max(len(prb), 1)), dtype)
    out_v = np.zeros((n_steps, max(len(ports), 1)), dtype)
    out_i = np.zeros((n_steps, max(len(ports), 1)), dtype)
    out_e = np.zeros(max(n_steps, 1), dtype)
    shapes = ((nx, ny), (nx, ny - 1), (nx - 1, ny))
    dft_full = [np.zeros((K,) + s, np.complex128) for s in shapes] if K and dft_monitors is None else [None] * 3
    mon_out = []
    mon_arr = (nt.DftMonitor * max(len(dft_monitors or ()), 1))()
    if dft_monitors is not None:
        for k, (comp, lo0, lo1, hi0, hi1) in enumerate(dft_monitors):
            t = np.zeros((K, hi0 - lo0, hi1 - lo1), np.complex128)
            mon_out.append(t)
            mon_arr[k].comp = comp
            mon_arr[k].lo[0], mon_arr[k].lo[1] = lo0, lo1
            mon_arr[k].hi[0], mon_arr[k].hi[1] = hi0, hi1
            mon_arr[k].out = t.ctypes.data

    prm = nt.TmParams()
    prm.nx, prm.ny, prm.npml, prm.n_steps = nx, ny, npml, n_steps
    prm.n_sources, prm.n_ports, prm.n_mx, prm.n_my = len(src), len(ports), len(mxi), len(myi)
    prm.n_probes, prm.n_freq, prm.record_energy = len(prb), K, int(record_energy)
    prm.dft_f64, prm.cw_sources = 1, int(cw is not None)
    prm.n_monitors = len(dft_monitors) if dft_monitors is not None else 0
    prm.dt, prm.dx, prm.dy, prm.dz, prm.mu0 = dt, grid.dx, grid.dy, onp.DZ, onp.MU0
    keep = []

    def col(a, c):
        v = np.ascontiguousarray(a[:, c], np.int32) if len(a) else np.zeros(1, np.int32)
        keep.append(v)
        return v.ctypes.data_as(nt.P_i32)

    pts = nt.TmPoints()
    for name, a in (("src", src), ("port", prt), ("mx", mxi), ("my", myi), ("probe", prb)):
        setattr(pts, f"{name}_i", col(a, 0))
        setattr(pts, f"{name}_j", col(a, 1))
    pts.monitors = mon_arr
    bufs = nt.TmBuffers()
    bufs.ca, bufs.cb, bufs.eps = _p(ca), _p(cb), _p(eps)
    for k, v in ik.items():
        setattr(bufs, k, _p(v))
    for k, v in tabs.items():
        setattr(bufs, k, _p(v))
    bufs.dt_mu, bufs.inv_dx, bufs.inv_dy = dt / onp.MU0, 1.0 / grid.dx, 1.0 / grid.dy
    sw, mw, yw = wav(source_current, len(src)), wav(mx_current, len(mxi)), wav(my_current, len(myi))
    bufs.cb_src, bufs.src_cur, bufs.cb_vs, bufs.port_vs = _p(cb_src if len(src) else np.zeros(1, dtype)), _p(sw), _p(cb_vs), _p(vs)
    bufs.mx_cur, bufs.my_cur = _p(mw), _p(yw)
    if cw is not None:
        env = np.ascontiguousarray(cw["env"], np.float64)
        ws_ = {k: (np.ascontiguousarray(np.asarray(cw[k]), np.complex128) if cw.get(k) is not None
                   else np.zeros(1, np.complex128)) for k in ("src_w", "mx_w", "my_w")}
        keep += [env, *ws_.values()]
        bufs.cw_env = _p(env)
        bufs.src_w, bufs.mx_w, bufs.my_w = _p(ws_["src_w"]), _p(ws_["mx_w"]), _p(ws_["my_w"])
    bufs.ph_e, bufs.ph_h = _p(ph_e), _p(ph_h)
    bufs.ez, bufs.hx, bufs.hy = _p(ez), _p(hx), _p(hy)
    bufs.out_probe, bufs.out_v, bufs.out_i, bufs.out_energy = _p(out_probe), _p(out_v), _p(out_i), _p(out_e)
    bufs.dft_ez, bufs.dft_hx, bufs.dft_hy = (_p(t) if t is not None else None for t in dft_full)
    fn = lib.oracle_tm_run_f64 if dtype == np.float64 else lib.oracle_tm_run_f32
    st = fn(ctypes.byref(prm), ctypes.byref(pts), ctypes.byref(bufs))
    if st != 0:
        raise RuntimeError(f"oracle C run failed: {st}")
    res = onp.SimResult(out_probe[:, :len(prb)], out_e[:n_steps] if record_energy else None, ez, hx, hy,
                        out_v[:, :len(ports)] if ports else None, out_i[:, :len(ports)] if ports else None,
                        *dft_full)
    return res, mon_out
