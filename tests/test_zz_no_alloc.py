"""The allocation-free entry point gdn_tm_run_noalloc_f32.

Some callers cannot allocate device memory while they run the solver (they
own the GPU's memory through their own pool, or run in a loop where
allocator calls are not allowed). For them the library offers
gdn_tm_run_noalloc_f32, which keeps its scratch in a fixed 32 MiB array
inside the library. This test plays such a caller: it allocates every input
and output once, up front, then calls the entry point through the C ABI
twice in a row and checks both results against gdn_tm_run_f32 on the same
inputs (the tolerance of the float32 parity tests: 1e-5 peak-normalised),
and that the device's free memory does not move across the second call. A
larger case with a full-grid DFT runs with a shortened monitor ring. The
documented capacity is checked at its edges, and an oversized run is
refused with a clear error.

The file is named to run last, so a failing run with -x has already run
every other test; it also passes on its own in a fresh process.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _case(dev, nx=70, ny=53, n_steps=300):
    """A prepared 2D TM run: CPML, a Jz source, a driven port and a passive
    port, probes, a full-grid complex64 DFT at two frequencies."""
    from gradenna_b200 import _native
    from gradenna_b200.constants import EPS0, MU0
    from gradenna_b200.cpml import CPMLSpec, axis_coefficients, slab_tables
    from gradenna_b200.grid import Grid2D

    g = Grid2D(nx, ny, 2e-3, 2e-3)
    npml = 8
    dt = g.dt
    f32 = np.float32
    t = (np.arange(n_steps) + 0.5) * dt
    u = (t - 20 * dt) / (6 * dt)
    wave = (-u * np.exp(0.5 * (1.0 - u**2))).astype(f32)
    src = np.array([[3 * nx // 7, 2 * ny // 5]], np.int32)
    ports = np.array([[4 * nx // 7, 4 * ny // 7], [5 * nx // 14, 2 * ny // 3]], np.int32)
    rs = np.array([50.0, 75.0])
    probes = np.array([[nx // 7, ny // 4], [5 * nx // 7, 3 * ny // 4], [0, 0]], np.int32)
    freqs = np.array([3e9, 5e9])

    eps = np.full((nx, ny), EPS0, f32)
    sig = np.zeros((nx, ny), f32)
    np.add.at(sig, (ports[:, 0], ports[:, 1]), (1.0 / (rs * g.dx * g.dy)).astype(f32))
    hl = sig * f32(dt) / (f32(2.0) * eps)
    ca = ((f32(1.0) - hl) / (f32(1.0) + hl)).astype(f32)
    cb = ((f32(dt) / eps) / (f32(1.0) + hl)).astype(f32)
    cb_src = (cb[src[:, 0], src[:, 1]] / (g.dx * g.dy)).astype(f32)
    cb_vs = (cb[ports[:, 0], ports[:, 1]] / (rs * g.dx * g.dy)).astype(f32)
    port_vs = np.stack([0.5 * wave, np.zeros_like(wave)], 1).astype(f32)
    spec = CPMLSpec(npml)
    ax = {k: axis_coefficients(n, d, dt, spec, half=h, dtype=f32)
          for k, (n, d, h) in {"xe": (nx, g.dx, False), "xh": (nx, g.dx, True),
                               "ye": (ny, g.dy, False), "yh": (ny, g.dy, True)}.items()}
    nn = np.arange(n_steps, dtype=np.float64)
    ph_e = np.exp(-2j * np.pi * np.outer(nn + 1.0, freqs) * dt)
    ph_h = np.exp(-2j * np.pi * np.outer(nn + 0.5, freqs) * dt)

    keep = {}

    def dv(name, a):
        keep[name] = torch.as_tensor(np.ascontiguousarray(a), device=dev)
        return keep[name].data_ptr()

    b = _native.TmBuffers()
    b.ca, b.cb, b.eps = dv("ca", ca), dv("cb", cb), dv("eps", eps)
    b.inv_kx_e, b.inv_ky_e = dv("ikxe", ax["xe"].inv_kappa[1:-1]), dv("ikye", ax["ye"].inv_kappa[1:-1])
    b.inv_kx_h, b.inv_ky_h = dv("ikxh", ax["xh"].inv_kappa), dv("ikyh", ax["yh"].inv_kappa)
    for key, (bb, cc) in {"ezx": (ax["xe"].b[1:-1], ax["xe"].c[1:-1]),
                          "ezy": (ax["ye"].b[1:-1], ax["ye"].c[1:-1]),
                          "hyx": (ax["xh"].b, ax["xh"].c), "hxy": (ax["yh"].b, ax["yh"].c)}.items():
        for nm, arr in zip(("b_%s_lo", "c_%s_lo", "b_%s_hi", "c_%s_hi"), slab_tables(bb, cc, npml)):
            setattr(b, nm % key, dv(nm % key, arr))
    b.dt_mu, b.inv_dx, b.inv_dy = dt / MU0, 1.0 / g.dx, 1.0 / g.dy
    b.cb_src, b.src_cur = dv("cb_src", cb_src), dv("src_cur", wave[:, None])
    b.cb_vs, b.port_vs = dv("cb_vs", cb_vs), dv("port_vs", port_vs)
    b.ph_e, b.ph_h = dv("ph_e", ph_e), dv("ph_h", ph_h)

    p = _native.TmParams()
    p.nx, p.ny, p.npml, p.n_steps = nx, ny, npml, n_steps
    p.n_sources, p.n_ports, p.n_probes, p.n_freq = 1, 2, 3, 2
    p.dt, p.dx, p.dy, p.dz, p.mu0 = dt, g.dx, g.dy, 1.0, MU0

    cols = {}

    def col(name, a, c):
        cols[(name, c)] = np.ascontiguousarray(a[:, c], np.int32)
        return cols[(name, c)].ctypes.data_as(_native.P_i32)

    pts = _native.TmPoints()
    pts.src_i, pts.src_j = col("s", src, 0), col("s", src, 1)
    pts.port_i, pts.port_j = col("p", ports, 0), col("p", ports, 1)
    pts.probe_i, pts.probe_j = col("q", probes, 0), col("q", probes, 1)
    return p, pts, b, (keep, cols), (nx, ny, n_steps)


def _outputs(b, dims, dev):
    nx, ny, n_steps = dims
    out = {
        "ez": torch.empty((nx, ny), device=dev), "hx": torch.empty((nx, ny - 1), device=dev),
        "hy": torch.empty((nx - 1, ny), device=dev),
        "probe": torch.empty((n_steps, 3), device=dev), "v": torch.empty((n_steps, 2), device=dev),
        "i": torch.empty((n_steps, 2), device=dev),
        "dft_ez": torch.empty((2, nx, ny), dtype=torch.complex64, device=dev),
        "dft_hx": torch.empty((2, nx, ny - 1), dtype=torch.complex64, device=dev),
        "dft_hy": torch.empty((2, nx - 1, ny), dtype=torch.complex64, device=dev),
    }
    _bind(b, out)
    return out


def _bind(b, out):
    """Point the buffer struct at one set of outputs (no allocation)."""
    b.ez, b.hx, b.hy = out["ez"].data_ptr(), out["hx"].data_ptr(), out["hy"].data_ptr()
    b.out_probe, b.out_v, b.out_i = out["probe"].data_ptr(), out["v"].data_ptr(), out["i"].data_ptr()
    b.dft_ez, b.dft_hx, b.dft_hy = (out[k].data_ptr() for k in ("dft_ez", "dft_hx", "dft_hy"))


def _rel(a, b):
    return float((a - b).abs().max() / (b.abs().max() + 1e-30))


def _noalloc(lib):
    fn = lib.gdn_tm_run_noalloc_f32
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(_native_mod().TmParams), ctypes.POINTER(_native_mod().TmPoints),
                   ctypes.POINTER(_native_mod().TmBuffers), ctypes.c_void_p]
    return fn


def _native_mod():
    from gradenna_b200 import _native

    return _native


def _compare_twice(nx, ny, n_steps):
    """The regular entry point once, then the allocation-free one twice in a
    row into separate outputs; every output of both calls must match, and
    the second call must leave the device's free memory unchanged."""
    _native = _native_mod()
    lib = _native.load()
    fn = _noalloc(lib)
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    p, pts, b, _keep, dims = _case(dev, nx, ny, n_steps)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

    want = _outputs(b, dims, dev)
    b.workspace, b.workspace_bytes = None, 0  # regular path: library-owned scratch
    _native.check(lib.gdn_tm_run_f32(ctypes.byref(p), ctypes.byref(pts), ctypes.byref(b), stream))
    torch.cuda.synchronize()
    assert float(want["dft_ez"].abs().max()) > 0.0 and float(want["v"].abs().max()) > 0.0

    outs = [_outputs(b, dims, dev) for _ in range(2)]  # allocated before the calls
    free = []
    for got in outs:  # the second call must not see the first call's state
        _bind(b, got)
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info(dev)[0])
        _native.check(fn(ctypes.byref(p), ctypes.byref(pts), ctypes.byref(b), stream))
        torch.cuda.synchronize()
        for k in want:
            assert _rel(got[k], want[k]) <= 1e-5, f"{k}: {_rel(got[k], want[k]):.2e}"
    free.append(torch.cuda.mem_get_info(dev)[0])
    # The first call may load the library's module on this device (lazy
    # loading); from then on a call allocates nothing on the device.
    assert free[2] == free[1], f"device free memory changed by {free[1] - free[2]} bytes"


def test_noalloc_matches_regular_entry_point_twice():
    _compare_twice(70, 53, 300)


def test_noalloc_full_grid_dft_with_a_shortened_ring():
    """At 420 x 420 with a full-grid DFT the monitor ring of 32 steps does not
    fit the fixed scratch; the entry point shortens the ring (and folds the
    DFT more often) and must still give the regular entry point's result."""
    _compare_twice(420, 420, 120)


def _status(nx, ny, dft):
    _native = _native_mod()
    lib = _native.load()
    fn = _noalloc(lib)
    dev = torch.device("cuda", 0)
    p, pts, b, _keep, dims = _case(dev, nx, ny, 8)
    _outputs(b, dims, dev)
    if not dft:
        p.n_freq = 0
    st = fn(ctypes.byref(p), ctypes.byref(pts), ctypes.byref(b), None)
    torch.cuda.synchronize()
    return st, lib.gdn_last_error().decode()


def test_noalloc_capacity_matches_the_documented_limits():
    """The header states about 670 x 670 cells without a DFT and about
    500 x 500 with a full-grid DFT (float32, default segment length)."""
    assert _status(664, 664, dft=False)[0] == 0
    assert _status(500, 500, dft=True)[0] == 0
    for n, dft in ((704, False), (528, True)):
        st, msg = _status(n, n, dft)
        assert st == 1 and "static scratch" in msg, (n, dft, st, msg)


def test_noalloc_rejects_runs_beyond_its_capacity():
    _native = _native_mod()
    lib = _native.load()
    fn = _noalloc(lib)
    p, pts, b, _keep, dims = _case(torch.device("cuda", 0))
    _outputs(b, dims, torch.device("cuda", 0))
    p.nx = p.ny = 4096  # ~200 MiB of scratch; checked before any device work
    p.n_probes, p.n_sources, p.n_ports = 0, 0, 0
    st = fn(ctypes.byref(p), ctypes.byref(pts), ctypes.byref(b), None)
    assert st == 1
    msg = lib.gdn_last_error().decode()
    assert "static scratch" in msg and "bytes" in msg
