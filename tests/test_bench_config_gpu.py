"""Parity of the benchmarked configurations against the oracle, at full size.

* The 2D benchmark workload exactly as ``bench.py`` builds it: 1024^2 at
  1 mm, CPML 16, 8000 steps, the seeded 512^2 design mapped to sigma, two
  50-ohm ports (a 4-tone CW drive with a 300-step ramp and a passive load),
  K = 4 complex128 DFT monitors on the design region, the Poynting box and
  the ports. The forward run on the GPU is compared with the C oracle
  (``oracle/tm2d_ref.c``, itself pinned to the reference's own outputs by
  ``tests/test_golden_oracle.py``), in float64 (<= 1e-9 peak-normalised on
  phasors, port V/I, P_rad and S11) and float32 (<= 1e-4). The float32 run's
  error against the float64 oracle is printed for every output and held to
  1e-4 as well.
* Every kernel configuration on a 384 x 320 grid (the shared-memory tile
  kernels under each forced tile shape, the row march under several segment
  lengths), so that each interior and boundary template runs on interior
  work well away from the CPML, against the C oracle.
* The 3D patch workload (160 x 160 x 64 at 0.5 mm, CPML 10) shortened to 200
  steps (the numpy oracle takes about half a second per step at this size),
  against the numpy oracle: port V/I, region phasors and port impedance.
"""

import numpy as np
import pytest
import torch

import bench
from oracle import fdtd2d_np as onp
from oracle.tm2d_c import build as build_c
from oracle.tm2d_c import simulate_tm_c

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / (np.max(np.abs(b)) + 1e-300))


def _c2_inputs():
    w = bench.workload(0, bench.N_GRID, bench.N_STEPS)
    g = w["grid"]
    sigma = np.zeros((g.nx, g.ny))
    sigma[w["design"]] = w["sigma_d"]
    (a0, a1), (b0, b1) = [(s.start, s.stop) for s in w["design"]]
    mons = [(0, a0, b0, a1, b1)] + bench.monitors_for(w)
    return w, sigma, mons


def _full(mons, outs, shape_of, K):
    """Scatter monitor boxes into full (K, ...) phasor arrays."""
    full = {c: np.zeros((K,) + shape_of[c], np.complex128) for c in range(3)}
    for (c, lo0, lo1, hi0, hi1), o in zip(mons, outs):
        full[c][:, lo0:hi0, lo1:hi1] = np.asarray(o)
    return full


def _objectives(w, full, v, i):
    g = onp.Grid2D(w["grid"].nx, w["grid"].ny, w["grid"].dx, w["grid"].dy)
    p = onp.poynting_flux_box_2d(full[0], full[1], full[2], g, w["box"])
    vh, ih = onp.port_dft(v[:, 0], i[:, 0], g.dt, bench.FREQS)
    return p, onp.s11_power_wave(vh, ih, bench.RS)


def _run_pair(dtype):
    import gradenna_b200 as gb

    w, sigma, mons = _c2_inputs()
    g = w["grid"]
    K = len(bench.FREQS)
    og = onp.Grid2D(g.nx, g.ny, g.dx, g.dy)
    shape_of = {0: (g.nx, g.ny), 1: (g.nx, g.ny - 1), 2: (g.nx - 1, g.ny)}
    r = gb.simulate_tm(gb.Grid2D(g.nx, g.ny, g.dx, g.dy), sigma=sigma,
                       ports=(gb.Port(w["ports"][0], bench.RS, w["vs"]),
                              gb.Port(w["ports"][1], bench.RS, None)),
                       dft_freqs=bench.FREQS, dft_dtype=np.complex128,
                       cpml=gb.CPMLSpec(bench.NPML), dtype=dtype, device="cuda:0",
                       dft_monitors=mons)
    torch.cuda.synchronize()
    gpu = dict(v=r.port_v.cpu().numpy(), i=r.port_i.cpu().numpy(),
               mons=[m.cpu().numpy() for m in r.monitors])
    build_c()
    o, omons = simulate_tm_c(og, sigma=sigma,
                             ports=(onp.Port(w["ports"][0], bench.RS, w["vs"]),
                                    onp.Port(w["ports"][1], bench.RS, None)),
                             dft_freqs=bench.FREQS, cpml=onp.CPMLSpec(bench.NPML), dtype=dtype,
                             dft_monitors=mons)
    ora = dict(v=o.port_v, i=o.port_i, mons=omons)
    for d in (gpu, ora):
        d["full"] = _full(mons, d["mons"], shape_of, K)
        d["p_rad"], d["s11"] = _objectives(w, d["full"], d["v"], d["i"])
    return gpu, ora


def _errs(a, b):
    out = {"port_v": rel(a["v"], b["v"]), "port_i": rel(a["i"], b["i"]),
           "p_rad": rel(a["p_rad"], b["p_rad"]), "s11": rel(a["s11"], b["s11"])}
    for k, (x, y) in enumerate(zip(a["mons"], b["mons"])):
        out[f"mon{k}"] = rel(x, y)
    return out


_CACHE = {}


def _pair(dtype):
    key = np.dtype(dtype).name
    if key not in _CACHE:
        _CACHE[key] = _run_pair(dtype)
    return _CACHE[key]


def test_c2_float64_matches_oracle():
    gpu, ora = _pair(np.float64)
    e = _errs(gpu, ora)
    print("\nC2 float64 GPU vs float64 oracle:", {k: f"{v:.1e}" for k, v in e.items()})
    assert max(e.values()) <= 1e-9, e


def test_c2_float32_matches_oracle_and_float64():
    gpu, ora = _pair(np.float32)
    e = _errs(gpu, ora)
    print("\nC2 float32 GPU vs float32 oracle:", {k: f"{v:.1e}" for k, v in e.items()})
    assert max(e.values()) <= 1e-4, e
    _, ora64 = _pair(np.float64)
    e64 = _errs(gpu, ora64)
    print("C2 float32 GPU vs FLOAT64 oracle:", {k: f"{v:.1e}" for k, v in e64.items()})
    assert max(e64.values()) <= 1e-4, e64


KERNELS = [("tile", str(t)) for t in range(5)] + [("march", s) for s in ("8", "16", "40", "64")]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("kernel", KERNELS, ids=lambda k: f"{k[0]}{k[1]}")
def test_every_kernel_config_large(kernel, dtype, monkeypatch):
    import gradenna_b200 as gb

    kind, val = kernel
    monkeypatch.setenv("GDN_TM_KERNEL", kind)
    monkeypatch.setenv("GDN_TM_TILE" if kind == "tile" else "GDN_TM_SEG", val)
    rng = np.random.default_rng(3)
    nx, ny, n = 384, 320, 600
    og = onp.Grid2D(nx, ny, 1e-3, 1e-3)
    eps = 1.0 + 2.0 * rng.uniform(size=(nx, ny))
    sig = np.zeros((nx, ny))
    sig[100:300, 90:250] = onp.sigma_from_density(rng.uniform(size=(200, 160)))
    t = (np.arange(n) + 0.5) * og.dt
    src = onp.gaussian_derivative(t, 20 * og.dt, 6 * og.dt)
    vs = np.clip(np.arange(n) / 100.0, 0, 1) * np.sin(2 * np.pi * 6e9 * t)
    mons = [(0, 96, 64, 224, 192), (1, 40, 40, 41, 280), (2, 300, 33, 302, 200)]
    kw = dict(eps_r=eps.astype(dtype), sigma=sig.astype(dtype), source_ij=((190, 160), (70, 250)),
              source_current=np.stack([src, -0.5 * src], 1).astype(dtype),
              probe_ij=((128, 128), (191, 64), (64, 255), (383, 0)), dft_freqs=(5e9, 7e9),
              dft_monitors=mons)
    r = gb.simulate_tm(gb.Grid2D(nx, ny, 1e-3, 1e-3),
                       ports=(gb.Port((256, 192), 50.0, vs.astype(dtype)),
                              gb.Port((150, 60), 50.0, None)),
                       cpml=gb.CPMLSpec(14), dtype=dtype, dft_dtype=np.complex128,
                       device="cuda:0", **kw)
    torch.cuda.synchronize()
    build_c()
    o, omons = simulate_tm_c(og, ports=(onp.Port((256, 192), 50.0, vs.astype(dtype)),
                                        onp.Port((150, 60), 50.0, None)),
                             cpml=onp.CPMLSpec(14), dtype=dtype, **kw)
    tol = 1e-12 if dtype == np.float64 else 1e-5
    tol_f = 1e-12 if dtype == np.float64 else 1e-4
    assert rel(r.probe_ez.cpu(), o.probe_ez) <= tol
    assert rel(r.port_v.cpu(), o.port_v) <= tol
    assert rel(r.port_i.cpu(), o.port_i) <= tol
    for a, b in zip(r.monitors, omons):
        assert rel(a.cpu(), b) <= tol
    for nm in ("ez", "hx", "hy"):
        assert rel(getattr(r, nm).cpu(), getattr(o, nm)) <= tol_f, nm


def test_patch3d_short_matches_oracle():
    """The 3D patch workload's forward run (160 x 160 x 64, CPML 10, region
    DFT over the design sheet, the NTFF box faces and the port), 200 steps."""
    import gradenna_b200 as gb
    from gradenna_b200 import dft_region as dr
    from gradenna_b200.fdtd3d import port_impedance, simulate_3d
    from oracle import fdtd3d_np as o3

    n = 200
    w = bench.workload3d(0, n)
    g = w["grid"]
    sig = np.array(w["sig_bg"])
    sig[w["design"]] = w["sigma_d"]
    shapes = dr.full_field_shapes(g.nx, g.ny, g.nz)
    regions = dr.union_regions(
        dr.union_regions(dr.design_region_to_slabs(w["design"], shapes),
                         dr.port_regions(w["port"], shapes)),
        dr.ntff_box_regions(g, bench.P3_BOX, shapes))
    kw = dict(eps_r=w["eps_bg"], sigma=sig, port_ijk=w["port"], port_voltage=w["vs"],
              port_resistance=bench.RS, dft_freqs=bench.P3_FREQS)
    r = simulate_3d(g, cpml=gb.CPMLSpec(bench.P3_NPML), dft_regions=regions,
                    dft_dtype=np.complex128, dtype=np.float64, device="cuda:0", **kw)
    torch.cuda.synchronize()
    comps = ("ex", "ey", "ez", "hx", "hy", "hz")
    og = o3.Grid3D(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz)
    regs = {c: (tuple(s.lo), tuple(s.hi)) for c, s in zip(comps, regions) if s is not None}
    o = o3.simulate_3d(og, cpml=onp.CPMLSpec(bench.P3_NPML), dft_regions=regs,
                       dtype=np.float64, **kw)
    assert rel(r.port_v.cpu(), o.port_v) <= 1e-12
    assert rel(r.port_i.cpu(), o.port_i) <= 1e-12
    for c in comps:
        a = getattr(r.dft, c)
        if a is not None:
            assert rel(a.cpu(), o.dft[c]) <= 1e-12, c
    z = port_impedance(r, g, bench.P3_FREQS).cpu().numpy()
    zo = o3.port_impedance(o, og, bench.P3_FREQS)
    assert rel(z, zo) <= 1e-10
