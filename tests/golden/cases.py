"""Golden-vector cases: seeded inputs and one runner per implementation.

Every case is a plain description (grid, materials, drives, monitors) built
from seeded numpy only, so that the same inputs can be handed to

  * the reference's own ``simulate_tm`` / ``simulate_3d`` and objective
    functions (run on the CPU through ``tests/golden/refload.py`` by
    ``make_golden.py``, which writes ``tests/golden/*.npz``),
  * the numpy oracle (``oracle/fdtd2d_np.py``, ``oracle/fdtd3d_np.py``,
    ``oracle/ntff_np.py``), checked against the fixtures on the CPU,
  * the CUDA library (``gradenna_b200``), checked against the fixtures on the
    GPU.

A fixture also stores a digest of its inputs, so a test fails loudly if the
inputs rebuilt here ever drift from the ones the fixture was made with.

Case sources: the reference's native-vs-XLA parity cases
(tests/test_native.py:66-153, tests/test_native3d.py:69-153), the README's
radiated-power example (README.md:24-39: 140^2 at 2 mm, 3500 steps, one
50-ohm port, 2.45 GHz, Poynting box (20, 120, 20, 120)), and seeded cases
that add metal-level conductivity, CW drives, magnetic currents, many tiles
and region-limited 3D monitors.
"""

from __future__ import annotations

import hashlib
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

F64, F32 = np.float64, np.float32


# ---------------------------------------------------------------------------
# Input helpers (restated here so the cases need nothing but numpy)
# ---------------------------------------------------------------------------

def gaussian_derivative(t, t0, tau):
    """sources.py: -(t - t0)/tau * exp(-((t - t0)/tau)^2 / 2)."""
    u = (t - t0) / tau
    return -u * np.exp(-0.5 * u * u)


def band_pulse(f_min, f_max, t):
    """sparams.py:121-139 (gaussian_pulse_for_band) evaluated at t."""
    f0, fc = 0.5 * (f_min + f_max), 0.5 * (f_max - f_min)
    sigma = 3.0 / (2.0 * math.sqrt(2.0) * math.pi * fc)
    t0 = 9.0 / (2.0 * math.pi * fc)
    u = t - t0
    return np.cos(2.0 * np.pi * f0 * u) * np.exp(-(u ** 2) / (2.0 * sigma ** 2))


def sigma_from_density(rho, sigma_min=1e-4, sigma_max=1e5):
    """materials.py:28-51."""
    lo, hi = math.log10(sigma_min), math.log10(sigma_max)
    return 10.0 ** ((hi - lo) * np.asarray(rho, np.float64) + lo)


def courant_dt(dx, dy, dz=None):
    """grid.py:33-36, 64-69 (Courant number 0.99)."""
    c0 = 299_792_458.0
    s = 1 / dx ** 2 + 1 / dy ** 2 + (0.0 if dz is None else 1 / dz ** 2)
    return 0.99 / (c0 * math.sqrt(s))


def _gauss(n, dt, dtype):
    t = (np.arange(n) + 0.5) * dt
    return np.asarray(gaussian_derivative(t, 20 * dt, 6 * dt), dtype)


def _smooth_noise(rng, shape, passes=3):
    a = rng.uniform(0.0, 1.0, shape)
    for _ in range(passes):
        a = 0.25 * (np.roll(a, 1, 0) + np.roll(a, -1, 0) + np.roll(a, 1, 1) + np.roll(a, -1, 1))
    a = (a - a.min()) / (a.max() - a.min())
    return a


def _cw(n, dt, freqs, amps, ramp, dtype):
    t = (np.arange(n) + 0.5) * dt
    env = np.clip(np.arange(n) / float(ramp), 0.0, 1.0)
    s = sum(a * np.sin(2 * np.pi * f * t) for f, a in zip(freqs, amps))
    return np.asarray(env * s, dtype)


# ---------------------------------------------------------------------------
# 2D TM cases
# ---------------------------------------------------------------------------
# A case: dict(name, kind="tm", grid=(nx, ny, dx, dy), dtype, npml, kw={...},
# ports=[(ij, R, voltage or None)], box=(il, ir, jb, jt) or None,
# sfreqs=frequencies for the port S11 or (), store=outputs kept).
# Final-field snapshots of the long float32 runs are not kept: after
# thousands of steps the snapshot is the decayed tail of the pulse, so its own
# peak is far below the rounding noise accumulated while the pulse was
# strong, and a peak-normalised comparison of it measures nothing (the
# reference holds final fields of its 400-500-step cases only).

def tm_cases():
    out = []
    for dt_ in (F64, F32):
        sfx = "f64" if dt_ is F64 else "f32"
        # tests/test_native.py:66-84 (test_basic_cpml)
        g = (48, 52, 1e-3, 1e-3)
        src = _gauss(400, courant_dt(1e-3, 1e-3), dt_)
        out.append(dict(name=f"tm_basic_cpml_{sfx}", kind="tm", grid=g, dtype=dt_, npml=8,
                        kw=dict(source_ij=(24, 26), source_current=src,
                                probe_ij=((12, 14), (30, 34)), record_energy=True),
                        ports=[], box=None, sfreqs=()))
        # tests/test_native.py:87-119 (test_multi_source_ports_dft)
        g = (44, 40, 2e-3, 2e-3)
        base = _gauss(500, courant_dt(2e-3, 2e-3), dt_)
        srcs = np.stack([base, 0.3 * base], axis=1).astype(dt_)
        vs = (0.5 * _gauss(500, courant_dt(2e-3, 2e-3), dt_)).astype(dt_)
        out.append(dict(name=f"tm_ports_dft_{sfx}", kind="tm", grid=g, dtype=dt_, npml=8,
                        kw=dict(source_ij=((15, 18), (25, 22)), source_current=srcs,
                                probe_ij=((10, 12), (30, 30)), dft_freqs=(3e9, 5e9),
                                dft_dtype=np.complex128),
                        ports=[((20, 20), 50.0, vs), ((22, 24), 75.0, None)], box=(8, 33, 8, 30),
                        sfreqs=(3e9, 5e9)))
    # tests/test_native.py:122-145 (test_magnetic_current_sources), float64
    g = (40, 40, 2e-3, 2e-3)
    base = _gauss(300, courant_dt(2e-3, 2e-3), F64)
    out.append(dict(name="tm_magnetic_f64", kind="tm", grid=g, dtype=F64, npml=8,
                    kw=dict(source_ij=(20, 20), source_current=base,
                            mx_ij=((18, 20), (22, 18)),
                            mx_current=np.stack([base, 0.5 * base], axis=1),
                            my_ij=(20, 22), my_current=0.7 * base, probe_ij=((15, 15),),
                            dft_freqs=(4e9,), dft_dtype=np.complex128),
                    ports=[], box=None, sfreqs=()))
    # tests/test_native.py:148-160 (test_no_pml_pec_box), float64
    g = (36, 36, 1e-3, 1e-3)
    out.append(dict(name="tm_pec_f64", kind="tm", grid=g, dtype=F64, npml=0,
                    kw=dict(source_ij=(18, 18), source_current=_gauss(250, courant_dt(1e-3, 1e-3), F64),
                            probe_ij=((10, 10),)),
                    ports=[], box=None, sfreqs=()))
    # README.md:24-39: the radiated-power example (forward part), float64 and
    # float32 fields with complex128 phasors.
    for dt_ in (F64, F32):
        sfx = "f64" if dt_ is F64 else "f32"
        dt = courant_dt(2e-3, 2e-3)
        v = np.asarray(band_pulse(2.0e9, 3.0e9, (np.arange(3500) + 0.5) * dt), dt_)
        sig = np.zeros((140, 140))
        sig[44:96, 60:112] = sigma_from_density(0.5 * np.ones((52, 52)))
        out.append(dict(name=f"tm_readme_{sfx}", kind="tm", grid=(140, 140, 2e-3, 2e-3), dtype=dt_,
                        npml=10, kw=dict(sigma=sig.astype(dt_), dft_freqs=(2.45e9,),
                                         dft_dtype=np.complex128),
                        ports=[((70, 55), 50.0, v)], box=(20, 120, 20, 120), sfreqs=(2.45e9,),
                        store=("probe_ez", "port_v", "port_i", "dft_ez", "p_rad", "s11")
                        + (("ez",) if dt_ is F64 else ())))
    # Heterogeneous medium: eps_r in [1, 4], a metal/air design from a
    # projected smooth density (up to 1e5 S/m), a CW two-tone port drive with
    # a ramp, a passive port, a Jz line source, Mx/My currents, three DFT
    # frequencies. float32 uses the default complex64 phasors.
    for dt_ in (F64, F32):
        sfx = "f64" if dt_ is F64 else "f32"
        rng = np.random.default_rng(7)
        nx, ny, n = 72, 64, 700
        dt = courant_dt(1.5e-3, 1.5e-3)
        eps = 1.0 + 3.0 * _smooth_noise(rng, (nx, ny))
        rho = _smooth_noise(rng, (24, 20))
        rho = 1.0 / (1.0 + np.exp(-16.0 * (rho - 0.5)))
        sig = np.zeros((nx, ny))
        sig[30:54, 24:44] = sigma_from_density(rho)
        vs = _cw(n, dt, (3.0e9, 4.5e9), (1.0, 0.6), 150, dt_)
        jz = (0.2 * _gauss(n, dt, F64)).astype(dt_)
        mx = (0.1 * _gauss(n, dt, F64)).astype(dt_)
        my = (-0.15 * _gauss(n, dt, F64)).astype(dt_)
        kw = dict(eps_r=eps.astype(dt_), sigma=sig.astype(dt_), source_ij=(40, 14),
                  source_current=jz, mx_ij=(20, 30), mx_current=mx, my_ij=(50, 50), my_current=my,
                  probe_ij=((15, 15), (60, 40), (36, 33)), dft_freqs=(3.0e9, 3.7e9, 4.5e9))
        if dt_ is F64:
            kw["dft_dtype"] = np.complex128
        out.append(dict(name=f"tm_media_cw_{sfx}", kind="tm", grid=(nx, ny, 1.5e-3, 1.5e-3),
                        dtype=dt_, npml=8, kw=kw,
                        ports=[((26, 20), 50.0, vs), ((58, 46), 50.0, None)],
                        box=(12, 58, 11, 51), sfreqs=(3.0e9, 4.5e9),
                        store=("probe_ez", "port_v", "port_i", "p_rad", "s11", "dft_ez",
                               "dft_hx_1") + (("ez", "hy") if dt_ is F64 else ())))
    # Several 64 x 64 tiles with ragged edges: 150 x 210, CPML 12, two ports,
    # three sources, probes on tile seams, two DFT frequencies.
    for dt_ in (F64, F32):
        sfx = "f64" if dt_ is F64 else "f32"
        nx, ny, n = 150, 210, 320
        dt = courant_dt(1e-3, 1e-3)
        base = _gauss(n, dt, F64)
        srcs = np.stack([base, -0.5 * base, 0.25 * base], axis=1).astype(dt_)
        vs = _cw(n, dt, (9e9,), (1.0,), 60, dt_)
        out.append(dict(name=f"tm_tiles_{sfx}", kind="tm", grid=(nx, ny, 1e-3, 1e-3), dtype=dt_,
                        npml=12,
                        kw=dict(source_ij=((64, 64), (100, 127), (40, 190)), source_current=srcs,
                                probe_ij=((63, 63), (64, 128), (127, 64), (20, 20), (140, 200)),
                                dft_freqs=(8e9, 11e9), dft_dtype=np.complex128),
                        ports=[((75, 100), 50.0, vs), ((128, 150), 50.0, None)],
                        box=(20, 129, 20, 189), sfreqs=(8e9, 11e9),
                        store=("probe_ez", "port_v", "port_i", "p_rad", "s11", "dft_ez_0")
                        + (("ez",) if dt_ is F64 else ())))
    return out


def run_tm(api, case, *, lib=False, oracle=False, device=None):
    """Run a 2D case through ``api`` (a namespace with Grid2D, CPMLSpec, Port,
    simulate_tm, poynting_flux_box_2d, port_dft, s11_power_wave) and return
    every output as numpy arrays (complex phasors as numpy complex)."""
    nx, ny, dx, dy = case["grid"]
    g = api.Grid2D(nx, ny, dx, dy)
    ports = [api.Port(ij, r, v) for ij, r, v in case["ports"]]
    kw = dict(case["kw"])
    extra = {}
    if lib:
        extra = dict(dtype=case["dtype"], device=device)
    elif oracle:
        extra = dict(dtype=case["dtype"])
    r = api.simulate_tm(g, ports=ports, cpml=api.CPMLSpec(case["npml"]), **kw, **extra)
    out = {}
    for k in ("probe_ez", "energy", "ez", "hx", "hy", "port_v", "port_i", "dft_ez", "dft_hx",
              "dft_hy"):
        v = getattr(r, k, None)
        if v is not None:
            out[k] = _np(v)
    if case["box"] is not None and "dft_ez" in out:
        p = api.poynting_flux_box_2d(r.dft_ez, r.dft_hx, r.dft_hy, g, case["box"])
        out["p_rad"] = _np(p)
    if case["sfreqs"] and "port_v" in out:
        vh, ih = api.port_dft(r.port_v[:, 0], r.port_i[:, 0], g.dt, case["sfreqs"])
        out["s11"] = _np(api.s11_power_wave(vh, ih, 50.0))
    return out


# ---------------------------------------------------------------------------
# 3D Yee cases
# ---------------------------------------------------------------------------

def yee_cases():
    out = []
    for dt_ in (F64, F32):
        sfx = "f64" if dt_ is F64 else "f32"
        # tests/test_native3d.py (CPML, Jz + Jx sources, probes, energy)
        g = (26, 28, 24, 1e-3, 1.1e-3, 0.9e-3)
        src = _gauss(200, courant_dt(1e-3, 1.1e-3, 0.9e-3), dt_)
        out.append(dict(name=f"yee_basic_{sfx}", kind="yee", grid=g, dtype=dt_, npml=7,
                        kw=dict(source_ijk=(13, 14, 12), source_current=src,
                                source_x_ijk=(9, 17, 15), source_x_current=(0.6 * src).astype(dt_),
                                probe_ijk=((10, 12, 8), (18, 16, 14)), record_energy=True),
                        regions=None, ntff=None, store=("probe_ez", "energy", "ez", "hx", "ey")))
        # every current channel plus the lumped port and a 2-frequency DFT
        g = (30, 28, 26, 1e-3, 1.1e-3, 0.9e-3)
        base = _gauss(240, courant_dt(1e-3, 1.1e-3, 0.9e-3), dt_)
        out.append(dict(name=f"yee_port_dft_{sfx}", kind="yee", grid=g, dtype=dt_, npml=6,
                        kw=dict(source_ijk=(10, 12, 9), source_current=base,
                                source_x_ijk=(14, 8, 15), source_x_current=(0.7 * base).astype(dt_),
                                source_y_ijk=(16, 15, 11), source_y_current=(0.4 * base).astype(dt_),
                                mx_ijk=(12, 10, 13), mx_current=(0.3 * base).astype(dt_),
                                my_ijk=(15, 14, 12), my_current=(0.2 * base).astype(dt_),
                                mz_ijk=(11, 16, 10), mz_current=(0.15 * base).astype(dt_),
                                port_ijk=(18, 18, 14), port_voltage=(0.5 * base).astype(dt_),
                                port_resistance=50.0, probe_ijk=((9, 9, 9), (20, 19, 16)),
                                dft_freqs=(20e9, 35e9), dft_dtype=np.complex128),
                        regions=None, ntff=(6 + 2, (0.0, 0.6, 1.2), (0.0, 1.0, 2.5)),
                        store=("probe_ez", "port_v", "port_i", "zin", "e_theta", "e_phi",
                               "directivity", "ez", "hz", "dft_ez_0", "dft_hx_1")))
    # A small patch: PEC-like ground sheet, 3-cell eps_r 4.4 substrate, a
    # seeded metal/air design sheet, a vertical port across the substrate;
    # region-limited DFT (design sheet + NTFF box faces + port), S11 and the
    # NTFF directivity at broadside. float64.
    rng = np.random.default_rng(11)
    nx, ny, nz, d, npml, n = 36, 34, 22, 1.0e-3, 6, 420
    eps = np.ones((nx, ny, nz))
    eps[:, :, 8:11] = 4.4
    sig = np.zeros((nx, ny, nz))
    sig[:, :, 8] = 1.0e7
    rho = _smooth_noise(rng, (14, 14))
    sig[11:25, 10:24, 11] = sigma_from_density(1.0 / (1.0 + np.exp(-12.0 * (rho - 0.45))))
    dtt = courant_dt(d, d, d)
    v = 0.8 * band_pulse(10e9, 30e9, (np.arange(n) + 0.5) * dtt)
    out.append(dict(name="yee_patch_regions_f64", kind="yee", grid=(nx, ny, nz, d, d, d),
                    dtype=F64, npml=npml,
                    kw=dict(eps_r=eps, sigma=sig, port_ijk=(18, 13, 10), port_voltage=v,
                            port_resistance=50.0, probe_ijk=((18, 17, 12),),
                            dft_freqs=(15e9, 20e9, 25e9), dft_dtype=np.complex128),
                    regions=dict(design=(slice(11, 25), slice(10, 24), slice(11, 12)),
                                 port=(18, 13, 10), box_margin=npml + 2),
                    ntff=(npml + 2, (0.0, 0.5), (0.0, 1.3)),
                    store=("probe_ez", "port_v", "port_i", "zin", "e_theta", "e_phi",
                           "directivity", "ez", "dft_ex", "dft_ey", "dft_ez", "dft_hz")))
    return out


def run_yee(api, case, *, lib=False, oracle=False, device=None):
    """Run a 3D case through ``api`` (namespace with Grid3D, CPMLSpec,
    simulate_3d, port_impedance, ntff_3d, and for region cases
    design_region_to_slabs, port_regions, ntff_box_regions, union_regions,
    full_field_shapes, scatter_full)."""
    nx, ny, nz, dx, dy, dz = case["grid"]
    g = api.Grid3D(nx, ny, nz, dx, dy, dz)
    kw = dict(case["kw"])
    extra = {}
    if lib:
        extra = dict(dtype=case["dtype"], device=device)
    elif oracle:
        extra = dict(dtype=case["dtype"])
    reg = case["regions"]
    if reg is not None:
        shapes = api.full_field_shapes(nx, ny, nz)
        regions = api.union_regions(
            api.union_regions(api.design_region_to_slabs(reg["design"], shapes),
                              api.port_regions(reg["port"], shapes)),
            api.ntff_box_regions(g, reg["box_margin"], shapes))
        kw["dft_regions"] = regions
    r = api.simulate_3d(g, cpml=api.CPMLSpec(case["npml"]), **kw, **extra)
    out = {}
    for k in ("probe_ez", "port_v", "port_i", "energy", "ex", "ey", "ez", "hx", "hy", "hz"):
        v = getattr(r, k, None)
        if v is not None:
            out[k] = _np(v)
    mon = r.dft
    if mon is not None:
        if reg is not None:
            for c in ("ex", "ey", "ez", "hx", "hy", "hz"):
                s = getattr(mon, c)
                if s is not None:
                    out[f"dft_{c}"] = _np(s)
            mon = api.scatter_full(mon, api.full_field_shapes(nx, ny, nz))
        else:
            for c in ("ex", "ey", "ez", "hx", "hy", "hz"):
                out[f"dft_{c}"] = _np(getattr(mon, c))
    if "port_v" in out and kw.get("dft_freqs"):
        out["zin"] = _np(api.port_impedance(r, g, kw["dft_freqs"]))
    if case["ntff"] is not None and mon is not None:
        m, th, ph = case["ntff"]
        et, ep = _ntff_pair(api.ntff_3d(mon, g, m, kw["dft_freqs"], th, ph))
        out["e_theta"], out["e_phi"] = et, ep
    return out


def _ntff_pair(res):
    if isinstance(res, tuple):
        return _np(res[0]), _np(res[1])
    a = _np(res)
    return a[..., 0], a[..., 1]


# ---------------------------------------------------------------------------
# Design transform and CPML tables
# ---------------------------------------------------------------------------

def design_cases():
    rng = np.random.default_rng(5)
    out = []
    for shape, radius, beta in (((40, 52), 3.0, 8.0), ((40, 52), 6.0, 64.0), ((33, 29), 1.0, 8.0),
                                ((104, 104), 6.0, 8.0), ((31, 47), 2.5, 32.0)):
        theta = rng.normal(0.0, 1.5, shape)
        out.append(dict(name=f"design_{shape[0]}x{shape[1]}_r{radius}_b{beta}", theta=theta,
                        radius=radius, beta=beta, eta=0.5))
    return out


def cpml_cases():
    return [dict(n=48, delta=1e-3, dt=courant_dt(1e-3, 1e-3), thickness=8),
            dict(n=140, delta=2e-3, dt=courant_dt(2e-3, 2e-3), thickness=10),
            dict(n=1024, delta=1e-3, dt=courant_dt(1e-3, 1e-3), thickness=16),
            dict(n=36, delta=1e-3, dt=courant_dt(1e-3, 1e-3, 1e-3), thickness=6)]


# ---------------------------------------------------------------------------
# Fixture I/O
# ---------------------------------------------------------------------------

def _np(x):
    try:
        import torch

        if isinstance(x, torch.Tensor):
            return x.detach().cpu().numpy()
    except ImportError:  # pragma: no cover
        pass
    return np.asarray(x)


def digest(obj) -> str:
    """SHA-256 over every array and scalar of a case description."""
    h = hashlib.sha256()

    def feed(v):
        if isinstance(v, dict):
            for k in sorted(v):
                h.update(str(k).encode())
                feed(v[k])
        elif isinstance(v, (list, tuple)):
            h.update(b"[")
            for x in v:
                feed(x)
            h.update(b"]")
        elif isinstance(v, np.ndarray):
            h.update(str(v.dtype).encode() + str(v.shape).encode())
            h.update(np.ascontiguousarray(v).tobytes())
        elif isinstance(v, slice):
            h.update(repr((v.start, v.stop, v.step)).encode())
        elif isinstance(v, type):
            h.update(v.__name__.encode())
        else:
            h.update(repr(v).encode())

    feed(obj)
    return h.hexdigest()


def fixture_path(name: str) -> str:
    return os.path.join(HERE, f"{name}.npz")


def select(case, outputs: dict) -> dict:
    """The outputs a fixture keeps: every output, or those named in the
    case's ``store`` list; ``name_k`` keeps frequency k of a phasor array."""
    keep = case.get("store") if isinstance(case, dict) else None
    if not keep:
        return dict(outputs)
    sel = {}
    for k in keep:
        base, _, idx = k.rpartition("_")
        if k in outputs:
            sel[k] = outputs[k]
        elif base in outputs and idx.isdigit():
            sel[k] = outputs[base][int(idx)]
    return sel


def save(name: str, case, outputs: dict):
    np.savez_compressed(fixture_path(name), __digest__=np.array(digest(case)),
                        **{k: np.asarray(v) for k, v in select(case, outputs).items()})


def load(name: str, case=None) -> dict:
    with np.load(fixture_path(name)) as z:
        d = {k: z[k] for k in z.files}
    if case is not None and str(d["__digest__"]) != digest(case):
        raise AssertionError(f"golden fixture {name}: inputs differ from the ones it was made with")
    d.pop("__digest__", None)
    return d


def rel(a, b) -> float:
    """Peak-normalised max error of a against the golden b."""
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        raise AssertionError(f"shape {a.shape} != golden {b.shape}")
    if b.size == 0:
        return 0.0
    return float(np.max(np.abs(a - b)) / (np.max(np.abs(b)) + 1e-300))
