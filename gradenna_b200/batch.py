"""Batched uneven 2D populations: many simulate_tm problems in shared launches.

A topology-optimisation population or a multiband sweep is many small,
uneven 2D problems. Run one at a time they leave most of the 148 SMs idle;
``simulate_tm_batch`` hands them to ``gdn_tm_run_batch_f32``, which advances
all of them with one launch per block of time steps and tile class (the work
list holds (problem, tile) pairs of the problems still running). Each
problem keeps its own grid, CPML, sources, ports, monitors and step count,
and its results equal a separate ``simulate_tm`` call with the same tile
configuration.

``autotune_tm_batch`` picks the tile shape and time-block depth (TB) by
timing a short prefix of the batch with every configuration, and caches the
choice per population signature. ``freq_adjoint_gradient_batch`` is the
frequency-domain adjoint gradient (gradenna_b200.freq_adjoint) of every
problem, with both FDTD passes batched.

No reference counterpart: the reference runs one simulation per call
(src/gradenna/fdtd2d.py:181, freq_adjoint.py:355).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from gradenna_b200 import _native
from gradenna_b200.fdtd2d import Port, _flatten, _prepare_tm

__all__ = ["N_CONFIGS", "simulate_tm_batch", "autotune_tm_batch", "freq_adjoint_gradient_batch"]

#: Tile configurations a batched run can use (GDN_TM_NCFG): 0 = 64x64
#: tiles / 4-step blocks, 1 = 32x64 / 4, 2 = 16x32 / 4, 3 = 64x64 / 2,
#: 4 = 32x64 / 2.
N_CONFIGS = 5


class TmProblem(ctypes.Structure):
    _fields_ = [("params", ctypes.POINTER(_native.TmParams)),
                ("points", ctypes.POINTER(_native.TmPoints)),
                ("buffers", ctypes.POINTER(_native.TmBuffers))]


_native.register("gdn_tm_run_batch_f32", ctypes.c_int,
                 [ctypes.POINTER(TmProblem), ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p])


def simulate_tm_batch(problems, *, tile_config: int | None = None, device=None):
    """Run a list of float32 2D TM problems together on the GPU.

    ``problems`` is a list of dicts of ``simulate_tm`` keyword arguments
    (``grid`` included; ``dtype`` must resolve to float32 and
    ``record_energy`` is not supported). ``tile_config`` in [0, N_CONFIGS)
    forces a tile configuration (see N_CONFIGS), None lets the library pick.
    Returns the list of SimResult, in order.
    """
    if not problems:
        return []
    dev = _native.require_cuda(device)
    lib = _native.load()
    preps = []
    for k, kw in enumerate(problems):
        kw = dict(kw)
        kw.setdefault("device", dev)
        if kw.get("record_energy"):
            raise ValueError(f"problem {k}: batched runs do not record the energy")
        grid = kw.pop("grid")
        p = _prepare_tm(grid, **kw)
        if p.f64:
            raise ValueError(f"problem {k}: batched runs are float32")
        preps.append(p)
    arr = (TmProblem * len(preps))()
    for k, p in enumerate(preps):
        # The workspace depends on the tile configuration the batch picks, so
        # the library allocates one stream-ordered block for all problems.
        p.bufs.workspace, p.bufs.workspace_bytes = None, 0
        arr[k].params = ctypes.pointer(p.params)
        arr[k].points = ctypes.pointer(p.pts)
        arr[k].buffers = ctypes.pointer(p.bufs)
    cfg = -1 if tile_config is None else int(tile_config)
    if not -1 <= cfg < N_CONFIGS:
        raise ValueError(f"tile_config must be in [0, {N_CONFIGS}) or None")
    stream = torch.cuda.current_stream(dev)
    with torch.cuda.device(dev):
        _native.check(lib.gdn_tm_run_batch_f32(arr, len(preps), cfg,
                                               ctypes.c_void_p(stream.cuda_stream)))
    for t in _flatten([p.keep for p in preps]):
        t.record_stream(stream)
    return [p.result for p in preps]


def _truncate(kw, n):
    """The same problem shortened to its first n time steps."""
    kw = dict(kw)
    for key in ("source_current", "mx_current", "my_current"):
        if kw.get(key) is not None:
            kw[key] = kw[key][:n]
    if kw.get("ports"):
        kw["ports"] = tuple(
            (p if isinstance(p, Port) else Port(*p))._replace(
                voltage=None if (p if isinstance(p, Port) else Port(*p)).voltage is None
                else (p if isinstance(p, Port) else Port(*p)).voltage[:n])
            for p in kw["ports"])
    cw = kw.get("cw_sources")
    if cw is not None:
        kw["cw_sources"] = dict(cw, env=np.asarray(cw["env"])[:n])
    return kw


_TUNE_CACHE: dict = {}


def _signature(problems):
    sig = []
    for kw in problems:
        g = kw["grid"]
        sig.append((g.nx, g.ny, len(tuple(kw.get("dft_freqs") or ())), len(kw.get("ports") or ())))
    return tuple(sorted(sig))


def autotune_tm_batch(problems, *, probe_steps: int = 64, repeats: int = 2, device=None,
                      configs=None, use_cache: bool = True):
    """Pick the tile configuration for a batch by timing its first
    ``probe_steps`` steps with every configuration: the device time of the
    time loops alone (CUDA events around the loops, gdn_tm_loop_stats), best
    of ``repeats``, so the per-call host set-up, which is the same for every
    configuration and dominates a short probe, does not decide. Returns
    (best_config, {config: seconds}); the choice is cached per population
    signature (grid sizes, frequency and port counts).
    """
    key = (_signature(problems), probe_steps)
    if use_cache and key in _TUNE_CACHE:
        return _TUNE_CACHE[key]
    dev = _native.require_cuda(device)
    short = [_truncate(kw, probe_steps) for kw in problems]
    timings = {}
    for cfg in (range(N_CONFIGS) if configs is None else configs):
        best = None
        simulate_tm_batch(short, tile_config=cfg, device=dev)  # warm-up
        for _ in range(repeats):
            torch.cuda.synchronize(dev)
            _native.tm_loop_stats(reset=True)
            simulate_tm_batch(short, tile_config=cfg, device=dev)
            torch.cuda.synchronize(dev)
            t = _native.tm_loop_stats(reset=True)[0] / 1e3
            best = t if best is None else min(best, t)
        timings[cfg] = best
    choice = (min(timings, key=timings.get), timings)
    _TUNE_CACHE[key] = choice
    return choice


def freq_adjoint_gradient_batch(specs, *, tile_config: int | None = None, device=None):
    """Frequency-domain adjoint gradients of many 2D problems, both FDTD
    passes batched (freq_adjoint.py:355-493 for each problem).

    ``specs`` is a list of dicts of ``freq_adjoint_gradient`` keyword
    arguments (``grid`` and ``objective`` included; ``dtype`` must be
    float32). Returns one {"sigma": ..., "eps_r": ...} dict per spec.
    """
    from gradenna_b200 import freq_adjoint as fa

    dev = _native.require_cuda(device)
    plans, designs = [], []
    for sp in specs:
        sp = dict(sp)
        grid = sp.pop("grid")
        objective = sp.pop("objective")
        ds, de = sp.pop("design_sigma", None), sp.pop("design_eps_r", None)
        plan = fa._make_plan(grid, sp["design_region"], sp["dft_freqs"], sp["env"],
                             sp.get("source_ij"), sp.get("source_current"), sp.get("ports", ()),
                             sp.get("cpml", fa.CPMLSpec()), sp.get("dtype", torch.float32), dev,
                             sp.get("objective_monitors"), sp.get("exact", True))
        if plan.dtype != torch.float32:
            raise ValueError("batched gradients are float32")
        eps_r, sigma = fa._full_eps_sigma(grid, ds, de, sp["design_region"], dev)
        plans.append((plan, objective, ds is not None, de is not None))
        designs.append((eps_r, sigma))
    fwd = simulate_tm_batch([fa._forward_kwargs(pl, e, s) for (pl, _, _, _), (e, s)
                             in zip(plans, designs)], tile_config=tile_config, device=dev)
    adj_kw, adj_at, cots = [], [], []
    for k, ((pl, obj, _, _), (e, s), res) in enumerate(zip(plans, designs, fwd)):
        _, srcs = fa._objective_sources(pl, obj, res)
        kw = fa._adjoint_kwargs(pl, e, s, srcs)
        if kw is not None:
            adj_at.append(k)
            adj_kw.append(kw)
    adj = dict(zip(adj_at, simulate_tm_batch(adj_kw, tile_config=tile_config, device=dev)))
    out = []
    for k, ((pl, _, want_s, want_e), (e, s), res) in enumerate(zip(plans, designs, fwd)):
        g = {}
        if k not in adj:
            shp = tuple(b - a for a, b in pl.bounds)
            if want_s:
                g["sigma"] = torch.zeros(shp, dtype=torch.float64, device=dev)
            if want_e:
                g["eps_r"] = torch.zeros(shp, dtype=torch.float64, device=dev)
        else:
            gs, ge = fa._contract(pl, e, s, res.monitors[0], adj[k].monitors[0], want_s, want_e)
            if gs is not None:
                g["sigma"] = gs
            if ge is not None:
                g["eps_r"] = ge
        out.append(g)
    return out
