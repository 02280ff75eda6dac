#!/usr/bin/env python
"""Benchmark: large 2D TM FDTD forward+adjoint design gradient on B200.

Workload (one "step" = one full design-gradient evaluation):
  Grid2D 1024 x 1024 at 1 mm, CPML 16, 8000 time steps, float32 fields;
  512 x 512 design region [256:768, 256:768] with a seeded density
  tanh_projection(conic_filter(U(0,1) noise, 3), beta=8, eta=0.5) mapped by
  sigma_from_density; two 50-ohm RVS ports at (200, 512) (driven, a 4-tone
  CW drive with a 300-step ramp) and (824, 512) (passive load); running DFT
  at 4 frequencies over 2.0-3.0 GHz (complex128 accumulators); objective =
  sum_k P_rad,k (Poynting box (150, 873, 150, 873)) - sum_k |S11_k|^2; its
  gradient over all 512^2 design cells by the frequency-domain adjoint
  (forward run + cotangents + adjoint run + contraction).
  Synthetic inputs (no dataset exists for this workload).

Metric: Gcell-steps/s fwd+adjoint = 2 * nx * ny * n_steps / time per step.

  value   device-resident inputs, CUDA events per step on the launching
          stream, L2 flushed (256 MiB write) before every timed step.
  e2e     the same through the public API from pinned HOST inputs: the
          design conductivity and the drive waveform are copied in, the
          gradient is read back, inside the timed region.
  roofline  dominant kernel tm_tb (one launch = a block of TB = 4 time steps;
          interior and boundary tiles run as two concurrent launches):
          algorithmic bytes per block = TB x 32 B per cell for float32 (Ez, Hx,
          Hy read + write, ca, cb read, per time step) / the block's mean
          duration inside the timed region: the library records CUDA events
          on the run's stream around every time loop (gdn_tm_loop_stats), so
          the duration covers the block launches and the DFT folds of both
          the forward and the adjoint run; peak = MEASURED_PEAKS.json
          hbm_gbs. traffic = ncu dram bytes of one block (both tile
          classes) at this workload, from profiles/tm_tb_1024.txt.
  cpu_baseline  the C oracle (restatement of the reference time loop, all
          host threads) on a bounded sample of the same workload.

Multi-GPU: one process per GPU (torchrun); every rank evaluates the gradient
of its own seeded design (a population member) - no data-path collective;
"scaling": "weak"; value = all ranks' cell-steps / max-over-ranks time. The
population workload instead splits ONE population over the ranks, longest
problems first (lpt_partition): "scaling": "strong", value = the
population's cell-steps / max-over-ranks time.

--impl reference: times the reference algorithm's CPU implementation here
(the C oracle port; the reference's own JAX/Rust paths cannot run on this
image) on the same config, each step a bounded sample; rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_GRID = 1024
N_STEPS = 8000
NPML = 16
FREQS = tuple(np.linspace(2.0e9, 3.0e9, 4))
DESIGN = (slice(256, 768), slice(256, 768))
PORTS = ((200, 512), (824, 512))
BOX = (150, 873, 150, 873)
RAMP = 300
RS = 50.0


# 3D patch workload (Yee, float32): 160 x 160 x 64 at 0.5 mm, CPML 10,
# 6000 steps, PEC-like ground sheet under a 4-cell eps_r = 4.4 substrate,
# 96 x 96 single-plane copper design sheet, vertical 50-ohm port, 11
# frequencies over 2-3 GHz.
P3_SHAPE = (160, 160, 64)
P3_D = 0.5e-3
P3_NPML = 10
P3_STEPS = 6000
P3_FREQS = tuple(np.linspace(2.0e9, 3.0e9, 11))
P3_NDES = 96
P3_SIG_FIXED = 1.0e7
P3_T_CU = 35e-6
P3_BOX = P3_NPML + 2
P3_THETAS = tuple(np.linspace(0.0, np.pi, 13))
P3_PHIS = tuple(np.linspace(0.0, 2 * np.pi, 16, endpoint=False))


# Surrogate workload: the 280 x 280 antenna-growth problem at 1 mm (104 x 104
# design, 7000 steps, 2.45 GHz CW port drive); the plain optimiser runs 200
# Adam iterations (beta 8 -> 64), the batched+surrogate optimiser runs until
# a verified design at beta 64 reaches the plain optimiser's final value.
SUR_SAMPLES = 20000
SUR_EPOCHS = 30
SUR_PLAIN_ITERS = 200
SUR_OUTER = 24


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--dtype", choices=("f32", "f64"), default="f32")
    ap.add_argument("--grid", type=int, default=N_GRID)
    ap.add_argument("--time-steps", type=int, default=None,
                    help="time steps per run (default: 8000 for tm2d, 6000 for patch3d)")
    ap.add_argument("--workload",
                    choices=("tm2d", "patch3d", "population", "surrogate", "unet"),
                    default="tm2d")
    ap.add_argument("--samples", type=int, default=SUR_SAMPLES,
                    help="surrogate workload: training designs solved by the batched kernel")
    ap.add_argument("--epochs", type=int, default=SUR_EPOCHS,
                    help="surrogate workload: training epochs")
    ap.add_argument("--seed", type=int, default=0,
                    help="surrogate workload: seed of the training designs")
    args = ap.parse_args()
    if args.time_steps is None:
        args.time_steps = {"tm2d": N_STEPS, "patch3d": P3_STEPS, "population": 0,
                           "surrogate": 0, "unet": 0}[args.workload]
    return args


def workload(seed: int, n_grid: int, n_steps: int):
    """Host (numpy) inputs of the workload for design `seed`."""
    import torch

    from gradenna_b200.grid import Grid2D
    from gradenna_b200.materials import sigma_from_density
    from gradenna_b200.topopt import seeded_density

    grid = Grid2D(n_grid, n_grid, 1e-3, 1e-3)
    s = n_grid / N_GRID
    design = tuple(slice(int(a.start * s), int(a.stop * s)) for a in DESIGN)
    shape = tuple(a.stop - a.start for a in design)
    rho = seeded_density(shape, seed=seed, radius_cells=3.0, beta=8.0, eta=0.5,
                         device="cpu", dtype=torch.float64).numpy()
    sigma_d = np.asarray(sigma_from_density(rho), np.float64)
    n = np.arange(n_steps)
    env = np.clip(n / float(RAMP), 0.0, 1.0)
    vs = env * sum(np.sin(2 * np.pi * f * (n + 0.5) * grid.dt) for f in FREQS)
    ports = tuple((int(i * s), int(j * s)) for i, j in PORTS)
    box = tuple(int(v * s) for v in BOX)
    return dict(grid=grid, design=design, sigma_d=sigma_d, env=env, vs=vs, ports=ports, box=box)


def workload3d(seed: int, n_steps: int):
    """Host inputs of the 3D patch workload for design `seed`."""
    import torch

    from gradenna_b200.grid import Grid3D
    from gradenna_b200.materials import sheet_conductivity, sigma_from_density
    from gradenna_b200.topopt import seeded_density

    nx, ny, nz = P3_SHAPE
    grid = Grid3D(nx, ny, nz, P3_D, P3_D, P3_D)
    kg = P3_NPML + 3          # ground sheet layer
    kp = kg + 4 + 1           # design (patch) layer above a 4-cell substrate
    d0 = (nx - P3_NDES) // 2
    d1 = d0 + P3_NDES
    g0, g1 = d0 - 6, d1 + 6
    eps_r = np.ones(P3_SHAPE)
    sigma = np.zeros(P3_SHAPE)
    eps_r[g0:g1, g0:g1, kg + 1:kp] = 4.4
    sigma[g0:g1, g0:g1, kg] = P3_SIG_FIXED
    pi, pj = (d0 + d1) // 2, d0 + P3_NDES // 4
    sigma[pi, pj, kg + 1:kp - 1] = P3_SIG_FIXED  # feed pin up to the port gap
    rho = seeded_density((P3_NDES, P3_NDES), seed=seed, radius_cells=3.0, beta=8.0, eta=0.5,
                         device="cpu", dtype=torch.float64).numpy()
    rho[pi - d0, pj - d0] = 1.0  # feed pad is metal
    sig_d = (sheet_conductivity(1.0, P3_T_CU, P3_D)
             * np.asarray(sigma_from_density(rho), np.float64))[:, :, None]
    n = np.arange(n_steps)
    env = np.clip(n / float(RAMP), 0.0, 1.0)
    vs = env * sum(np.sin(2 * np.pi * f * (n + 0.5) * grid.dt) for f in P3_FREQS)
    design = (slice(d0, d1), slice(d0, d1), slice(kp, kp + 1))
    return dict(grid=grid, design=design, sigma_d=sig_d, env=env, vs=vs, port=(pi, pj, kp - 1),
                eps_bg=eps_r, sig_bg=sigma)


def make_objective3d(grid):
    """sum_k |S11_k|^2 - mean_k D_k(theta = 0) from the NTFF of the box."""
    import torch

    from gradenna_b200.fdtd3d import DFTMonitor
    from gradenna_b200.ntff import directivity_3d, ntff_3d
    from gradenna_b200.sparams import s11_power_wave

    def obj(ph):
        s = s11_power_wave(ph.port_v[:, 0], ph.port_i[:, 0], RS)
        mon = DFTMonitor(torch.tensor(P3_FREQS), ph.dft_ex, ph.dft_ey, ph.dft_ez, ph.dft_hx,
                         ph.dft_hy, ph.dft_hz)
        ef = ntff_3d(mon, grid, P3_BOX, P3_FREQS, P3_THETAS, P3_PHIS)
        d = directivity_3d(ef[..., 0], ef[..., 1], P3_THETAS, P3_PHIS)
        return (s.real**2 + s.imag**2).sum() - d[:, 0, 0].mean()

    return obj


def gradient_call3d(w, sigma_dev, vs_dev, dtype):
    import gradenna_b200 as gb
    from gradenna_b200.freq_adjoint3d import freq_adjoint_gradient_3d

    grid = w["grid"]
    return freq_adjoint_gradient_3d(
        grid, make_objective3d(grid), design_sigma=sigma_dev, design_region=w["design"],
        dft_freqs=P3_FREQS, env=w["env"], port_ijk=w["port"], port_voltage=vs_dev,
        port_resistance=RS, cpml=gb.CPMLSpec(P3_NPML), dtype=dtype,
        objective_kind=("port", "ntff_box"), box_margin=P3_BOX,
        eps_r_background=w["eps_bg"], sigma_background=w["sig_bg"])["sigma"]


POP_N = 64


def population(seed: int, n_problems: int = POP_N, max_steps: int = 0):
    """64 seeded uneven 2D TM problems: square grids U{128..512} at 1 mm,
    CPML U{10..16}, U{2000..6000} steps (capped by max_steps when > 0),
    1-4 ports (the first driven by a CW sum of the problem's tones under a
    300-step ramp, the others passive 50-ohm loads), 1-8 frequencies in
    1-6 GHz, a seeded filtered/projected density on the central square of
    half the side mapped by sigma_from_density, and the objective
    sum_k P_rad,k (Poynting box 4 cells inside the CPML) - sum_k |S11_k|^2."""
    import torch

    import gradenna_b200 as gb
    from gradenna_b200.materials import sigma_from_density
    from gradenna_b200.monitors import poynting_box_monitors, port_monitors
    from gradenna_b200.objectives import RadiatedPowerS11
    from gradenna_b200.topopt import seeded_density

    rng = np.random.default_rng(1000 + seed)
    specs = []
    for q in range(n_problems):
        n = int(rng.integers(128, 513))
        npml = int(rng.integers(10, 17))
        steps = int(rng.integers(2000, 6001))
        if max_steps > 0:
            steps = min(steps, max_steps)
        k = int(rng.integers(1, 9))
        freqs = tuple(float(f) for f in np.sort(rng.uniform(1e9, 6e9, k)))
        grid = gb.Grid2D(n, n, 1e-3, 1e-3)
        d0, d1 = n // 4, n // 4 + n // 2
        rho = seeded_density((n // 2, n // 2), seed=int(rng.integers(1 << 30)), radius_cells=3.0,
                             beta=8.0, eta=0.5, device="cpu", dtype=torch.float64).numpy()
        sig_d = np.asarray(sigma_from_density(rho), np.float64)
        nn = np.arange(steps)
        env = np.clip(nn / float(RAMP), 0.0, 1.0)
        vs = env * sum(np.sin(2 * np.pi * f * (nn + 0.5) * grid.dt) for f in freqs)
        lo, hi = npml + 3, d0 - 2
        ports = []
        for m in range(int(rng.integers(1, 5))):
            ij = (int(rng.integers(lo, hi)), int(rng.integers(lo, n - lo)))
            ports.append(gb.Port(ij, RS, vs if m == 0 else None))
        b = npml + 4
        box = (b, n - b - 1, b, n - b - 1)
        mons = poynting_box_monitors(box)
        for pt in ports:
            mons += port_monitors(pt.ij)

        # sum_k P_rad,k - sum_k |S11_k|^2 of the first port, fused on the device
        obj = RadiatedPowerS11(grid, box, ports[0].ij, freqs, resistance=RS, w_prad=1.0,
                               w_s11=-1.0)
        specs.append(dict(grid=grid, objective=obj, design_sigma=sig_d,
                          design_region=(slice(d0, d1), slice(d0, d1)), dft_freqs=freqs, env=env,
                          ports=tuple(ports), cpml=gb.CPMLSpec(npml), dtype=torch.float32,
                          objective_monitors=mons))
    return specs


def pop_cells(specs):
    return sum(sp["grid"].nx * sp["grid"].ny * len(sp["env"]) for sp in specs)


def lpt_partition(costs, n_parts):
    """Longest-processing-time-first split of items with the given costs over
    n_parts workers: items in decreasing cost, each to the least-loaded
    worker (ties to the lower index). Returns one sorted index list per
    worker; the largest load is within 4/3 of the optimum."""
    loads = [0.0] * n_parts
    parts = [[] for _ in range(n_parts)]
    for i in sorted(range(len(costs)), key=lambda q: (-costs[q], q)):
        w = min(range(n_parts), key=lambda r: (loads[r], r))
        parts[w].append(i)
        loads[w] += costs[i]
    return [sorted(p) for p in parts]


def make_objective(grid, box, port_ij):
    """sum_k P_rad,k - sum_k |S11_k|^2 of port 0: the built-in objective, whose
    value and adjoint weights come from one fused kernel on the forward
    run's monitor boxes (gradenna_b200.objectives)."""
    from gradenna_b200.objectives import RadiatedPowerS11

    return RadiatedPowerS11(grid, box, port_ij, FREQS, resistance=RS, w_prad=1.0, w_s11=-1.0)


def monitors_for(w):
    from gradenna_b200.monitors import port_monitors, poynting_box_monitors

    mons = poynting_box_monitors(w["box"])
    for p in w["ports"]:
        mons += port_monitors(p)
    return mons


def gradient_call(w, sigma_dev, vs_dev, dtype, mons):
    import gradenna_b200 as gb
    from gradenna_b200.freq_adjoint import freq_adjoint_gradient

    grid = w["grid"]
    ports = (gb.Port(w["ports"][0], RS, vs_dev), gb.Port(w["ports"][1], RS, None))
    return freq_adjoint_gradient(
        grid, make_objective(grid, w["box"], w["ports"][0]), design_sigma=sigma_dev,
        design_region=w["design"],
        dft_freqs=FREQS, env=w["env"], ports=ports, cpml=gb.CPMLSpec(NPML), dtype=dtype,
        objective_monitors=mons)["sigma"]


# ---------------------------------------------------------------------------
# CPU baseline: the C oracle on a bounded sample of the workload
# ---------------------------------------------------------------------------


def cpu_sample(w, dtype_np, target_s: float = 10.0):
    """Time forward + adjoint-shaped C-oracle runs of n_s steps on the full
    grid (all host threads); n_s is sized so the sample takes ~target_s."""
    from oracle import fdtd2d_np as onp
    from oracle.tm2d_c import simulate_tm_c

    g = w["grid"]
    og = onp.Grid2D(g.nx, g.ny, g.dx, g.dy)
    sigma = np.zeros((g.nx, g.ny))
    sigma[w["design"]] = w["sigma_d"]
    (a0, a1), (b0, b1) = [(s.start, s.stop) for s in w["design"]]
    mons = [(0, a0, b0, a1, b1)] + monitors_for(w)

    def run(n_s):
        kw = dict(sigma=sigma, ports=(onp.Port(w["ports"][0], RS, w["vs"][:n_s]),
                                      onp.Port(w["ports"][1], RS, None)),
                  dft_freqs=FREQS, cpml=onp.CPMLSpec(NPML), dtype=dtype_np, dft_monitors=mons)
        t0 = time.perf_counter()
        simulate_tm_c(og, **kw)  # forward run
        simulate_tm_c(og, **kw)  # adjoint-shaped run (same stencil work)
        return time.perf_counter() - t0

    probe = 10
    t = run(probe)
    n_s = int(np.clip(target_s / max(t, 1e-6) * probe, 20, len(w["vs"])))
    t = run(n_s)
    cells = g.nx * g.ny
    return 2 * cells * n_s / t / 1e9, n_s, t


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int, interval_ms: int = 200):
        self.index = index
        self.interval_ms = int(interval_ms)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", str(self.interval_ms)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=10)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out = ""

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(name):
    """DRAM bytes per block of the dominant kernel from a committed ncu summary
    (its traffic_bytes_per_launch line), or None."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return int(float(line.split(":", 1)[1].split()[0]))
    except OSError:
        pass
    return None


def max_over_ranks(pg, values, device):
    """Element-wise max of per-rank floats over the process group (identity
    without one): every rank's timings reduce to the slowest rank's."""
    if pg is None:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------


def run_reference(args):
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return 0
    if args.workload == "unet":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned "
                          "surrogate, so there is no U-Net training step to time"}), flush=True)
        return 0
    if args.workload == "surrogate":
        P, spec = _hero_cpu_spec()
        vals = []
        for k in range(args.warmup + args.steps):
            v, n_s, t_s = cpu_sample_pop(spec)
            if k >= args.warmup:
                vals.append(v)
        v = float(np.mean(vals))
        secs = SUR_PLAIN_ITERS * 2 * P.nx * P.ny * P.n_steps / (v * 1e9)
        line = {
            "impl": "reference",
            "metric": "GPU-seconds to the plain optimiser's final radiated fraction",
            "value": secs, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": secs * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "antenna growth (see the GPU arm): the reference's plain "
                                   f"optimiser, {SUR_PLAIN_ITERS} forward + adjoint iterations"},
            "cpu_baseline": {"value": secs, "unit": "s", "cores": os.cpu_count(), "kind": "port",
                             "sample": f"C oracle, forward + adjoint-shaped runs of {n_s} steps "
                                       f"({t_s:.1f} s) per step, extrapolated to "
                                       f"{SUR_PLAIN_ITERS} iterations"},
            "e2e": {"value": secs, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return 0
    if args.workload == "population":
        specs = population(0, max_steps=args.time_steps)
        g0 = specs[0]["grid"]
        case = dict(cells=pop_cells(specs) / (args.time_steps or 1),
                    cpu=lambda dt: cpu_sample_pop(specs[0]),
                    cpu_what=lambda n_s, t: (f"C oracle, forward + adjoint-shaped runs of {n_s} "
                                             f"steps of population member 0 ({g0.nx}^2, {t:.1f} s)"),
                    config={"workload": f"batched uneven population of {len(specs)} 2D TM "
                                        "problems (see the GPU arm)",
                            "problems": len(specs), "cell_steps_per_step": 2 * pop_cells(specs)})
    else:
        case = make_case(args, 0)
    dt_np = np.float32 if args.dtype == "f32" else np.float64
    vals = []
    n_s = None
    for k in range(args.warmup + args.steps):
        v, n_s, t_s = case["cpu"](dt_np)
        if k >= args.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    cores = os.cpu_count() if args.workload != "patch3d" else 1
    line = {
        "impl": "reference", "metric": "Gcell-steps/s fwd+adjoint", "value": value,
        "unit": "Gcell-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": (2 * pop_cells(specs) if args.workload == "population"
                        else 2 * case["cells"] * args.time_steps) / value / 1e6,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": args.dtype,
        "data": "synthetic",
        "config": case["config"],
        "cpu_baseline": {"value": value, "unit": "Gcell-steps/s", "cores": cores, "kind": "port",
                         "sample": case["cpu_what"](n_s, t_s) + " per step"},
        "e2e": {"value": value, "unit": "Gcell-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def config_dict(args, w):
    g = w["grid"]
    return {
        "workload": f"2D TM {g.nx}x{g.ny} @1mm, CPML {NPML}, {args.time_steps} steps, 2 RVS ports, "
                    f"K={len(FREQS)} DFT (complex128), P_rad - |S11|^2 objective, freq-adjoint "
                    f"gradient over a {w['sigma_d'].shape[0]}x{w['sigma_d'].shape[1]} design",
        "grid": [g.nx, g.ny], "time_steps": args.time_steps, "n_freq": len(FREQS),
        "design_cells": int(w["sigma_d"].size), "parallelism": f"replicas x{args.gpus}",
        "l2": "flushed (256 MiB write) before every timed step",
    }


def cpu_sample3d(w, dtype_np, target_s: float = 10.0):
    """Time n_s steps of the numpy 3D oracle on the full patch grid (one
    forward run: ground, substrate, design sheet, port); n_s is sized so the
    sample takes about target_s."""
    from oracle import fdtd2d_np as onp
    from oracle import fdtd3d_np as o3

    g = w["grid"]
    og = o3.Grid3D(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz)
    sigma = w["sig_bg"].copy()
    sigma[w["design"]] = w["sigma_d"]

    def run(n_s):
        t0 = time.perf_counter()
        o3.simulate_3d(og, eps_r=w["eps_bg"], sigma=sigma, port_ijk=w["port"],
                       port_voltage=w["vs"][:n_s], port_resistance=RS,
                       cpml=onp.CPMLSpec(P3_NPML), dtype=dtype_np)
        return time.perf_counter() - t0

    probe = 2
    t = run(probe)
    n_s = int(np.clip(target_s / max(t, 1e-6) * probe, 2, len(w["vs"])))
    t = run(n_s)
    return g.nx * g.ny * g.nz * n_s / t / 1e9, n_s, t


def make_case(args, seed):
    """The workload's inputs and per-workload figures for the JSON line."""
    if args.workload == "tm2d":
        w = workload(seed, args.grid, args.time_steps)
        mons = monitors_for(w)
        g = w["grid"]
        # DFT cells per run: the design's Ez in both runs, the objective's
        # boxes in the forward run only.
        obj_cells = sum((hi0 - lo0) * (hi1 - lo1) for _, lo0, lo1, hi0, hi1 in mons)
        return dict(
            w=w, call=lambda s_, v_, fdt: gradient_call(w, s_, v_, fdt, mons),
            cells=g.nx * g.ny, tb=4, words=8, config=config_dict(args, w),
            dft_cells=int(w["sigma_d"].size) + obj_cells / 2, n_freq=len(FREQS),
            kernel="tm_tb 4-step block over the grid (time loop incl. DFT folds)",
            traffic=profiled_traffic("tm_tb_1024.txt"),
            cpu=lambda dt: cpu_sample(w, dt),
            cpu_what=lambda n_s, t: (f"C oracle, forward + adjoint-shaped runs of {n_s} steps on "
                                     f"the full {g.nx}^2 grid ({t:.1f} s)"))
    w = workload3d(seed, args.time_steps)
    g = w["grid"]
    return dict(
        w=w, call=lambda s_, v_, fdt: gradient_call3d(w, s_, v_, fdt),
        cells=g.nx * g.ny * g.nz, tb=1, words=14, config=config3d(args, w),
        dft_cells=dft_cells3d(w), n_freq=len(P3_FREQS),
        kernel="yee_h + yee_e, one time step over the volume (time loop incl. DFT folds)",
        traffic=profiled_traffic("yee_patch3d.txt"),
        cpu=lambda dt: cpu_sample3d(w, dt),
        cpu_what=lambda n_s, t: (f"numpy 3D oracle, one forward run of {n_s} steps on the full "
                                 f"{g.nx}x{g.ny}x{g.nz} grid ({t:.1f} s)"))


def dft_cells3d(w):
    """Monitored cells per run of the 3D gradient: the design E slabs in both
    runs, the port and NTFF face boxes in the forward run only."""
    from gradenna_b200 import dft_region as dr
    from gradenna_b200.freq_adjoint3d import _objective_boxes

    g = w["grid"]
    shapes = dr.full_field_shapes(g.nx, g.ny, g.nz)

    def cells(boxes):
        return sum(int(np.prod(np.subtract(hi, lo))) for _, lo, hi in boxes)

    design = cells(dr.region_boxes(dr.design_region_to_slabs(w["design"], shapes)))
    obj = cells(_objective_boxes(g, ("port", "ntff_box"), port_ijk=w["port"], box_margin=P3_BOX))
    return design + obj / 2


def config3d(args, w):
    g = w["grid"]
    return {
        "workload": f"3D Yee patch {g.nx}x{g.ny}x{g.nz} @0.5mm, CPML {P3_NPML}, "
                    f"{args.time_steps} steps, ground sheet + 4-cell eps_r 4.4 substrate, "
                    f"{P3_NDES}x{P3_NDES} design sheet, 50-ohm port, K={len(P3_FREQS)} DFT "
                    f"(complex128, port + NTFF faces + design), objective sum|S11|^2 - mean "
                    f"D(theta=0), freq-adjoint gradient",
        "grid": [g.nx, g.ny, g.nz], "time_steps": args.time_steps, "n_freq": len(P3_FREQS),
        "design_cells": int(w["sigma_d"].size), "parallelism": f"replicas x{args.gpus}",
        "l2": "flushed (256 MiB write) before every timed step",
    }


def _pop_forward_kwargs(specs, dev):
    """simulate_tm keyword arguments of the forward runs of a population."""
    from gradenna_b200 import freq_adjoint as fa

    out = []
    for sp in specs:
        plan = fa._make_plan(sp["grid"], sp["design_region"], sp["dft_freqs"], sp["env"], None,
                             None, sp["ports"], sp["cpml"], sp["dtype"], dev,
                             sp["objective_monitors"])
        eps_r, sigma = fa._full_eps_sigma(sp["grid"], sp["design_sigma"], None,
                                          sp["design_region"], dev)
        out.append(fa._forward_kwargs(plan, eps_r, sigma))
    return out


def cpu_sample_pop(spec, target_s: float = 10.0):
    """C-oracle forward + adjoint-shaped runs of one population member for a
    bounded number of steps (all host threads)."""
    from oracle import fdtd2d_np as onp
    from oracle.tm2d_c import simulate_tm_c

    g = spec["grid"]
    og = onp.Grid2D(g.nx, g.ny, g.dx, g.dy)
    sigma = np.zeros((g.nx, g.ny))
    sigma[spec["design_region"]] = np.asarray(spec["design_sigma"])
    (a0, a1), (b0, b1) = [(r.start, r.stop) for r in spec["design_region"]]
    mons = [(0, a0, b0, a1, b1)] + list(spec["objective_monitors"])

    def run(n_s):
        ports = tuple(onp.Port(p.ij, p.resistance,
                               None if p.voltage is None else np.asarray(p.voltage)[:n_s])
                      for p in spec["ports"])
        kw = dict(sigma=sigma, ports=ports, dft_freqs=spec["dft_freqs"],
                  cpml=onp.CPMLSpec(spec["cpml"].thickness), dtype=np.float32, dft_monitors=mons)
        t0 = time.perf_counter()
        simulate_tm_c(og, **kw)
        simulate_tm_c(og, **kw)
        return time.perf_counter() - t0

    t = run(10)
    n_s = int(np.clip(target_s / max(t, 1e-6) * 10, 20, len(spec["env"])))
    t = run(n_s)
    return 2 * g.nx * g.ny * n_s / t / 1e9, n_s, t


def run_population(args):
    """Batched forward + adjoint design gradients of a 64-member population."""
    import torch

    from gradenna_b200 import _native
    from gradenna_b200.batch import autotune_tm_batch, freq_adjoint_gradient_batch
    from gradenna_b200.freq_adjoint import freq_adjoint_gradient

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    # One population; its problems are split over the ranks by cell-steps,
    # longest first, so N GPUs share the fixed total work.
    all_specs = population(0, max_steps=args.time_steps)
    share = lpt_partition([pop_cells([sp]) for sp in all_specs], world)[rank]
    specs = [all_specs[q] for q in share]
    dev_specs = [dict(sp, design_sigma=torch.as_tensor(sp["design_sigma"], device=dev))
                 for sp in specs]
    t0 = time.perf_counter()
    best, tune = autotune_tm_batch(_pop_forward_kwargs(dev_specs, dev), probe_steps=128)
    t_tune = time.perf_counter() - t0
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def call(sp):
        return freq_adjoint_gradient_batch(sp, tile_config=best)

    for _ in range(args.warmup):
        call(dev_specs)
    torch.cuda.synchronize()

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    times = []
    barrier()
    l0 = _native.kernel_launches()
    _native.tm_loop_stats(reset=True)
    # The population's step is host-bound (tens of thousands of launches); a
    # 5 Hz nvidia-smi poll measurably slows it, so clocks are sampled at 1 Hz.
    with ClockSampler(local, interval_ms=1000) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            g = call(dev_specs)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
    launches = (_native.kernel_launches() - l0) // args.steps
    loop_ms, loop_cells, _ = _native.tm_loop_stats(reset=True)
    barrier()
    t_step = float(np.mean(times))
    assert all(torch.isfinite(x["sigma"]).all() for x in g)

    # e2e: designs from pinned host memory, gradients read back.
    hosts = [torch.as_tensor(sp["design_sigma"]).pin_memory() for sp in specs]
    outs = [torch.empty(h.shape, dtype=torch.float64).pin_memory() for h in hosts]
    e2e_times = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sp_e = [dict(sp, design_sigma=h.to(dev, non_blocking=True)) for sp, h in zip(specs, hosts)]
        gg = call(sp_e)
        for o, x in zip(outs, gg):
            o.copy_(x["sigma"], non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        e2e_times.append(e0.elapsed_time(e1) / 1e3)
    t_e2e = float(np.mean(e2e_times))

    # The same population one problem at a time (no batching), for reference.
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for sp in dev_specs:
        sp = dict(sp)
        freq_adjoint_gradient(sp.pop("grid"), sp.pop("objective"), **sp)
    e1.record()
    torch.cuda.synchronize()
    t_single = e0.elapsed_time(e1) / 1e3

    t_step, t_e2e = max_over_ranks(pg, [t_step, t_e2e], dev)
    cell_steps = 2 * pop_cells(all_specs)
    value = cell_steps / t_step / 1e9
    e2e = cell_steps / t_e2e / 1e9
    achieved = 8 * 4 * loop_cells / (loop_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    h2d = sum(h.numel() * h.element_size() for h in hosts)
    cpu = None
    if rank == 0:
        v_cpu, n_s, t_cpu = cpu_sample_pop(all_specs[0])
        cpu = {"value": v_cpu, "unit": "Gcell-steps/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"C oracle, forward + adjoint-shaped runs of {n_s} steps of population "
                         f"member 0 ({all_specs[0]['grid'].nx}^2, {t_cpu:.1f} s)"}
        sides = [sp["grid"].nx for sp in all_specs]
        line = {
            "metric": "Gcell-steps/s fwd+adjoint", "value": value, "unit": "Gcell-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {
                "workload": f"batched uneven population: {len(all_specs)} 2D TM problems, square "
                            f"grids {min(sides)}-{max(sides)} at 1 mm, CPML 10-16, 2000-6000 "
                            "steps, 1-4 ports, 1-8 DFT frequencies in 1-6 GHz, seeded "
                            "filtered/projected designs; freq-adjoint gradient of each",
                "problems": len(all_specs), "problems_on_rank0": len(specs),
                "cell_steps_per_step": cell_steps,
                "autotuned_tile_config": best,
                "autotune_s": t_tune, "autotune_probe_s": {str(k): v for k, v in tune.items()},
                "unbatched_ms": t_single * 1e3,
                "unbatched_value": 2 * pop_cells(specs) / t_single / 1e9,
                "parallelism": f"longest-first partition over {world} GPU(s)",
                "l2": "flushed (256 MiB write) before every timed step"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "tm_tb_batch block launches of both passes (time loops incl. "
                                   "DFT folds; 32 B per cell-step)",
                         "peak_source": peak_kind,
                         "loop_share_of_step": loop_ms / 1e3 / (t_step * args.steps)},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "Gcell-steps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(h2d)},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def _hero_cpu_spec():
    """The antenna problem at its gray start, as a cpu_sample_pop spec."""
    import torch

    from gradenna_b200.fdtd2d import Port
    from gradenna_b200.monitors import poynting_box_monitors
    from gradenna_b200.surrogate import AntennaProblem

    P = AntennaProblem()
    v, env = P.drive()
    sig = P.design_sigma(torch.full(P.design_shape, 0.5, dtype=torch.float64)).numpy()
    return P, dict(grid=P.grid, design_region=P.design_region, design_sigma=sig,
                   objective_monitors=poynting_box_monitors(P.flux_box),
                   ports=(Port(P.port_ij, P.resistance, v.astype(np.float32)),),
                   dft_freqs=(P.f0,), cpml=P.cpml, env=env)


def _unet_level(name: str) -> int:
    """Resolution level at which a U-Net layer runs (up-convolutions run at
    the coarser level)."""
    if name == "head":
        return 0
    if name.startswith("up"):
        return int(name[2:]) + 1
    return int(name[3:-1])


def run_surrogate(args):
    """Batched+surrogate optimiser against the plain optimiser on the antenna
    problem (one "step" = one complete optimisation by each method)."""
    import torch

    from gradenna_b200 import _native
    from gradenna_b200 import surrogate as S

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
        pg = dist
    P = S.AntennaProblem()
    # Offline: training data from the batched kernel, then training.
    data = S.generate_dataset(P, args.samples, seed=args.seed + rank, device=dev)
    # Several GPUs: data-parallel training (every rank solved its own seeded
    # designs; gradients all-reduced over NCCL before each Adam step).
    sur, hist = S.train_surrogate(data, epochs=args.epochs, lr=5e-4, device=dev,
                                  data_parallel=world > 1)
    fwd_flops = 2 * sum(
        ly.taps * ly.cin * ly.cout * (P.design_shape[0] >> _unet_level(ly.name))
        * (P.design_shape[1] >> _unet_level(ly.name)) for ly in sur.net.layers)
    # Warm-up: short runs of both methods (tile configurations, allocations).
    for _ in range(max(1, args.warmup)):
        S.optimize_plain(P, n_iters=2, device=dev)
        S.optimize_surrogate(P, sur, n_outer=1, n_inner=4, device=dev)
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    rows = []
    l0 = _native.kernel_launches()
    _native.tm_loop_stats(reset=True)
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            pl = S.optimize_plain(P, n_iters=SUR_PLAIN_ITERS, device=dev)
            target = float(pl["fraction"][-1])
            su = S.optimize_surrogate(P, sur, n_outer=SUR_OUTER, target=target, device=dev)
            hit = np.nonzero((su["fraction"] >= target) & (su["beta"] == su["beta"].max()))[0]
            rows.append((pl, su, target, hit))
    launches = (_native.kernel_launches() - l0) // max(1, args.steps)
    loop_ms, loop_cells, _ = _native.tm_loop_stats(reset=True)
    lin = S.optimize_surrogate(P, None, use_network=False, n_outer=SUR_OUTER, device=dev)
    pl, su, target, hit = rows[-1]
    t_plain = float(np.mean([r[0]["seconds"][-1] for r in rows]))
    t_hit = [float(r[1]["seconds"][r[3][0]]) if len(r[3]) else float(r[1]["seconds"][-1])
             for r in rows]
    t_sur = float(np.mean(t_hit))
    t_sur, t_plain = max_over_ranks(pg, [t_sur, t_plain], dev)
    achieved = 8 * 4 * loop_cells / (loop_ms / 1e3) / 1e9 if loop_ms > 0 else 0.0
    peak, peak_kind = measured_peak()
    if rank == 0:
        _, spec = _hero_cpu_spec()
        v_cpu, n_s, t_cpu = cpu_sample_pop(spec)
        cpu_plain = SUR_PLAIN_ITERS * 2 * P.nx * P.ny * P.n_steps / (v_cpu * 1e9)
        cpu = {"value": cpu_plain, "unit": "s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"C oracle, forward + adjoint-shaped runs of {n_s} steps of the "
                         f"antenna problem ({t_cpu:.1f} s), extrapolated to the plain "
                         f"optimiser's {SUR_PLAIN_ITERS} iterations"}
        line = {
            # When the surrogate run never reaches the target, value is the
            # whole run's time and config.surrogate.reached is false.
            "metric": "GPU-seconds to the plain optimiser's final radiated fraction",
            "value": t_sur, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": (t_sur + t_plain) * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": "antenna growth, 280 x 280 at 1 mm, CPML 8, 104 x 104 design, "
                            "7000 steps, 2.45 GHz CW port drive, radiated fraction through "
                            "the (40, 240, 40, 240) Poynting box; exact freq-adjoint gradients",
                "plain": {"iterations": SUR_PLAIN_ITERS, "seconds": t_plain,
                          "final_fraction": target,
                          "iters_per_s": SUR_PLAIN_ITERS / t_plain,
                          "fdtd_runs": int(pl["fdtd_runs"][-1])},
                "surrogate": {"reached": bool(len(hit)), "seconds_to_target": t_sur,
                              "outer_iterations": int(len(su["fraction"])),
                              "iters_per_s": len(su["fraction"]) / float(su["seconds"][-1]),
                              "final_fraction": float(su["fraction"][-1]),
                              "fdtd_runs": int(su["fdtd_runs"][-1]),
                              "accepted": [str(a) for a in su["accepted"]],
                              "trajectory": [float(f) for f in su["fraction"]]},
                # only meaningful when the surrogate run reached the target
                "speedup_vs_plain": (t_plain / t_sur) if len(hit) else None,
                # The same comparison with the offline work (solving the
                # training designs, training the network) counted in: one
                # problem, nothing amortised.
                "seconds_incl_offline": t_sur + data["seconds"] + hist["seconds"],
                "speedup_vs_plain_incl_offline": (
                    t_plain / (t_sur + data["seconds"] + hist["seconds"]) if len(hit) else None),
                "seed": args.seed,
                "linear_model_ablation": {"final_fraction": float(lin["fraction"][-1]),
                                          "seconds": float(lin["seconds"][-1]),
                                          "reached": bool(np.any(lin["fraction"] >= target))},
                "offline": {"samples": args.samples, "dataset_s": data["seconds"],
                            "training_s": hist["seconds"], "epochs": args.epochs,
                            "train_steps": hist["steps"],
                            "train_tflops": 3 * fwd_flops * 32 * hist["steps"]
                            / hist["seconds"] / 1e12,
                            "val_r2_log_fraction": hist["val_r2_log"][-1],
                            "val_r2_fraction": hist["val_r2"][-1],
                            "val_field_rel": hist["val_field_rel"][-1]},
                "parallelism": (f"data-parallel surrogate training + optimiser replicas x{world}"
                                if world > 1 else "1 GPU")},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "tm_tb / tm_tb_batch time loops of all FDTD runs of both "
                                   "optimisers (32 B per cell-step)", "peak_source": peak_kind},
            "cpu_baseline": cpu,
            "e2e": {"value": t_sur, "unit": "s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0,
                    "note": "the optimisers are host-driven end to end; value is their "
                            "synchronised wall time"},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


UNET_BATCH = 32


def unet_step_flops(net) -> float:
    """Convolution FLOPs of one training step: forward, input gradients
    (all but the first layer) and weight gradients, 2 per multiply-add."""
    spec = net.spec
    total = 0.0
    for ly in net.layers:
        lev = _unet_level(ly.name)
        px = (spec.height >> lev) * (spec.width >> lev)
        f = 2.0 * px * ly.taps * ly.cin * ly.cout
        total += f * (2 if ly.name == "enc0a" else 3)
    return total


def cpu_sample_unet(target_s: float = 10.0, batch: int = 2):
    """The oracle U-Net (torch float32 on the host cores, bf16 rounding off)
    training step: forward, loss, autograd backward, for about target_s
    seconds. Returns (TFLOP/s, steps, seconds, threads)."""
    import torch

    from gradenna_b200.unet import UNet, UNetSpec, unet_layers
    from oracle.unet_torch import unet_loss

    spec = UNetSpec()
    layers, n = unet_layers(spec)
    theta = torch.as_tensor(UNet.init_params(spec, 0)).requires_grad_(True)
    g = torch.Generator().manual_seed(0)
    x = torch.rand((batch, spec.height, spec.width), generator=g)
    tf = torch.randn((batch, spec.height, spec.width, 2), generator=g)
    tp = torch.rand(batch, generator=g)
    lt = [tuple(ly) for ly in layers]

    class _Net:  # unet_step_flops reads .spec and .layers
        pass

    net = _Net()
    net.spec, net.layers = spec, layers
    flops = unet_step_flops(net) * batch
    steps, t0 = 0, time.perf_counter()
    while True:
        loss = unet_loss(theta, lt, spec.levels, x, tf, tp, bf16=False)
        theta.grad = None
        loss.backward()
        steps += 1
        el = time.perf_counter() - t0
        if el >= target_s or steps >= 1000:
            break
    return flops * steps / el / 1e12, steps, el, torch.get_num_threads()


def run_unet(args):
    """Training step of the 104 x 104 surrogate U-Net (batch 32) on its own
    BF16 tensor-core kernels: forward, head loss, backward, Adam."""
    import torch

    from gradenna_b200 import _native
    from gradenna_b200.unet import UNet, UNetSpec

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    spec = UNetSpec()
    net = UNet(spec, seed=rank, device=dev, learning_rate=1e-4)
    g = torch.Generator(device="cpu").manual_seed(rank)
    n = UNET_BATCH
    x_h = torch.rand((n, spec.height, spec.width), generator=g).pin_memory()
    tf_h = torch.randn((n, spec.height, spec.width, 2), generator=g).pin_memory()
    tp_h = torch.rand((n,), generator=g).pin_memory()
    x, tf, tp = x_h.to(dev), tf_h.to(dev), tp_h.to(dev)
    loss_h = torch.empty((), dtype=torch.float32).pin_memory()
    flops = unet_step_flops(net) * n
    for _ in range(args.warmup):
        net.train_step(x, tf, tp)
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    stream = torch.cuda.current_stream(dev)
    l0 = _native.kernel_launches()
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            net.train_step(x, tf, tp)
        e1.record(stream)
        torch.cuda.synchronize()
        t_step = e0.elapsed_time(e1) / 1e3 / args.steps
        launches = (_native.kernel_launches() - l0) // args.steps
        # e2e: the batch copied in from pinned host memory, the loss read back.
        e0.record(stream)
        for _ in range(args.steps):
            xd = x_h.to(dev, non_blocking=True)
            tfd = tf_h.to(dev, non_blocking=True)
            tpd = tp_h.to(dev, non_blocking=True)
            loss_h.copy_(net.train_step(xd, tfd, tpd), non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        t_e2e = e0.elapsed_time(e1) / 1e3 / args.steps
    t_step, t_e2e = max_over_ranks(pg, [t_step, t_e2e], dev)
    if rank == 0:
        v_cpu, n_cpu, t_cpu, threads = cpu_sample_unet()
        cpu = {"value": v_cpu, "unit": "TFLOP/s", "cores": threads, "kind": "port",
               "sample": f"oracle U-Net (torch float32 on the host), {n_cpu} training steps "
                         f"of batch 2 at 104^2 in {t_cpu:.1f} s"}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
            peak, kind = float(peaks["bf16_tflops"]), "measured (cuBLAS bf16 burst)"
        except (OSError, KeyError, ValueError):
            peak, kind = 1590.0, "fallback"
        value = world * flops / t_step / 1e12
        line = {
            "metric": "U-Net training TFLOP/s", "value": value, "unit": "TFLOP/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
            "config": {"workload": "surrogate U-Net training step: 104 x 104 densities, "
                                   "4 levels, 32 base channels, batch 32, BF16 weights and "
                                   "activations, FP32 accumulation and master weights, Adam",
                       "params": net.n_params, "flops_per_step": flops,
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs (35 MB of activations) below L2; not flushed"},
            "roofline": {"bound": "tensor", "achieved": value / world, "peak": peak,
                         "unit": "TFLOP/s", "frac": value / world / peak, "traffic": None,
                         "kernel": "all convolution kernels of the step (conv_fwd, conv_wgrad) "
                                   "plus their elementwise kernels", "peak_source": kind},
            "cpu_baseline": cpu,
            "e2e": {"value": world * flops / t_e2e / 1e12, "unit": "TFLOP/s",
                    "h2d_bytes_per_step": int(x_h.nbytes + tf_h.nbytes + tp_h.nbytes),
                    "d2h_bytes_per_step": 4},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def run_ours(args):
    import torch

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
        pg = dist

    from gradenna_b200 import _native

    fdt = torch.float32 if args.dtype == "f32" else torch.float64
    case = make_case(args, rank)
    w = case["w"]
    sigma_dev = torch.as_tensor(w["sigma_d"], device=dev)
    vs_dev = torch.as_tensor(w["vs"], device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    for _ in range(args.warmup):
        case["call"](sigma_dev, vs_dev, fdt)
    torch.cuda.synchronize()

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    times = []
    barrier()
    l0 = _native.kernel_launches()
    _native.tm_loop_stats(reset=True)
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            g = case["call"](sigma_dev, vs_dev, fdt)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
    launches = (_native.kernel_launches() - l0) // args.steps
    # Dominant kernel: the TB-step block launches of the forward and adjoint
    # time loops inside the timed region, timed by events on their stream.
    loop_ms, loop_cells, loop_blocks = _native.tm_loop_stats(reset=True)
    barrier()
    t_step = float(np.mean(times))
    assert torch.isfinite(g).all()

    # e2e: public API from pinned host inputs, gradient read back.
    sig_h = torch.as_tensor(w["sigma_d"]).pin_memory()
    vs_h = torch.as_tensor(w["vs"]).pin_memory()
    out_h = torch.empty(w["sigma_d"].shape, dtype=torch.float64).pin_memory()
    e2e_times = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sd = sig_h.to(dev, non_blocking=True)
        vd = vs_h.to(dev, non_blocking=True)
        gg = case["call"](sd, vd, fdt)
        out_h.copy_(gg, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        e2e_times.append(e0.elapsed_time(e1) / 1e3)
    t_e2e = float(np.mean(e2e_times))

    t_block = loop_ms / 1e3 / max(loop_blocks, 1)

    t_step, t_e2e = max_over_ranks(pg, [t_step, t_e2e], dev)

    cell_steps = 2 * case["cells"] * args.time_steps
    value = world * cell_steps / t_step / 1e9
    e2e = world * cell_steps / t_e2e / 1e9
    esize = 4 if fdt == torch.float32 else 8
    # Words per cell-step: 2D 8 (Ez/Hx/Hy read + written, ca/cb read), 3D 14
    # (six fields read + written, ca/cb read); one block = tb time steps.
    algo_bytes = case["tb"] * case["words"] * esize * case["cells"]
    achieved = algo_bytes / t_block / 1e9
    # The survey's per-cell-step figure with the DFT counted in: each
    # monitored cell's complex128 accumulators read and written per step and
    # frequency (the ring-and-fold design touches them once per R steps,
    # which is why this can exceed the peak).
    dft_bytes = case["tb"] * case["dft_cells"] * case["n_freq"] * 2 * 16
    peak, peak_kind = measured_peak()
    h2d = w["sigma_d"].nbytes + w["vs"].nbytes
    d2h = w["sigma_d"].nbytes

    cpu = None
    if rank == 0:
        v_cpu, n_s, t_cpu = case["cpu"](np.float32 if fdt == torch.float32 else np.float64)
        cpu = {"value": v_cpu, "unit": "Gcell-steps/s",
               "cores": os.cpu_count() if args.workload == "tm2d" else 1, "kind": "port",
               "sample": case["cpu_what"](n_s, t_cpu)}
    if rank == 0:
        line = {
            "metric": "Gcell-steps/s fwd+adjoint", "value": value, "unit": "Gcell-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.dtype, "data": "synthetic",
            "config": case["config"],
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": case["traffic"],
                         "kernel": case["kernel"], "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": algo_bytes,
                         "frac_incl_dft": (algo_bytes + dft_bytes) / t_block / 1e9 / peak,
                         "algorithmic_bytes_incl_dft_per_launch": int(algo_bytes + dft_bytes),
                         "launch_us": t_block * 1e6,
                         "loop_share_of_step": loop_ms / 1e3 / (t_step * args.steps)},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "Gcell-steps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "population":
        return run_population(args)
    if args.workload == "surrogate":
        return run_surrogate(args)
    if args.workload == "unet":
        return run_unet(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
