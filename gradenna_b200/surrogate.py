"""Learned design surrogate with the FDTD solver as verifier.

A BF16 U-Net (gradenna_b200.unet) is trained on density -> field pairs that
the batched 2D solver itself generates, and then proposes design updates
for a topology optimisation whose every accepted step is verified by a full
FDTD forward + adjoint run. No reference counterpart: the reference
optimises with plain Adam on jax.grad of the FDTD objective
(scripts/export_viz.py:118-171, examples/optimize_2d_antenna.py:130-171).

The problem is the reference's antenna-growth demo (export_viz.py:118-171):
a 280 x 280 grid of 1 mm cells, CPML 8 with alpha_max for 1.5 GHz, a 50 ohm
lumped port at (140, 100) inside a 104 x 104 design region [88:192, 80:184],
a Poynting box (40, 240, 40, 240), sigma = sigma_from_density(rho, 1e-4,
1e5) with the feed cell kept free of design conductivity, a conic filter of
radius 6, beta 8 -> 64 and the figure of merit P_rad(f0) / P_avail(f0) at
f0 = 2.45 GHz. The reference drives a broadband pulse and differentiates the
time loop; here the port is driven by a 2.45 GHz CW voltage under a raised-
cosine turn-on so that the frequency-domain adjoint (two FDTD runs) gives
the exact gradient (``exact``: both runs include the port resistor and the
contraction carries the loss factor 1 + sigma dt / (2 eps), which matters at
metal-level conductivities).

Pieces:

* ``AntennaProblem`` - the problem (``AntennaProblem()`` = the 1 mm hero,
  ``AntennaProblem.coarse()`` = the same geometry at 3 mm for tests);
* ``evaluate`` - the FDTD verifier: radiated fractions, design-region Ez
  phasors and exact gradients of many designs, both runs batched;
* ``random_densities`` / ``generate_dataset`` - seeded filtered/projected
  densities solved by the batched kernel;
* ``Surrogate`` / ``train_surrogate`` - the network with its output scaling,
  trained by its own CUDA kernels;
* ``optimize_plain`` - the reference's method: Adam (lr 0.15) with beta
  continuation on the exact gradient, one forward + adjoint per iteration;
* ``optimize_surrogate`` - the batched+surrogate method: at each outer
  iteration a batch of inner Adam trajectories (different step sizes) on the
  surrogate model corrected to match the verified value and gradient at the
  current design (m(rho) = S(rho) + f_k - S(rho_k) + (g_k - dS_k).(rho -
  rho_k)), the candidates verified together by one batched forward run, the
  best improving one accepted and its adjoint run giving the next gradient.
  ``use_network=False`` drops S (the same loop on the linear model), which
  isolates what the trained network contributes.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass

import numpy as np
import torch
import torch.nn.functional as F

from gradenna_b200 import _native
from gradenna_b200 import freq_adjoint as fa
from gradenna_b200.batch import simulate_tm_batch
from gradenna_b200.cpml import CPMLSpec, alpha_max_for_fmin
from gradenna_b200.fdtd2d import Port
from gradenna_b200.grid import Grid2D
from gradenna_b200.materials import sigma_from_density
from gradenna_b200.monitors import poynting_box_monitors, poynting_flux_box_2d
from gradenna_b200.sparams import half_step_dft
from gradenna_b200.topopt import beta_schedule, conic_kernel, tanh_projection
from gradenna_b200.unet import UNet, UNetSpec

__all__ = ["AntennaProblem", "forward_batch", "adjoint_batch", "evaluate", "design_transform",
           "random_densities", "generate_dataset", "Surrogate", "train_surrogate",
           "optimize_plain", "optimize_surrogate"]


@dataclass(frozen=True)
class AntennaProblem:
    nx: int = 280
    ny: int = 280
    dx: float = 1e-3
    cpml_cells: int = 8
    f_min: float = 1.5e9
    f0: float = 2.45e9
    n_steps: int = 7000
    ramp_steps: int = 700
    port_ij: tuple = (140, 100)
    resistance: float = 50.0
    design: tuple = (88, 192, 80, 184)  # i0, i1, j0, j1
    flux_box: tuple = (40, 240, 40, 240)
    sigma_min: float = 1e-4
    sigma_max: float = 1e5
    filter_radius: float = 6.0
    drive_kind: str = "cw"  # "cw" (frequency-domain adjoint) or "pulse" (time-domain adjoint)
    f_max: float = 3.5e9    # upper band edge of the pulse drive

    @classmethod
    def coarse(cls) -> "AntennaProblem":
        """The same physical layout at 3 mm cells: 96 x 96 grid, 2400 steps
        (the same 16.8 ns), filter radius 2 (the same 6 mm), and a 32 x 32
        design (96 mm, a multiple of 8 cells for the U-Net, centred where
        the hero's 104 mm region is)."""
        return cls(nx=96, ny=96, dx=3e-3, n_steps=2400, ramp_steps=240, port_ij=(47, 33),
                   design=(31, 63, 28, 60), flux_box=(13, 80, 13, 80), filter_radius=2.0)

    @property
    def grid(self) -> Grid2D:
        return Grid2D(self.nx, self.ny, self.dx, self.dx)

    @property
    def cpml(self) -> CPMLSpec:
        return CPMLSpec(self.cpml_cells, alpha_max=alpha_max_for_fmin(self.f_min))

    @property
    def design_region(self):
        i0, i1, j0, j1 = self.design
        return (slice(i0, i1), slice(j0, j1))

    @property
    def design_shape(self) -> tuple[int, int]:
        i0, i1, j0, j1 = self.design
        return (i1 - i0, j1 - j0)

    def drive(self):
        """(v, env): the port voltage sampled at (n + 1/2) dt and its turn-on
        envelope. CW: a 2.45 GHz sine under a raised-cosine ramp. Pulse: the
        reference's band pulse gaussian_pulse_for_band(f_min, f_max)
        (export_viz.py:136-138), envelope all ones (unused)."""
        n = np.arange(self.n_steps, dtype=np.float64)
        if self.drive_kind == "pulse":
            from gradenna_b200.sparams import gaussian_pulse_for_band

            v = gaussian_pulse_for_band(self.f_min, self.f_max)((n + 0.5) * self.grid.dt)
            return np.asarray(v, np.float64), np.ones(self.n_steps)
        if self.drive_kind != "cw":
            raise ValueError(f"drive_kind must be 'cw' or 'pulse', got {self.drive_kind!r}")
        env = np.where(n < self.ramp_steps, 0.5 - 0.5 * np.cos(np.pi * n / self.ramp_steps), 1.0)
        v = env * np.sin(2 * np.pi * self.f0 * (n + 0.5) * self.grid.dt)
        return v, env

    def p_avail(self) -> float:
        """|Vs(f0)|^2 / (8 Rs) (export_viz.py:141)."""
        v, _ = self.drive()
        vs = half_step_dft(torch.as_tensor(v), self.grid.dt, (self.f0,))[0]
        return float(abs(vs) ** 2 / (8.0 * self.resistance))

    def design_mask(self, device=None) -> torch.Tensor:
        """True on design cells that carry conductivity (the feed cell does not)."""
        m = torch.ones(self.design_shape, dtype=torch.bool, device=device)
        i0, _, j0, _ = self.design
        m[self.port_ij[0] - i0, self.port_ij[1] - j0] = False
        return m

    def design_sigma(self, rho: torch.Tensor) -> torch.Tensor:
        s = sigma_from_density(rho.to(torch.float64), self.sigma_min, self.sigma_max)
        return torch.where(self.design_mask(rho.device), s, torch.zeros_like(s))

    def plan(self, device):
        v, env = self.drive()
        ports = (Port(tuple(self.port_ij), self.resistance, v.astype(np.float32)),)
        return fa._make_plan(self.grid, self.design_region, (self.f0,), env, None, None, ports,
                             self.cpml, torch.float32, device, poynting_box_monitors(self.flux_box),
                             exact=True)

    def objective(self):
        grid, box, pa = self.grid, self.flux_box, self.p_avail()

        def radiated_fraction(ph):
            return poynting_flux_box_2d(ph.dft_ez, ph.dft_hx, ph.dft_hy, grid, box)[0] / pa

        return radiated_fraction


class _Verifier:
    """Cached plan and objective of a problem on a device (and, for the
    pulse drive, the time-domain adjoint plan)."""

    _cache: dict = {}

    @classmethod
    def get(cls, problem: AntennaProblem, dev):
        key = (problem, str(dev))
        if key not in cls._cache:
            cls._cache[key] = (problem.plan(dev), problem.objective())
        return cls._cache[key]

    @classmethod
    def tplan(cls, problem: AntennaProblem, dev):
        key = ("t", problem, str(dev))
        if key not in cls._cache:
            from gradenna_b200.time_adjoint import _TPlan

            v, _ = problem.drive()
            ports = (Port(tuple(problem.port_ij), problem.resistance, v.astype(np.float32)),)
            cls._cache[key] = _TPlan(problem.grid, problem.design_region, (problem.f0,), None,
                                     None, ports, problem.cpml, torch.float32, dev,
                                     poynting_box_monitors(problem.flux_box))
        return cls._cache[key]


class _Forward:
    """Forward runs of a batch of designs, kept for later adjoint runs."""

    def __init__(self, problem, dev, designs, fwd, full, fraction, ez):
        self.problem, self.dev, self.designs, self.fwd, self.full = problem, dev, designs, fwd, full
        self.fraction, self.ez = fraction, ez


def forward_batch(problem: AntennaProblem, rhos, *, device=None,
                  tile_config: int | None = None) -> _Forward:
    """Forward runs of designs ``rhos`` (B, H, W), batched; the result holds
    the radiated fractions (B,) and design-region Ez phasors (and, for the
    pulse drive, the design cells' Ez histories for the time-domain
    adjoint)."""
    dev = _native.require_cuda(device)
    plan, obj = _Verifier.get(problem, dev)
    rhos = torch.as_tensor(rhos, device=dev).to(torch.float64).reshape((-1,) + problem.design_shape)
    designs = [fa._full_eps_sigma(problem.grid, problem.design_sigma(rho), None,
                                  problem.design_region, dev) for rho in rhos]
    kws = [fa._forward_kwargs(plan, e, s) for e, s in designs]
    if problem.drive_kind == "pulse":
        cells = _Verifier.tplan(problem, dev).cells  # design-cell Ez histories
        for kw in kws:
            kw["probe_ij"] = cells
    fwd = simulate_tm_batch(kws, tile_config=tile_config, device=dev)
    full = [fa._scatter_full(plan, res) for res in fwd]
    fr = torch.stack([fa._objective_value(plan, obj, fu, res).detach().to(torch.float64).reshape(())
                      for fu, res in zip(full, fwd)])
    ez = torch.stack([res.monitors[0][0] for res in fwd])
    return _Forward(problem, dev, designs, fwd, full, fr, ez)


def adjoint_batch(state: _Forward, which, *, tile_config: int | None = None) -> list:
    """Exact d fraction / d rho (H, W) float64 of the designs ``which`` of a
    forward batch: their adjoint runs batched, then the contraction (the
    frequency-domain adjoint for the CW drive, the time-domain adjoint of
    gradenna_b200.time_adjoint for the pulse drive)."""
    problem, dev = state.problem, state.dev
    plan, obj = _Verifier.get(problem, dev)
    pulse = problem.drive_kind == "pulse"
    if pulse:
        from gradenna_b200 import time_adjoint as ta

        tp = _Verifier.tplan(problem, dev)
    which = list(which)
    kws, at = [], []
    for k in which:
        e, s = state.designs[k]
        _, cot = fa._cotangents(plan, obj, state.full[k], state.fwd[k])
        if pulse:
            jz_i, jz, mx_i, mx, my_i, my = ta._adjoint_sources(tp, cot)
            kw = None
            if jz_i is not None or mx_i is not None or my_i is not None:
                kw = dict(grid=problem.grid, source_ij=jz_i,
                          source_current=None if jz is None else jz.float(), mx_ij=mx_i,
                          mx_current=None if mx is None else mx.float(), my_ij=my_i,
                          my_current=None if my is None else my.float(), eps_r=e, sigma=s,
                          ports=tuple(Port(p.ij, p.resistance, None) for p in tp.ports),
                          probe_ij=tp.cells, cpml=problem.cpml, dtype=torch.float32,
                          device=dev)
        else:
            kw = fa._adjoint_kwargs(plan, e, s, fa._adjoint_sources(plan, cot))
        if kw is not None:
            kws.append(kw)
            at.append(k)
    adj = simulate_tm_batch(kws, tile_config=tile_config, device=dev) if kws else []
    lo, hi = math.log10(problem.sigma_min), math.log10(problem.sigma_max)
    out = []
    for k in which:
        if k not in at:
            out.append(torch.zeros(problem.design_shape, dtype=torch.float64, device=dev))
            continue
        e, s = state.designs[k]
        if pulse:
            gs = ta._contract(tp, e, ta._total_sigma(tp, s), state.fwd[k].probe_ez,
                              adj[at.index(k)].probe_ez, True, False)["sigma"]
        else:
            gs, _ = fa._contract(plan, e, s, state.fwd[k].monitors[0],
                                 adj[at.index(k)].monitors[0], True, False)
        # d sigma / d rho of sigma_from_density (zero on the feed cell).
        out.append(gs * s[problem.design_region] * (math.log(10.0) * (hi - lo)))
    return out


def evaluate(problem: AntennaProblem, rhos, *, gradient: bool = True, device=None,
             tile_config: int | None = None):
    """FDTD verification of designs ``rhos`` (B, H, W): (fraction (B,) float64,
    ez (B, H, W) complex128 design-region phasor, grads) with grads a list
    of d fraction / d rho (H, W) float64 per design (None without
    ``gradient``). Forward runs batched, then adjoint runs batched."""
    st = forward_batch(problem, rhos, device=device, tile_config=tile_config)
    grads = adjoint_batch(st, range(len(st.designs)), tile_config=tile_config) if gradient else None
    return st.fraction, st.ez, grads


def design_transform(theta: torch.Tensor, beta, radius: float, eta: float = 0.5) -> torch.Tensor:
    """theta (B, H, W) -> sigmoid -> conic filter -> tanh projection: the
    batched form of topopt.DesignTransform (topopt.py:109-127), on the
    library's fused kernels for float64 CUDA tensors
    (topopt.design_transform_batch)."""
    from gradenna_b200.topopt import design_transform_batch

    return design_transform_batch(theta, beta, radius, eta)


def random_densities(n: int, shape, *, seed: int = 0, radius_range=(2.0, 12.0),
                     device=None) -> torch.Tensor:
    """Seeded filtered/projected densities (n, H, W) float32 in [0, 1]:
    U(0, 1) noise -> conic filter of a random radius -> standardised to
    0.5 + 0.2 z -> tanh projection with beta in {2, ..., 64} and eta in
    [0.3, 0.7]; one in eight is a near-uniform gray level."""
    dev = torch.device("cpu") if device is None else torch.device(device)
    rng = np.random.default_rng(seed)
    out = torch.empty((n,) + tuple(shape), dtype=torch.float32, device=dev)
    for k in range(n):
        noise = torch.as_tensor(rng.uniform(0.0, 1.0, shape), dtype=torch.float64, device=dev)
        radius = float(rng.uniform(*radius_range))
        kern = torch.as_tensor(conic_kernel(radius, 2), dtype=torch.float64, device=dev)
        pad = kern.shape[0] // 2
        f = F.conv2d(noise[None, None], kern[None, None], padding=pad)[0, 0]
        f = f / F.conv2d(torch.ones_like(noise)[None, None], kern[None, None], padding=pad)[0, 0]
        z = (f - f.mean()) / (f.std() + 1e-12)
        if rng.uniform() < 0.125:
            rho = (float(rng.uniform(0.2, 0.8)) + 0.05 * z).clamp(0.0, 1.0)
        else:
            base = (0.5 + 0.2 * z).clamp(0.0, 1.0)
            beta = float(rng.choice([2.0, 4.0, 8.0, 16.0, 32.0, 64.0]))
            rho = tanh_projection(base, beta, float(rng.uniform(0.3, 0.7)))
        out[k] = rho.to(torch.float32)
    return out


def generate_dataset(problem: AntennaProblem, n: int, *, seed: int = 0, batch: int = 64,
                     device=None, tile_config: int | None = None) -> dict:
    """n seeded densities solved by the batched FDTD kernel (forward runs).

    Feature radii are drawn from [1, 6] x the problem's filter radius, so the
    designs have the same physical feature sizes at any cell size. Returns
    {"rho": (n, H, W) float32, "fraction": (n,) float32, "ez": (n, H, W, 2)
    float32 = asinh(Re, Im of the design-region Ez phasor / "ez_scale"),
    "ez_scale": float (the median per-design RMS field), "seconds": solve
    time}. The asinh keeps the few strongly driven designs from dominating
    the field loss.
    """
    dev = _native.require_cuda(device)
    r = problem.filter_radius
    rho = random_densities(n, problem.design_shape, seed=seed, radius_range=(r, 6.0 * r),
                           device=dev)
    frac = torch.empty(n, dtype=torch.float64, device=dev)
    ez = torch.empty((n,) + problem.design_shape, dtype=torch.complex128, device=dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for s in range(0, n, batch):
        f, e, _ = evaluate(problem, rho[s:s + batch], gradient=False, device=dev,
                           tile_config=tile_config)
        frac[s:s + batch] = f
        ez[s:s + batch] = e
    torch.cuda.synchronize(dev)
    seconds = time.perf_counter() - t0
    rms = torch.sqrt(torch.mean(ez.abs() ** 2, dim=(1, 2)))
    scale = float(torch.median(rms)) or 1.0
    ez_ri = torch.asinh(torch.stack([ez.real, ez.imag], dim=-1) / scale)
    return {"rho": rho, "fraction": frac.to(torch.float32), "ez": ez_ri.to(torch.float32),
            "ez_scale": scale, "seconds": seconds}


class Surrogate:
    """A trained U-Net with the scaling of its outputs: channel 2's mean is
    (log(fraction + power_floor) - power_mean) / power_std (the radiated
    fraction of random designs spans orders of magnitude), channels 0, 1 are
    asinh(Ez / ez_scale)."""

    def __init__(self, net: UNet, power_mean: float = 0.0, power_std: float = 1.0,
                 ez_scale: float = 1.0, power_floor: float = 1e-6):
        self.net, self.power_mean, self.power_std = net, power_mean, power_std
        self.ez_scale, self.power_floor = ez_scale, power_floor

    def _fraction(self, p):
        return torch.exp(p * self.power_std + self.power_mean) - self.power_floor

    def predict(self, rho):
        """(fraction (B,), ez (B, H, W) complex) predicted for densities rho."""
        out, p = self.net.forward(torch.as_tensor(rho, dtype=torch.float32))
        ez = torch.complex(torch.sinh(out[..., 0]), torch.sinh(out[..., 1])) * self.ez_scale
        return self._fraction(p), ez

    def fraction_grad(self, rho, weight=None):
        """(fraction (B,), d fraction / d rho (B, H, W)) from the network's
        own forward and input-gradient kernels."""
        p, g = self.net.power_grad(torch.as_tensor(rho, dtype=torch.float32), weight)
        f = self._fraction(p)
        return f, g * ((f + self.power_floor) * self.power_std)[:, None, None]

    def state_dict(self) -> dict:
        return dict(self.net.state_dict(), power_mean=self.power_mean, power_std=self.power_std,
                    ez_scale=self.ez_scale, power_floor=self.power_floor)


def train_surrogate(data: dict, *, spec: UNetSpec | None = None, epochs: int = 30,
                    batch: int = 32, lr: float = 1e-3, lr_final: float = 5e-5,
                    warmup: int = 300, field_weight: float = 1.0, power_weight: float = 4.0,
                    val_fraction: float = 0.1, seed: int = 0, device=None,
                    data_parallel: bool = False) -> tuple:
    """Train a U-Net surrogate on ``generate_dataset`` output with its own
    CUDA kernels (linear warmup over ``warmup`` steps, then cosine decay from
    lr to lr_final). The power target is log(fraction + floor), floor = 1e-3
    of the largest fraction, standardised. Returns (Surrogate, history) with
    per-epoch training loss, the validation R^2 of the fraction and of its
    log, the fraction RMSE and the field relative error, plus the time.

    With ``data_parallel`` (inside an initialised torch.distributed process
    group), every rank trains on its own data with the same initial weights
    and the gradients are averaged over the ranks before each Adam step
    (``unet.allreduce_mean``); the output scaling (log-fraction mean and
    spread, field scale) is averaged the same way first, so all ranks hold
    the same network. Every rank must take the same number of steps: pass
    datasets of equal size.
    """
    dev = _native.require_cuda(device)
    rho = data["rho"].to(dev)
    n, h, w = rho.shape
    spec = spec or UNetSpec(height=h, width=w)
    net = UNet(spec, seed=seed, device=dev, learning_rate=lr)
    frac = data["fraction"].to(dev).to(torch.float32)
    ez = data["ez"].to(dev)
    gen = torch.Generator(device="cpu").manual_seed(seed)
    perm = torch.randperm(n, generator=gen).to(dev)
    n_val = max(1, int(round(val_fraction * n))) if n > 1 else 0
    val, tr = perm[:n_val], perm[n_val:]
    hook = None
    ez_scale = data.get("ez_scale", 1.0)
    fmax = float(frac.max())
    if data_parallel:
        import torch.distributed as dist

        from gradenna_b200.unet import allreduce_mean

        hook = allreduce_mean()
        t = torch.tensor([fmax], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        fmax = float(t[0])
    floor = max(1e-3 * fmax, 1e-30)
    lt = torch.log(frac.to(torch.float64) + floor)
    mu, sd = float(lt[tr].mean()), float(lt[tr].std()) or 1.0
    if data_parallel:
        t = torch.tensor([mu, sd, ez_scale], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        t /= dist.get_world_size()
        mu, sd, common = float(t[0]), float(t[1]), float(t[2])
        # re-express this rank's field targets in the common field scale
        ez = torch.asinh(torch.sinh(ez.to(torch.float64)) * (ez_scale / common)).to(torch.float32)
        ez_scale = common
    tp_all = ((lt - mu) / sd).to(torch.float32)
    steps_per_epoch = max(1, len(tr) // batch)
    total = epochs * steps_per_epoch
    warmup = min(warmup, max(1, total // 5))
    hist = {"loss": [], "val_rmse": [], "val_r2": [], "val_r2_log": [], "val_field_rel": []}
    sur = Surrogate(net, mu, sd, ez_scale, floor)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    step = 0
    for _ in range(epochs):
        order = tr[torch.randperm(len(tr), generator=gen).to(dev)]
        acc = torch.zeros((), dtype=torch.float32, device=dev)
        for b in range(steps_per_epoch):
            idx = order[b * batch:(b + 1) * batch]
            if step < warmup:
                net.set_learning_rate(lr * (step + 1) / warmup)
            else:
                c = (step - warmup) / max(1, total - warmup)
                net.set_learning_rate(lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * c)))
            acc += net.train_step(rho[idx], ez[idx], tp_all[idx], field_weight=field_weight,
                                  power_weight=power_weight, grad_hook=hook)
            step += 1
        hist["loss"].append(float(acc) / steps_per_epoch)
        if n_val:
            pf, pl, pe, tf_, te = [], [], [], frac[val], ez[val]
            for s in range(0, n_val, 256):
                out, p = net.forward(rho[val[s:s + 256]])
                pl.append(p)
                pf.append(sur._fraction(p))
                pe.append(out[..., :2])
            pf, pl, pe = torch.cat(pf), torch.cat(pl), torch.cat(pe)
            tl = tp_all[val]
            hist["val_rmse"].append(float(torch.sqrt(torch.mean((pf - tf_) ** 2))))
            hist["val_r2"].append(float(1 - torch.mean((pf - tf_) ** 2) / torch.var(tf_)))
            hist["val_r2_log"].append(float(1 - torch.mean((pl - tl) ** 2) / torch.var(tl)))
            hist["val_field_rel"].append(float(torch.linalg.vector_norm(pe - te)
                                               / torch.linalg.vector_norm(te)))
    torch.cuda.synchronize(dev)
    hist["seconds"] = time.perf_counter() - t0
    hist["steps"] = step
    return sur, hist


def _clock(dev):
    torch.cuda.synchronize(dev)
    return time.perf_counter()


def optimize_plain(problem: AntennaProblem, *, n_iters: int = 200,
                   betas=(8.0, 16.0, 32.0, 64.0), learning_rate: float = 0.15, device=None,
                   tile_config: int | None = None) -> dict:
    """The reference's optimiser (export_viz.py:147-190): theta0 = 0, Adam
    (lr 0.15, optax defaults) on -fraction with beta continuation, one
    verified forward + adjoint per iteration. Returns per-iteration
    "fraction" (of the design before the update), "seconds" (wall clock of
    the GPU, synchronised) and "fdtd_runs", plus "theta" and "rho"."""
    dev = _native.require_cuda(device)
    theta = torch.zeros(problem.design_shape, dtype=torch.float64, device=dev, requires_grad=True)
    opt = torch.optim.Adam([theta], lr=learning_rate, betas=(0.9, 0.999), eps=1e-8)
    sched = beta_schedule(betas, max(1, n_iters // len(betas)))
    fr, secs, runs = [], [], []
    t0 = _clock(dev)
    for i in range(n_iters):
        beta = sched(i)
        opt.zero_grad(set_to_none=True)
        rho = design_transform(theta[None], beta, problem.filter_radius)[0]
        f, _, g = evaluate(problem, rho.detach()[None], gradient=True, device=dev,
                           tile_config=tile_config)
        rho.backward(-g[0])
        opt.step()
        fr.append(float(f[0]))
        secs.append(_clock(dev) - t0)
        runs.append(2 * (i + 1))
    with torch.no_grad():
        rho = design_transform(theta[None], sched(n_iters - 1), problem.filter_radius)[0]
    return {"fraction": np.asarray(fr), "seconds": np.asarray(secs), "fdtd_runs": np.asarray(runs),
            "theta": theta.detach(), "rho": rho}


def optimize_surrogate(problem: AntennaProblem, surrogate: Surrogate | None, *,
                       n_outer: int = 24, n_inner: int = 30, inner_lrs=(0.1, 0.3, 1.0),
                       betas=(8.0, 16.0, 32.0, 64.0), iters_per_beta: int = 3,
                       use_network: bool = True, target: float | None = None, device=None,
                       tile_config: int | None = None) -> dict:
    """The batched+surrogate optimiser (see the module docstring).

    Each outer iteration runs inner Adam trajectories of ``n_inner`` steps
    from the current design, one per (model, step size): the corrected
    surrogate model (when ``use_network``) and the linear model, each with
    every step size in ``inner_lrs``. The network trajectories advance
    together (one network batch per inner step); all end points are verified
    together by one batched FDTD forward run. The best candidate is accepted
    if it improves the verified fraction (its adjoint run then gives the next
    gradient, and if it used the largest step size the step sizes grow by
    1.5x); otherwise the step sizes halve. The beta stage advances every
    ``iters_per_beta`` outer iterations up to the last one, which then holds
    for the remaining iterations (the current design is re-verified at each
    new beta). With ``target``, the loop stops once a verified design at the
    final beta reaches it. Returns "fraction" / "seconds" /
    "fdtd_runs" per outer iteration (the accepted design's verified
    fraction), "beta", "accepted" (model of the accepted candidate, or ""),
    "theta", "rho".
    """
    dev = _native.require_cuda(device)
    if use_network and surrogate is None:
        raise ValueError("use_network needs a trained surrogate")
    H, W = problem.design_shape
    theta = torch.zeros((H, W), dtype=torch.float64, device=dev)
    lr0 = torch.as_tensor(inner_lrs, dtype=torch.float64, device=dev)
    kinds = (["net"] if use_network else []) + ["lin"]
    use_net = torch.as_tensor([k == "net" for k in kinds for _ in inner_lrs], device=dev)
    B = int(use_net.numel())
    n_net = int(use_net.sum())
    scale = 1.0
    sched = beta_schedule(betas, max(1, int(iters_per_beta)))
    fr, secs, runs, bh, acc = [], [], [], [], []
    n_runs = 0
    t0 = _clock(dev)
    beta_k = None
    f_k = g_k = rho_k = None
    for k in range(n_outer):
        beta = sched(k)
        if beta != beta_k:
            beta_k = beta
            rho_k = design_transform(theta[None], beta, problem.filter_radius)[0]
            f, _, g = evaluate(problem, rho_k[None], gradient=True, device=dev,
                               tile_config=tile_config)
            f_k, g_k = float(f[0]), g[0]
            n_runs += 2
        corr_net = None
        if n_net:
            _, gs_k = surrogate.fraction_grad(rho_k[None])
            corr_net = g_k - gs_k[0].to(torch.float64)
        lrs = (lr0.repeat(len(kinds)) * scale)[:, None, None]
        th = theta[None].repeat(B, 1, 1).requires_grad_(True)
        m = torch.zeros_like(th)
        v = torch.zeros_like(th)
        base = g_k[None].expand(B, H, W).clone()
        if n_net:
            base[use_net] = corr_net[None].expand(n_net, H, W)
        for j in range(n_inner):
            rho = design_transform(th, beta, problem.filter_radius)
            dm = base
            if n_net:
                _, gs = surrogate.fraction_grad(rho[use_net].detach())
                dm = base.clone()
                dm[use_net] += gs.to(torch.float64)
            (gth,) = torch.autograd.grad(rho, th, grad_outputs=-dm)
            with torch.no_grad():
                m.mul_(0.9).add_(gth, alpha=0.1)
                v.mul_(0.999).addcmul_(gth, gth, value=0.001)
                mh = m / (1 - 0.9 ** (j + 1))
                vh = v / (1 - 0.999 ** (j + 1))
                th -= lrs * mh / (vh.sqrt() + 1e-8)
        with torch.no_grad():
            cand = design_transform(th.detach(), beta, problem.filter_radius)
        st = forward_batch(problem, cand, device=dev, tile_config=tile_config)
        n_runs += B
        best = int(torch.argmax(st.fraction))
        accepted = float(st.fraction[best]) > f_k
        if accepted:
            theta = th[best].detach().clone()
            rho_k = cand[best]
            f_k = float(st.fraction[best])
            g_k = adjoint_batch(st, [best], tile_config=tile_config)[0]
            n_runs += 1
            if best % len(inner_lrs) == len(inner_lrs) - 1:
                scale *= 1.5
        else:
            scale *= 0.5
        fr.append(f_k)
        secs.append(_clock(dev) - t0)
        runs.append(n_runs)
        bh.append(beta)
        acc.append(kinds[best // len(inner_lrs)] if accepted else "")
        if target is not None and beta == float(betas[-1]) and f_k >= target:
            break
    return {"fraction": np.asarray(fr), "seconds": np.asarray(secs), "fdtd_runs": np.asarray(runs),
            "beta": np.asarray(bh), "accepted": np.asarray(acc), "theta": theta, "rho": rho_k}
