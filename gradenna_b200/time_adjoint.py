r"""Exact time-domain adjoint gradient of 2D TM objectives on the GPU.

The reference differentiates broadband (pulse-driven) objectives with
jax.grad through the whole time loop (freq_adjoint.py:269-309,
scripts/export_viz.py:181-186); its frequency-domain adjoint needs a CW
drive. This module gives the exact gradient of the discrete time loop for
any drive, with two FDTD runs of this library and no reverse-mode tape:

1. Forward run: the objective's DFT phasors (full grid or the objective's
   monitor boxes) plus the Ez history of every design cell (one probe per
   cell: n_steps x design cells values).
2. Cotangents of the objective with respect to the phasors (torch autograd
   of the user objective). A phasor X_k = dt sum_n x^n exp(-i w_k t_n) makes
   the time-domain force on a field sample x^n equal to
   f^n = dt sum_k Re(c_k exp(-i w_k t_n)), c_k the conjugated cotangent
   (t_n = (n + 1) dt for Ez^{n+1}, (n + 1/2) dt for H^{n+1/2}).
3. Adjoint run: the same medium (lumped ports kept as passive loads), driven
   by the forces played backwards in time: at step k a Jz source
   -f_E^{N-1-k} / cb0 on every E cell the objective reads (cb0 =
   (dt / eps0) / (dx dy), the vacuum source coefficient, whatever the
   cell's medium), and Mx/My sources
   (Q_MAG / (-dt / mu0)) f_H^{N-k} on every H cell (one step later than the
   E forces: the H samples sit half a step before the E samples they
   pair with). Q_MAG = -eps0 / mu0 as in the frequency-domain adjoint.
4. Contraction on each design cell (the Yee update's reciprocity makes the
   adjoint variable of the step-n update equal to eps_r (1 + h) times the
   adjoint run's Ez at step N - n, h = sigma dt / (2 eps)):
       dL/dtheta = eps_r (1 + h) sum_n L^{N-n} (dca E^n + dcb curl^{n+1/2}),
       curl^{n+1/2} = (E^{n+1} - ca E^n) / cb,
   with the closed-form dca, dcb of the frequency-domain contraction
   (freq_adjoint.py:186-206), evaluated with the cell's total conductivity.

It matches torch autograd through the oracle's time loop to rounding
(relative 1e-15 in float64) for lossy, metal, permittivity and port-driven
designs: tests/test_time_adjoint_gpu.py. Memory: two float histories of
n_steps x design cells on the device (the forward and adjoint Ez), e.g.
300 MB for a 104^2 design over 7000 steps in float32.
"""

from __future__ import annotations

import numpy as np
import torch

from gradenna_b200 import _native
from gradenna_b200 import freq_adjoint as fa
from gradenna_b200.constants import EPS0, MU0
from gradenna_b200.cpml import CPMLSpec
from gradenna_b200.fdtd2d import Port, simulate_tm
from gradenna_b200.grid import Grid2D

__all__ = ["time_domain_gradient", "TimeAdjointObjective", "time_domain_objective"]


class _TPlan:
    """Run description of a time-domain gradient."""

    def __init__(self, grid, design_region, dft_freqs, source_ij, source_current, ports, cpml,
                 dtype, device, objective_monitors):
        self.dev = _native.require_cuda(device)
        self.grid = grid
        self.freqs = tuple(float(f) for f in dft_freqs)
        self.bounds = fa._region_bounds(design_region, grid.shape)
        self.design_region = tuple(design_region)
        self.source_ij = source_ij
        self.source_current = source_current
        self.ports = tuple(p if isinstance(p, Port) else Port(*p) for p in ports)
        self.cpml = cpml
        self.dtype = dtype
        self.objective_monitors = objective_monitors
        (a0, a1), (b0, b1) = self.bounds
        ii, jj = np.meshgrid(np.arange(a0, a1), np.arange(b0, b1), indexing="ij")
        self.cells = np.stack([ii.ravel(), jj.ravel()], 1).astype(np.int32)
        if source_current is not None:
            self.n_steps = int(np.shape(source_current)[0])
        else:
            lens = [len(p.voltage) for p in self.ports if p.voltage is not None]
            if not lens:
                raise ValueError("need source_current or a driven port")
            self.n_steps = int(lens[0])
        # a frequency-domain plan for the monitor / scatter / cotangent helpers
        self.fplan = fa._make_plan(grid, design_region, self.freqs, np.ones(self.n_steps),
                                   source_ij, source_current, self.ports, cpml, dtype, self.dev,
                                   objective_monitors)


def _total_sigma(plan: _TPlan, sigma):
    """sigma plus the lumped ports' conductance DZ / (R dx dy) on their cells."""
    s = sigma.clone()
    g = plan.grid
    for p in plan.ports:
        s[p.ij[0], p.ij[1]] += fa.DZ / (float(p.resistance) * g.dx * g.dy)
    return s


def _forward(plan: _TPlan, eps_r, sigma):
    kw = fa._forward_kwargs(plan.fplan, eps_r, sigma)
    kw["dft_monitors"] = kw["dft_monitors"][1:]  # no design-region phasor needed
    kw["probe_ij"] = plan.cells
    g = kw.pop("grid")
    res = simulate_tm(g, **kw)
    # _scatter_full expects the design monitor first
    res = res._replace(monitors=[None] + list(res.monitors))
    return res


def _forces(plan: _TPlan, w, half: bool):
    """(n_steps, m) float64 time-domain forces of phasor cotangents w (K, m)."""
    dt = plan.grid.dt
    om = torch.as_tensor(2 * np.pi * np.asarray(plan.freqs), dtype=torch.float64, device=plan.dev)
    n = torch.arange(plan.n_steps, dtype=torch.float64, device=plan.dev) + (0.5 if half else 1.0)
    ph = torch.exp(-1j * torch.outer(n, om) * dt)  # (N, K)
    return (ph @ w.to(torch.complex128)).real * dt


def _adjoint_sources(plan: _TPlan, cot):
    """Time-reversed adjoint waveforms: (jz_idx, jz, mx_idx, mx, my_idx, my)."""
    g = plan.grid
    dt = g.dt
    dt_mu = dt / MU0
    out = []
    for comp, w in enumerate(cot):
        active = torch.any(w.abs() > 0, dim=0)
        idx = torch.nonzero(active)
        if idx.shape[0] == 0:
            out += [None, None]
            continue
        wv = w[:, idx[:, 0], idx[:, 1]]  # (K, m)
        f = _forces(plan, wv, half=comp != 0)  # (N, m)
        rev = torch.flip(f, [0])
        if comp == 0:
            # Vacuum source coefficient on every cell: the injection uses the
            # cell's own c_b = (dt / eps) / (1 + h), and the adjoint scaling
            # eps_r (1 + h) of that cell cancels everything but dt / eps0.
            wave = rev / (-(dt / EPS0) / (g.dx * g.dy))
        else:
            wave = torch.zeros_like(rev)
            wave[1:] = rev[:-1]
            wave = wave * (fa.Q_MAG / (-dt_mu))
        out += [idx.cpu().numpy().astype(np.int32), wave.contiguous()]
    return out


def _adjoint(plan: _TPlan, eps_r, sigma, srcs):
    jz_i, jz, mx_i, mx, my_i, my = srcs
    if jz_i is None and mx_i is None and my_i is None:
        return None
    fdt = plan.dtype
    ports = tuple(Port(p.ij, p.resistance, None) for p in plan.ports)
    return simulate_tm(plan.grid, source_ij=jz_i, source_current=None if jz is None else jz.to(fdt),
                       mx_ij=mx_i, mx_current=None if mx is None else mx.to(fdt), my_ij=my_i,
                       my_current=None if my is None else my.to(fdt), eps_r=eps_r, sigma=sigma,
                       ports=ports, probe_ij=plan.cells, cpml=plan.cpml, dtype=fdt,
                       device=plan.dev)


def _contract(plan: _TPlan, eps_r, sig_tot, e_hist, l_hist, want_sigma, want_eps, chunk=1024):
    """eps_r (1 + h) sum_n L^{N-n} (dca E^n + dcb (E^{n+1} - ca E^n) / cb)
    per design cell; e_hist / l_hist are the (N, cells) probe series
    (E^{n+1} and L^{k+1} at row n, k)."""
    g = plan.grid
    dt = g.dt
    dr = plan.design_region
    er = eps_r[dr].reshape(-1).to(torch.float64)
    sg = sig_tot[dr].reshape(-1).to(torch.float64)
    eps = EPS0 * er
    h = sg * dt / (2 * eps)
    ca = (1 - h) / (1 + h)
    cb = (dt / eps) / (1 + h)
    den = (1 + h) ** 2
    N = e_hist.shape[0]
    # S0 = sum_n L^{N-n} E^n, S1 = sum_n L^{N-n} E^{n+1}; L^{N-n} = l_hist[N-1-n],
    # E^n = e_hist[n-1] (E^0 = 0), E^{n+1} = e_hist[n].
    s0 = torch.zeros_like(er)
    s1 = torch.zeros_like(er)
    for a in range(0, N, chunk):
        b = min(N, a + chunk)
        lam = torch.flip(l_hist[N - b:N - a], [0]).to(torch.float64)  # rows n = a .. b-1
        s1 += (lam * e_hist[a:b].to(torch.float64)).sum(0)
        if a == 0:
            s0 += (lam[1:] * e_hist[0:b - 1].to(torch.float64)).sum(0)
        else:
            s0 += (lam * e_hist[a - 1:b - 1].to(torch.float64)).sum(0)
    scale = er * (1 + h)
    shape = tuple(b - a for a, b in plan.bounds)
    out = {}
    if want_sigma:
        dca = (-dt / eps) / den
        dcb = (-(dt / eps) * (dt / (2 * eps))) / den
        out["sigma"] = (scale * ((dca - dcb * ca / cb) * s0 + dcb / cb * s1)).reshape(shape)
    if want_eps:
        dca = EPS0 * ((sg * dt / (eps * eps)) / den)
        dcb = EPS0 * ((-(dt / (eps * eps))) / den)
        out["eps_r"] = (scale * ((dca - dcb * ca / cb) * s0 + dcb / cb * s1)).reshape(shape)
    return out


def time_domain_gradient(grid: Grid2D, objective, *, design_sigma=None, design_eps_r=None,
                         design_region, dft_freqs, source_ij=None, source_current=None,
                         ports=(), cpml: CPMLSpec = CPMLSpec(), dtype=torch.float32,
                         device=None, objective_monitors=None, return_value: bool = False):
    """Exact gradient of ``objective(FreqPhasors)`` through the time loop,
    for any drive (pulse, multi-tone, CW): one forward and one adjoint run.

    Arguments as ``freq_adjoint_gradient`` (``objective_monitors`` limits the
    forward DFT to the boxes the objective reads), without ``env``: the
    drive's own waveform defines the run. Returns {"sigma": ..., "eps_r":
    ...} float64 tensors of the design shape (and the objective value with
    ``return_value``).
    """
    if design_sigma is None and design_eps_r is None:
        raise ValueError("give design_sigma and/or design_eps_r")
    plan = _TPlan(grid, design_region, dft_freqs, source_ij, source_current, ports, cpml, dtype,
                  device, objective_monitors)
    eps_r, sigma = fa._full_eps_sigma(grid, design_sigma, design_eps_r, design_region, plan.dev)
    val, grads = _gradient(plan, objective, eps_r, sigma, design_sigma is not None,
                           design_eps_r is not None)
    return (grads, val) if return_value else grads


def _gradient(plan: _TPlan, objective, eps_r, sigma, want_sigma, want_eps, fwd=None):
    if fwd is None:
        fwd = _forward(plan, eps_r, sigma)
    full = fa._scatter_full(plan.fplan, fwd)
    val, cot = fa._cotangents(plan.fplan, objective, full, fwd)
    sig_tot = _total_sigma(plan, sigma)
    adj = _adjoint(plan, eps_r, sigma, _adjoint_sources(plan, cot))
    if adj is None:
        shape = tuple(b - a for a, b in plan.bounds)
        z = torch.zeros(shape, dtype=torch.float64, device=plan.dev)
        out = {}
        if want_sigma:
            out["sigma"] = z
        if want_eps:
            out["eps_r"] = z.clone()
        return val, out
    return val, _contract(plan, eps_r, sig_tot, fwd.probe_ez, adj.probe_ez, want_sigma,
                          want_eps)


class TimeAdjointObjective(torch.autograd.Function):
    """objective(design_sigma) whose backward is the exact time-domain
    adjoint (forward run in ``forward``; adjoint run and contraction in
    ``backward``)."""

    @staticmethod
    def forward(ctx, design_sigma, plan, objective):
        eps_r, sigma = fa._full_eps_sigma(plan.grid, design_sigma, None, plan.design_region,
                                          plan.dev)
        fwd = _forward(plan, eps_r, sigma)
        full = fa._scatter_full(plan.fplan, fwd)
        val = fa._objective_value(plan.fplan, objective, full, fwd)
        ctx.plan, ctx.objective = plan, objective
        ctx.state = (eps_r, sigma, fwd)
        return val.detach().to(torch.float64)

    @staticmethod
    def backward(ctx, g):
        eps_r, sigma, fwd = ctx.state
        _, grads = _gradient(ctx.plan, ctx.objective, eps_r, sigma, True, False, fwd=fwd)
        return g * grads["sigma"], None, None


def time_domain_objective(design_sigma, grid: Grid2D, objective, *, design_region, dft_freqs,
                          source_ij=None, source_current=None, ports=(),
                          cpml: CPMLSpec = CPMLSpec(), dtype=torch.float32, device=None,
                          objective_monitors=None):
    """Differentiable objective value: ``.backward()`` runs the exact
    time-domain adjoint."""
    plan = _TPlan(grid, design_region, dft_freqs, source_ij, source_current, ports, cpml, dtype,
                  device, objective_monitors)
    return TimeAdjointObjective.apply(design_sigma, plan, objective)
