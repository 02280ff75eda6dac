r"""Frequency-domain (Meep-type) adjoint for the 2D TM solver on B200.

Same method and conventions as the reference (src/gradenna/freq_adjoint.py):
one forward CW run records the design-region (and objective) phasors, the
objective's cotangents with respect to the phasors become CW adjoint sources
(Jz for E cotangents, Mx/My with the Yee transpose constant ``Q_MAG`` for H
cotangents, freq_adjoint.py:317-352), one adjoint run records the adjoint Ez
phasor on the design region, and the gradient is the per-frequency
contraction (freq_adjoint.py:85-91, 454-493)

    dL/dtheta_i = sum_k 2/(N_eff dt) eps_r Re[conj(Lambda_ki) conj(G_ki)],
    G = dca E/z + dcb (E - ca E/z)/cb,  z = exp(i w dt),  N_eff = sum env^2.

What runs where: both FDTD runs are ``gdn_tm_run_*`` calls (the adjoint
sources are synthesised on the device from their CW phasor weights, so no
(n_steps x n_sources) waveform table is built); the cotangents come from
torch autograd of the user objective on the phasors (the objective
reductions themselves are CUDA kernels, see monitors.py); the contraction is
``gdn_tm_adjoint_contract``. The backward-pass state is O(design x freq),
independent of the number of steps.

torch's complex gradient of a real loss is dL/dRe + i dL/dIm, the complex
conjugate of the value jax.grad returns; the adjoint weights below take the
conjugate so the source phases match the reference.
"""

from __future__ import annotations

import ctypes
from typing import NamedTuple

import numpy as np
import torch

from gradenna_b200 import _native
from gradenna_b200.constants import EPS0, MU0
from gradenna_b200.cpml import CPMLSpec
from gradenna_b200.fdtd2d import DZ, Port, simulate_tm
from gradenna_b200.grid import Grid2D

__all__ = [
    "Q_MAG", "FreqPhasors", "simulate_tm_freq", "freq_adjoint_gradient", "FreqAdjointObjective",
    "freq_adjoint_objective",
]

#: Yee transpose constant coupling a magnetic-current cotangent into the
#: adjoint Ez phasor, Q_MAG = -eps0/mu0 (freq_adjoint.py:141-154).
Q_MAG = -EPS0 / MU0

_native.register("gdn_tm_adjoint_contract", ctypes.c_int, [
    ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
    ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p])

#: gdn_tm_adjoint_contract flag: scale by eps_r (1 + h) instead of eps_r.
CONTRACT_EXACT_LOSS = 1


class FreqPhasors(NamedTuple):
    """Phasors handed to objectives (freq_adjoint.py:157-171)."""

    dft_ez: torch.Tensor
    dft_hx: torch.Tensor
    dft_hy: torch.Tensor
    port_v: torch.Tensor | None = None
    port_i: torch.Tensor | None = None


def _region_bounds(design_region, shape):
    out = []
    for s, n in zip(design_region, shape):
        if not isinstance(s, slice) or s.step not in (None, 1):
            raise ValueError("design_region must be a tuple of step-1 slices")
        a, b, _ = s.indices(n)
        out.append((a, b))
    return out


def _full_eps_sigma(grid, design_sigma, design_eps_r, design_region, device):
    """Vacuum background with the design values on design_region (freq_adjoint.py:214-221)."""
    eps_r = torch.ones(grid.shape, dtype=torch.float64, device=device)
    sigma = torch.zeros(grid.shape, dtype=torch.float64, device=device)
    if design_eps_r is not None:
        eps_r[design_region] = torch.as_tensor(design_eps_r, dtype=torch.float64, device=device)
    if design_sigma is not None:
        sigma[design_region] = torch.as_tensor(design_sigma, dtype=torch.float64, device=device)
    return eps_r, sigma


def _port_cells(ports):
    return [tuple(int(v) for v in (p if isinstance(p, Port) else Port(*p)).ij) for p in ports]


def ports_from_fields(dft_ez, dft_hx, dft_hy, grid, port_cells, freqs):
    """(V_hat, I_hat) rebuilt from the field phasors (freq_adjoint.py:536-558):
    V = -DZ z^{-1/2} (E/z + E)/2, I = (Hy[i]-Hy[i-1]) dy - (Hx[j]-Hx[j-1]) dx."""
    om = torch.as_tensor(2 * np.pi * np.asarray(freqs, np.float64), device=dft_ez.device)
    z = torch.exp(1j * om * grid.dt)
    half = torch.exp(0.5j * om * grid.dt)
    vh, ih = [], []
    for (i, j) in port_cells:
        ez = dft_ez[:, i, j]
        vh.append(-DZ * 0.5 * (ez / z + ez) * half)
        ih.append((dft_hy[:, i, j] - dft_hy[:, i - 1, j]) * grid.dy
                  - (dft_hx[:, i, j] - dft_hx[:, i, j - 1]) * grid.dx)
    return torch.stack(vh, dim=1), torch.stack(ih, dim=1)


def simulate_tm_freq(grid: Grid2D, *, design_sigma=None, design_eps_r=None, design_region,
                     dft_freqs, source_ij=None, source_current=None, ports=(),
                     cpml: CPMLSpec = CPMLSpec(), dtype=torch.float64, device=None) -> FreqPhasors:
    """Forward run returning full-grid complex128 phasors (freq_adjoint.py:224-261)."""
    dev = _native.require_cuda(device)
    eps_r, sigma = _full_eps_sigma(grid, design_sigma, design_eps_r, design_region, dev)
    res = simulate_tm(grid, source_ij=source_ij, source_current=source_current, eps_r=eps_r,
                      sigma=sigma, ports=ports, dft_freqs=dft_freqs, dft_dtype=np.complex128,
                      cpml=cpml, dtype=dtype, device=dev)
    port_v = port_i = None
    if res.port_v is not None:
        from gradenna_b200.sparams import port_dft

        port_v, port_i = port_dft(res.port_v, res.port_i, grid.dt, dft_freqs)
    return FreqPhasors(res.dft_ez, res.dft_hx, res.dft_hy, port_v, port_i)


class _Plan(NamedTuple):
    grid: Grid2D
    freqs: tuple
    env: np.ndarray
    design_region: tuple
    bounds: list
    source_ij: object
    source_current: object
    ports: tuple
    cpml: CPMLSpec
    dtype: torch.dtype
    device: torch.device
    objective_monitors: list | None
    exact: bool = True


def _forward_kwargs(plan: _Plan, eps_r, sigma):
    """simulate_tm keyword arguments of the forward CW run: design-region Ez
    plus the objective's phasors."""
    g = plan.grid
    (a0, a1), (b0, b1) = plan.bounds
    mons = [(0, a0, b0, a1, b1)]
    if plan.objective_monitors is None:
        mons += [(0, 0, 0, g.nx, g.ny), (1, 0, 0, g.nx, g.ny - 1), (2, 0, 0, g.nx - 1, g.ny)]
    else:
        mons += list(plan.objective_monitors)
    return dict(grid=g, source_ij=plan.source_ij, source_current=plan.source_current,
                eps_r=eps_r, sigma=sigma, ports=plan.ports, dft_freqs=plan.freqs,
                dft_dtype=np.complex128, cpml=plan.cpml, dtype=plan.dtype, device=plan.device,
                dft_monitors=mons)


def _forward(plan: _Plan, eps_r, sigma):
    """Forward CW run: design-region Ez plus the objective's phasors."""
    kw = _forward_kwargs(plan, eps_r, sigma)
    return simulate_tm(kw.pop("grid"), **kw)


def _scatter_full(plan: _Plan, res):
    """Objective phasors on full grids (zero outside the recorded boxes)."""
    g = plan.grid
    K = len(plan.freqs)
    shapes = ((g.nx, g.ny), (g.nx, g.ny - 1), (g.nx - 1, g.ny))
    full = [torch.zeros((K,) + s, dtype=torch.complex128, device=plan.device) for s in shapes]
    mons = ([(0, 0, 0, g.nx, g.ny), (1, 0, 0, g.nx, g.ny - 1), (2, 0, 0, g.nx - 1, g.ny)]
            if plan.objective_monitors is None else plan.objective_monitors)
    for (comp, lo0, lo1, hi0, hi1), t in zip(mons, res.monitors[1:]):
        full[comp][:, lo0:hi0, lo1:hi1] = t
    return full


def _objective_value(plan: _Plan, objective, full, fwd_res):
    pv = pi = None
    cells = _port_cells(plan.ports)
    if cells:
        pv, pi = ports_from_fields(full[0], full[1], full[2], plan.grid, cells, plan.freqs)
    return objective(FreqPhasors(full[0], full[1], full[2], pv, pi))


def _cotangents(plan: _Plan, objective, full, fwd_res):
    leaves = [t.detach().requires_grad_(True) for t in full]
    with torch.enable_grad():
        val = _objective_value(plan, objective, leaves, fwd_res)
        grads = torch.autograd.grad(val, leaves, allow_unused=True)
    out = []
    for t, gr in zip(leaves, grads):
        out.append(torch.zeros_like(t) if gr is None else gr.conj())
    return val.detach(), out


def _adjoint_sources(plan: _Plan, cot):
    """CW adjoint source cells and weights (freq_adjoint.py:317-352)."""
    g = plan.grid
    dt = g.dt
    cb_src = (dt / EPS0) / (g.dx * g.dy)
    dt_mu = dt / MU0
    out = []
    for w, basis in ((cot[0], 1.0 / (-cb_src)), (cot[1], Q_MAG / (-dt_mu)),
                     (cot[2], Q_MAG / (-dt_mu))):
        active = torch.any(w.abs() > 0, dim=0)
        idx = torch.nonzero(active)
        if idx.shape[0] == 0:
            out.append((None, None))
            continue
        wv = w[:, idx[:, 0], idx[:, 1]].T.contiguous() * basis  # (M, K)
        out.append((idx.cpu().numpy().astype(np.int32), wv))
    return out


def _fusable(plan: _Plan, objective):
    """True when the objective has a fused device evaluation for this run:
    its frequencies are the run's and the forward run recorded boxes."""
    return (getattr(objective, "fused_tm", None) is not None
            and plan.objective_monitors is not None
            and tuple(getattr(objective, "freqs", ())) == plan.freqs)


def _objective_sources(plan: _Plan, objective, fwd):
    """(objective value, adjoint CW sources) of the forward run. An objective
    with a fused device evaluation (gradenna_b200.objectives) takes one
    kernel launch on the recorded monitor boxes; any other objective goes
    through full-grid phasors and torch autograd."""
    if _fusable(plan, objective):
        val, _, _, lists = objective.fused_tm(list(plan.objective_monitors),
                                              list(fwd.monitors[1:]), plan.device)
        return val, [(idx, w) if len(idx) else (None, None) for idx, w in lists]
    full = _scatter_full(plan, fwd)
    val, cot = _cotangents(plan, objective, full, fwd)
    return val, _adjoint_sources(plan, cot)


def _adjoint_kwargs(plan: _Plan, eps_r, sigma, srcs):
    """simulate_tm keyword arguments of the adjoint run (None without sources)."""
    (a0, a1), (b0, b1) = plan.bounds
    (jz_idx, jz_w), (mx_idx, mx_w), (my_idx, my_w) = srcs
    if jz_idx is None and mx_idx is None and my_idx is None:
        return None
    # The reference's adjoint run has no ports (freq_adjoint.py:437-450). A
    # lumped port is a resistor in the medium, so the exact adjoint keeps it
    # as a passive load (no source voltage).
    ports = tuple(Port(p.ij, p.resistance, None) for p in plan.ports) if plan.exact else ()
    return dict(grid=plan.grid, source_ij=jz_idx, eps_r=eps_r, sigma=sigma, mx_ij=mx_idx,
                my_ij=my_idx, ports=ports, dft_freqs=plan.freqs, dft_dtype=np.complex128,
                cpml=plan.cpml, dtype=plan.dtype, device=plan.device,
                dft_monitors=[(0, a0, b0, a1, b1)],
                cw_sources=dict(env=plan.env, src_w=jz_w, mx_w=mx_w, my_w=my_w))


def _adjoint_run(plan: _Plan, eps_r, sigma, srcs):
    kw = _adjoint_kwargs(plan, eps_r, sigma, srcs)
    if kw is None:
        return None
    return simulate_tm(kw.pop("grid"), **kw)


def _contract(plan: _Plan, eps_r, sigma, e_d, lam_d, want_sigma, want_eps):
    g = plan.grid
    dt = g.dt
    K = len(plan.freqs)
    n_eff = float(np.sum(plan.env**2))
    k_norm = 2.0 / (n_eff * dt)
    om = 2 * np.pi * np.asarray(plan.freqs, np.float64)
    z = torch.as_tensor(np.exp(1j * om * dt), device=plan.device)
    dr = plan.design_region
    er = eps_r[dr].contiguous().reshape(-1)
    sg = sigma[dr].contiguous().reshape(-1)
    n_cells = er.numel()
    e = e_d.reshape(K, -1).contiguous()
    lam = lam_d.reshape(K, -1).contiguous()
    gs = torch.empty(n_cells, dtype=torch.float64, device=plan.device) if want_sigma else None
    ge = torch.empty(n_cells, dtype=torch.float64, device=plan.device) if want_eps else None
    lib = _native.load()
    stream = torch.cuda.current_stream(plan.device).cuda_stream
    with torch.cuda.device(plan.device):
        _native.check(lib.gdn_tm_adjoint_contract(
            n_cells, K, dt, k_norm, e.data_ptr(), lam.data_ptr(), er.data_ptr(), sg.data_ptr(),
            z.data_ptr(), _native.ptr(gs), _native.ptr(ge),
            CONTRACT_EXACT_LOSS if plan.exact else 0, stream))
    shape = e_d.shape[1:]
    return (None if gs is None else gs.reshape(shape)), (None if ge is None else ge.reshape(shape))


def _make_plan(grid, design_region, dft_freqs, env, source_ij, source_current, ports, cpml,
               dtype, device, objective_monitors, exact=True):
    dev = _native.require_cuda(device)
    freqs = tuple(float(f) for f in dft_freqs)
    env = np.asarray(env.detach().cpu() if isinstance(env, torch.Tensor) else env, np.float64)
    bounds = _region_bounds(design_region, grid.shape)
    ports = tuple(p if isinstance(p, Port) else Port(*p) for p in ports)
    return _Plan(grid, freqs, env, tuple(design_region), bounds, source_ij, source_current, ports,
                 cpml, dtype, dev, objective_monitors, bool(exact))


def freq_adjoint_gradient(grid: Grid2D, objective, *, design_sigma=None, design_eps_r=None,
                          design_region, dft_freqs, env, source_ij=None, source_current=None,
                          ports=(), cpml: CPMLSpec = CPMLSpec(), backend: str = "cuda",
                          dtype=torch.float64, device=None, objective_monitors=None,
                          exact: bool = True):
    """Two-run frequency-domain adjoint gradient (freq_adjoint.py:355-493).

    ``objective`` maps FreqPhasors (torch complex128 on the device) to a real
    scalar tensor. ``source_current`` must be a CW drive at ``dft_freqs``
    under the turn-on envelope ``env``. Returns {"sigma": ..., "eps_r": ...}
    for the design variables supplied (float64 tensors on the device).

    ``backend`` is accepted for signature compatibility ("xla", "native",
    "cuda"); every run is the CUDA path. ``objective_monitors`` optionally
    lists the boxes (comp, lo_i, lo_j, hi_i, hi_j) the objective reads (like
    the reference's 3D DFTRegions); other phasors are then zero and the
    forward run records far less DFT data. ``dtype`` is the field dtype of
    both runs (float64 like the reference's freq-adjoint solves).
    ``exact`` (default) keeps the ports in the adjoint run as passive
    resistive loads and scales the contraction by eps_r (1 + sigma dt /
    (2 eps)), which makes the gradient match the exact time-domain gradient
    for port-driven and lossy designs; ``exact=False`` reproduces the
    reference's formulas (port-less adjoint run, eps_r scaling), which agree
    only for small sigma and no ports.
    """
    if backend not in ("xla", "native", "cuda"):
        raise ValueError(f"backend must be 'xla', 'native' or 'cuda', got {backend!r}")
    plan = _make_plan(grid, design_region, dft_freqs, env, source_ij, source_current, ports,
                      cpml, dtype, device, objective_monitors, exact)
    eps_r, sigma = _full_eps_sigma(grid, design_sigma, design_eps_r, design_region, plan.device)
    fwd = _forward(plan, eps_r, sigma)
    _, srcs = _objective_sources(plan, objective, fwd)
    adj = _adjoint_run(plan, eps_r, sigma, srcs)
    out = {}
    if adj is None:
        shp = tuple(b - a for a, b in plan.bounds)
        if design_sigma is not None:
            out["sigma"] = torch.zeros(shp, dtype=torch.float64, device=plan.device)
        if design_eps_r is not None:
            out["eps_r"] = torch.zeros(shp, dtype=torch.float64, device=plan.device)
        return out
    gs, ge = _contract(plan, eps_r, sigma, fwd.monitors[0], adj.monitors[0],
                       design_sigma is not None, design_eps_r is not None)
    if gs is not None:
        out["sigma"] = gs
    if ge is not None:
        out["eps_r"] = ge
    return out


class FreqAdjointObjective(torch.autograd.Function):
    """objective(design_sigma) whose backward is the two-run adjoint.

    forward: one CW forward run + the objective value; backward: cotangents,
    one adjoint run and the design contraction, scaled by the incoming grad.
    """

    @staticmethod
    def forward(ctx, design_sigma, plan, objective):
        eps_r, sigma = _full_eps_sigma(plan.grid, design_sigma, None, plan.design_region,
                                       plan.device)
        fwd = _forward(plan, eps_r, sigma)
        if _fusable(plan, objective):
            val, srcs = _objective_sources(plan, objective, fwd)
        else:
            srcs = None
            val = _objective_value(plan, objective, _scatter_full(plan, fwd), fwd)
        ctx.plan, ctx.objective = plan, objective
        ctx.state = (eps_r, sigma, fwd, srcs)
        return val.detach().to(torch.float64)

    @staticmethod
    def backward(ctx, g):
        plan = ctx.plan
        eps_r, sigma, fwd, srcs = ctx.state
        if srcs is None:
            _, srcs = _objective_sources(plan, ctx.objective, fwd)
        adj = _adjoint_run(plan, eps_r, sigma, srcs)
        if adj is None:
            return torch.zeros_like(sigma[plan.design_region]), None, None
        gs, _ = _contract(plan, eps_r, sigma, fwd.monitors[0], adj.monitors[0], True, False)
        return g * gs, None, None


def freq_adjoint_objective(design_sigma, grid: Grid2D, objective, *, design_region, dft_freqs,
                           env, source_ij=None, source_current=None, ports=(),
                           cpml: CPMLSpec = CPMLSpec(), dtype=torch.float64, device=None,
                           objective_monitors=None, exact: bool = True):
    """Differentiable objective value: ``.backward()`` runs the adjoint."""
    plan = _make_plan(grid, design_region, dft_freqs, env, source_ij, source_current, ports,
                      cpml, dtype, device, objective_monitors, exact)
    return FreqAdjointObjective.apply(design_sigma, plan, objective)


_3D_NAMES = ("FreqPhasors3D", "simulate_3d_freq", "port_dft_3d", "freq_adjoint_gradient_3d")


def __getattr__(name):
    # The reference keeps its 3D adjoint in this module (freq_adjoint.py:560-1065);
    # here it lives in freq_adjoint3d and is re-exported lazily.
    if name in _3D_NAMES:
        from gradenna_b200 import freq_adjoint3d

        return getattr(freq_adjoint3d, name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
