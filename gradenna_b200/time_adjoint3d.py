r"""Exact time-domain adjoint gradient of 3D objectives, with checkpointing.

The reference differentiates 3D objectives with jax.grad through the whole
time loop (exact_design_gradient_3d, freq_adjoint.py:724-771), keeping the
reverse-mode tape in ``checkpoint_segments`` segments (fdtd3d.py:735-749);
its frequency-domain adjoint needs a CW drive. This module gives the exact
gradient of the discrete 3D loop for any drive (pulse, multi-tone, CW) with
runs of this library's CUDA solver and no tape:

1. Forward run: the objective's DFT phasors (the boxes it reads, or every
   component) and the history of Ex, Ey and Ez on every design node.
2. Cotangents of the objective with respect to the phasors (torch autograd
   of the user objective). A phasor X_k = dt sum_n x^n exp(-i w_k t_n) puts
   the time-domain force f^n = dt sum_k Re(c_k exp(-i w_k t_n)) on the field
   sample x^n, c_k the conjugated cotangent (t_n = (n + 1) dt for E^{n+1},
   (n + 1/2) dt for H^{n+1/2}).
3. Adjoint run in the same medium (a lumped port stays as a passive load),
   driven by the forces played backwards in time: at adjoint step a, Jx / Jy
   / Jz sources -f_E^{N-1-a} / cb0 on every updated E edge the objective
   reads (cb0 = (dt / eps0) / area, area = dy dz, dx dz, dx dy: the vacuum
   source coefficient, whatever the cell's medium), and Mx / My / Mz sources
   (Q_MAG / (-dt / mu0)) f_H^{N-a} on every H edge it reads (one step after
   the E forces, Q_MAG = -eps0 / mu0, as in the frequency-domain adjoint).
4. Contraction on each design node, summed over its three E edges (the
   Yee update's reciprocity makes the adjoint variable of the step-n update
   of an edge eps_r (1 + h) times the adjoint run's field there at step
   N - n, h = sigma dt / (2 eps)):
       dL/dtheta = sum_edges eps_r (1 + h) sum_n L^{N-n}
                   (dca E^n + dcb (E^{n+1} - ca E^n) / cb),
   with the closed-form dca, dcb of freq_adjoint.py:186-206 evaluated with
   the edge's total conductivity (on the port's Ez edge the port's
   dz / (R dx dy) is added, which makes the port's semi-implicit update,
   drive included, the same formula).

The reciprocity that step 4 rests on holds for fields the objective reads
outside the CPML slabs (the design region is outside them too); inside a
slab the stretched update is not its own adjoint, and the gradient is
approximate there (a warning is issued), as for the frequency-domain
adjoint.

Checkpointing. With ``checkpoint_segments`` = S (it must divide n_steps, as
in the reference) the histories are never held whole: the forward pass
keeps the complete solver state (six fields and twelve CPML psi arrays, the
resumable state of gdn_yee_run_*) at the start of every segment; the
adjoint then runs segment by segment, and before each adjoint segment the
matching forward segment is recomputed from its checkpoint. Device memory
is S - 1 states plus two segment histories instead of two whole histories:
for a volumetric design of D nodes over N steps that is
(S - 1) * state + 2 * (N / S) * 3 D values, smallest near S = sqrt(N). The
price is one more forward pass (S - 1 recomputed segments). S = 1 (the
default) keeps the whole histories and needs one forward and one adjoint
run.

It matches torch autograd through the oracle's 3D loop (oracle/fdtd3d_ad.py)
to rounding in float64, for lossy and permittivity designs, CPML, E and H
objectives and a driven port inside the design region:
tests/test_time_adjoint3d_gpu.py.
"""

from __future__ import annotations

import warnings

import numpy as np
import torch

from gradenna_b200 import _native
from gradenna_b200 import dft_region as dr
from gradenna_b200 import freq_adjoint3d as fa3
from gradenna_b200.constants import EPS0, MU0
from gradenna_b200.cpml import CPMLSpec
from gradenna_b200.fdtd3d import simulate_3d
from gradenna_b200.freq_adjoint import Q_MAG
from gradenna_b200.grid import Grid3D

__all__ = ["time_domain_gradient_3d", "segment_bounds", "design_probes_3d"]

_NAMES = {0: ("source_x_ijk", "source_x_current"), 1: ("source_y_ijk", "source_y_current"),
          2: ("source_ijk", "source_current"), 3: ("mx_ijk", "mx_current"),
          4: ("my_ijk", "my_current"), 5: ("mz_ijk", "mz_current")}


def segment_bounds(n_steps: int, checkpoint_segments) -> list[tuple[int, int]]:
    """[(start, stop), ...] of the checkpoint segments; the count must divide
    n_steps (fdtd3d.py:738-741)."""
    s = 1 if checkpoint_segments is None else int(checkpoint_segments)
    if s <= 0 or n_steps % s != 0:
        raise ValueError(f"checkpoint_segments={checkpoint_segments} must divide "
                         f"n_steps={n_steps}")
    m = n_steps // s
    return [(q * m, (q + 1) * m) for q in range(s)]


def _updated_box(c, nx, ny, nz):
    """[lo, hi) of the E edges of component c that the update writes (the
    rest are PEC and stay zero)."""
    if c == 0:
        return (0, 1, 1), (nx - 1, ny - 1, nz - 1)
    if c == 1:
        return (1, 0, 1), (nx - 1, ny - 1, nz - 1)
    return (1, 1, 0), (nx - 1, ny - 1, nz - 1)


def design_probes_3d(grid: Grid3D, bounds):
    """Probe list of the design region's updated E edges.

    ``bounds`` = ((a0, a1), (b0, b1), (c0, c1)). Returns (ijk (P, 3) int32,
    comp (P,) int32 in 0..2, node (P,) int64 = the node's flat index in the
    design box)."""
    (a0, a1), (b0, b1), (c0, c1) = bounds
    ii, jj, kk = np.meshgrid(np.arange(a0, a1), np.arange(b0, b1), np.arange(c0, c1),
                             indexing="ij")
    cells = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], 1)
    node = np.arange(cells.shape[0], dtype=np.int64)
    ijk, comp, pos = [], [], []
    for c in range(3):
        lo, hi = _updated_box(c, grid.nx, grid.ny, grid.nz)
        ok = np.all((cells >= lo) & (cells < hi), axis=1)
        ijk.append(cells[ok])
        comp.append(np.full(int(ok.sum()), c, np.int32))
        pos.append(node[ok])
    return (np.ascontiguousarray(np.concatenate(ijk), np.int32), np.concatenate(comp),
            np.concatenate(pos))


def _adjoint_channels(grid: Grid3D, cot, npml: int = 0):
    """{comp: (idx (m, 3) int32, w (K, m) complex128)} of the cotangents'
    active edges (E edges only where the update writes them). Warns when an
    active edge lies within reach of a CPML slab."""
    out = {}
    lim = np.array([grid.nx, grid.ny, grid.nz]) - 2 - npml
    for c, w in enumerate(cot):
        if w is None:
            continue
        active = torch.any(w.abs() > 0, dim=0)
        if c < 3:
            lo, hi = _updated_box(c, grid.nx, grid.ny, grid.nz)
            keep = torch.zeros_like(active)
            keep[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = True
            active &= keep
        idx = torch.nonzero(active)
        if idx.shape[0] == 0:
            continue
        ijk = idx.cpu().numpy().astype(np.int32)
        if npml > 0 and np.any((ijk < npml + 1) | (ijk > lim)):
            warnings.warn("the objective reads fields inside the CPML; the time-domain "
                          "adjoint is exact only outside the absorbing slabs", stacklevel=3)
        out[c] = (ijk, w[:, idx[:, 0], idx[:, 1], idx[:, 2]].to(torch.complex128).contiguous())
    return out


def _adjoint_waves(grid: Grid3D, chans, freqs, n_steps, a0, a1, dtype, device):
    """simulate_3d keyword arguments of the adjoint drive for adjoint steps
    a0 .. a1 - 1 (time-reversed forces, H forces one step later)."""
    dt = grid.dt
    om = torch.as_tensor(2 * np.pi * np.asarray(freqs, np.float64), device=device)
    a = torch.arange(a0, a1, dtype=torch.float64, device=device)
    area = (grid.dy * grid.dz, grid.dx * grid.dz, grid.dx * grid.dy)
    kw = {}
    for c, (idx, w) in chans.items():
        if c < 3:
            t = (n_steps - 1 - a) + 1.0            # E^{n+1}, n = N - 1 - a
            basis = 1.0 / (-(dt / EPS0) / area[c])
        else:
            t = (n_steps - a) + 0.5                # H^{n+1/2}, n = N - a
            basis = Q_MAG / (-(dt / MU0))
        ph = torch.exp(-1j * torch.outer(t, om) * dt)          # (rows, K)
        wave = (ph @ w).real * (dt * basis)
        if c >= 3 and a0 == 0:
            wave[0] = 0.0                          # no H force at the first adjoint step
        kw[_NAMES[c][0]] = idx
        kw[_NAMES[c][1]] = wave.to(dtype).contiguous()
    return kw


def _coefficients(eps_r_p, sig_p, dt):
    """Per-edge scale eps_r (1 + h) and the sigma / eps_r contraction weights
    of E^n and E^{n+1}: d/dtheta = scale (u0 S0 + u1 S1)."""
    eps = EPS0 * eps_r_p
    h = sig_p * dt / (2 * eps)
    ca = (1 - h) / (1 + h)
    cb = (dt / eps) / (1 + h)
    den = (1 + h) ** 2
    scale = eps_r_p * (1 + h)
    out = {}
    dca = (-dt / eps) / den
    dcb = (-(dt / eps) * (dt / (2 * eps))) / den
    out["sigma"] = (dca - dcb * ca / cb, dcb / cb)
    dca = EPS0 * ((sig_p * dt / (eps * eps)) / den)
    dcb = EPS0 * ((-(dt / (eps * eps))) / den)
    out["eps_r"] = (dca - dcb * ca / cb, dcb / cb)
    return scale, out


def _sum_into(acc, new):
    if acc is None:
        return list(new)
    return [a if b is None else (b if a is None else a + b) for a, b in zip(acc, new)]


def time_domain_gradient_3d(grid: Grid3D, objective, *, design_sigma=None, design_eps_r=None,
                            design_region, dft_freqs, source_ijk=None, source_current=None,
                            port_ijk=None, port_voltage=None, port_resistance: float = 50.0,
                            cpml: CPMLSpec = CPMLSpec(), checkpoint_segments=None,
                            dtype=torch.float64, device=None, eps_r_background=None,
                            sigma_background=None, objective_kind=None, box_margin=None,
                            monitor_region=None, return_value: bool = False):
    """Exact gradient of ``objective(FreqPhasors3D)`` through the 3D time
    loop, for any drive.

    Arguments as ``freq_adjoint_gradient_3d`` without ``env`` (the drive's
    own waveform defines the run), plus ``checkpoint_segments`` (the
    reference's name, fdtd3d.py:735-749): None or 1 keeps whole design
    histories; S > 1 keeps S - 1 solver states and recomputes each segment
    (module docstring). ``objective_kind`` / ``box_margin`` /
    ``monitor_region`` limit the forward DFT to what the objective reads.
    Returns {"sigma": ..., "eps_r": ...} float64 tensors of the design shape
    for the design variables given (and the objective value with
    ``return_value``).
    """
    if design_sigma is None and design_eps_r is None:
        raise ValueError("give design_sigma and/or design_eps_r")
    dev = _native.require_cuda(device)
    freqs = tuple(float(f) for f in dft_freqs)
    if source_current is not None:
        n_steps = int(np.shape(source_current)[0])
    elif port_voltage is not None:
        n_steps = int(np.size(port_voltage) if not isinstance(port_voltage, torch.Tensor)
                      else port_voltage.numel())
    else:
        raise ValueError("need source_current or a driven port")
    segs = segment_bounds(n_steps, checkpoint_segments)
    fdt = dtype
    eps_r, sigma = fa3._full_eps_sigma_3d(grid, design_sigma, design_eps_r, design_region, dev,
                                          eps_r_background, sigma_background)
    bounds = [s.indices(n)[:2] for s, n in zip(design_region, grid.shape)]
    shape = tuple(b - a for a, b in bounds)
    pijk, pcomp, pnode = design_probes_3d(grid, bounds)
    shapes = dr.full_field_shapes(grid.nx, grid.ny, grid.nz)
    boxes = None
    if objective_kind is not None:
        boxes = fa3._objective_boxes(grid, objective_kind, port_ijk=port_ijk,
                                     box_margin=box_margin, monitor_region=monitor_region)
    port = None if port_ijk is None else tuple(int(v) for v in np.asarray(port_ijk).reshape(3))

    def rows(a, s0, s1):
        if a is None:
            return None
        t = a if isinstance(a, torch.Tensor) else torch.as_tensor(np.asarray(a))
        return t[s0:s1]

    common = dict(eps_r=eps_r, sigma=sigma, cpml=cpml, dtype=fdt, device=dev,
                  probe_ijk=pijk, probe_comp=pcomp)

    def forward_segment(q, state, keep_state, with_dft):
        s0, s1 = segs[q]
        kw = dict(source_ijk=source_ijk, source_current=rows(source_current, s0, s1))
        if port is not None:
            kw.update(port_ijk=port, port_voltage=rows(port_voltage, s0, s1),
                      port_resistance=port_resistance)
        if with_dft:
            kw.update(dft_freqs=freqs, dft_dtype=np.complex128, dft_monitors=boxes,
                      dft_step0=s0)
        return simulate_3d(grid, state_in=state, return_state=keep_state, **kw, **common)

    # Forward pass: phasors, port records, checkpoints, the design E at each
    # segment's end and the last segment's whole history.
    S = len(segs)
    ckpt = [None] * S
    e_end = [None] * S
    phas = None
    pv_t, pi_t = [], []
    state = None
    last_hist = None
    for q in range(S):
        r = forward_segment(q, state, q < S - 1, True)
        if boxes is None:
            d = r.dft
            new = [d.ex, d.ey, d.ez, d.hx, d.hy, d.hz]
        else:
            ft = torch.as_tensor(np.asarray(freqs), device=dev)
            d = dr.boxes_to_full(ft, boxes, r.monitors, shapes)
            new = [d.ex, d.ey, d.ez, d.hx, d.hy, d.hz]
        phas = _sum_into(phas, new)
        if r.port_v is not None:
            pv_t.append(r.port_v)
            pi_t.append(r.port_i)
        e_end[q] = r.probe_ez[-1].clone()
        if q == S - 1:
            last_hist = r.probe_ez
        state = r.state
        if q < S - 1:
            ckpt[q + 1] = r.state
        del r
    ckpt[0] = None

    # Objective value and cotangents (torch's complex gradient is the
    # conjugate of jax's).
    comps = [p if p is not None else torch.zeros((len(freqs),) + tuple(s), dtype=torch.complex128,
                                                 device=dev)
             for p, s in zip(phas, shapes)]
    leaves = [t.detach().requires_grad_(True) for t in comps]
    with torch.enable_grad():
        pv = pi = None
        if port is not None:
            pv, pi = fa3._port_v_i_3d(leaves[2], leaves[3], leaves[4], grid, port, freqs)
        val = objective(fa3.FreqPhasors3D(*leaves, pv, pi))
        grads = torch.autograd.grad(val, leaves, allow_unused=True)
    cot = [None if g is None else g.conj().resolve_conj() for g in grads]
    chans = _adjoint_channels(grid, cot, cpml.thickness)

    out = {}
    want = [k for k, v in (("sigma", design_sigma), ("eps_r", design_eps_r)) if v is not None]
    if not chans or pijk.shape[0] == 0:
        for k in want:
            out[k] = torch.zeros(shape, dtype=torch.float64, device=dev)
        return (out, float(val.detach())) if return_value else out

    # Per-edge coefficients; the port's Ez edge carries the port conductance.
    ii = torch.as_tensor(pijk.astype(np.int64), device=dev)
    er_p = eps_r[ii[:, 0], ii[:, 1], ii[:, 2]].to(torch.float64)
    sg_p = sigma[ii[:, 0], ii[:, 1], ii[:, 2]].to(torch.float64).clone()
    if port is not None:
        on_port = torch.as_tensor((pcomp == 2) & np.all(pijk == np.asarray(port), axis=1),
                                  device=dev)
        sg_p[on_port] += grid.dz / (float(port_resistance) * grid.dx * grid.dy)
    scale, u = _coefficients(er_p, sg_p, grid.dt)

    # Adjoint pass, segment by segment in adjoint time (forward segments in
    # reverse), each paired with its recomputed forward history.
    acc0 = torch.zeros_like(er_p)
    acc1 = torch.zeros_like(er_p)
    astate = None
    for p in range(S):
        q = S - 1 - p
        a0, a1 = p * (n_steps // S), (p + 1) * (n_steps // S)
        if q == S - 1:
            e_seg = last_hist
        else:
            e_seg = forward_segment(q, ckpt[q], False, False).probe_ez
            ckpt[q + 1] = None  # the state after segment q is no longer needed
        e_prev = e_end[q - 1] if q > 0 else torch.zeros_like(e_end[0])
        kw = _adjoint_waves(grid, chans, freqs, n_steps, a0, a1, fdt, dev)
        if port is not None:
            kw.update(port_ijk=port, port_voltage=torch.zeros(a1 - a0, dtype=fdt, device=dev),
                      port_resistance=port_resistance)
        ar = simulate_3d(grid, state_in=astate, return_state=p < S - 1, **kw, **common)
        lam = torch.flip(ar.probe_ez, [0]).to(torch.float64)   # rows n = start .. stop - 1
        e1 = e_seg.to(torch.float64)                            # E^{n+1}
        e0 = torch.cat([e_prev[None], e_seg[:-1]]).to(torch.float64)  # E^n
        acc1 += (lam * e1).sum(0)
        acc0 += (lam * e0).sum(0)
        astate = ar.state
        del ar, e_seg
    node = torch.as_tensor(pnode, device=dev)
    n_nodes = int(np.prod(shape))
    for k in want:
        u0, u1 = u[k]
        edge = scale * (u0 * acc0 + u1 * acc1)
        g = torch.zeros(n_nodes, dtype=torch.float64, device=dev)
        g.index_add_(0, node, edge)
        out[k] = g.reshape(shape)
    return (out, float(val.detach())) if return_value else out
