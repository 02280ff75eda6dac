"""Test infrastructure: the exact time-domain gradient of the 2D TM solver.

The reference's gradient oracle is jax.grad through simulate_tm, i.e. the
reverse sweep of the whole discrete time loop
(src/gradenna/freq_adjoint.py:269-309 exact_design_gradient, and
README.md:24-39). jax is not available here, so this module restates the
same time loop (the numpy oracle's, oracle/fdtd2d_np.py, which follows
fdtd2d.py:343-487 line for line) in torch float64 on the CPU and lets torch
autograd form the reverse sweep. Segments of ``segment`` steps are
recomputed in the backward pass (torch.utils.checkpoint), the sqrt(N)
checkpointing of fdtd3d.py:735-749, so memory stays O(N / segment + segment)
states.

Only tests use it, as the checker of the GPU frequency-domain adjoint.
"""

from __future__ import annotations

import numpy as np
import torch
from torch.utils.checkpoint import checkpoint

from oracle import fdtd2d_np as onp

DT = torch.float64


def _psi_step(psi, diff, b, c, m, axis, inv_kappa):
    """cpml.py:120-158 on both slabs of `axis` (restates onp.psi_step)."""
    if m == 0:
        return psi, diff
    n = diff.shape[axis]
    lo, mid, hi = diff.narrow(axis, 0, m), diff.narrow(axis, m, n - 2 * m), diff.narrow(axis, n - m, m)
    shape = [1, 1]
    shape[axis] = m
    p_lo = b[:m].reshape(shape) * psi[0] + c[:m].reshape(shape) * lo
    p_hi = b[n - m:].reshape(shape) * psi[1] + c[n - m:].reshape(shape) * hi
    k_lo = inv_kappa.narrow(axis, 0, m)
    k_hi = inv_kappa.narrow(axis, n - m, m)
    term = torch.cat([lo * k_lo + p_lo, mid, hi * k_hi + p_hi], dim=axis)
    return (p_lo, p_hi), term


def simulate_tm_ad(grid, *, eps_r, sigma, source_ij=None, source_current=None, ports=(),
                   dft_freqs=(), cpml=onp.CPMLSpec(), segment: int = 200):
    """Differentiable float64 restatement of simulate_tm (fdtd2d.py:343-487).

    ``eps_r`` and ``sigma`` are (nx, ny) torch tensors (they may require
    grad); everything runs on their device (plain torch operations, so a
    CUDA device only makes the checker faster). Returns (dft_ez, dft_hx, dft_hy, port_v, port_i) with complex128
    full-grid phasors and (n_steps, n_ports) series.
    """
    nx, ny = grid.nx, grid.ny
    dt = grid.dt
    dev = sigma.device
    T = lambda a: torch.as_tensor(a, device=dev)  # noqa: E731
    ports = tuple(p if isinstance(p, onp.Port) else onp.Port(*p) for p in ports)
    src = None
    if source_current is not None:
        cur = T(np.asarray(source_current, np.float64))
        cur = cur[:, None] if cur.ndim == 1 else cur
        sidx = np.asarray(source_ij, np.int64).reshape(-1, 2)
        src = (sidx, cur)
        n_steps = cur.shape[0]
    for p in ports:
        if p.voltage is not None:
            n_steps = len(p.voltage)
    eps = onp.EPS0 * eps_r
    sig = sigma.clone()
    if ports:
        pidx = np.asarray([p.ij for p in ports], np.int64)
        rs = T(np.asarray([float(p.resistance) for p in ports], np.float64))
        sig = sig.index_put((T(pidx[:, 0]), T(pidx[:, 1])),
                            onp.DZ / (rs * grid.dx * grid.dy), accumulate=True)
        vs = torch.stack([torch.zeros(n_steps, dtype=DT, device=dev) if p.voltage is None
                          else T(np.asarray(p.voltage, np.float64)) for p in ports], 1)
    half = sig * dt / (2.0 * eps)
    ca = (1.0 - half) / (1.0 + half)
    cb = (dt / eps) / (1.0 + half)
    m = cpml.thickness
    tab = {}
    for key, (n, d, hf) in {"x_e": (nx, grid.dx, False), "x_h": (nx, grid.dx, True),
                            "y_e": (ny, grid.dy, False), "y_h": (ny, grid.dy, True)}.items():
        a = onp.axis_coefficients(n, d, dt, cpml, half=hf, dtype=np.float64)
        tab[key] = tuple(T(np.ascontiguousarray(v)) for v in (a.b, a.c, a.inv_kappa))
    kx_e = tab["x_e"][2][1:-1, None]
    ky_e = tab["y_e"][2][None, 1:-1]
    kx_h = tab["x_h"][2][:, None]
    ky_h = tab["y_h"][2][None, :]
    inv_dx, inv_dy = 1.0 / grid.dx, 1.0 / grid.dy
    dt_mu = dt / onp.MU0
    if src is not None:
        si, sj = T(src[0][:, 0]), T(src[0][:, 1])
        cb_src = cb[si, sj] * (inv_dx * inv_dy)
    if ports:
        pi, pj = T(pidx[:, 0]), T(pidx[:, 1])
        cb_vs = cb[pi, pj] / (rs * grid.dx * grid.dy)
    fr = np.asarray(dft_freqs, np.float64)
    nn = np.arange(n_steps, dtype=np.float64)
    ph_e = T(np.exp(-2j * np.pi * np.outer(nn + 1.0, fr) * dt))
    ph_h = T(np.exp(-2j * np.pi * np.outer(nn + 0.5, fr) * dt))
    K = len(fr)

    def step_range(n0, n1, ca, cb, state):
        (ez, hx, hy, pxy0, pxy1, pyx0, pyx1, pzx0, pzx1, pzy0, pzy1, ae_r, ae_i, ax_r, ax_i,
         ay_r, ay_i) = state
        ae = torch.complex(ae_r, ae_i)
        ax = torch.complex(ax_r, ax_i)
        ay = torch.complex(ay_r, ay_i)
        vv, ii = [], []
        for n in range(n0, n1):
            dez_dy = (ez[:, 1:] - ez[:, :-1]) * inv_dy
            (pxy0, pxy1), t_hx = _psi_step((pxy0, pxy1), dez_dy, tab["y_h"][0], tab["y_h"][1], m,
                                           1, ky_h)
            hx = hx - dt_mu * t_hx
            dez_dx = (ez[1:, :] - ez[:-1, :]) * inv_dx
            (pyx0, pyx1), t_hy = _psi_step((pyx0, pyx1), dez_dx, tab["x_h"][0], tab["x_h"][1], m,
                                           0, kx_h)
            hy = hy + dt_mu * t_hy
            if ports:
                i_port = ((hy[pi, pj] - hy[pi - 1, pj]) * grid.dy
                          - (hx[pi, pj] - hx[pi, pj - 1]) * grid.dx)
                ez_before = ez[pi, pj]
            dhy_dx = (hy[1:, 1:-1] - hy[:-1, 1:-1]) * inv_dx
            dhx_dy = (hx[1:-1, 1:] - hx[1:-1, :-1]) * inv_dy
            (pzx0, pzx1), tx = _psi_step((pzx0, pzx1), dhy_dx, tab["x_e"][0][1:-1],
                                         tab["x_e"][1][1:-1], m, 0, kx_e)
            (pzy0, pzy1), ty = _psi_step((pzy0, pzy1), dhx_dy, tab["y_e"][0][1:-1],
                                         tab["y_e"][1][1:-1], m, 1, ky_e)
            inner = ca[1:-1, 1:-1] * ez[1:-1, 1:-1] + cb[1:-1, 1:-1] * (tx - ty)
            ez = torch.nn.functional.pad(inner, (1, 1, 1, 1))
            if src is not None:
                ez = ez.index_put((si, sj), -cb_src * src[1][n], accumulate=True)
            if ports:
                ez = ez.index_put((pi, pj), -cb_vs * vs[n], accumulate=True)
                vv.append(-0.5 * onp.DZ * (ez_before + ez[pi, pj]))
                ii.append(i_port)
            if K:
                ae = ae + ph_e[n][:, None, None] * ez
                ax = ax + ph_h[n][:, None, None] * hx
                ay = ay + ph_h[n][:, None, None] * hy
        vt = torch.stack(vv) if vv else torch.zeros((n1 - n0, 0), dtype=DT, device=dev)
        it = torch.stack(ii) if ii else torch.zeros((n1 - n0, 0), dtype=DT, device=dev)
        return (ez, hx, hy, pxy0, pxy1, pyx0, pyx1, pzx0, pzx1, pzy0, pzy1, ae.real, ae.imag,
                ax.real, ax.imag, ay.real, ay.imag, vt, it)

    z = lambda *s: torch.zeros(s, dtype=DT, device=dev)  # noqa: E731
    state = (z(nx, ny), z(nx, ny - 1), z(nx - 1, ny), z(nx, m), z(nx, m), z(m, ny), z(m, ny),
             z(m, ny - 2), z(m, ny - 2), z(nx - 2, m), z(nx - 2, m), z(K, nx, ny), z(K, nx, ny),
             z(K, nx, ny - 1), z(K, nx, ny - 1), z(K, nx - 1, ny), z(K, nx - 1, ny))
    vs_out, is_out = [], []
    for n0 in range(0, n_steps, segment):
        n1 = min(n_steps, n0 + segment)
        out = checkpoint(step_range, n0, n1, ca, cb, state, use_reentrant=False)
        state, vt, it = out[:17], out[17], out[18]
        vs_out.append(vt)
        is_out.append(it)
    dft_ez = torch.complex(state[11], state[12]) * dt
    dft_hx = torch.complex(state[13], state[14]) * dt
    dft_hy = torch.complex(state[15], state[16]) * dt
    pv = torch.cat(vs_out) if ports else None
    pcur = torch.cat(is_out) if ports else None
    return dft_ez, dft_hx, dft_hy, pv, pcur


def exact_design_gradient(grid, objective, *, design_sigma=None, design_eps_r=None, design_region,
                          dft_freqs, source_ij=None, source_current=None, ports=(),
                          cpml=onp.CPMLSpec(), segment: int = 200, device="cpu"):
    """d objective / d design through the whole time loop (the reference's
    exact_design_gradient, freq_adjoint.py:269-309, with torch autograd in
    place of jax.grad). ``objective(dft_ez, dft_hx, dft_hy, port_v, port_i)``
    returns a real scalar tensor; port_v / port_i are the time series.
    Returns {"sigma": ..., "eps_r": ...} numpy arrays for the design
    variables given.
    """
    nx, ny = grid.nx, grid.ny
    leaves = {}
    eps_r = torch.ones((nx, ny), dtype=DT, device=device)
    sigma = torch.zeros((nx, ny), dtype=DT, device=device)
    idx = tuple(t.to(device) for t in _region_index(design_region, nx, ny))
    if design_sigma is not None:
        leaves["sigma"] = torch.as_tensor(np.asarray(design_sigma, np.float64),
                                          device=device).requires_grad_(True)
        sigma = sigma.index_put(idx, leaves["sigma"].reshape(-1))
    if design_eps_r is not None:
        leaves["eps_r"] = torch.as_tensor(np.asarray(design_eps_r, np.float64),
                                          device=device).requires_grad_(True)
        eps_r = eps_r.index_put(idx, leaves["eps_r"].reshape(-1))
    out = simulate_tm_ad(grid, eps_r=eps_r, sigma=sigma, source_ij=source_ij,
                         source_current=source_current, ports=ports, dft_freqs=dft_freqs,
                         cpml=cpml, segment=segment)
    val = objective(*out)
    grads = torch.autograd.grad(val, list(leaves.values()))
    return {k: g.detach().cpu().numpy() for k, g in zip(leaves, grads)}, float(val.detach())


def _region_index(region, nx, ny):
    ii = np.arange(nx)[region[0]]
    jj = np.arange(ny)[region[1]]
    I, J = np.meshgrid(ii, jj, indexing="ij")
    return torch.as_tensor(I.reshape(-1)), torch.as_tensor(J.reshape(-1))


def half_step_dft_t(x_t, dt, freqs):
    """sparams.py:24-46 in torch (differentiable)."""
    fr = np.atleast_1d(np.asarray(freqs, np.float64))
    t = (np.arange(x_t.shape[0]) + 0.5) * dt
    kern = torch.as_tensor(np.exp(-2j * np.pi * fr[:, None] * t[None, :]) * dt, device=x_t.device)
    return kern @ x_t.to(torch.complex128)


def poynting_flux_box_2d_t(dft_ez, dft_hx, dft_hy, grid, box):
    """monitors.py:20-70 in torch (restates onp.poynting_flux_box_2d)."""
    il, ir, jb, jt = (int(v) for v in box)
    dx, dy = grid.dx, grid.dy
    js, isl = slice(jb + 1, jt + 1), slice(il + 1, ir + 1)
    re = lambda a, b: torch.real(a * torch.conj(b))  # noqa: E731
    p = -0.5 * re(0.5 * (dft_ez[:, ir, js] + dft_ez[:, ir + 1, js]), dft_hy[:, ir, js]).sum(-1) * dy
    p = p + 0.5 * re(0.5 * (dft_ez[:, il, js] + dft_ez[:, il + 1, js]), dft_hy[:, il, js]).sum(-1) * dy
    p = p + 0.5 * re(0.5 * (dft_ez[:, isl, jt] + dft_ez[:, isl, jt + 1]), dft_hx[:, isl, jt]).sum(-1) * dx
    p = p - 0.5 * re(0.5 * (dft_ez[:, isl, jb] + dft_ez[:, isl, jb + 1]), dft_hx[:, isl, jb]).sum(-1) * dx
    return p



