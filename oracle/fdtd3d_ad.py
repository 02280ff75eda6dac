"""Test infrastructure: the exact time-domain gradient of the 3D Yee solver.

The reference's 3D gradient oracle is jax.grad through simulate_3d
(src/gradenna/freq_adjoint.py:724-771, exact_design_gradient_3d), with the
time loop wrapped in jax.checkpoint segments (fdtd3d.py:735-749). jax is not
available here, so this module restates the same loop (the numpy oracle's,
oracle/fdtd3d_np.py, which follows fdtd3d.py:462-679 line for line,
including the port overwrite of fdtd3d.py:517-525, 627-633) in torch
float64 and lets torch autograd form the reverse sweep. Segments of
``segment`` steps are recomputed in the backward pass
(torch.utils.checkpoint): the sqrt(N) checkpointing of fdtd3d.py:735-749.

Only tests use it, as the checker of the GPU frequency-domain adjoint in 3D.
"""

from __future__ import annotations

import numpy as np
import torch
from torch.utils.checkpoint import checkpoint

from oracle import fdtd2d_np as o2
from oracle import fdtd3d_np as o3

DT = torch.float64
COMPS = ("ex", "ey", "ez", "hx", "hy", "hz")
PSI = ("exy", "exz", "eyx", "eyz", "ezx", "ezy", "hxy", "hxz", "hyx", "hyz", "hzx", "hzy")


def _psi_step(psi, diff, b, c, m, axis, inv_kappa):
    """cpml.py:120-158 on both slabs of `axis` (restates o2.psi_step)."""
    if m == 0:
        return psi, diff
    n = diff.shape[axis]
    lo, mid, hi = diff.narrow(axis, 0, m), diff.narrow(axis, m, n - 2 * m), diff.narrow(axis, n - m, m)
    shape = [1, 1, 1]
    shape[axis] = m
    p_lo = b[:m].reshape(shape) * psi[0] + c[:m].reshape(shape) * lo
    p_hi = b[n - m:].reshape(shape) * psi[1] + c[n - m:].reshape(shape) * hi
    k_lo = inv_kappa.narrow(axis, 0, m)
    k_hi = inv_kappa.narrow(axis, n - m, m)
    term = torch.cat([lo * k_lo + p_lo, mid, hi * k_hi + p_hi], dim=axis)
    return (p_lo, p_hi), term


def simulate_3d_ad(grid, *, eps_r, sigma, source_ijk=None, source_current=None, port_ijk=None,
                   port_voltage=None, port_resistance=50.0, dft_freqs=(), dft_regions=None,
                   cpml=o2.CPMLSpec(), segment: int = 100):
    """Differentiable float64 restatement of simulate_3d (fdtd3d.py:462-679).

    ``eps_r`` and ``sigma`` are (nx, ny, nz) torch tensors (they may require
    grad); everything runs on their device. Jz line sources and one RVS port.
    ``dft_regions``: dict comp -> (lo, hi) boxes (default: full grid).
    Returns (dft dict comp -> complex128 phasors scaled by dt, port_v,
    port_i).
    """
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    dx, dy, dz, dt = grid.dx, grid.dy, grid.dz, grid.dt
    dev = sigma.device
    T = lambda a: torch.as_tensor(a, device=dev)  # noqa: E731
    n_steps = None
    if source_current is not None:
        cur = T(np.asarray(source_current, np.float64))
        cur = cur[:, None] if cur.ndim == 1 else cur
        sidx = np.asarray(source_ijk, np.int64).reshape(-1, 3)
        n_steps = cur.shape[0]
    has_port = port_ijk is not None
    if has_port:
        vport = T(np.asarray(port_voltage, np.float64).reshape(-1))
        n_steps = vport.shape[0]
        pi, pj, pk = (int(v) for v in np.asarray(port_ijk).reshape(3))
    eps = o3.EPS0 * eps_r
    half = sigma * dt / (2.0 * eps)
    ca = (1.0 - half) / (1.0 + half)
    cb = (dt / eps) / (1.0 + half)
    m = cpml.thickness
    tab = {}
    for key, (n, d, hf) in {"xe": (nx, dx, False), "ye": (ny, dy, False), "ze": (nz, dz, False),
                            "xh": (nx, dx, True), "yh": (ny, dy, True), "zh": (nz, dz, True)}.items():
        a = o2.axis_coefficients(n, d, dt, cpml, half=hf, dtype=np.float64)
        tab[key] = tuple(T(np.ascontiguousarray(v)) for v in (a.b, a.c, a.inv_kappa))
    kx_e = tab["xe"][2][1:-1, None, None]
    ky_e = tab["ye"][2][None, 1:-1, None]
    kz_e = tab["ze"][2][None, None, 1:-1]
    kx_h = tab["xh"][2][:, None, None]
    ky_h = tab["yh"][2][None, :, None]
    kz_h = tab["zh"][2][None, None, :]
    bx_e, cx_e = tab["xe"][0][1:-1], tab["xe"][1][1:-1]
    by_e, cy_e = tab["ye"][0][1:-1], tab["ye"][1][1:-1]
    bz_e, cz_e = tab["ze"][0][1:-1], tab["ze"][1][1:-1]
    bx_h, cx_h = tab["xh"][0], tab["xh"][1]
    by_h, cy_h = tab["yh"][0], tab["yh"][1]
    bz_h, cz_h = tab["zh"][0], tab["zh"][1]
    inv_dx, inv_dy, inv_dz = 1 / dx, 1 / dy, 1 / dz
    dt_mu = dt / o3.MU0
    if source_current is not None:
        si, sj, sk = (T(sidx[:, q]) for q in range(3))
        cb_src = cb[si, sj, sk] * (inv_dx * inv_dy)
    if has_port:
        eps_p = eps[pi, pj, pk]
        h_p = sigma[pi, pj, pk] * dt / (2.0 * eps_p)
        beta = dt * dz / (2.0 * port_resistance * eps_p * dx * dy)
        denom = 1.0 + h_p + beta
        a_port = (1.0 - h_p - beta) / denom
        b_port = (dt / eps_p) / denom
        c_port = -dt / (port_resistance * eps_p * dx * dy * denom)
    fr = np.atleast_1d(np.asarray(dft_freqs, np.float64))
    K = len(fr)
    nn = np.arange(n_steps, dtype=np.float64)
    ph_e = T(np.exp(-2j * np.pi * np.outer(nn + 1.0, fr) * dt))
    ph_h = T(np.exp(-2j * np.pi * np.outer(nn + 0.5, fr) * dt))
    shapes = o3.full_shapes(nx, ny, nz)
    regions = dft_regions if dft_regions is not None else {k: ((0, 0, 0), s)
                                                           for k, s in shapes.items()}
    regions = {k: v for k, v in regions.items() if v is not None}
    racc = list(regions)
    psi_shapes = dict(
        exy=(nx - 1, m, nz - 2), exz=(nx - 1, ny - 2, m), eyx=(m, ny - 1, nz - 2),
        eyz=(nx - 2, ny - 1, m), ezx=(m, ny - 2, nz - 1), ezy=(nx - 2, m, nz - 1),
        hxy=(nx, m, nz - 1), hxz=(nx, ny - 1, m), hyx=(m, ny, nz - 1), hyz=(nx - 1, ny, m),
        hzx=(m, ny - 1, nz), hzy=(nx - 1, m, nz))

    def pad_e(inner, lead):
        """Ex/Ey/Ez with their PEC-tangential border cells (fdtd3d.py:602-621)."""
        return torch.nn.functional.pad(inner, lead)

    def step_range(n0, n1, ca, cb, state):
        f = dict(zip(COMPS, state[:6]))
        psi = {k: (state[6 + 2 * q], state[7 + 2 * q]) for q, k in enumerate(PSI)}
        acc = {k: torch.complex(state[30 + 2 * q], state[31 + 2 * q]) for q, k in enumerate(racc)}
        ex, ey, ez, hx, hy, hz = (f[c] for c in COMPS)
        vv, ii = [], []
        ca_ex, cb_ex = ca[:-1, 1:-1, 1:-1], cb[:-1, 1:-1, 1:-1]
        ca_ey, cb_ey = ca[1:-1, :-1, 1:-1], cb[1:-1, :-1, 1:-1]
        ca_ez, cb_ez = ca[1:-1, 1:-1, :-1], cb[1:-1, 1:-1, :-1]
        for n in range(n0, n1):
            dey_dz = (ey[:, :, 1:] - ey[:, :, :-1]) * inv_dz
            dez_dy = (ez[:, 1:, :] - ez[:, :-1, :]) * inv_dy
            psi["hxz"], t_hxz = _psi_step(psi["hxz"], dey_dz, bz_h, cz_h, m, 2, kz_h)
            psi["hxy"], t_hxy = _psi_step(psi["hxy"], dez_dy, by_h, cy_h, m, 1, ky_h)
            hx = hx + dt_mu * (t_hxz - t_hxy)
            dez_dx = (ez[1:, :, :] - ez[:-1, :, :]) * inv_dx
            dex_dz = (ex[:, :, 1:] - ex[:, :, :-1]) * inv_dz
            psi["hyx"], t_hyx = _psi_step(psi["hyx"], dez_dx, bx_h, cx_h, m, 0, kx_h)
            psi["hyz"], t_hyz = _psi_step(psi["hyz"], dex_dz, bz_h, cz_h, m, 2, kz_h)
            hy = hy + dt_mu * (t_hyx - t_hyz)
            dex_dy = (ex[:, 1:, :] - ex[:, :-1, :]) * inv_dy
            dey_dx = (ey[1:, :, :] - ey[:-1, :, :]) * inv_dx
            psi["hzy"], t_hzy = _psi_step(psi["hzy"], dex_dy, by_h, cy_h, m, 1, ky_h)
            psi["hzx"], t_hzx = _psi_step(psi["hzx"], dey_dx, bx_h, cx_h, m, 0, kx_h)
            hz = hz + dt_mu * (t_hzy - t_hzx)
            if has_port:  # fdtd3d.py:590-594
                i_loop = (hy[pi, pj, pk] - hy[pi - 1, pj, pk]) * dy + (
                    hx[pi, pj - 1, pk] - hx[pi, pj, pk]) * dx
            dhz_dy = (hz[:, 1:, :] - hz[:, :-1, :])[:, :, 1:-1] * inv_dy
            dhy_dz = (hy[:, :, 1:] - hy[:, :, :-1])[:, 1:-1, :] * inv_dz
            psi["exy"], t_exy = _psi_step(psi["exy"], dhz_dy, by_e, cy_e, m, 1, ky_e)
            psi["exz"], t_exz = _psi_step(psi["exz"], dhy_dz, bz_e, cz_e, m, 2, kz_e)
            ex = pad_e(ca_ex * ex[:, 1:-1, 1:-1] + cb_ex * (t_exy - t_exz), (1, 1, 1, 1, 0, 0))
            dhx_dz = (hx[:, :, 1:] - hx[:, :, :-1])[1:-1, :, :] * inv_dz
            dhz_dx = (hz[1:, :, :] - hz[:-1, :, :])[:, :, 1:-1] * inv_dx
            psi["eyz"], t_eyz = _psi_step(psi["eyz"], dhx_dz, bz_e, cz_e, m, 2, kz_e)
            psi["eyx"], t_eyx = _psi_step(psi["eyx"], dhz_dx, bx_e, cx_e, m, 0, kx_e)
            ey = pad_e(ca_ey * ey[1:-1, :, 1:-1] + cb_ey * (t_eyz - t_eyx), (1, 1, 0, 0, 1, 1))
            dhy_dx = (hy[1:, :, :] - hy[:-1, :, :])[:, 1:-1, :] * inv_dx
            dhx_dy = (hx[:, 1:, :] - hx[:, :-1, :])[1:-1, :, :] * inv_dy
            psi["ezx"], t_ezx = _psi_step(psi["ezx"], dhy_dx, bx_e, cx_e, m, 0, kx_e)
            psi["ezy"], t_ezy = _psi_step(psi["ezy"], dhx_dy, by_e, cy_e, m, 1, ky_e)
            curl_z = t_ezx - t_ezy
            ez_prev = ez
            ez = pad_e(ca_ez * ez[1:-1, 1:-1, :] + cb_ez * curl_z, (0, 0, 1, 1, 1, 1))
            if source_current is not None:
                ez = ez.index_put((si, sj, sk), -cb_src * cur[n], accumulate=True)
            if has_port:  # fdtd3d.py:627-633
                newv = (a_port * ez_prev[pi, pj, pk] + b_port * curl_z[pi - 1, pj - 1, pk]
                        + c_port * vport[n])
                ez = ez.index_put((T([pi]), T([pj]), T([pk])), newv.reshape(1))
                vv.append(-0.5 * dz * (ez_prev[pi, pj, pk] + ez[pi, pj, pk]))
                ii.append(i_loop)
            if K:
                fields = dict(ex=ex, ey=ey, ez=ez, hx=hx, hy=hy, hz=hz)
                for k in racc:
                    lo, hi = regions[k]
                    ph = ph_e[n] if k[0] == "e" else ph_h[n]
                    patch = fields[k][lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
                    acc[k] = acc[k] + ph[:, None, None, None] * patch[None]
        vt = torch.stack(vv) if vv else torch.zeros(n1 - n0, dtype=DT, device=dev)
        it = torch.stack(ii) if ii else torch.zeros(n1 - n0, dtype=DT, device=dev)
        out = [ex, ey, ez, hx, hy, hz]
        for k in PSI:
            out += list(psi[k])
        for k in racc:
            out += [acc[k].real, acc[k].imag]
        return tuple(out) + (vt, it)

    z = lambda s: torch.zeros(s, dtype=DT, device=dev)  # noqa: E731
    state = [z(shapes[c]) for c in COMPS]
    for k in PSI:
        state += [z(psi_shapes[k]), z(psi_shapes[k])]
    for k in racc:
        lo, hi = regions[k]
        shp = (K,) + tuple(h - l for l, h in zip(lo, hi))
        state += [z(shp), z(shp)]
    state = tuple(state)
    nst = len(state)
    vs_out, is_out = [], []
    for n0 in range(0, n_steps, segment):
        n1 = min(n_steps, n0 + segment)
        out = checkpoint(step_range, n0, n1, ca, cb, state, use_reentrant=False)
        state, vt, it = out[:nst], out[nst], out[nst + 1]
        vs_out.append(vt)
        is_out.append(it)
    dft = {k: torch.complex(state[30 + 2 * q], state[31 + 2 * q]) * dt for q, k in enumerate(racc)}
    pv = torch.cat(vs_out) if has_port else None
    pcur = torch.cat(is_out) if has_port else None
    return dft, pv, pcur


def exact_design_gradient_3d(grid, objective, *, design_sigma=None, design_eps_r=None,
                             design_region, dft_freqs, eps_r_background=1.0,
                             sigma_background=0.0, segment: int = 100, device="cpu", **kw):
    """d objective / d design through the whole 3D time loop (the
    reference's exact_design_gradient_3d, freq_adjoint.py:724-771, with torch
    autograd in place of jax.grad). ``objective(dft, port_v, port_i)``
    returns a real scalar tensor. Returns ({"sigma"/"eps_r": numpy array},
    objective value)."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    leaves = {}
    eps_r = torch.as_tensor(np.broadcast_to(np.asarray(eps_r_background, np.float64),
                                            (nx, ny, nz)).copy(), device=device)
    sigma = torch.as_tensor(np.broadcast_to(np.asarray(sigma_background, np.float64),
                                            (nx, ny, nz)).copy(), device=device)
    if design_sigma is not None:
        leaves["sigma"] = torch.as_tensor(np.asarray(design_sigma, np.float64),
                                          device=device).requires_grad_(True)
        sigma = sigma.clone()
        sigma[design_region] = leaves["sigma"]
    if design_eps_r is not None:
        leaves["eps_r"] = torch.as_tensor(np.asarray(design_eps_r, np.float64),
                                          device=device).requires_grad_(True)
        eps_r = eps_r.clone()
        eps_r[design_region] = leaves["eps_r"]
    dft, pv, pcur = simulate_3d_ad(grid, eps_r=eps_r, sigma=sigma, dft_freqs=dft_freqs,
                                   segment=segment, **kw)
    val = objective(dft, pv, pcur)
    grads = torch.autograd.grad(val, list(leaves.values()))
    return {k: g.detach().cpu().numpy() for k, g in zip(leaves, grads)}, float(val.detach())
