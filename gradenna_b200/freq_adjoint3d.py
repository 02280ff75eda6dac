r"""Frequency-domain (Meep-type) adjoint for the 3D Yee solver on B200.

Same method and conventions as the reference's 3D extension
(src/gradenna/freq_adjoint.py:560-1065): one forward CW run records the
design-region E phasors (and what the objective reads), torch autograd of
the objective on the six phasor components gives the cotangents, and those
become CW adjoint sources:

* E cotangents drive Jx / Jy / Jz with the vacuum basis 1/(-c_b,src) and the
  component's own transverse area (dy dz, dx dz, dx dy);
* H cotangents drive Mx / My / Mz with the single basis Q_MAG / (-dt/mu0),
  Q_MAG = -eps0/mu0 (freq_adjoint.py:774-822).

One adjoint run records the adjoint E phasors on the design cells, and the
gradient is the sum over the three E components of the 2D contraction
(freq_adjoint.py:1034-1065),

    dL/dtheta = sum_alpha sum_k 2/(N_eff dt) eps_r Re[conj(Lambda_a) conj(G_a)],

evaluated by the same device kernel as 2D (gdn_tm_adjoint_contract), once
per component. Both runs are gdn_yee_run_f64 calls whose adjoint drive is
synthesised on the device from the CW phasor weights.
"""

from __future__ import annotations

from typing import NamedTuple

import numpy as np
import torch

from gradenna_b200 import _native
from gradenna_b200 import dft_region as dr
from gradenna_b200.constants import EPS0, MU0
from gradenna_b200.cpml import CPMLSpec
from gradenna_b200.fdtd3d import simulate_3d, time_series_dft
from gradenna_b200.freq_adjoint import Q_MAG
from gradenna_b200.grid import Grid3D

__all__ = ["FreqPhasors3D", "simulate_3d_freq", "port_dft_3d", "freq_adjoint_gradient_3d"]


class FreqPhasors3D(NamedTuple):
    """Full-grid phasors handed to 3D objectives (freq_adjoint.py:592-608)."""

    dft_ex: torch.Tensor
    dft_ey: torch.Tensor
    dft_ez: torch.Tensor
    dft_hx: torch.Tensor
    dft_hy: torch.Tensor
    dft_hz: torch.Tensor
    port_v: torch.Tensor | None = None
    port_i: torch.Tensor | None = None


def _full_eps_sigma_3d(grid, design_sigma, design_eps_r, design_region, device,
                       eps_r_background=None, sigma_background=None):
    """Background (vacuum unless given) with the design values on design_region
    (freq_adjoint.py:611-617)."""
    def bg(a, fill):
        if a is None:
            return torch.full(grid.shape, fill, dtype=torch.float64, device=device)
        return torch.as_tensor(a, dtype=torch.float64, device=device).expand(grid.shape).clone()

    eps_r = bg(eps_r_background, 1.0)
    sigma = bg(sigma_background, 0.0)
    if design_eps_r is not None:
        eps_r[design_region] = torch.as_tensor(design_eps_r, dtype=torch.float64, device=device)
    if design_sigma is not None:
        sigma[design_region] = torch.as_tensor(design_sigma, dtype=torch.float64, device=device)
    return eps_r, sigma


def _port_v_i_3d(dft_ez, dft_hx, dft_hy, grid, pijk, freqs):
    """(V_hat, I_hat) of the z-directed RVS port rebuilt from the phasors
    (freq_adjoint.py:620-649): V = -dz (E/z + E)/2 z^{1/2},
    I = (Hy[i] - Hy[i-1]) dy + (Hx[j-1] - Hx[j]) dx."""
    om = torch.as_tensor(2 * np.pi * np.asarray(freqs, np.float64), device=dft_ez.device)
    z = torch.exp(1j * om * grid.dt)
    half = torch.exp(0.5j * om * grid.dt)
    i, j, k = pijk
    ez = dft_ez[:, i, j, k]
    v = -grid.dz * 0.5 * (ez / z + ez) * half
    cur = ((dft_hy[:, i, j, k] - dft_hy[:, i - 1, j, k]) * grid.dy
           + (dft_hx[:, i, j - 1, k] - dft_hx[:, i, j, k]) * grid.dx)
    return v[:, None], cur[:, None]


def port_dft_3d(v_t, i_t, dt, freqs):
    """Half-step DFT of the 3D port V/I series (freq_adjoint.py:715-719)."""
    v_hat = time_series_dft(v_t, dt, freqs, t0=0.5 * dt)
    i_hat = time_series_dft(i_t, dt, freqs, t0=0.5 * dt)
    return v_hat[:, None], i_hat[:, None]


def _full_phasors(res, grid):
    d = res.dft
    if getattr(d, "regions", None) is not None:
        d = dr.scatter_full(d, dr.full_field_shapes(grid.nx, grid.ny, grid.nz))
    return d


def simulate_3d_freq(grid: Grid3D, *, design_sigma=None, design_eps_r=None, design_region,
                     dft_freqs, source_ijk=None, source_current=None, port_ijk=None,
                     port_voltage=None, port_resistance: float = 50.0,
                     cpml: CPMLSpec = CPMLSpec(), checkpoint_segments=None, dft_regions=None,
                     dtype=torch.float64, device=None) -> FreqPhasors3D:
    """3D forward run returning full-grid complex128 phasors (freq_adjoint.py:652-712).

    With ``dft_regions`` only the slabs are accumulated and the result is
    zero-filled back to full grids, as in the reference.
    """
    dev = _native.require_cuda(device)
    eps_r, sigma = _full_eps_sigma_3d(grid, design_sigma, design_eps_r, design_region, dev)
    res = simulate_3d(grid, eps_r=eps_r, sigma=sigma, source_ijk=source_ijk,
                      source_current=source_current, port_ijk=port_ijk,
                      port_voltage=port_voltage, port_resistance=port_resistance,
                      dft_freqs=dft_freqs, dft_dtype=np.complex128, dft_regions=dft_regions,
                      cpml=cpml, checkpoint_segments=checkpoint_segments, dtype=dtype,
                      device=dev)
    d = _full_phasors(res, grid)
    port_v = port_i = None
    if res.port_v is not None:
        port_v, port_i = port_dft_3d(res.port_v, res.port_i, grid.dt, dft_freqs)
    return FreqPhasors3D(d.ex, d.ey, d.ez, d.hx, d.hy, d.hz, port_v, port_i)


def _objective_boxes(grid, objective_kind, *, port_ijk=None, box_margin=None,
                     monitor_region=None):
    """DFT monitor boxes (comp, lo, hi) of what an objective reads:
    objective_kind "port", "ntff_box" or "field", or a tuple of them."""
    shapes = dr.full_field_shapes(grid.nx, grid.ny, grid.nz)
    kinds = (objective_kind,) if isinstance(objective_kind, str) else tuple(objective_kind)
    boxes = []
    for kind in kinds:
        if kind == "port":
            if port_ijk is None:
                raise ValueError("objective_kind='port' requires port_ijk")
            boxes += dr.region_boxes(dr.port_regions(port_ijk, shapes))
        elif kind == "ntff_box":
            if box_margin is None:
                raise ValueError("objective_kind='ntff_box' requires box_margin")
            boxes += dr.ntff_face_boxes(grid, box_margin)
        elif kind == "field":
            if monitor_region is None:
                raise ValueError("objective_kind='field' requires monitor_region")
            boxes += dr.region_boxes(dr.field_regions(monitor_region, shapes))
        else:
            raise ValueError("objective_kind must be 'port', 'ntff_box' or 'field' (or a "
                             f"tuple of them), got {kind!r}")
    return boxes


def _adjoint_channels(grid, cot):
    """Adjoint source cells and CW weights per channel (freq_adjoint.py:774-822).

    Returns {key: (idx (M, 3) int32, W (M, K) complex128)} for the active
    channels, key in simulate_3d's source naming (src = Jz).
    """
    dt = grid.dt
    dx, dy, dz = grid.dx, grid.dy, grid.dz
    m_basis = Q_MAG / (-(dt / MU0))
    out = {}
    for key, w, basis in (
        ("jx", cot[0], 1.0 / (-(dt / EPS0) / (dy * dz))),
        ("jy", cot[1], 1.0 / (-(dt / EPS0) / (dx * dz))),
        ("src", cot[2], 1.0 / (-(dt / EPS0) / (dx * dy))),
        ("mx", cot[3], m_basis),
        ("my", cot[4], m_basis),
        ("mz", cot[5], m_basis),
    ):
        if w is None:
            continue
        active = torch.any(w.abs() > 0, dim=0)
        idx = torch.nonzero(active)
        if idx.shape[0] == 0:
            continue
        wv = w[:, idx[:, 0], idx[:, 1], idx[:, 2]].T.contiguous() * basis
        out[key] = (idx.cpu().numpy().astype(np.int32), wv)
    return out


def _contract(grid, freqs, env, eps_d, sig_d, e_fwd, lam, want_sigma, want_eps, exact=True):
    """Per-cell gradient of one E component (gdn_tm_adjoint_contract; with
    ``exact`` the contraction carries the loss factor 1 + sigma dt / (2 eps))."""
    dt = grid.dt
    K = len(freqs)
    n_eff = float(np.sum(np.asarray(env, np.float64) ** 2))
    z = torch.as_tensor(np.exp(1j * 2 * np.pi * np.asarray(freqs, np.float64) * dt),
                        device=e_fwd.device)
    er = eps_d.contiguous().reshape(-1)
    sg = sig_d.contiguous().reshape(-1)
    n = er.numel()
    e = e_fwd.reshape(K, -1).contiguous()
    lm = lam.reshape(K, -1).contiguous()
    gs = torch.empty(n, dtype=torch.float64, device=e.device) if want_sigma else None
    ge = torch.empty(n, dtype=torch.float64, device=e.device) if want_eps else None
    stream = torch.cuda.current_stream(e.device).cuda_stream
    with torch.cuda.device(e.device):
        _native.check(_native.load().gdn_tm_adjoint_contract(
            n, K, dt, 2.0 / (n_eff * dt), e.data_ptr(), lm.data_ptr(), er.data_ptr(),
            sg.data_ptr(), z.data_ptr(), _native.ptr(gs), _native.ptr(ge),
            1 if exact else 0, stream))
    return gs, ge


def freq_adjoint_gradient_3d(grid: Grid3D, objective, *, design_sigma=None, design_eps_r=None,
                             design_region, dft_freqs, env, source_ijk=None, source_current=None,
                             port_ijk=None, port_voltage=None, port_resistance: float = 50.0,
                             cpml: CPMLSpec = CPMLSpec(), backend: str = "cuda",
                             objective_kind: str | None = None, box_margin: int | None = None,
                             monitor_region=None, dtype=torch.float64, device=None,
                             eps_r_background=None, sigma_background=None, exact: bool = True):
    """Two-run 3D frequency-domain adjoint gradient (freq_adjoint.py:864-1065).

    ``objective`` maps FreqPhasors3D (torch complex128 on the device) to a
    real scalar tensor; the source/port drive must be CW at ``dft_freqs``
    under the turn-on envelope ``env``. ``objective_kind`` ("port",
    "ntff_box" or "field", with ``box_margin`` / ``monitor_region``, or a
    tuple of them) limits the forward DFT to the design E slabs plus what
    the objective reads and the adjoint DFT to the design slabs, as in the
    reference; the gradient is unchanged. Where the reference records one
    bounding slab per component (for the NTFF box: the whole box volume),
    this records exact boxes (for the NTFF box: the face layers ntff_3d
    reads). ``eps_r_background`` / ``sigma_background`` (nx, ny, nz)
    replace the reference's vacuum background (an addition: fixed structures
    such as a substrate and ground plane around the design); the design
    values overwrite them on design_region. ``exact`` (default) keeps the
    port in the adjoint run as a passive load and scales the contraction by
    eps_r (1 + sigma dt / (2 eps)); ``exact=False`` reproduces the
    reference's formulas, which hold only for small sigma and no port.
    ``backend`` is accepted for signature compatibility
    ("xla", "native", "cuda"); every run is the CUDA path. Returns
    {"sigma": ..., "eps_r": ...} (float64 tensors of the design shape) for
    the design variables supplied.
    """
    if backend not in ("xla", "native", "cuda"):
        raise ValueError(f"backend must be 'xla', 'native' or 'cuda', got {backend!r}")
    if design_sigma is None and design_eps_r is None:
        raise ValueError("give design_sigma and/or design_eps_r")
    dev = _native.require_cuda(device)
    freqs = tuple(float(f) for f in dft_freqs)
    env = np.asarray(env.detach().cpu() if isinstance(env, torch.Tensor) else env, np.float64)
    eps_r, sigma = _full_eps_sigma_3d(grid, design_sigma, design_eps_r, design_region, dev,
                                      eps_r_background, sigma_background)
    shapes = dr.full_field_shapes(grid.nx, grid.ny, grid.nz)

    # Region-limited DFT: exact monitor boxes (the design E slabs, plus what
    # the objective reads in the forward run). The objective and the
    # contraction see zero-filled full grids, so the gradient is unchanged.
    fwd_boxes = adj_boxes = None
    if objective_kind is not None:
        adj_boxes = dr.region_boxes(dr.design_region_to_slabs(design_region, shapes))
        fwd_boxes = list(adj_boxes) + _objective_boxes(grid, objective_kind, port_ijk=port_ijk,
                                                       box_margin=box_margin,
                                                       monitor_region=monitor_region)

    def phasors(res, boxes):
        if boxes is None:
            return res.dft
        ft = torch.as_tensor(np.asarray(freqs), device=dev)
        return dr.boxes_to_full(ft, boxes, res.monitors, shapes)

    common = dict(eps_r=eps_r, sigma=sigma, dft_freqs=freqs, dft_dtype=np.complex128, cpml=cpml,
                  dtype=dtype, device=dev)
    fwd = simulate_3d(grid, source_ijk=source_ijk, source_current=source_current,
                      port_ijk=port_ijk, port_voltage=port_voltage,
                      port_resistance=port_resistance, dft_monitors=fwd_boxes, **common)
    fd = phasors(fwd, fwd_boxes)
    comps = [fd.ex, fd.ey, fd.ez, fd.hx, fd.hy, fd.hz]

    # Objective cotangents; torch's complex gradient is the conjugate of jax's.
    pijk = None if port_ijk is None else tuple(int(v) for v in np.asarray(port_ijk).reshape(3))
    leaves = [t.detach().requires_grad_(True) for t in comps]
    with torch.enable_grad():
        pv = pi = None
        if pijk is not None:
            pv, pi = _port_v_i_3d(leaves[2], leaves[3], leaves[4], grid, pijk, freqs)
        val = objective(FreqPhasors3D(*leaves, pv, pi))
        grads = torch.autograd.grad(val, leaves, allow_unused=True)
    cot = [None if g is None else g.conj() for g in grads]

    chans = _adjoint_channels(grid, cot)
    shp = tuple(s.indices(n)[1] - s.indices(n)[0] for s, n in zip(design_region, grid.shape))
    out = {}
    if not chans:
        if design_sigma is not None:
            out["sigma"] = torch.zeros(shp, dtype=torch.float64, device=dev)
        if design_eps_r is not None:
            out["eps_r"] = torch.zeros(shp, dtype=torch.float64, device=dev)
        return out
    kw = {}
    cw = dict(env=env)
    names = {"src": ("source_ijk", "source_current"), "jx": ("source_x_ijk", "source_x_current"),
             "jy": ("source_y_ijk", "source_y_current"), "mx": ("mx_ijk", "mx_current"),
             "my": ("my_ijk", "my_current"), "mz": ("mz_ijk", "mz_current")}
    for key, (idx, w) in chans.items():
        kw[names[key][0]] = idx
        cw[f"{key}_w"] = w
    if exact and pijk is not None:
        # The lumped port is a resistor in the medium: the exact adjoint run
        # keeps it as a passive load (the reference's adjoint run drops it).
        kw.update(port_ijk=pijk, port_resistance=port_resistance,
                  port_voltage=np.zeros(len(np.asarray(env)), np.float64))
    adj = simulate_3d(grid, dft_monitors=adj_boxes, cw_sources=cw, **kw, **common)
    ad = phasors(adj, adj_boxes)

    sel = (slice(None),) + tuple(design_region)
    eps_d, sig_d = eps_r[design_region], sigma[design_region]
    gs_tot = ge_tot = None
    for e_full, l_full in ((fd.ex, ad.ex), (fd.ey, ad.ey), (fd.ez, ad.ez)):
        gs, ge = _contract(grid, freqs, env, eps_d, sig_d, e_full[sel], l_full[sel],
                           design_sigma is not None, design_eps_r is not None, exact)
        if gs is not None:
            gs_tot = gs if gs_tot is None else gs_tot + gs
        if ge is not None:
            ge_tot = ge if ge_tot is None else ge_tot + ge
    if gs_tot is not None:
        out["sigma"] = gs_tot.reshape(shp)
    if ge_tot is not None:
        out["eps_r"] = ge_tot.reshape(shp)
    return out
