"""CPU check of the time-domain adjoint method itself, independent of the
GPU code: the recipe of gradenna_b200.time_adjoint restated in numpy over
runs of the numpy oracle (oracle/fdtd2d_np.py: forward with probes on the
design cells, adjoint with waveform Jz / Mx / My sources and the port as a
passive load) equals autograd through the oracle's time loop
(oracle/fdtd2d_ad.py) to rounding. The recipe:

* forces f^n = dt sum_k Re(c_k exp(-i w_k t_n)) of the conjugated phasor
  cotangents c, t_n = (n + 1) dt on Ez, (n + 1/2) dt on H;
* adjoint sources played backwards: Jz at step k = -f_E^{N-1-k} / cb0 with
  the vacuum cb0 = (dt / eps0) / (dx dy); Mx / My at step k =
  (Q_MAG / (-dt / mu0)) f_H^{N-k} (one step later), Q_MAG = -eps0 / mu0;
* gradient = eps_r (1 + h) sum_n L^{N-n} (dca E^n + dcb (E^{n+1} - ca E^n) / cb).

Sizes are small (40 x 40, 500 steps) so the case runs in seconds.
"""

import numpy as np
import torch

from oracle import fdtd2d_ad as ad
from oracle import fdtd2d_np as onp

EPS0, MU0 = onp.EPS0, onp.MU0
Q_MAG = -EPS0 / MU0
N = 500
REG = (slice(18, 26), slice(18, 26))
BOX = (12, 29, 12, 29)


def _recipe_gradient(g, sigma, epsr, F, drive, G, cells, E, port_ij=None, rs=50.0):
    dt = g.dt
    nn = np.arange(N)
    om = 2 * np.pi * np.asarray(F)
    ph_e = np.exp(-1j * np.outer(nn + 1.0, om) * dt)
    ph_h = np.exp(-1j * np.outer(nn + 0.5, om) * dt)

    def srcs(Gc, ph, e_basis):
        idx = np.argwhere(np.any(np.abs(Gc) > 0, axis=0))
        w = Gc[:, idx[:, 0], idx[:, 1]]
        f = np.real(np.conj(w)[None] * dt * ph[:, :, None]).sum(1)  # torch grad -> conj
        rev = f[::-1].copy()
        if e_basis:
            return [tuple(x) for x in idx], rev / (-(dt / EPS0) / (g.dx * g.dy))
        rev = np.roll(rev, 1, axis=0)
        rev[0] = 0.0
        return [tuple(x) for x in idx], rev * (Q_MAG / (-dt / MU0))

    jz_i, jz = srcs(G[0], ph_e, True)
    mx_i, mx = srcs(G[1], ph_h, False)
    my_i, my = srcs(G[2], ph_h, False)
    ports = (onp.Port(port_ij, rs, None),) if port_ij else ()
    adj = onp.simulate_tm(g, source_ij=jz_i, source_current=jz, mx_ij=mx_i, mx_current=mx,
                          my_ij=my_i, my_current=my, sigma=sigma, eps_r=epsr, ports=ports,
                          probe_ij=cells, cpml=onp.CPMLSpec(8))
    L = np.vstack([np.zeros((1, len(cells))), np.asarray(adj.probe_ez)])
    eps = EPS0 * epsr[REG].ravel()
    s_ = sigma[REG].ravel()
    h = s_ * dt / (2 * eps)
    ca, cb, den = (1 - h) / (1 + h), (dt / eps) / (1 + h), (1 + h) ** 2
    dca, dcb = (-dt / eps) / den, (-(dt / eps) * (dt / (2 * eps))) / den
    curl = (E[1:] - ca * E[:-1]) / cb
    return (epsr[REG].ravel() * (1 + h)) * np.sum(L[N - nn] * (dca * E[:-1] + dcb * curl), axis=0)


def _case(sig_d, use_port, F):
    g = onp.Grid2D(40, 40, 2e-3, 2e-3)
    t = (np.arange(N) + 0.5) * g.dt
    pulse = np.sin(2 * np.pi * 3e9 * t) * np.exp(-((t - 100 * g.dt) / (35 * g.dt)) ** 2)
    sigma = np.zeros((40, 40))
    sigma[REG] = sig_d
    epsr = np.ones((40, 40))
    cells = [(i, j) for i in range(18, 26) for j in range(18, 26)]
    drive = (dict(ports=(onp.Port((15, 22), 50.0, pulse),)) if use_port
             else dict(source_ij=(14, 22), source_current=pulse))
    fw = onp.simulate_tm(g, sigma=sigma, probe_ij=cells, dft_freqs=F, cpml=onp.CPMLSpec(8),
                         **drive)
    E = np.vstack([np.zeros((1, 64)), np.asarray(fw.probe_ez)])
    tz = [torch.tensor(np.asarray(a), requires_grad=True) for a in (fw.dft_ez, fw.dft_hx,
                                                                    fw.dft_hy)]
    ad.poynting_flux_box_2d_t(*tz, g, BOX).sum().backward()
    G = [a.grad.numpy() for a in tz]
    got = _recipe_gradient(g, sigma, epsr, F, drive, G, cells, E,
                           port_ij=(15, 22) if use_port else None)
    ex, _ = ad.exact_design_gradient(
        g, lambda ez, hx, hy, pv, pi: ad.poynting_flux_box_2d_t(ez, hx, hy, g, BOX).sum(),
        design_sigma=sig_d, design_region=REG, dft_freqs=F, cpml=onp.CPMLSpec(8), segment=250,
        **drive)
    want = ex["sigma"].ravel()
    return float(np.linalg.norm(got - want) / np.linalg.norm(want))


def test_recipe_lossy_design_pulse_source():
    assert _case(np.random.default_rng(0).uniform(0, 30, (8, 8)), False, (3e9,)) <= 1e-10


def test_recipe_metal_design_port_two_frequencies():
    sig = 10.0 ** (-4 + 9 * np.random.default_rng(1).uniform(0, 1, (8, 8)))
    assert _case(sig, True, (2.5e9, 3.5e9)) <= 1e-10
