"""The exact time-domain gradient oracle (oracle/fdtd2d_ad.py): its forward
equals the numpy oracle to 1e-13 (last-bit rounding of the material
coefficients), and its reverse sweep (torch autograd
with segment recomputation) equals central finite differences of the numpy
oracle, as the reference pins jax.grad (tests/test_gradients.py:48-73)."""

import numpy as np
import torch

from oracle import fdtd2d_ad as ad
from oracle import fdtd2d_np as onp

G = onp.Grid2D(24, 22, 2e-3, 2e-3)
N = 160
CPML = onp.CPMLSpec(5)


def _case():
    n = np.arange(N)
    cur = np.sin(2 * np.pi * 4e9 * (n + 0.5) * G.dt) * np.exp(-((n - 50) / 20.0) ** 2)
    ports = (onp.Port((7, 11), 50.0, cur), onp.Port((17, 10), 50.0, None))
    return cur, ports


def test_forward_equals_numpy_oracle():
    cur, ports = _case()
    sig = np.zeros((24, 22))
    sig[9:14, 8:13] = 0.4
    eps = np.ones((24, 22))
    eps[10:12, 12:15] = 2.5
    o = onp.simulate_tm(G, source_ij=(12, 16), source_current=cur, sigma=sig, eps_r=eps,
                        ports=ports, dft_freqs=(3e9, 5e9), cpml=CPML)
    r = ad.simulate_tm_ad(G, eps_r=torch.as_tensor(eps), sigma=torch.as_tensor(sig),
                          source_ij=(12, 16), source_current=cur, ports=ports,
                          dft_freqs=(3e9, 5e9), cpml=CPML, segment=37)
    for a, b in ((o.dft_ez, r[0]), (o.dft_hx, r[1]), (o.dft_hy, r[2]), (o.port_v, r[3]),
                 (o.port_i, r[4])):
        b = b.detach().numpy()
        assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()


def test_exact_gradient_matches_finite_differences():
    cur, ports = _case()
    region = (slice(9, 13), slice(8, 11))
    box = (3, 19, 3, 17)

    def obj_t(ez, hx, hy, pv, pi):
        p = ad.poynting_flux_box_2d_t(ez, hx, hy, G, box).sum()
        v = ad.half_step_dft_t(pv[:, 0], G.dt, (4e9,))
        i = ad.half_step_dft_t(pi[:, 0], G.dt, (4e9,))
        s = (v - 50.0 * i) / (v + 50.0 * i)
        return p * 1e9 + (s.real**2 + s.imag**2).sum()

    def obj_np(sig_d):
        sig = np.zeros((24, 22))
        sig[region] = sig_d
        o = onp.simulate_tm(G, sigma=sig, ports=ports, dft_freqs=(4e9,), cpml=CPML)
        p = onp.poynting_flux_box_2d(o.dft_ez, o.dft_hx, o.dft_hy, G, box).sum()
        v, i = onp.port_dft(o.port_v[:, 0], o.port_i[:, 0], G.dt, (4e9,))
        s = onp.s11_power_wave(v, i)
        return p * 1e9 + float((np.abs(s) ** 2).sum())

    sig0 = 0.3 + 0.1 * np.arange(12).reshape(4, 3) / 12
    g, val = ad.exact_design_gradient(G, obj_t, design_sigma=sig0, design_region=region,
                                      dft_freqs=(4e9,), ports=ports, cpml=CPML, segment=50)
    assert np.isclose(val, obj_np(sig0), rtol=1e-12)
    for idx in [(0, 0), (2, 1), (3, 2)]:
        h = 1e-4
        sp, sm = sig0.copy(), sig0.copy()
        sp[idx] += h
        sm[idx] -= h
        fd = (obj_np(sp) - obj_np(sm)) / (2 * h)
        assert abs(g["sigma"][idx] - fd) <= 1e-6 * abs(fd) + 1e-12, (idx, g["sigma"][idx], fd)
