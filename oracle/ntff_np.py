"""Test infrastructure: numpy restatement of the reference's near-to-far-field
transforms (src/gradenna/ntff.py). Only the tests, the smoke check and the
CPU baseline leg of the benchmark use this module, as the checker.

Every function follows the reference line for line in what it computes (the
surface sampling, Yee averages, signs, quadrature and prefactors), written
as plain numpy sums so a reader can compare it with ntff.py directly:

  periodic_trapezoid_weights  ntff.py:64-84
  trapezoid_weights           ntff.py:87-92
  ntff_2d                     ntff.py:100-232
  radiated_power_2d           ntff.py:235-244
  directivity_2d              ntff.py:247-256
  ntff_3d                     ntff.py:262-431
  radiated_power_3d           ntff.py:441-455
  directivity_3d              ntff.py:458-466
  gain                        ntff.py:469-484

Parity pins: the reference's own acceptance tests (tests/test_ntff.py) are
restated on this oracle in tests/test_oracle_ntff_known_answers.py (line
current isotropy and power, broadside and endfire array patterns, the
z-dipole's D(90 deg) = 1.5, sin^2 pattern and radiation resistance).
"""

from __future__ import annotations

import math

import numpy as np

C0 = 299792458.0  # constants.py:3-6
MU0 = 1.25663706212e-06
ETA0 = MU0 * C0


def periodic_trapezoid_weights(angles, period):
    a = np.asarray(angles, np.float64)
    if a.ndim != 1 or a.shape[0] < 2:
        raise ValueError("need a 1D array of at least 2 angles")
    return 0.5 * (np.mod(np.roll(a, -1) - a, period) + np.mod(a - np.roll(a, 1), period))


def trapezoid_weights(x):
    x = np.asarray(x, np.float64)
    d = np.diff(x)
    return 0.5 * np.concatenate([d[:1], d[:-1] + d[1:], d[-1:]])


def ntff_2d(dft_ez, dft_hx, dft_hy, nx, ny, dx, dy, contour_margin, freqs, angles):
    """Pattern amplitude E_far (n_freq, n_angles) of the TM contour transform."""
    dft_ez, dft_hx, dft_hy = (np.asarray(a) for a in (dft_ez, dft_hx, dft_hy))
    freqs = np.atleast_1d(np.asarray(freqs, np.float64))
    angles = np.atleast_1d(np.asarray(angles, np.float64))
    m = int(contour_margin)
    i0, i1, j0, j1 = m, nx - 1 - m, m, ny - 1 - m
    xn = (np.arange(nx) - 0.5 * (nx - 1)) * dx
    yn = (np.arange(ny) - 0.5 * (ny - 1)) * dy

    def sw(n, dl):
        w = np.full(n, dl)
        w[0] *= 0.5
        w[-1] *= 0.5
        return w

    jr, ir = slice(j0, j1 + 1), slice(i0, i1 + 1)
    nj, ni = j1 - j0 + 1, i1 - i0 + 1
    sides = [
        (np.full(nj, xn[i1]), yn[jr], 1.0, 0.0, sw(nj, dy),
         0.5 * (dft_hy[:, i1 - 1, jr] + dft_hy[:, i1, jr]), dft_ez[:, i1, jr]),
        (np.full(nj, xn[i0]), yn[jr], -1.0, 0.0, sw(nj, dy),
         -0.5 * (dft_hy[:, i0 - 1, jr] + dft_hy[:, i0, jr]), dft_ez[:, i0, jr]),
        (xn[ir], np.full(ni, yn[j1]), 0.0, 1.0, sw(ni, dx),
         -0.5 * (dft_hx[:, ir, j1 - 1] + dft_hx[:, ir, j1]), dft_ez[:, ir, j1]),
        (xn[ir], np.full(ni, yn[j0]), 0.0, -1.0, sw(ni, dx),
         0.5 * (dft_hx[:, ir, j0 - 1] + dft_hx[:, ir, j0]), dft_ez[:, ir, j0]),
    ]
    x = np.concatenate([s[0] for s in sides])
    y = np.concatenate([s[1] for s in sides])
    n_x = np.concatenate([np.full(s[0].shape, s[2]) for s in sides])
    n_y = np.concatenate([np.full(s[0].shape, s[3]) for s in sides])
    w = np.concatenate([s[4] for s in sides])
    jz = np.concatenate([s[5] for s in sides], axis=1).astype(np.complex128)
    ez = np.concatenate([s[6] for s in sides], axis=1).astype(np.complex128)
    k = 2.0 * np.pi * freqs / C0
    ca, sa = np.cos(angles), np.sin(angles)
    proj = x[None, :] * ca[:, None] + y[None, :] * sa[:, None]
    mdir = n_x[None, :] * ca[:, None] + n_y[None, :] * sa[:, None]
    phase = np.exp(1j * k[:, None, None] * proj[None])
    integrand = ETA0 * jz[:, None, :] - mdir[None] * ez[:, None, :]
    total = np.sum(w * integrand * phase, axis=-1)
    return -np.sqrt(1j * k / (8.0 * np.pi))[:, None] * total


def radiated_power_2d(e_far, angles):
    w = periodic_trapezoid_weights(angles, 2.0 * math.pi)
    return np.sum(w * np.abs(e_far) ** 2, axis=-1) / (2.0 * ETA0)


def directivity_2d(e_far, angles):
    e2 = np.abs(e_far) ** 2
    w = periodic_trapezoid_weights(angles, 2.0 * math.pi)
    return 2.0 * np.pi * e2 / np.sum(w * e2, axis=-1, keepdims=True)


def box_currents_3d(mon, nx, ny, nz, dx, dy, dz, box_margin):
    """(pos (n_pts, 3), w (n_pts,), J, M (n_freq, n_pts, 3)) on the six faces.

    ``mon`` maps 'ex'..'hz' to full-grid (n_freq, ...) phasor arrays.
    """
    ex, ey, ez, hx, hy, hz = (np.asarray(mon[c]) for c in ("ex", "ey", "ez", "hx", "hy", "hz"))
    m = int(box_margin)
    i0, i1, j0, j1, k0, k1 = m, nx - 1 - m, m, ny - 1 - m, m, nz - 1 - m
    ic, icp = slice(i0, i1), slice(i0 + 1, i1 + 1)
    jc, jcp = slice(j0, j1), slice(j0 + 1, j1 + 1)
    kc, kcp = slice(k0, k1), slice(k0 + 1, k1 + 1)
    xn = (np.arange(nx) - 0.5 * (nx - 1)) * dx
    yn = (np.arange(ny) - 0.5 * (ny - 1)) * dy
    zn = (np.arange(nz) - 0.5 * (nz - 1)) * dz
    xc, yc, zc = xn[i0:i1] + 0.5 * dx, yn[j0:j1] + 0.5 * dy, zn[k0:k1] + 0.5 * dz
    P, W, J, M = [], [], [], []

    def add(X, Y, Z, area, jv, mv):
        P.append(np.stack([X.ravel(), Y.ravel(), Z.ravel()], -1))
        W.append(np.full(X.size, area))
        nf = jv[0].shape[0]
        J.append(np.stack([c.reshape(nf, -1) for c in jv], -1))
        M.append(np.stack([c.reshape(nf, -1) for c in mv], -1))

    for i, s in ((i1, 1.0), (i0, -1.0)):
        ey_f = 0.5 * (ey[:, i, jc, kc] + ey[:, i, jc, kcp])
        ez_f = 0.5 * (ez[:, i, jc, kc] + ez[:, i, jcp, kc])
        hy_f = 0.25 * (hy[:, i - 1, jc, kc] + hy[:, i, jc, kc]
                       + hy[:, i - 1, jcp, kc] + hy[:, i, jcp, kc])
        hz_f = 0.25 * (hz[:, i - 1, jc, kc] + hz[:, i, jc, kc]
                       + hz[:, i - 1, jc, kcp] + hz[:, i, jc, kcp])
        yy, zz = np.meshgrid(yc, zc, indexing="ij")
        o = np.zeros_like(hz_f)
        add(np.full_like(yy, xn[i]), yy, zz, dy * dz, (o, -s * hz_f, s * hy_f),
            (o, s * ez_f, -s * ey_f))
    for j, s in ((j1, 1.0), (j0, -1.0)):
        ex_f = 0.5 * (ex[:, ic, j, kc] + ex[:, ic, j, kcp])
        ez_f = 0.5 * (ez[:, ic, j, kc] + ez[:, icp, j, kc])
        hx_f = 0.25 * (hx[:, ic, j - 1, kc] + hx[:, ic, j, kc]
                       + hx[:, icp, j - 1, kc] + hx[:, icp, j, kc])
        hz_f = 0.25 * (hz[:, ic, j - 1, kc] + hz[:, ic, j, kc]
                       + hz[:, ic, j - 1, kcp] + hz[:, ic, j, kcp])
        xx, zz = np.meshgrid(xc, zc, indexing="ij")
        o = np.zeros_like(hz_f)
        add(xx, np.full_like(xx, yn[j]), zz, dx * dz, (s * hz_f, o, -s * hx_f),
            (-s * ez_f, o, s * ex_f))
    for kk, s in ((k1, 1.0), (k0, -1.0)):
        ex_f = 0.5 * (ex[:, ic, jc, kk] + ex[:, ic, jcp, kk])
        ey_f = 0.5 * (ey[:, ic, jc, kk] + ey[:, icp, jc, kk])
        hx_f = 0.25 * (hx[:, ic, jc, kk - 1] + hx[:, ic, jc, kk]
                       + hx[:, icp, jc, kk - 1] + hx[:, icp, jc, kk])
        hy_f = 0.25 * (hy[:, ic, jc, kk - 1] + hy[:, ic, jc, kk]
                       + hy[:, ic, jcp, kk - 1] + hy[:, ic, jcp, kk])
        xx, yy = np.meshgrid(xc, yc, indexing="ij")
        o = np.zeros_like(hx_f)
        add(xx, yy, np.full_like(xx, zn[kk]), dx * dy, (-s * hy_f, s * hx_f, o),
            (s * ey_f, -s * ex_f, o))
    return (np.concatenate(P), np.concatenate(W), np.concatenate(J, 1).astype(np.complex128),
            np.concatenate(M, 1).astype(np.complex128))


def project_3d(pos, w, J, M, freqs, thetas, phis):
    """(n_freq, n_theta, n_phi, 2) pattern amplitudes of surface currents J, M."""
    k = 2.0 * np.pi * np.atleast_1d(np.asarray(freqs, np.float64)) / C0
    coef = 1j * k / (4.0 * np.pi)
    thetas = np.atleast_1d(np.asarray(thetas, np.float64))
    phis = np.atleast_1d(np.asarray(phis, np.float64))
    out = np.zeros((k.shape[0], thetas.shape[0], phis.shape[0], 2), np.complex128)
    for a, th in enumerate(thetas):
        ct, st = np.cos(th), np.sin(th)
        for b, phi in enumerate(phis):
            cp, sp = np.cos(phi), np.sin(phi)
            rhat = np.array([st * cp, st * sp, ct])
            ph = w * np.exp(1j * k[:, None] * (pos @ rhat)[None, :])
            nv = np.einsum("fp,fpc->fc", ph, J)
            lv = np.einsum("fp,fpc->fc", ph, M)
            n_th = (nv[:, 0] * cp + nv[:, 1] * sp) * ct - nv[:, 2] * st
            n_ph = -nv[:, 0] * sp + nv[:, 1] * cp
            l_th = (lv[:, 0] * cp + lv[:, 1] * sp) * ct - lv[:, 2] * st
            l_ph = -lv[:, 0] * sp + lv[:, 1] * cp
            out[:, a, b, 0] = -coef * (l_ph + ETA0 * n_th)
            out[:, a, b, 1] = coef * (l_th - ETA0 * n_ph)
    return out


def ntff_3d(mon, nx, ny, nz, dx, dy, dz, box_margin, freqs, thetas, phis):
    pos, w, J, M = box_currents_3d(mon, nx, ny, nz, dx, dy, dz, box_margin)
    return project_3d(pos, w, J, M, freqs, thetas, phis)


def radiated_power_3d(e_theta, e_phi, thetas, phis):
    u = (np.abs(e_theta) ** 2 + np.abs(e_phi) ** 2) / (2.0 * ETA0)
    u_phi = np.sum(u * periodic_trapezoid_weights(phis, 2.0 * math.pi), axis=-1)
    th = np.asarray(thetas, np.float64)
    return np.sum(u_phi * trapezoid_weights(th) * np.sin(th), axis=-1)


def directivity_3d(e_theta, e_phi, thetas, phis):
    u = (np.abs(e_theta) ** 2 + np.abs(e_phi) ** 2) / (2.0 * ETA0)
    return 4.0 * np.pi * u / radiated_power_3d(e_theta, e_phi, thetas, phis)[:, None, None]


def gain(directivity, p_rad, p_in):
    d = np.asarray(directivity)
    eff = np.asarray(p_rad) / np.asarray(p_in)
    return d * eff.reshape(eff.shape + (1,) * (d.ndim - eff.ndim))
