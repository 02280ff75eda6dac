"""GPU checks of the near-to-far-field transforms (gradenna_b200.ntff).

* Parity: the CUDA projection against the numpy oracle (oracle/ntff_np.py,
  a restatement of src/gradenna/ntff.py) on the same seeded phasors, in
  complex128 (relative 1e-12 of the pattern maximum) and complex64 (1e-5).
* Adjoint: the backward kernels satisfy Re<A^H c, v> = Re<c, A v> with A v
  evaluated by the oracle, which pins the gradient without finite
  differences.
* Known answers: the reference's acceptance tests (tests/test_ntff.py) run
  through the GPU solvers and the GPU transform.
* Region monitors: ntff_3d on the slab spectra of ``ntff_box_regions``
  equals ntff_3d on the full-grid spectra.
* A directivity objective differentiates through the frequency-domain
  adjoint and matches central finite differences.
"""

import functools
import types

import numpy as np
import pytest
import torch

from oracle import ntff_np as on
from tests import known_ntff as kn

pytestmark = pytest.mark.gpu


def _cplx(rng, *shape):
    return rng.normal(size=shape) + 1j * rng.normal(size=shape)


def _fields2(rng, K, nx, ny):
    return _cplx(rng, K, nx, ny), _cplx(rng, K, nx, ny - 1), _cplx(rng, K, nx - 1, ny)


def _fields3(rng, K, nx, ny, nz):
    from gradenna_b200.dft_region import full_field_shapes

    names = ("ex", "ey", "ez", "hx", "hy", "hz")
    return {n: _cplx(rng, K, *s) for n, s in zip(names, full_field_shapes(nx, ny, nz))}


FREQS = (2.0e9, 2.9e9, 4.1e9)


@pytest.mark.parametrize("cdt,tol", [(torch.complex128, 1e-12), (torch.complex64, 1e-5)])
def test_ntff_2d_matches_oracle(cdt, tol):
    import gradenna_b200 as gb
    from gradenna_b200.ntff import ntff_2d

    rng = np.random.default_rng(1)
    nx, ny, m = 41, 37, 5
    ez, hx, hy = _fields2(rng, 3, nx, ny)
    ang = np.sort(rng.uniform(0, 2 * np.pi, 77))
    want = on.ntff_2d(ez, hx, hy, nx, ny, 1.5e-3, 2e-3, m, FREQS, ang)
    t = [torch.tensor(a, device="cuda").to(cdt) for a in (ez, hx, hy)]
    got = ntff_2d(*t, gb.Grid2D(nx, ny, 1.5e-3, 2e-3), m, FREQS, ang)
    assert got.dtype == cdt and got.shape == (3, 77)
    err = np.abs(got.cpu().numpy() - want).max() / np.abs(want).max()
    assert err <= tol, err


@pytest.mark.parametrize("cdt,tol", [(torch.complex128, 1e-12), (torch.complex64, 1e-5)])
def test_ntff_3d_matches_oracle(cdt, tol):
    import gradenna_b200 as gb
    from gradenna_b200.fdtd3d import DFTMonitor
    from gradenna_b200.ntff import ntff_3d

    rng = np.random.default_rng(2)
    nx, ny, nz, m = 22, 19, 17, 3
    dx, dy, dz = 2e-3, 2.5e-3, 3e-3
    f = _fields3(rng, 3, nx, ny, nz)
    th = np.linspace(0, np.pi, 13)
    ph = np.linspace(0, 2 * np.pi, 10, endpoint=False)
    want = on.ntff_3d(f, nx, ny, nz, dx, dy, dz, m, FREQS, th, ph)
    mon = DFTMonitor(torch.tensor(FREQS), *(torch.tensor(f[c], device="cuda").to(cdt)
                                           for c in ("ex", "ey", "ez", "hx", "hy", "hz")))
    got = ntff_3d(mon, gb.Grid3D(nx, ny, nz, dx, dy, dz), m, FREQS, th, ph)
    assert got.dtype == cdt and got.shape == (3, 13, 10, 2)
    err = np.abs(got.cpu().numpy() - want).max() / np.abs(want).max()
    assert err <= tol, err


def _re_dot(a, b):
    return float(np.sum(np.real(np.conj(a) * b)))


def test_ntff_2d_adjoint_identity():
    import gradenna_b200 as gb
    from gradenna_b200.ntff import ntff_2d

    rng = np.random.default_rng(3)
    nx, ny, m = 30, 34, 4
    x = _fields2(rng, 3, nx, ny)
    v = _fields2(rng, 3, nx, ny)
    ang = np.linspace(0, 2 * np.pi, 50, endpoint=False)
    c = _cplx(rng, 3, 50)
    t = [torch.tensor(a, device="cuda", requires_grad=True) for a in x]
    out = ntff_2d(*t, gb.Grid2D(nx, ny, 2e-3, 2e-3), m, FREQS, ang)
    loss = torch.sum(torch.real(torch.conj(torch.tensor(c, device="cuda")) * out))
    loss.backward()
    lhs = sum(_re_dot(tt.grad.cpu().numpy(), vv) for tt, vv in zip(t, v))
    rhs = _re_dot(c, on.ntff_2d(*v, nx, ny, 2e-3, 2e-3, m, FREQS, ang))
    assert abs(lhs - rhs) <= 1e-11 * abs(rhs), (lhs, rhs)


def test_ntff_3d_adjoint_identity():
    import gradenna_b200 as gb
    from gradenna_b200.fdtd3d import DFTMonitor
    from gradenna_b200.ntff import ntff_3d

    rng = np.random.default_rng(4)
    nx, ny, nz, m = 16, 15, 14, 3
    names = ("ex", "ey", "ez", "hx", "hy", "hz")
    x = _fields3(rng, 3, nx, ny, nz)
    v = _fields3(rng, 3, nx, ny, nz)
    th = np.linspace(0, np.pi, 9)
    ph = np.linspace(0, 2 * np.pi, 8, endpoint=False)
    c = _cplx(rng, 3, 9, 8, 2)
    t = [torch.tensor(x[n], device="cuda", requires_grad=True) for n in names]
    out = ntff_3d(DFTMonitor(torch.tensor(FREQS), *t), gb.Grid3D(nx, ny, nz, 1e-3, 1e-3, 1e-3),
                  m, FREQS, th, ph)
    torch.sum(torch.real(torch.conj(torch.tensor(c, device="cuda")) * out)).backward()
    lhs = sum(_re_dot(tt.grad.cpu().numpy(), v[n]) for tt, n in zip(t, names))
    rhs = _re_dot(c, on.ntff_3d(v, nx, ny, nz, 1e-3, 1e-3, 1e-3, m, FREQS, th, ph))
    assert abs(lhs - rhs) <= 1e-11 * abs(rhs), (lhs, rhs)


def test_ntff_bad_arguments():
    import gradenna_b200 as gb
    from gradenna_b200.ntff import ntff_2d

    g = gb.Grid2D(20, 20, 1e-3, 1e-3)
    ez = torch.zeros((1, 20, 20), dtype=torch.complex128, device="cuda")
    hx = torch.zeros((1, 20, 19), dtype=torch.complex128, device="cuda")
    hy = torch.zeros((1, 19, 20), dtype=torch.complex128, device="cuda")
    with pytest.raises(ValueError):
        ntff_2d(ez, hx, hy, g, 0, (1e9,), [0.0, 1.0])
    with pytest.raises(ValueError):
        ntff_2d(ez, hx, hy, g, 9, (1e9,), [0.0, 1.0])
    with pytest.raises(ValueError):
        ntff_2d(ez, hx, hy, g, 3, (1e9, 2e9), [0.0, 1.0])


# --- known answers through the GPU solvers ---------------------------------


def _np(t):
    return t.detach().cpu().numpy()


def _mod():
    import gradenna_b200 as gb
    from gradenna_b200 import ntff as nt

    def ntff2(res, grid, margin, freqs, angles):
        return _np(nt.ntff_2d(res.dft_ez, res.dft_hx, res.dft_hy, grid, margin, freqs, angles))

    def ntff3(res, grid, margin, freqs, thetas, phis):
        return _np(nt.ntff_3d(res.dft, grid, margin, freqs, thetas, phis))

    def dev(a):
        return torch.as_tensor(a, device="cuda")

    return types.SimpleNamespace(
        Grid2D=gb.Grid2D, Grid3D=gb.Grid3D, CPMLSpec=gb.CPMLSpec,
        alpha_max_for_fmin=gb.alpha_max_for_fmin, simulate_tm=gb.simulate_tm,
        simulate_3d=gb.simulate_3d, ntff2=ntff2, ntff3=ntff3,
        power2=lambda e, a: _np(nt.radiated_power_2d(dev(e), a)),
        power3=lambda a, b, t, p: _np(nt.radiated_power_3d(dev(a), dev(b), t, p)),
        directivity3=lambda a, b, t, p: _np(nt.directivity_3d(dev(a), dev(b), t, p)))


@functools.lru_cache(maxsize=3)
def _run2(kind):
    return kn.run_2d(_mod(), kind)


def test_line_current_isotropy_and_power():
    grid, cur, e_far = _run2("single")
    kn.check_isotropy(e_far)
    kn.check_line_power(_mod(), grid, cur, e_far)


def test_broadside_and_endfire_patterns():
    kn.check_pair(_run2("pair")[2])
    kn.check_endfire(_run2("endfire")[2])


def test_dipole_3d_known_answers_and_region_monitor():
    import gradenna_b200 as gb
    from gradenna_b200.dft_region import full_field_shapes, ntff_box_regions
    from gradenna_b200.ntff import ntff_3d

    mod = _mod()
    grid, cur, e_far = kn.run_3d(mod)
    kn.check_dipole_3d(mod, grid, cur, e_far)

    # Same run with only the NTFF box recorded.
    c = kn.N3 // 2
    tau = 6.0 / (2.0 * np.pi * kn.F3)
    t = (np.arange(kn.STEPS3) + 0.5) * grid.dt
    regions = ntff_box_regions(grid, kn.MARGIN3, full_field_shapes(grid.nx, grid.ny, grid.nz))
    res = gb.simulate_3d(grid, source_ijk=(c, c, c),
                         source_current=kn.modulated_gaussian(t, kn.F3, 5.0 * tau, tau),
                         dft_freqs=np.array([kn.F3]), dft_regions=regions,
                         cpml=gb.CPMLSpec(thickness=10,
                                          alpha_max=gb.alpha_max_for_fmin(kn.F3 / 2.0)))
    e_reg = _np(ntff_3d(res.dft, grid, kn.MARGIN3, (kn.F3,), kn.THETAS3, kn.PHIS3))
    assert np.allclose(e_reg, e_far, rtol=0, atol=1e-12 * np.abs(e_far).max())


def test_directivity_gradient_through_freq_adjoint():
    """d D(phi=0) / d eps_r of a dielectric patch (test_ntff.py:241-273 as a
    CW frequency-domain objective) against central finite differences."""
    import gradenna_b200 as gb
    from gradenna_b200.freq_adjoint import freq_adjoint_gradient, simulate_tm_freq
    from gradenna_b200.ntff import directivity_2d, ntff_2d

    grid = gb.Grid2D(44, 44, 2e-3, 2e-3)
    f0 = 3e9
    n = np.arange(8000)
    env = np.clip(n / 300.0, 0.0, 1.0)
    cur = env * np.sin(2.0 * np.pi * f0 * (n + 0.5) * grid.dt)
    angles = np.linspace(0.0, 2.0 * np.pi, 72, endpoint=False)
    region = (slice(24, 30), slice(19, 25))

    def obj(ph):
        e_far = ntff_2d(ph.dft_ez, ph.dft_hx, ph.dft_hy, grid, 12, (f0,), angles)
        return directivity_2d(e_far, angles)[0, 0]

    common = dict(design_region=region, dft_freqs=(f0,), source_ij=(20, 22),
                  source_current=cur, cpml=gb.CPMLSpec(8))
    theta0 = 2.0 * np.ones((6, 6))
    g = freq_adjoint_gradient(grid, obj, design_eps_r=theta0, env=env, **common)["eps_r"]
    g = g.cpu().numpy()
    assert np.all(np.isfinite(g)) and np.abs(g).max() > 0.0

    def value(th):
        return float(obj(simulate_tm_freq(grid, design_eps_r=th, **common)))

    rng = np.random.default_rng(0)
    v = rng.normal(size=theta0.shape)
    v /= np.linalg.norm(v)
    h = 1e-3
    d_fd = (value(theta0 + h * v) - value(theta0 - h * v)) / (2 * h)
    d_adj = float(np.sum(g * v))
    assert abs(d_adj - d_fd) <= 2e-2 * abs(d_fd), (d_adj, d_fd)
