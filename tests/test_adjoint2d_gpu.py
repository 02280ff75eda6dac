"""GPU checks of the 2D objective reductions and the frequency-domain adjoint.

* Poynting flux (CUDA reduction) against the oracle's numpy restatement of
  monitors.py:20-70, and its CUDA cotangent against torch autograd of the
  same formula written in torch.
* freq_adjoint_gradient against the central finite-difference gradient of
  the same objective through the same solver, on the reference's own
  acceptance cases (tests/test_freq_adjoint.py:37-230: 44x44 grid, CW drive
  with a 300-step ramp, 10000 steps, 8x8 design). The reference compares
  against jax.grad of simulate_tm (unavailable here); the FD gradient of the
  discrete solver is the same quantity up to FD error. Tolerances are the
  reference's: cosine >= 0.999 and directional relative error <= 1e-2
  (2e-2 for the two-tone case).
"""

import numpy as np
import pytest
import torch

from oracle import fdtd2d_np as ref

pytestmark = pytest.mark.gpu

GRID_ARGS = (44, 44, 2e-3, 2e-3)
NPML = 8
F0 = 3e9
N_STEPS = 10000
RAMP = 300
FLUX_REGION = (slice(18, 26), slice(18, 26))
FLUX_BOX = (12, 31, 12, 31)
FLUX_SRC = (14, 22)
S11_REGION = (slice(20, 28), slice(18, 26))
RS = 50.0


def _cw(grid, freqs=(F0,)):
    n = np.arange(N_STEPS)
    env = np.clip(n / float(RAMP), 0.0, 1.0)
    cur = env * sum(np.sin(2.0 * np.pi * f * (n + 0.5) * grid.dt) for f in freqs)
    return cur, env


def test_poynting_kernel_matches_oracle_and_autograd():
    import gradenna_b200 as gb
    from gradenna_b200.monitors import poynting_flux_box_2d

    g = gb.Grid2D(30, 27, 1e-3, 2e-3)
    rng = np.random.default_rng(0)
    K = 3

    def cplx(*shape):
        return rng.normal(size=shape) + 1j * rng.normal(size=shape)

    ez, hx, hy = cplx(K, 30, 27), cplx(K, 30, 26), cplx(K, 29, 27)
    box = (3, 25, 2, 20)
    want = ref.poynting_flux_box_2d(ez, hx, hy, ref.Grid2D(30, 27, 1e-3, 2e-3), box)
    t = [torch.tensor(a, device="cuda", requires_grad=True) for a in (ez, hx, hy)]
    got = poynting_flux_box_2d(*t, g, box)
    assert np.allclose(got.detach().cpu().numpy(), want, rtol=1e-12, atol=0)

    # Cotangent: same formula in plain torch ops, autograd.
    w = torch.tensor([0.3, -1.2, 2.0], device="cuda", dtype=torch.float64)
    (got * w).sum().backward()
    t2 = [torch.tensor(a, device="cuda", requires_grad=True) for a in (ez, hx, hy)]
    il, ir, jb, jt = box
    E, X, Y = t2
    js, isl = slice(jb + 1, jt + 1), slice(il + 1, ir + 1)
    p = -0.5 * torch.real(0.5 * (E[:, ir, js] + E[:, ir + 1, js]) * Y[:, ir, js].conj()).sum(-1) * g.dy
    p = p + 0.5 * torch.real(0.5 * (E[:, il, js] + E[:, il + 1, js]) * Y[:, il, js].conj()).sum(-1) * g.dy
    p = p + 0.5 * torch.real(0.5 * (E[:, isl, jt] + E[:, isl, jt + 1]) * X[:, isl, jt].conj()).sum(-1) * g.dx
    p = p - 0.5 * torch.real(0.5 * (E[:, isl, jb] + E[:, isl, jb + 1]) * X[:, isl, jb].conj()).sum(-1) * g.dx
    (p * w).sum().backward()
    for a, b in zip(t, t2):
        assert torch.allclose(a.grad, b.grad, rtol=1e-12, atol=1e-15)

    # complex64 phasors go through the float kernel.
    got32 = poynting_flux_box_2d(*(x.detach().to(torch.complex64) for x in t), g, box)
    assert np.allclose(got32.cpu().numpy(), want, rtol=1e-5)


def _fd_gradient(value_fn, theta, rel_step=1e-3):
    th = theta.copy()
    grad = np.zeros_like(th)
    for idx in np.ndindex(th.shape):
        h = rel_step * max(abs(th[idx]), 1e-3)
        tp, tm = th.copy(), th.copy()
        tp[idx] += h
        tm[idx] -= h
        grad[idx] = (value_fn(tp) - value_fn(tm)) / (2 * h)
    return grad


def _compare(g_or, g_fa, seed=0):
    g_or, g_fa = np.asarray(g_or).ravel(), np.asarray(g_fa).ravel()
    assert np.all(np.isfinite(g_fa))
    cos = float(np.dot(g_or, g_fa) / (np.linalg.norm(g_or) * np.linalg.norm(g_fa)))
    v = np.random.default_rng(seed).normal(size=g_or.shape)
    v /= np.linalg.norm(v)
    d_or, d_fa = float(np.dot(g_or, v)), float(np.dot(g_fa, v))
    return cos, abs(d_fa - d_or) / max(abs(d_or), 1e-30)


def _flux_case(design_key, theta0, freqs=(F0,)):
    import gradenna_b200 as gb
    from gradenna_b200.freq_adjoint import freq_adjoint_gradient, simulate_tm_freq
    from gradenna_b200.monitors import poynting_flux_box_2d

    grid = gb.Grid2D(*GRID_ARGS)
    cur, env = _cw(grid, freqs)

    def obj(ph):
        p = poynting_flux_box_2d(ph.dft_ez, ph.dft_hx, ph.dft_hy, grid, FLUX_BOX)
        return p.sum()

    common = dict(design_region=FLUX_REGION, dft_freqs=freqs, source_ij=FLUX_SRC,
                  source_current=cur, cpml=gb.CPMLSpec(NPML))

    def value(th):
        ph = simulate_tm_freq(grid, **{f"design_{design_key}": th}, **common)
        return float(obj(ph))

    g_fa = freq_adjoint_gradient(grid, obj, **{f"design_{design_key}": theta0}, env=env,
                                 **common)[design_key].cpu().numpy()
    g_fd = _fd_gradient(value, theta0)
    return g_fd, g_fa


def test_flux_sigma_matches_fd():
    g_fd, g_fa = _flux_case("sigma", 0.01 * np.ones((8, 8)))
    cos, rel = _compare(g_fd, g_fa)
    assert cos >= 0.999, f"flux/sigma cosine {cos:.5f}"
    assert rel <= 1e-2, f"flux/sigma directional rel. error {rel:.2e}"


def test_flux_two_frequencies():
    g_fd, g_fa = _flux_case("sigma", 0.01 * np.ones((8, 8)), freqs=(2.6e9, 3.4e9))
    cos, rel = _compare(g_fd, g_fa)
    assert cos >= 0.999, f"flux 2-freq cosine {cos:.5f}"
    assert rel <= 2e-2, f"flux 2-freq directional rel. error {rel:.2e}"


def test_flux_eps_r_nonuniform():
    rng = np.random.default_rng(3)
    g_fd, g_fa = _flux_case("eps_r", 1.0 + 1.5 * rng.random((8, 8)))
    cos, rel = _compare(g_fd, g_fa)
    assert cos >= 0.999, f"flux/eps_r cosine {cos:.5f}"
    assert rel <= 1e-2
    per = np.abs(g_fd - g_fa) / np.maximum(np.abs(g_fd), 1e-30)
    assert np.median(per) < 2e-2


def test_s11_sigma_matches_fd():
    import gradenna_b200 as gb
    from gradenna_b200.freq_adjoint import freq_adjoint_gradient, simulate_tm_freq
    from gradenna_b200.sparams import s11_power_wave

    grid = gb.Grid2D(*GRID_ARGS)
    cur, env = _cw(grid)
    port = gb.Port((14, 22), RS, cur)

    def obj(ph):
        s = s11_power_wave(ph.port_v[0, 0], ph.port_i[0, 0], RS)
        return s.real**2 + s.imag**2

    common = dict(design_region=S11_REGION, dft_freqs=(F0,), ports=(port,),
                  cpml=gb.CPMLSpec(NPML))
    theta0 = 0.02 * np.ones((8, 8))

    def value(th):
        # The objective reads port phasors rebuilt from the field phasors,
        # exactly as the adjoint path differentiates it.
        from gradenna_b200.freq_adjoint import ports_from_fields

        ph = simulate_tm_freq(grid, design_sigma=th, **common)
        pv, pi = ports_from_fields(ph.dft_ez, ph.dft_hx, ph.dft_hy, grid, [(14, 22)], (F0,))
        return float(obj(ph._replace(port_v=pv, port_i=pi)))

    g_fa = freq_adjoint_gradient(grid, obj, design_sigma=theta0, env=env, **common)["sigma"]
    g_fd = _fd_gradient(value, theta0)
    cos, rel = _compare(g_fd, g_fa.cpu().numpy())
    assert cos >= 0.999, f"S11/sigma cosine {cos:.5f}"
    assert rel <= 1e-2, f"S11/sigma directional rel. error {rel:.2e}"


def test_autograd_function_and_region_monitors():
    """freq_adjoint_objective(...).backward() == freq_adjoint_gradient, and
    recording only the contour boxes gives the same value and gradient."""
    import gradenna_b200 as gb
    from gradenna_b200.freq_adjoint import freq_adjoint_gradient, freq_adjoint_objective
    from gradenna_b200.monitors import poynting_flux_box_2d

    grid = gb.Grid2D(*GRID_ARGS)
    cur, env = _cw(grid)

    def obj(ph):
        return poynting_flux_box_2d(ph.dft_ez, ph.dft_hx, ph.dft_hy, grid, FLUX_BOX)[0]

    il, ir, jb, jt = FLUX_BOX
    mons = [(0, il, jb, ir + 2, jt + 2), (1, il + 1, jb, ir + 1, jt + 1),
            (2, il, jb + 1, ir + 1, jt + 1)]
    common = dict(design_region=FLUX_REGION, dft_freqs=(F0,), source_ij=FLUX_SRC,
                  source_current=cur, cpml=gb.CPMLSpec(NPML), env=env)
    sig = torch.full((8, 8), 0.01, dtype=torch.float64, device="cuda", requires_grad=True)
    val = freq_adjoint_objective(sig, grid, obj, **common)
    val.backward()
    g_ref = freq_adjoint_gradient(grid, obj, design_sigma=0.01 * np.ones((8, 8)), **common)["sigma"]
    assert torch.allclose(sig.grad, g_ref, rtol=1e-12, atol=0)
    sig2 = sig.detach().clone().requires_grad_(True)
    val2 = freq_adjoint_objective(sig2, grid, obj, objective_monitors=mons, **common)
    val2.backward()
    assert torch.allclose(val2, val, rtol=1e-12, atol=0)
    assert torch.allclose(sig2.grad, sig.grad, rtol=1e-10, atol=0)
