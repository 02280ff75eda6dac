"""The 3D frequency-domain adjoint against the exact 3D gradient.

The reference validates freq_adjoint_gradient_3d against jax.grad of its own
3D solve (exact_design_gradient_3d, freq_adjoint.py:724-771,
tests/test_freq_adjoint3d.py). Here oracle/fdtd3d_ad.py stands in for
jax.grad: the same 3D time loop in torch float64 with an autograd reverse
sweep and segment recomputation (the sqrt(N) checkpointing of
fdtd3d.py:735-749), itself checked against the numpy oracle and central
differences (tests/test_oracle_ad3d.py). The oracle runs its torch
operations on the GPU only to be fast; it is not the library.

Cases follow the reference's acceptance setup: 30^3 at 3 mm, CPML 6, CW at
4 GHz with a 300-step ramp, 6000 steps, a 6^3 design box. Bars are the
reference's: cosine >= 0.9999 where the whole gradient is compared, and a
random-direction relative error <= 1.5e-2.
"""

import numpy as np
import pytest
import torch

from oracle import fdtd2d_np as o2
from oracle import fdtd3d_ad as ad
from oracle import fdtd3d_np as o3
from tests.test_adjoint3d_gpu import (CENTER, DR, DR_SHAPE, F0, FLUX_BOX, NPML, _adjoint, _cw,
                                      _flux_box_3d, _grid)

pytestmark = pytest.mark.gpu


def _exact(obj_oracle, key, theta, cur, **kw):
    g = _grid()
    og = o3.Grid3D(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz)
    grads, _ = ad.exact_design_gradient_3d(
        og, obj_oracle, **{f"design_{key}": theta}, design_region=DR, dft_freqs=(F0,),
        source_current=cur, cpml=o2.CPMLSpec(NPML), segment=200, device="cuda", **kw)
    return grads[key]


def _compare(g, g_ref, full):
    cos = float(np.dot(g.ravel(), g_ref.ravel()) / (np.linalg.norm(g) * np.linalg.norm(g_ref)))
    v = np.random.default_rng(0).normal(size=DR_SHAPE)
    rel = abs(np.sum(g * v) - np.sum(g_ref * v)) / abs(np.sum(g_ref * v))
    print(f"\ncosine {cos:.7f}, directional error {rel:.2e}")
    if full:
        assert cos >= 0.9999, cos
    assert rel <= 1.5e-2, rel


@pytest.mark.parametrize("key,theta0", [("sigma", 0.02), ("eps_r", 2.0)])
def test_point_field_gradient_matches_exact(key, theta0):
    import gradenna_b200 as gb

    grid = _grid()
    cur, env = _cw(grid)
    theta = theta0 * np.ones(DR_SHAPE)

    def obj(ph):
        e = ph.dft_ez[0, 19, 15, 15]
        return e.real**2 + e.imag**2

    common = dict(design_region=DR, dft_freqs=(F0,), source_ijk=(11, 15, 15),
                  source_current=cur, cpml=gb.CPMLSpec(NPML))
    g = _adjoint(grid, obj, key, theta, env, common)

    def obj_oracle(dft, pv, pi):
        e = dft["ez"][0, 0, 0, 0]
        return e.real**2 + e.imag**2

    g_ref = _exact(obj_oracle, key, theta, cur, source_ijk=(11, 15, 15),
                   dft_regions={"ez": ((19, 15, 15), (20, 16, 16))})
    _compare(g, g_ref, full=key == "sigma")


def test_flux_gradient_matches_exact():
    import gradenna_b200 as gb
    from gradenna_b200.fdtd3d import DFTMonitor  # noqa: F401

    grid = _grid()
    cur, env = _cw(grid)
    sig0 = 0.02 * np.ones(DR_SHAPE)

    def obj(ph):
        return _flux_box_3d(ph, grid, FLUX_BOX).sum()

    common = dict(design_region=DR, dft_freqs=(F0,), source_ijk=CENTER, source_current=cur,
                  cpml=gb.CPMLSpec(NPML))
    g = _adjoint(grid, obj, "sigma", sig0, env, common)

    class Ph:
        pass

    def obj_oracle(dft, pv, pi):
        ph = Ph()
        for c in ("ex", "ey", "ez", "hx", "hy", "hz"):
            setattr(ph, f"dft_{c}", dft[c])
        return _flux_box_3d(ph, grid, FLUX_BOX).sum()

    g_ref = _exact(obj_oracle, "sigma", sig0, cur, source_ijk=CENTER)
    _compare(g, g_ref, full=True)
