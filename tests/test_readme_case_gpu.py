"""The reference README's own example (README.md:24-39): a 140 x 140 grid
at 2 mm, a 50 ohm port at (70, 55) driven by gaussian_pulse_for_band(2,
3 GHz) for 3500 steps, CPML 10, copper design
sigma_from_density(rho) on [44:96, 60:112], and the gradient of the negative
radiated power at 2.45 GHz through the box (20, 120, 20, 120) with respect
to rho = 0.5 (52 x 52): written with this library's surface
(time_domain_objective + torch autograd in place of jax.grad) and compared
with autograd through the oracle's time loop (the stand-in for jax.grad)."""

import math

import numpy as np
import pytest
import torch

from oracle import fdtd2d_ad as ad
from oracle import fdtd2d_np as onp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-9), (torch.float32, 5e-3)])
def test_readme_gradient(dtype, tol):
    import gradenna_b200 as gb
    from gradenna_b200.materials import sigma_from_density
    from gradenna_b200.monitors import poynting_flux_box_2d
    from gradenna_b200.sparams import gaussian_pulse_for_band
    from gradenna_b200.time_adjoint import time_domain_objective

    grid = gb.Grid2D(nx=140, ny=140, dx=2e-3, dy=2e-3)
    pulse = gaussian_pulse_for_band(2.0e9, 3.0e9)
    v = pulse((np.arange(3500) + 0.5) * grid.dt)
    region = (slice(44, 96), slice(60, 112))

    def radiated(ph):
        return poynting_flux_box_2d(ph.dft_ez, ph.dft_hx, ph.dft_hy, grid,
                                    (20, 120, 20, 120))[0]

    rho = torch.full((52, 52), 0.5, dtype=torch.float64, device="cuda", requires_grad=True)
    loss = -time_domain_objective(sigma_from_density(rho), grid, radiated, design_region=region,
                                  dft_freqs=(2.45e9,), ports=(gb.Port((70, 55), 50.0, v),),
                                  cpml=gb.CPMLSpec(thickness=10), dtype=dtype)
    loss.backward()
    got = rho.grad.cpu().numpy()

    og = onp.Grid2D(140, 140, 2e-3, 2e-3)
    sig = sigma_from_density(np.full((52, 52), 0.5))
    ex, val = ad.exact_design_gradient(
        og, lambda ez, hx, hy, pv, pi: ad.poynting_flux_box_2d_t(ez, hx, hy, og,
                                                                  (20, 120, 20, 120)).sum(),
        design_sigma=sig, design_region=region, dft_freqs=(2.45e9,),
        ports=(onp.Port((70, 55), 50.0, v),), cpml=onp.CPMLSpec(10), segment=500, device="cuda")
    want = -ex["sigma"] * sig * math.log(10.0) * 9.0  # d sigma / d rho, log10 span 1e-4 .. 1e5
    assert abs(float(loss) + val) <= 1e-6 * abs(val)
    rel = float(np.linalg.norm(got - want) / np.linalg.norm(want))
    assert rel <= tol, rel
