"""CPU checks of the surrogate pipeline's host logic (no CUDA work):

* the batched design transform equals topopt.DesignTransform per design;
* seeded random densities are reproducible, lie in [0, 1] and span gray to
  nearly binary designs;
* the 3 mm antenna problem has the hero's physical layout within two cells
  (port inside the design region, flux box outside the CPML, the same
  duration), and the
  feed cell carries no design conductivity;
* the surrogate's fraction and its gradient follow the log-fraction output
  scaling (chain rule against autograd).
"""

import math

import numpy as np
import torch


def test_batched_transform_matches_design_transform():
    from gradenna_b200.surrogate import design_transform
    from gradenna_b200.topopt import DesignTransform

    rng = np.random.default_rng(0)
    th = torch.as_tensor(rng.normal(size=(3, 20, 24)))
    for radius in (1.0, 2.0, 6.0):
        got = design_transform(th, 16.0, radius)
        tr = DesignTransform(radius_cells=radius)
        for b in range(3):
            torch.testing.assert_close(got[b], tr(th[b], 16.0), rtol=1e-12, atol=1e-12)


def test_random_densities_reproducible_and_varied():
    from gradenna_b200.surrogate import random_densities

    a = random_densities(40, (32, 32), seed=3)
    b = random_densities(40, (32, 32), seed=3)
    c = random_densities(40, (32, 32), seed=4)
    assert torch.equal(a, b) and not torch.equal(a, c)
    assert float(a.min()) >= 0.0 and float(a.max()) <= 1.0
    gray = (4 * a * (1 - a)).mean(dim=(1, 2))
    assert float(gray.min()) < 0.3 and float(gray.max()) > 0.8


def test_coarse_problem_matches_hero_layout():
    from gradenna_b200.surrogate import AntennaProblem

    hero, coarse = AntennaProblem(), AntennaProblem.coarse()
    for P in (hero, coarse):
        i0, i1, j0, j1 = P.design
        assert i0 <= P.port_ij[0] < i1 and j0 <= P.port_ij[1] < j1
        il, ir, jb, jt = P.flux_box
        assert min(il, jb) >= P.cpml_cells + 2 and max(ir, jt) <= P.nx - P.cpml_cells - 3
        assert P.p_avail() > 0
        m = P.design_mask()
        assert int((~m).sum()) == 1 and not bool(m[P.port_ij[0] - i0, P.port_ij[1] - j0])
        s = P.design_sigma(torch.ones(P.design_shape, dtype=torch.float64))
        assert float(s[P.port_ij[0] - i0, P.port_ij[1] - j0]) == 0.0
        assert math.isclose(float(s.max()), P.sigma_max, rel_tol=1e-12)
    # same physical layout within two coarse cells (the coarse design is 32
    # cells = 96 mm wide, a multiple of 8 for the U-Net, against 104 mm) and
    # the same duration within 5 %
    for attr in ("design", "flux_box"):
        hv = np.asarray(getattr(hero, attr)) * hero.dx
        cv = np.asarray(getattr(coarse, attr)) * coarse.dx
        assert np.all(np.abs(hv - cv) <= 2 * coarse.dx + 1e-12)
    assert abs(hero.n_steps * hero.grid.dt - coarse.n_steps * coarse.grid.dt) < 0.05 * hero.n_steps * hero.grid.dt


def test_surrogate_scaling_chain_rule():
    from gradenna_b200.surrogate import Surrogate

    class FakeNet:
        """power_grad of p(x) = mean(x^2) per design, gradient 2x / HW."""

        def power_grad(self, x, weight=None):
            x = torch.as_tensor(x, dtype=torch.float32)
            return (x ** 2).mean(dim=(1, 2)), 2 * x / (x.shape[1] * x.shape[2])

    sur = Surrogate(FakeNet(), power_mean=-6.0, power_std=1.7, ez_scale=1.0, power_floor=1e-4)
    x = torch.rand(2, 5, 6, dtype=torch.float32)
    f, g = sur.fraction_grad(x)
    xr = x.clone().requires_grad_(True)
    fr = torch.exp((xr ** 2).mean(dim=(1, 2)) * 1.7 - 6.0) - 1e-4
    fr.sum().backward()
    torch.testing.assert_close(f, fr.detach(), rtol=1e-6, atol=1e-12)
    torch.testing.assert_close(g, xr.grad, rtol=1e-5, atol=1e-12)
