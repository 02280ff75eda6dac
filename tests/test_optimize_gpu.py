"""GPU check of the topology-optimisation driver on an FDTD objective: Adam
with beta continuation over a sigma_from_density design, the loss and its
gradient from freq_adjoint_objective (forward run + two-run adjoint on the
GPU), improves the radiated flux of a CW source within a few iterations."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_optimize_flux_with_freq_adjoint():
    import gradenna_b200 as gb
    from gradenna_b200.freq_adjoint import freq_adjoint_objective
    from gradenna_b200.materials import sigma_from_density
    from gradenna_b200.monitors import poynting_box_monitors, poynting_flux_box_2d
    from gradenna_b200.topopt import DesignTransform, optimize

    grid = gb.Grid2D(44, 44, 2e-3, 2e-3)
    f0 = 3e9
    n = np.arange(6000)
    env = np.clip(n / 300.0, 0.0, 1.0)
    cur = env * np.sin(2 * np.pi * f0 * (n + 0.5) * grid.dt)
    box = (12, 31, 12, 31)

    def flux(ph):
        return poynting_flux_box_2d(ph.dft_ez, ph.dft_hx, ph.dft_hy, grid, box).sum()

    def loss_fn(rho, beta):
        sig = sigma_from_density(rho)
        p = freq_adjoint_objective(sig, grid, flux, design_region=(slice(18, 26), slice(18, 26)),
                                   dft_freqs=(f0,), env=env, source_ij=(14, 22),
                                   source_current=cur, cpml=gb.CPMLSpec(8),
                                   objective_monitors=poynting_box_monitors(box))
        return -p / 1e-9

    theta0 = torch.zeros((8, 8), dtype=torch.float64, device="cuda")
    out = optimize(loss_fn, theta0, n_steps=8, betas=(4.0, 8.0), learning_rate=0.3,
                   transform=DesignTransform(radius_cells=2.0), n_snapshots=2)
    assert np.all(np.isfinite(out["loss"]))
    assert out["loss"][-1] < out["loss"][0]
    assert out["rho"].shape == (8, 8) and out["theta"].device.type == "cuda"
