"""GPU checks of the antenna problem under the reference's pulse drive
(AntennaProblem(drive_kind="pulse"): gaussian_pulse_for_band(1.5, 3.5 GHz)
at the port, export_viz.py:136-138), verified with the exact time-domain
adjoint: the batched verifier's gradient equals time_domain_gradient chained
through sigma_from_density, and a few plain Adam iterations on it raise the
radiated fraction."""

import dataclasses
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_pulse_verifier_gradient_and_plain_steps():
    from gradenna_b200 import surrogate as S
    from gradenna_b200.fdtd2d import Port
    from gradenna_b200.monitors import poynting_box_monitors
    from gradenna_b200.time_adjoint import time_domain_gradient

    P = dataclasses.replace(S.AntennaProblem.coarse(), drive_kind="pulse")
    rho = S.random_densities(1, P.design_shape, seed=5, radius_range=(2.0, 8.0), device="cuda")
    f, _, g = S.evaluate(P, rho, gradient=True)
    assert torch.isfinite(f).all() and float(f[0]) >= 0
    sig = P.design_sigma(rho[0].double())
    v, _ = P.drive()
    gs = time_domain_gradient(P.grid, P.objective(), design_sigma=sig,
                              design_region=P.design_region, dft_freqs=(P.f0,),
                              ports=(Port(P.port_ij, P.resistance, v.astype(np.float32)),),
                              cpml=P.cpml, dtype=torch.float32,
                              objective_monitors=poynting_box_monitors(P.flux_box))["sigma"]
    lo, hi = math.log10(P.sigma_min), math.log10(P.sigma_max)
    want = gs * sig * (math.log(10.0) * (hi - lo))
    rel = float(torch.linalg.vector_norm(g[0] - want) / torch.linalg.vector_norm(want))
    assert rel <= 1e-3, rel
    pl = S.optimize_plain(P, n_iters=6)
    assert np.all(np.isfinite(pl["fraction"])) and pl["fraction"][-1] > pl["fraction"][0]
