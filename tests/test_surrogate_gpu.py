"""GPU checks of the learned design surrogate on the antenna problem at 3 mm
cells (AntennaProblem.coarse(): 96 x 96 grid, 32 x 32 design, 2400 steps):

* the batched training-data generator labels every design with the same
  radiated fraction as the FDTD verifier evaluating it alone;
* the U-Net trained by its own kernels on 1024 solver-labelled designs
  predicts the held-out log radiated fraction (R^2 >= 0.7);
* what the trained network gains: with the same outer-iteration budget the
  batched+surrogate optimiser reaches a verified radiated fraction at least
  3x that of the identical loop without the network (linear model only,
  which stalls near the gray start; measured margins 8-18x).
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    from gradenna_b200 import surrogate as S

    P = S.AntennaProblem.coarse()
    data = S.generate_dataset(P, 1024, seed=0)
    sur, hist = S.train_surrogate(data, epochs=30)
    return P, data, sur, hist


def test_dataset_labels_match_single_evaluation(trained):
    from gradenna_b200 import surrogate as S

    P, data, _, _ = trained
    assert data["rho"].shape == (1024, 32, 32) and data["ez"].shape == (1024, 32, 32, 2)
    assert torch.isfinite(data["fraction"]).all() and float(data["fraction"].max()) > 0
    for k in (0, 7):
        f, ez, _ = S.evaluate(P, data["rho"][k][None], gradient=False)
        assert abs(float(f[0]) - float(data["fraction"][k])) <= 1e-4 * float(data["fraction"].max())
        ez_ri = torch.asinh(torch.stack([ez[0].real, ez[0].imag], -1) / data["ez_scale"])
        assert float((ez_ri.float() - data["ez"][k].to(ez_ri.device)).abs().max()) <= 1e-3


def test_trained_network_predicts_fraction(trained):
    _, _, _, hist = trained
    assert np.all(np.isfinite(hist["loss"])) and hist["loss"][-1] < hist["loss"][0]
    assert hist["val_r2_log"][-1] >= 0.7, hist["val_r2_log"]


def test_network_gain_over_linear_model(trained):
    from gradenna_b200 import surrogate as S

    P, _, sur, _ = trained
    su = S.optimize_surrogate(P, sur, n_outer=6, iters_per_beta=2)
    lin = S.optimize_surrogate(P, None, use_network=False, n_outer=6, iters_per_beta=2)
    pl = S.optimize_plain(P, n_iters=60)
    f_su, f_lin = float(su["fraction"][-1]), float(lin["fraction"][-1])
    # The same loop without the network stalls near the gray start.
    assert f_su >= 3.0 * f_lin, (f_su, f_lin)
    # The plain optimiser is the reference point the benchmark measures
    # against (bench.py --workload surrogate, at the 1 mm hero size); at this
    # coarse size how far the 6-iteration surrogate run gets depends on the
    # training run, so only its progress is checked here.
    assert np.all(np.isfinite(pl["fraction"])) and f_su > float(pl["fraction"][0])
    # every accepted step was verified: the recorded fractions never decrease
    # within a beta stage
    for b in np.unique(su["beta"]):
        fb = su["fraction"][su["beta"] == b]
        assert np.all(np.diff(fb) >= 0)
