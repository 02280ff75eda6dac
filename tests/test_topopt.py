"""Host checks of the topology-optimisation helpers (src/gradenna/topopt.py):
the Adam + beta-continuation driver against a plain numpy Adam on an
analytic loss, the filter on 1D/2D/3D, the gray indicator and the
fabrication checks (tests/test_topopt.py of the reference: connectivity and
minimum-feature screens)."""

import numpy as np
import torch

from gradenna_b200.topopt import (DesignTransform, conic_filter, connected_to_seed,
                                  gray_indicator, minimum_feature_size, optimize)


def _adam_np(grad_fn, x, lr, steps, b1=0.9, b2=0.999, eps=1e-8):
    m = np.zeros_like(x)
    v = np.zeros_like(x)
    for t in range(1, steps + 1):
        g = grad_fn(x, t - 1)
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        x = x - lr * (m / (1 - b1**t)) / (np.sqrt(v / (1 - b2**t)) + eps)
    return x


def test_optimize_matches_numpy_adam_on_analytic_loss():
    rng = np.random.default_rng(0)
    target = rng.uniform(0, 1, (6, 7))
    theta0 = rng.normal(size=(6, 7))
    tr = DesignTransform(radius_cells=1.0)  # identity filter: rho = projected sigmoid

    def loss_fn(rho, beta):
        return torch.sum((rho - torch.as_tensor(target)) ** 2)

    out = optimize(loss_fn, torch.as_tensor(theta0), n_steps=12, betas=(2.0, 4.0),
                   learning_rate=0.05, transform=tr, n_snapshots=3)

    def grad_np(th, i):
        beta = 2.0 if i < 6 else 4.0
        t = torch.as_tensor(th).requires_grad_(True)
        loss_fn(tr(t, beta), beta).backward()
        return t.grad.numpy()

    want = _adam_np(grad_np, theta0.copy(), 0.05, 12)
    assert np.allclose(out["theta"].numpy(), want, rtol=1e-10, atol=1e-12)
    assert list(out["beta"]) == [2.0] * 6 + [4.0] * 6
    assert out["loss"][-1] < out["loss"][0]
    assert [s for s, _ in out["snapshots"]] == [0, 6, 11]  # round(5.5) -> 6
    assert np.allclose(out["rho"].numpy(), tr(out["theta"], 4.0).numpy())
    assert out["gray"].shape == (12,)


def test_conic_filter_preserves_constants_in_1d_2d_3d():
    for shape in ((17,), (9, 11), (6, 7, 8)):
        x = torch.full(shape, 0.37, dtype=torch.float64)
        assert torch.allclose(conic_filter(x, 2.5), x, atol=1e-14)


def test_gray_indicator():
    assert float(gray_indicator(torch.tensor([0.0, 1.0]))) == 0.0
    assert float(gray_indicator(torch.tensor([0.5, 0.5]))) == 1.0


def test_connectivity_and_minimum_feature():
    rho = np.zeros((12, 12))
    rho[2:5, 2:10] = 1.0   # bar connected to the seed
    rho[8:10, 8:11] = 1.0  # island
    m = connected_to_seed(rho, (3, 3))
    assert m[3, 8] and not m[9, 9]
    assert not connected_to_seed(rho, (0, 0)).any()
    thin = np.zeros((12, 12))
    thin[5, 1:11] = 1.0    # one-cell line
    thin[1:5, 1:5] = 1.0   # 4x4 square
    bad = minimum_feature_size(thin, 3)
    assert bad[5, 6] and not bad[2, 2]
    assert not minimum_feature_size(thin, 1).any()
