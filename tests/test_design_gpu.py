"""GPU check of the fused design-transform kernels (gdn_design_forward /
gdn_design_backward): rho and d(sum g rho)/dtheta equal the torch form of
topopt's sigmoid -> conic filter -> tanh projection with autograd, for
filter radii with and without a window, two betas, ragged sizes and a
batch, in float64 (1e-12)."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("radius,beta,shape", [(1.0, 8.0, (3, 17, 23)), (2.0, 64.0, (2, 32, 32)),
                                               (6.0, 16.0, (3, 40, 29)), (3.5, 8.0, (1, 104, 104))])
def test_fused_transform_matches_torch(radius, beta, shape):
    from gradenna_b200.topopt import design_transform_batch

    rng = np.random.default_rng(int(radius * 10))
    th = torch.as_tensor(rng.normal(0, 1.5, shape), device="cuda")
    g = torch.as_tensor(rng.normal(size=shape), device="cuda")
    a = th.clone().requires_grad_(True)
    rho = design_transform_batch(a, beta, radius)
    (rho * g).sum().backward()
    b = th.cpu().clone().requires_grad_(True)
    ref = design_transform_batch(b, beta, radius)  # torch form on the CPU
    (ref * g.cpu()).sum().backward()
    torch.testing.assert_close(rho.detach().cpu(), ref.detach(), rtol=1e-12, atol=1e-12)
    torch.testing.assert_close(a.grad.cpu(), b.grad, rtol=1e-10, atol=1e-12)
