"""GPU checks of the BF16 U-Net surrogate kernels against the torch float32
CPU oracle (oracle/unet_torch.py, which rounds weights and stored
activations to bfloat16 at the same points):

* forward output within 2e-2 of the output's peak, on the full 104 x 104
  4-level network and on a small 3-level network whose pixel count is not a
  multiple of the 64-pixel tile;
* loss, weight gradient and input gradient of the training loss: cosine
  >= 0.995 and relative norm error <= 5e-2 against autograd (the CUDA
  gradients are stored in bfloat16 between layers);
* power_grad equals autograd of the summed power prediction;
* a few hundred Adam steps on a fixed batch reduce the loss tenfold.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def _cos(a, b):
    return float(torch.dot(a.flatten(), b.flatten())
                 / (torch.linalg.vector_norm(a) * torch.linalg.vector_norm(b)))


def _data(spec, n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, 1, (n, spec.height, spec.width)).astype(np.float32)
    tf = rng.normal(0, 0.5, (n, spec.height, spec.width, 2)).astype(np.float32)
    tp = rng.uniform(0, 1, n).astype(np.float32)
    return x, tf, tp


@pytest.mark.parametrize("spec_kw,n", [(dict(), 2), (dict(height=20, width=28, base=32, levels=3), 3)])
def test_forward_matches_oracle(spec_kw, n):
    from gradenna_b200.unet import UNet, UNetSpec
    from oracle.unet_torch import unet_forward

    spec = UNetSpec(**spec_kw)
    net = UNet(spec, seed=3)
    x, _, _ = _data(spec, n, 0)
    out, power = net.forward(torch.as_tensor(x, device="cuda"))
    ref = unet_forward(net.theta.cpu(), [tuple(ly) for ly in net.layers], spec.levels,
                       torch.as_tensor(x)).permute(0, 2, 3, 1)
    scale = float(ref.abs().max())
    assert float((out.cpu() - ref).abs().max()) <= 2e-2 * scale
    np.testing.assert_allclose(power.cpu().numpy(), ref[..., 2].mean(dim=(1, 2)).numpy(),
                               atol=2e-2 * scale)


@pytest.mark.parametrize("spec_kw,n", [(dict(height=20, width=28, base=32, levels=3), 3),
                                       (dict(height=32, width=32, base=32, levels=4), 2)])
def test_gradients_match_oracle(spec_kw, n):
    from gradenna_b200.unet import UNet, UNetSpec
    from oracle.unet_torch import unet_loss

    spec = UNetSpec(**spec_kw)
    net = UNet(spec, seed=5)
    x, tf, tp = _data(spec, n, 1)
    loss, g_theta, g_x = net.gradients(torch.as_tensor(x, device="cuda"), tf, tp,
                                       field_weight=1.0, power_weight=3.0)
    theta = net.theta.cpu().clone().requires_grad_(True)
    xt = torch.as_tensor(x).clone().requires_grad_(True)
    ref = unet_loss(theta, [tuple(ly) for ly in net.layers], spec.levels, xt,
                    torch.as_tensor(tf), torch.as_tensor(tp), 1.0, 3.0)
    ref.backward()
    assert abs(float(loss) - float(ref)) <= 1e-2 * float(ref)
    gt = g_theta.cpu()
    assert _cos(gt, theta.grad) >= 0.995 and _rel(gt, theta.grad) <= 5e-2
    for ly in net.layers:  # every layer's weight gradient, not just the total
        sl = slice(ly.w_off, ly.w_off + ly.taps * ly.cin * ly.cout)
        assert _cos(gt[sl], theta.grad[sl]) >= 0.99, ly.name
        bs = slice(ly.b_off, ly.b_off + ly.cout)
        assert _cos(gt[bs], theta.grad[bs]) >= 0.99, ly.name
    assert _cos(g_x.cpu(), xt.grad) >= 0.99 and _rel(g_x.cpu(), xt.grad) <= 1e-1


def test_power_grad_matches_oracle():
    from gradenna_b200.unet import UNet, UNetSpec
    from oracle.unet_torch import unet_forward

    spec = UNetSpec(height=24, width=24, levels=3)
    net = UNet(spec, seed=7)
    x, _, _ = _data(spec, 4, 2)
    w = np.array([1.0, -0.5, 2.0, 0.25], np.float32)
    p, gx = net.power_grad(torch.as_tensor(x, device="cuda"), weight=w)
    xt = torch.as_tensor(x).clone().requires_grad_(True)
    out = unet_forward(net.theta.cpu(), [tuple(ly) for ly in net.layers], spec.levels, xt)
    pr = out[:, 2].mean(dim=(1, 2))
    (pr * torch.as_tensor(w)).sum().backward()
    np.testing.assert_allclose(p.cpu().numpy(), pr.detach().numpy(),
                               atol=2e-2 * float(pr.abs().max()))
    assert _cos(gx.cpu(), xt.grad) >= 0.99


def test_training_reduces_loss():
    from gradenna_b200.unet import UNet, UNetSpec

    spec = UNetSpec(height=32, width=32, levels=3)
    net = UNet(spec, seed=0, learning_rate=2e-3)
    x, _, _ = _data(spec, 16, 3)
    xs = torch.as_tensor(x, device="cuda")
    # a learnable target: smooth functions of the density
    sm = torch.nn.functional.avg_pool2d(xs[:, None], 5, 1, 2)[:, 0]
    tf = torch.stack([sm - 0.5, (xs - sm) * 2], dim=-1)
    tp = xs.mean(dim=(1, 2)) * 2
    losses = [float(net.train_step(xs, tf, tp)) for _ in range(300)]
    assert np.all(np.isfinite(losses))
    assert np.mean(losses[-10:]) < 0.1 * np.mean(losses[:3])
