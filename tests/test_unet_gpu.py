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


@pytest.mark.parametrize("cin,cout,taps,hw,n", [(32, 32, 9, (20, 28), 3), (64, 64, 9, (13, 13), 5),
                                                (128, 256, 9, (26, 26), 2), (64, 32, 9, (52, 52), 1),
                                                (256, 128, 1, (13, 13), 4), (32, 3, 1, (24, 24), 2),
                                                (96, 40, 9, (17, 11), 2)])
def test_tensor_core_conv_matches_mma_conv(cin, cout, taps, hw, n):
    """gdn_sur_conv_fwd_tc (tcgen05, TMEM accumulators) against gdn_sur_conv_fwd
    (mma.sync) on the same bf16 operands: channel slices in and out, bias,
    leaky ReLU and the backward mask, ragged pixel counts and channel counts
    that are not multiples of the tile; FP32 results within 2e-3 of the peak
    (the two sum the same products in different orders)."""
    import ctypes

    from gradenna_b200 import _native
    from gradenna_b200.unet import tc_timeouts

    lib = _native.load()
    h, w = hw
    g = torch.Generator(device="cpu").manual_seed(cin * 7 + cout)
    stride_in, c0_in = cin + 16, 8
    x = torch.randn((n, h, w, stride_in), generator=g).to(torch.bfloat16).cuda()
    wt = (torch.randn((taps * cin, cout), generator=g) / (taps * cin) ** 0.5).to(torch.bfloat16).cuda()
    bias = torch.randn(cout, generator=g).cuda()
    mask = torch.randn((n, h, w, cout), generator=g).to(torch.bfloat16).cuda()
    wk = torch.empty_like(wt)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _native.check(lib.gdn_sur_weights_kmajor(wt.data_ptr(), cin, cout, taps, 0, wk.data_ptr(), s))
    outs = []
    tc_timeouts(reset=True)
    for fn, wp in ((lib.gdn_sur_conv_fwd, wt), (lib.gdn_sur_conv_fwd_tc, wk)):
        res = []
        for relu, use_mask in ((1, False), (0, True)):
            o16 = torch.zeros((n, h, w, cout + 8), dtype=torch.bfloat16, device="cuda")
            o32 = torch.zeros((n * h * w, cout), dtype=torch.float32, device="cuda")
            _native.check(fn(x.data_ptr(), stride_in, c0_in, n, h, w, cin, taps, wp.data_ptr(),
                             bias.data_ptr(), cout, relu, 0.1, o16.data_ptr(), cout + 8, 8,
                             o32.data_ptr(), mask.data_ptr() if use_mask else None,
                             cout if use_mask else 0, 0, s))
            res.append((o16, o32))
        outs.append(res)
    torch.cuda.synchronize()
    assert tc_timeouts(reset=True) == 0
    for (a16, a32), (b16, b32) in zip(outs[0], outs[1]):
        scale = float(a32.abs().max())
        assert float((a32 - b32).abs().max()) <= 2e-3 * scale
        assert float((a16[..., 8:].float() - b16[..., 8:].float()).abs().max()) <= 1e-2 * scale
        assert torch.equal(a16[..., :8], b16[..., :8])  # untouched channels


def test_tensor_core_flipped_weights_give_input_gradient():
    """gdn_sur_weights_kmajor(flip=1) + gdn_sur_conv_fwd_tc equals the
    mma.sync input-gradient convolution with gdn_sur_flip_weights."""
    import ctypes

    from gradenna_b200 import _native

    lib = _native.load()
    cin, cout, taps, n, h, w = 64, 128, 9, 2, 26, 26
    g = torch.Generator(device="cpu").manual_seed(3)
    gy = torch.randn((n, h, w, cout), generator=g).to(torch.bfloat16).cuda()
    wt = (torch.randn((taps * cin, cout), generator=g) / 24).to(torch.bfloat16).cuda()
    flip = torch.empty_like(wt)
    fk = torch.empty_like(wt)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _native.check(lib.gdn_sur_flip_weights(wt.data_ptr(), cin, cout, taps, flip.data_ptr(), s))
    _native.check(lib.gdn_sur_weights_kmajor(wt.data_ptr(), cin, cout, taps, 1, fk.data_ptr(), s))
    o = [torch.zeros((n * h * w, cin), dtype=torch.float32, device="cuda") for _ in range(2)]
    for fn, wp, out in ((lib.gdn_sur_conv_fwd, flip, o[0]), (lib.gdn_sur_conv_fwd_tc, fk, o[1])):
        _native.check(fn(gy.data_ptr(), cout, 0, n, h, w, cout, taps, wp.data_ptr(), None, cin, 0,
                         0.1, None, 0, 0, out.data_ptr(), None, 0, 0, s))
    torch.cuda.synchronize()
    assert float((o[0] - o[1]).abs().max()) <= 2e-3 * float(o[0].abs().max())


@pytest.mark.parametrize("step", [0, 3, 8])
def test_tensor_core_conv_abort_path(step):
    """A tensor-core convolution whose bounded wait runs out (injected at
    reduction step 0, 3 or 8 of 9, with MMAs of earlier steps possibly still
    in flight) drains them, releases TMEM and returns: the launch writes no
    results, gdn_sur_status counts it, the context stays usable and the next
    convolution is correct."""
    import ctypes

    from gradenna_b200 import _native
    from gradenna_b200.unet import tc_timeouts

    lib = _native.load()
    cin, cout, taps, n, h, w = 64, 64, 9, 2, 26, 26  # 9 reduction steps of 64
    g = torch.Generator(device="cpu").manual_seed(11)
    x = torch.randn((n, h, w, cin), generator=g).to(torch.bfloat16).cuda()
    wt = (torch.randn((taps * cin, cout), generator=g) / 24).to(torch.bfloat16).cuda()
    wk = torch.empty_like(wt)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _native.check(lib.gdn_sur_weights_kmajor(wt.data_ptr(), cin, cout, taps, 0, wk.data_ptr(), s))

    def conv(fn, wp):
        out = torch.full((n * h * w, cout), 7.0, dtype=torch.float32, device="cuda")
        _native.check(fn(x.data_ptr(), cin, 0, n, h, w, cin, taps, wp.data_ptr(), None, cout, 0,
                         0.1, None, 0, 0, out.data_ptr(), None, 0, 0, s))
        return out

    tc_timeouts(reset=True)
    try:
        _native.check(lib.gdn_sur_inject_timeout(step))
        bad = conv(lib.gdn_sur_conv_fwd_tc, wk)
        torch.cuda.synchronize()
    finally:
        _native.check(lib.gdn_sur_inject_timeout(-1))
    assert tc_timeouts(reset=True) == 1
    assert bool((bad == 7.0).all())  # nothing written
    good = conv(lib.gdn_sur_conv_fwd_tc, wk)
    ref = conv(lib.gdn_sur_conv_fwd, wt)
    torch.cuda.synchronize()
    assert tc_timeouts(reset=True) == 0
    assert float((good - ref).abs().max()) <= 2e-3 * float(ref.abs().max())
