"""CPU checks of the surrogate network's host logic and of the identities
its CUDA kernels rely on (no device work):

* the layer table: channel counts, 8-element aligned offsets and a
  parameter count near 2M for the default 104 x 104, 4-level, 32-channel
  network;
* the input gradient of a convolution equals the convolution of the output
  gradient with the point-reflected, transposed weights that
  gdn_sur_flip_weights writes (restated here in numpy);
* the activation-mask rule: multiplying the input gradient of every
  convolution by (input > 0 ? 1 : slope) reproduces autograd through the
  leaky ReLUs, pooling, upsampling and concatenation of the U-Net (checked
  on the oracle network in float64).
"""

import numpy as np
import torch
import torch.nn.functional as F


def test_layer_table():
    from gradenna_b200.unet import UNetSpec, unet_layers

    layers, n = unet_layers(UNetSpec())
    assert 1.8e6 < n < 2.2e6
    assert all(ly.w_off % 8 == 0 and ly.b_off % 8 == 0 for ly in layers)
    names = [ly.name for ly in layers]
    assert names[:2] == ["enc0a", "enc0b"] and names[-1] == "head"
    by = {ly.name: ly for ly in layers}
    assert by["enc0a"].cin == 1 and by["enc3b"].cout == 256 and by["dec0a"].cin == 64
    assert by["head"].taps == 1 and not by["head"].relu
    end = max(ly.b_off + ly.cout for ly in layers)
    assert end <= n
    import pytest

    with pytest.raises(ValueError):
        unet_layers(UNetSpec(height=100))


def _flip_np(w, cin, cout, taps):
    """gdn_sur_flip_weights: wt[(taps-1-tap)*cout + co][ci] = w[tap*cin + ci][co]."""
    w = w.reshape(taps, cin, cout)
    wt = np.empty((taps, cout, cin), w.dtype)
    for tap in range(taps):
        wt[taps - 1 - tap] = w[tap].T
    return wt.reshape(taps * cout, cin)


def _conv_nhwc(x, w, cin, cout, taps):
    """The kernel's convolution: out[p, co] = sum x[p + d(tap), ci] w[tap*cin+ci][co]."""
    k = 3 if taps == 9 else 1
    wt = torch.as_tensor(w.reshape(k, k, cin, cout)).permute(3, 2, 0, 1)
    return F.conv2d(x.permute(0, 3, 1, 2), wt, padding=k // 2).permute(0, 2, 3, 1)


def test_flipped_weights_give_the_input_gradient():
    rng = np.random.default_rng(0)
    for taps in (9, 1):
        cin, cout = 5, 7
        w = rng.normal(size=(taps * cin, cout))
        x = torch.tensor(rng.normal(size=(2, 6, 9, cin)), requires_grad=True)
        g = torch.tensor(rng.normal(size=(2, 6, 9, cout)))
        (_conv_nhwc(x, w, cin, cout, taps) * g).sum().backward()
        via_flip = _conv_nhwc(g, _flip_np(w, cin, cout, taps), cout, cin, taps)
        np.testing.assert_allclose(via_flip.numpy(), x.grad.numpy(), rtol=1e-10, atol=1e-10)


def test_relu_mask_rule_matches_autograd():
    """Backward through the oracle network using only 'input gradient of each
    conv times (its input > 0 ? 1 : slope)' equals autograd (float64, no
    rounding)."""
    from gradenna_b200.unet import UNetSpec, unet_layers
    from oracle.unet_torch import unet_forward

    spec = UNetSpec(height=8, width=12, base=4, levels=3)
    layers, n = unet_layers(spec)
    rng = np.random.default_rng(1)
    theta = torch.tensor(rng.normal(0, 0.4, n))
    x = torch.tensor(rng.uniform(0, 1, (2, 8, 12)), requires_grad=True)
    out = unet_forward(theta, [tuple(ly) for ly in layers], spec.levels, x, bf16=False)
    gout = torch.tensor(rng.normal(size=out.shape))
    (out * gout).sum().backward()
    want = x.grad.clone()

    # Manual backward with the mask rule, mirroring gradenna_b200.unet._backward.
    by = {ly.name: ly for ly in layers}

    def wb(ly):
        w = theta[ly.w_off:ly.w_off + ly.taps * ly.cin * ly.cout].numpy()
        return w, theta[ly.b_off:ly.b_off + ly.cout]

    def conv(ly, h):
        w, b = wb(ly)
        y = _conv_nhwc(h, w, ly.cin, ly.cout, ly.taps) + b
        return F.leaky_relu(y, spec.neg_slope) if ly.relu else y

    def tconv(ly, g, mask):
        w, _ = wb(ly)
        gi = _conv_nhwc(g, _flip_np(w, ly.cin, ly.cout, ly.taps), ly.cout, ly.cin, ly.taps)
        if mask is None:
            return gi
        return gi * (1.0 - (1.0 - spec.neg_slope) * (mask <= 0).to(gi.dtype))

    L = spec.levels
    with torch.no_grad():
        xs, as_, cats, ds, dps, us, skips = {}, {}, {}, {}, {}, {}, {}
        h = x.detach()[..., None]
        for lev in range(L):
            xs[lev] = h
            as_[lev] = conv(by[f"enc{lev}a"], h)
            s = conv(by[f"enc{lev}b"], as_[lev])
            if lev < L - 1:
                skips[lev] = s
                h = F.max_pool2d(s.permute(0, 3, 1, 2), 2).permute(0, 2, 3, 1)
            else:
                ds[lev] = s
        for lev in range(L - 2, -1, -1):
            us[lev] = conv(by[f"up{lev}"], ds[lev + 1])
            up = F.interpolate(us[lev].permute(0, 3, 1, 2), scale_factor=2,
                               mode="nearest").permute(0, 2, 3, 1)
            cats[lev] = torch.cat([skips[lev], up], dim=-1)
            dps[lev] = conv(by[f"dec{lev}a"], cats[lev])
            ds[lev] = conv(by[f"dec{lev}b"], dps[lev])
        g = gout.permute(0, 2, 3, 1)
        gd = {0: tconv(by["head"], g, ds[0])}
        gcat = {}
        for lev in range(L - 1):
            gdp = tconv(by[f"dec{lev}b"], gd[lev], dps[lev])
            gcat[lev] = tconv(by[f"dec{lev}a"], gdp, cats[lev])
            c = spec.channels(lev)
            gu_full = gcat[lev][..., c:]
            n_, hh, ww, _ = gu_full.shape
            gu = gu_full.reshape(n_, hh // 2, 2, ww // 2, 2, c).sum(dim=(2, 4))
            gd[lev + 1] = tconv(by[f"up{lev}"], gu, ds[lev + 1])
        for lev in range(L - 1, -1, -1):
            gs = gcat[lev][..., :spec.channels(lev)] if lev < L - 1 else gd[lev]
            ga = tconv(by[f"enc{lev}b"], gs, as_[lev])
            gx = tconv(by[f"enc{lev}a"], ga, xs[lev] if lev > 0 else None)
            if lev > 0:
                # route to the pooling winner (first maximum in the window)
                s = skips[lev - 1]
                n_, hh, ww, c = s.shape
                win = s.reshape(n_, hh // 2, 2, ww // 2, 2, c).permute(0, 1, 3, 5, 2, 4)
                win = win.reshape(n_, hh // 2, ww // 2, c, 4)
                arg = win.argmax(dim=-1)
                routed = F.one_hot(arg, 4).to(gx.dtype) * gx[..., None]
                routed = routed.reshape(n_, hh // 2, ww // 2, c, 2, 2).permute(0, 1, 4, 2, 5, 3)
                gcat[lev - 1][..., :c] += routed.reshape(n_, hh, ww, c)
            else:
                got = gx[..., 0]
    np.testing.assert_allclose(got.numpy(), want.numpy(), rtol=1e-9, atol=1e-12)


def test_bench_cpu_sample_of_the_unet():
    """bench.py's CPU baseline of the unet workload: the oracle network's
    training step on the host cores, a bounded sample."""
    import bench

    tflops, steps, seconds, threads = bench.cpu_sample_unet(target_s=0.5, batch=1)
    assert steps >= 1 and seconds > 0 and threads >= 1 and 0 < tflops < 50
