"""Test infrastructure: a torch float32 CPU restatement of the surrogate U-Net.

The design surrogate has no counterpart in the reference, so its checker is
the same network written with torch.nn.functional on the CPU (conv2d with
zero padding, max_pool2d, nearest upsampling, concatenation) and
differentiated by torch autograd. It reads the flat parameter vector through
a layer table [(name, cin, cout, taps, relu, w_off, b_off)], weights laid out
[tap * cin + ci][co] with tap = (dy + 1) * 3 + (dx + 1).

With ``bf16=True`` the weights and every stored activation are rounded to
bfloat16 at the points where the CUDA kernels store them (straight-through
in the backward pass), so the remaining differences come from FP32
accumulation order and from the BF16 rounding of the CUDA path's gradients.

Only tests use it.
"""

from __future__ import annotations

import torch
import torch.nn.functional as F


def _round(x, bf16):
    if not bf16:
        return x
    return x + (x.to(torch.bfloat16).to(x.dtype) - x).detach()


def _weight(theta, ly, bf16):
    name, cin, cout, taps, relu, w_off, b_off = ly
    w = theta[w_off:w_off + taps * cin * cout].reshape(taps, cin, cout)
    w = _round(w, bf16)
    k = 3 if taps == 9 else 1
    # [ky*3+kx, ci, co] -> [co, ci, ky, kx] (conv2d is a cross-correlation:
    # out[y, x] = sum w[ky, kx] in[y + ky - 1, x + kx - 1]).
    w = w.reshape(k, k, cin, cout).permute(3, 2, 0, 1)
    b = theta[b_off:b_off + cout]
    return w, b


def _conv(theta, ly, x, bf16, slope, out_round=True):
    w, b = _weight(theta, ly, bf16)
    y = F.conv2d(x, w, b, padding=w.shape[-1] // 2)
    if ly[4]:
        y = F.leaky_relu(y, slope)
    return _round(y, bf16) if out_round else y


def unet_forward(theta, layers, levels, x, *, bf16=True, slope=0.1):
    """Head output (N, C, H, W) float32 for densities x (N, H, W); the
    activations are leaky ReLUs of negative slope ``slope``."""
    by = {ly[0]: ly for ly in layers}
    h = _round(x[:, None], bf16)
    skips = []
    for lev in range(levels):
        h = _conv(theta, by[f"enc{lev}a"], h, bf16, slope)
        h = _conv(theta, by[f"enc{lev}b"], h, bf16, slope)
        if lev < levels - 1:
            skips.append(h)
            h = F.max_pool2d(h, 2)
    for lev in range(levels - 2, -1, -1):
        u = _conv(theta, by[f"up{lev}"], h, bf16, slope)
        u = F.interpolate(u, scale_factor=2, mode="nearest")
        h = torch.cat([skips[lev], u], dim=1)
        h = _conv(theta, by[f"dec{lev}a"], h, bf16, slope)
        h = _conv(theta, by[f"dec{lev}b"], h, bf16, slope)
    return _conv(theta, by["head"], h, bf16, slope, out_round=False)


def unet_loss(theta, layers, levels, x, target_field, target_power, field_weight=1.0,
              power_weight=1.0, bf16=True, slope=0.1):
    """The training loss of the CUDA head kernel:
    wf * mean (out[:2] - tf)^2 + wp * mean_n (mean_hw out[2] - tp)^2."""
    out = unet_forward(theta, layers, levels, x, bf16=bf16, slope=slope)
    field = out[:, :2].permute(0, 2, 3, 1)
    power = out[:, 2].mean(dim=(1, 2))
    return (field_weight * ((field - target_field) ** 2).mean()
            + power_weight * ((power - target_power) ** 2).mean())
