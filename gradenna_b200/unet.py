"""BF16 U-Net over 2D design densities, run by this library's own kernels.

The design surrogate maps a density image (N, H, W) to three output
channels per pixel: the real and imaginary part of the (normalised) Ez
phasor on the design region, and a power-density channel whose spatial mean
is the predicted radiated power. No reference counterpart: the reference
has no learned component.

Architecture (``UNetSpec``, defaults 104 x 104, 4 levels, 32 base
channels, about 2M parameters, leaky-ReLU slope 0.1 written "ReLU" below):
level l has c_l = base * 2^l channels at
H / 2^l; the encoder applies two 3x3 convolutions + ReLU per level and 2x2
max pooling between levels; the decoder computes a 3x3 convolution + ReLU of
the coarser level's output at the coarse resolution, upsamples it (nearest,
x2) into the upper half of the level's concatenation buffer (whose lower
half already holds the encoder output), and applies two 3x3 convolutions +
ReLU; a 1x1 head gives the output channels (no activation).

Everything runs in ``gdn_sur_*`` kernels (gradenna_b200/csrc/surrogate.cu):
BF16 tensor-core implicit-GEMM convolutions with FP32 accumulation, their
input gradients (flipped-weight convolutions whose epilogue applies the ReLU
mask) and weight gradients (split-K over pixels), pooling, upsampling, the
head loss and Adam on FP32 master weights with a BF16 copy. torch provides
device memory and the stream only.

Parameters live in one flat FP32 vector; layer ``i`` owns
``theta[w_off : w_off + taps * cin * cout]`` laid out [tap * cin + ci][co]
(tap = (dy + 1) * 3 + (dx + 1)) and ``theta[b_off : b_off + cout]``.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import NamedTuple

import numpy as np
import torch

from gradenna_b200 import _native

__all__ = ["UNetSpec", "Layer", "unet_layers", "UNet", "allreduce_mean", "tc_timeouts"]

_v, _i, _f = ctypes.c_void_p, ctypes.c_int32, ctypes.c_float
_native.register("gdn_sur_conv_fwd", ctypes.c_int,
                 [_v, _i, _i, _i, _i, _i, _i, _i, _v, _v, _i, _i, _f, _v, _i, _i, _v, _v, _i, _i, _v])
_native.register("gdn_sur_conv_wgrad", ctypes.c_int,
                 [_v, _i, _i, _i, _i, _i, _i, _i, _v, _i, _i, _i, _v, _v, _v])
_native.register("gdn_sur_flip_weights", ctypes.c_int, [_v, _i, _i, _i, _v, _v])
_native.register("gdn_sur_maxpool2", ctypes.c_int, [_v, _i, _i, _i, _i, _i, _i, _v, _v, _v])
_native.register("gdn_sur_maxpool2_grad_acc", ctypes.c_int,
                 [_v, _v, _i, _i, _i, _i, _v, _i, _i, _v])
_native.register("gdn_sur_upsample2", ctypes.c_int, [_v, _i, _i, _i, _i, _v, _i, _i, _v])
_native.register("gdn_sur_upsample2_grad", ctypes.c_int, [_v, _i, _i, _i, _i, _i, _i, _v, _v])
_native.register("gdn_sur_head_grad", ctypes.c_int,
                 [_v, _i, _i, _i, _v, _v, _v, _f, _f, _v, _v, _v, _v])
_native.register("gdn_sur_adam", ctypes.c_int,
                 [_v, _v, _v, _v, _v, ctypes.c_int64, _v, _f, _f, _f, _v])
_native.register("gdn_sur_to_bf16", ctypes.c_int, [_v, _v, ctypes.c_int64, _v])
_native.register("gdn_sur_conv_fwd_tc", ctypes.c_int,
                 [_v, _i, _i, _i, _i, _i, _i, _i, _v, _v, _i, _i, _f, _v, _i, _i, _v, _v, _i, _i, _v])
_native.register("gdn_sur_weights_kmajor", ctypes.c_int, [_v, _i, _i, _i, _i, _v, _v])
_native.register("gdn_sur_status", ctypes.c_int, [ctypes.POINTER(ctypes.c_int32), _i])
_native.register("gdn_sur_inject_timeout", ctypes.c_int, [_i])


def tc_timeouts(reset: bool = True) -> int:
    """Number of tensor-core convolutions that gave up on a bounded wait
    since the last reset (gdn_sur_status); 0 in normal operation."""
    v = ctypes.c_int32()
    _native.check(_native.load().gdn_sur_status(ctypes.byref(v), int(reset)))
    return int(v.value)


def allreduce_mean(group=None):
    """A train_step gradient hook for data-parallel training: the sum of the
    ranks' flat FP32 gradients over torch.distributed (NCCL over NVLink on
    GPUs), divided by the world size, in place. Every rank then applies the
    same Adam step, so the replicas stay identical."""
    import torch.distributed as dist

    world = dist.get_world_size(group)

    def hook(grad):
        dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
        grad.div_(world)

    return hook


@dataclass(frozen=True)
class UNetSpec:
    height: int = 104
    width: int = 104
    base: int = 32
    levels: int = 4
    out_channels: int = 3
    neg_slope: float = 0.1  # leaky-ReLU slope (0 = ReLU)

    def channels(self, level: int) -> int:
        return self.base * 2**level

    def size(self, level: int) -> tuple[int, int]:
        return self.height >> level, self.width >> level


class Layer(NamedTuple):
    name: str
    cin: int
    cout: int
    taps: int
    relu: bool
    w_off: int
    b_off: int


def unet_layers(spec: UNetSpec) -> tuple[list[Layer], int]:
    """Layer table in forward order and the flat parameter count (offsets
    aligned to 8 elements so every BF16 weight block starts on 16 bytes)."""
    div = 2 ** (spec.levels - 1)
    if spec.height % div or spec.width % div:
        raise ValueError(f"height and width must be multiples of {div} for {spec.levels} levels")
    if spec.levels < 2 or spec.out_channels < 3:
        raise ValueError("the U-Net needs at least 2 levels and 3 output channels")
    shapes = []
    L = spec.levels
    for lev in range(L):
        c = spec.channels(lev)
        shapes.append((f"enc{lev}a", 1 if lev == 0 else spec.channels(lev - 1), c, 9, True))
        shapes.append((f"enc{lev}b", c, c, 9, True))
    for lev in range(L - 2, -1, -1):
        c = spec.channels(lev)
        shapes.append((f"up{lev}", spec.channels(lev + 1), c, 9, True))
        shapes.append((f"dec{lev}a", 2 * c, c, 9, True))
        shapes.append((f"dec{lev}b", c, c, 9, True))
    shapes.append(("head", spec.channels(0), spec.out_channels, 1, False))
    layers, off = [], 0
    for name, cin, cout, taps, relu in shapes:
        w_off = off
        off = (off + taps * cin * cout + 7) // 8 * 8
        b_off = off
        off = (off + cout + 7) // 8 * 8
        layers.append(Layer(name, cin, cout, taps, relu, w_off, b_off))
    return layers, off


class _Ws:
    """Activation and gradient buffers of one batch size (NHWC bfloat16)."""

    def __init__(self, spec: UNetSpec, n: int, dev):
        bf = dict(dtype=torch.bfloat16, device=dev)
        L = spec.levels
        self.n = n
        self.x = [None] * L       # level inputs (density, then pool outputs)
        self.a = [None] * L       # first encoder conv outputs
        self.cat = [None] * L     # [skip | upsampled] buffers (levels < L-1)
        self.arg = [None] * L     # pool winners of level l (at level l+1's size)
        self.u = [None] * L       # up-conv outputs (coarse size)
        self.dp = [None] * L
        self.d = [None] * L
        self.g_x, self.g_a, self.g_cat, self.g_u, self.g_dp, self.g_d = ([None] * L for _ in range(6))
        for lev in range(L):
            h, w = spec.size(lev)
            c = spec.channels(lev)
            cin = 1 if lev == 0 else spec.channels(lev - 1)
            self.x[lev] = torch.zeros((n, h, w, cin), **bf)
            self.g_x[lev] = torch.zeros((n, h, w, cin), **bf)
            self.a[lev] = torch.zeros((n, h, w, c), **bf)
            self.g_a[lev] = torch.zeros((n, h, w, c), **bf)
            if lev < L - 1:
                self.cat[lev] = torch.zeros((n, h, w, 2 * c), **bf)
                self.g_cat[lev] = torch.zeros((n, h, w, 2 * c), **bf)
                hc, wc = spec.size(lev + 1)
                self.arg[lev] = torch.zeros((n, hc, wc, c), dtype=torch.uint8, device=dev)
                self.u[lev] = torch.zeros((n, hc, wc, c), **bf)
                self.g_u[lev] = torch.zeros((n, hc, wc, c), **bf)
                self.dp[lev] = torch.zeros((n, h, w, c), **bf)
                self.g_dp[lev] = torch.zeros((n, h, w, c), **bf)
            # d[L-1] is the bottom encoder output; d[l] (l < L-1) the decoder output.
            self.d[lev] = torch.zeros((n, h, w, c), **bf)
            self.g_d[lev] = torch.zeros((n, h, w, c), **bf)
        h, w = spec.size(0)
        self.out32 = torch.zeros((n, h, w, spec.out_channels), dtype=torch.float32, device=dev)
        self.g_out = torch.zeros((n, h, w, spec.out_channels), **bf)
        self.g_in32 = torch.zeros((n, h, w, 1), dtype=torch.float32, device=dev)
        self.mean = torch.zeros(n, dtype=torch.float32, device=dev)
        self.loss = torch.zeros(1, dtype=torch.float32, device=dev)
        self.x32 = torch.zeros((n, h, w), dtype=torch.float32, device=dev)


class UNet:
    """The surrogate network: parameters, Adam state and per-batch workspaces.

    ``forward(x)`` returns (out, power) for densities x (N, H, W) float32 on
    the device: out = (N, H, W, out_channels) float32 head output and power =
    (N,) the spatial mean of channel 2. ``train_step`` runs forward, the
    head loss, backward and one Adam step; ``power_grad`` returns the
    predicted power and its gradient with respect to the input densities.
    """

    def __init__(self, spec: UNetSpec = UNetSpec(), *, seed: int = 0, device=None,
                 learning_rate: float = 1e-3, betas=(0.9, 0.999), eps: float = 1e-8,
                 tensor_cores: bool | None = None):
        self.dev = _native.require_cuda(device)
        self.lib = _native.load()
        self.spec = spec
        self.layers, self.n_params = unet_layers(spec)
        self.by_name = {ly.name: ly for ly in self.layers}
        f32 = dict(dtype=torch.float32, device=self.dev)
        self.theta = torch.as_tensor(self.init_params(spec, seed), **f32)
        self.theta16 = torch.zeros(self.n_params, dtype=torch.bfloat16, device=self.dev)
        self.flip16 = torch.zeros(self.n_params, dtype=torch.bfloat16, device=self.dev)
        # K-major copies for the tcgen05 convolutions: forward and flipped.
        self.wk16 = torch.zeros(self.n_params, dtype=torch.bfloat16, device=self.dev)
        self.fk16 = torch.zeros(self.n_params, dtype=torch.bfloat16, device=self.dev)
        if tensor_cores is None:
            import os

            # The tcgen05 convolutions are the default (measured on B200: 5.01
            # against 5.18 ms per training step of the 104^2, batch-32 U-Net);
            # GDN_SUR_TC=0 selects the mma.sync ones.
            tensor_cores = os.environ.get("GDN_SUR_TC", "1") != "0"
        self.tensor_cores = bool(tensor_cores)
        self._kmajor = False
        self.grad = torch.zeros(self.n_params, **f32)
        self.m = torch.zeros(self.n_params, **f32)
        self.v = torch.zeros(self.n_params, **f32)
        self.hyper = torch.tensor([0.0, learning_rate, 1.0, 1.0], **f32)
        self.betas, self.eps = (float(betas[0]), float(betas[1])), float(eps)
        self._ws: dict[int, _Ws] = {}
        self._flipped = False
        self.sync_params()

    # ----------------------------------------------------------- parameters
    @staticmethod
    def init_params(spec: UNetSpec, seed: int) -> np.ndarray:
        """He-normal weights (std sqrt(2 / fan_in)), zero biases; the head
        starts at std sqrt(1 / fan_in)."""
        layers, n = unet_layers(spec)
        rng = np.random.default_rng(seed)
        theta = np.zeros(n, np.float32)
        for ly in layers:
            fan_in = ly.taps * ly.cin
            std = np.sqrt((2.0 if ly.relu else 1.0) / fan_in)
            theta[ly.w_off:ly.w_off + fan_in * ly.cout] = rng.normal(0.0, std, fan_in * ly.cout)
        return theta

    def _s(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    def sync_params(self) -> None:
        """Refresh the BF16 copy after the FP32 parameters were set."""
        with torch.cuda.device(self.dev):
            _native.check(self.lib.gdn_sur_to_bf16(self.theta.data_ptr(), self.theta16.data_ptr(),
                                                   self.n_params, self._s()))
        self._flipped = False
        self._kmajor = False

    def set_learning_rate(self, lr: float) -> None:
        self.hyper[1].fill_(float(lr))

    def state_dict(self) -> dict:
        return {"spec": self.spec.__dict__.copy(), "theta": self.theta.detach().cpu().clone()}

    def load_state_dict(self, state: dict) -> None:
        if UNetSpec(**state["spec"]) != self.spec:
            raise ValueError("state was saved for a different UNetSpec")
        self.theta.copy_(state["theta"].to(self.dev))
        self.sync_params()

    # ------------------------------------------------------------ kernels
    def _w16(self, ly: Layer, flipped: bool = False) -> int:
        base = self.flip16 if flipped else self.theta16
        return base.data_ptr() + 2 * ly.w_off

    def _bias(self, ly: Layer) -> int:
        return self.theta.data_ptr() + 4 * ly.b_off

    def _conv(self, ly: Layer, src, n, h, w, dst, *, out32=None, mask=None, transpose=False,
              stream=None):
        """Forward convolution of layer ``ly`` (or, with ``transpose``, its
        input gradient). ``src``/``dst``/``mask`` are (tensor, c0) with the
        tensor's last dimension as the row stride."""
        cin, cout = (ly.cout, ly.cin) if transpose else (ly.cin, ly.cout)
        st, sc0 = src
        dt_, dc0 = dst if dst is not None else (None, 0)
        mt, mc0 = mask if mask is not None else (None, 0)
        use_tc = (self.tensor_cores and cin % 8 == 0 and st.shape[-1] % 8 == 0 and sc0 % 8 == 0
                  and cout >= 8)
        fn = self.lib.gdn_sur_conv_fwd_tc if use_tc else self.lib.gdn_sur_conv_fwd
        if use_tc:
            wbase = (self.fk16 if transpose else self.wk16).data_ptr() + 2 * ly.w_off
        else:
            wbase = self._w16(ly, transpose)
        _native.check(fn(
            st.data_ptr(), st.shape[-1], sc0, n, h, w, cin, ly.taps, wbase,
            None if transpose else self._bias(ly), cout, int(ly.relu and not transpose),
            float(self.spec.neg_slope), _native.ptr(dt_), 0 if dt_ is None else dt_.shape[-1], dc0, _native.ptr(out32),
            _native.ptr(mt), 0 if mt is None else mt.shape[-1], mc0, stream))

    def _wgrad(self, ly: Layer, src, g, n, h, w, stream):
        st, sc0 = src
        gt, gc0 = g
        _native.check(self.lib.gdn_sur_conv_wgrad(
            st.data_ptr(), st.shape[-1], sc0, n, h, w, ly.cin, ly.taps, gt.data_ptr(),
            gt.shape[-1], gc0, ly.cout, self.grad.data_ptr() + 4 * ly.w_off,
            self.grad.data_ptr() + 4 * ly.b_off, stream))

    def _flip_all(self, stream) -> None:
        for ly in self.layers:
            _native.check(self.lib.gdn_sur_flip_weights(self._w16(ly), ly.cin, ly.cout, ly.taps,
                                                        self._w16(ly, True), stream))
            if self.tensor_cores:
                _native.check(self.lib.gdn_sur_weights_kmajor(
                    self._w16(ly), ly.cin, ly.cout, ly.taps, 1,
                    self.fk16.data_ptr() + 2 * ly.w_off, stream))
        self._flipped = True

    def _kmajor_all(self, stream) -> None:
        if self.tensor_cores:
            for ly in self.layers:
                _native.check(self.lib.gdn_sur_weights_kmajor(
                    self._w16(ly), ly.cin, ly.cout, ly.taps, 0,
                    self.wk16.data_ptr() + 2 * ly.w_off, stream))
        self._kmajor = True

    def workspace(self, n: int) -> _Ws:
        ws = self._ws.get(n)
        if ws is None:
            ws = self._ws[n] = _Ws(self.spec, n, self.dev)
        return ws

    # ------------------------------------------------------------ passes
    def _forward(self, ws: _Ws, stream) -> None:
        spec, lib, L, n = self.spec, self.lib, self.spec.levels, ws.n
        B = self.by_name
        if not self._kmajor:
            self._kmajor_all(stream)
        h0, w0 = spec.size(0)
        _native.check(lib.gdn_sur_to_bf16(ws.x32.data_ptr(), ws.x[0].data_ptr(), n * h0 * w0,
                                          stream))
        for lev in range(L):
            h, w = spec.size(lev)
            c = spec.channels(lev)
            self._conv(B[f"enc{lev}a"], (ws.x[lev], 0), n, h, w, (ws.a[lev], 0), stream=stream)
            out = (ws.cat[lev], 0) if lev < L - 1 else (ws.d[lev], 0)
            self._conv(B[f"enc{lev}b"], (ws.a[lev], 0), n, h, w, out, stream=stream)
            if lev < L - 1:
                _native.check(lib.gdn_sur_maxpool2(ws.cat[lev].data_ptr(), 2 * c, 0, n, h, w, c,
                                                   ws.x[lev + 1].data_ptr(),
                                                   ws.arg[lev].data_ptr(), stream))
        for lev in range(L - 2, -1, -1):
            h, w = spec.size(lev)
            hc, wc = spec.size(lev + 1)
            c = spec.channels(lev)
            self._conv(B[f"up{lev}"], (ws.d[lev + 1], 0), n, hc, wc, (ws.u[lev], 0), stream=stream)
            _native.check(lib.gdn_sur_upsample2(ws.u[lev].data_ptr(), n, hc, wc, c,
                                                ws.cat[lev].data_ptr(), 2 * c, c, stream))
            self._conv(B[f"dec{lev}a"], (ws.cat[lev], 0), n, h, w, (ws.dp[lev], 0), stream=stream)
            self._conv(B[f"dec{lev}b"], (ws.dp[lev], 0), n, h, w, (ws.d[lev], 0), stream=stream)
        self._conv(B["head"], (ws.d[0], 0), n, h0, w0, None, out32=ws.out32, stream=stream)

    def _backward(self, ws: _Ws, stream, *, weights: bool, input_grad: bool) -> None:
        """Backward from ws.g_out: weight gradients into self.grad (added)
        and/or the input gradient into ws.g_in32."""
        spec, lib, L, n = self.spec, self.lib, self.spec.levels, ws.n
        B = self.by_name
        if not self._flipped:
            self._flip_all(stream)
        h0, w0 = spec.size(0)
        head = B["head"]
        if weights:
            self._wgrad(head, (ws.d[0], 0), (ws.g_out, 0), n, h0, w0, stream)
        self._conv(head, (ws.g_out, 0), n, h0, w0, (ws.g_d[0], 0), mask=(ws.d[0], 0),
                   transpose=True, stream=stream)
        for lev in range(L - 1):
            h, w = spec.size(lev)
            hc, wc = spec.size(lev + 1)
            c = spec.channels(lev)
            db, da, up = B[f"dec{lev}b"], B[f"dec{lev}a"], B[f"up{lev}"]
            if weights:
                self._wgrad(db, (ws.dp[lev], 0), (ws.g_d[lev], 0), n, h, w, stream)
            self._conv(db, (ws.g_d[lev], 0), n, h, w, (ws.g_dp[lev], 0), mask=(ws.dp[lev], 0),
                       transpose=True, stream=stream)
            if weights:
                self._wgrad(da, (ws.cat[lev], 0), (ws.g_dp[lev], 0), n, h, w, stream)
            self._conv(da, (ws.g_dp[lev], 0), n, h, w, (ws.g_cat[lev], 0),
                       mask=(ws.cat[lev], 0), transpose=True, stream=stream)
            _native.check(lib.gdn_sur_upsample2_grad(ws.g_cat[lev].data_ptr(), 2 * c, c, n, hc,
                                                     wc, c, ws.g_u[lev].data_ptr(), stream))
            if weights:
                self._wgrad(up, (ws.d[lev + 1], 0), (ws.g_u[lev], 0), n, hc, wc, stream)
            self._conv(up, (ws.g_u[lev], 0), n, hc, wc, (ws.g_d[lev + 1], 0),
                       mask=(ws.d[lev + 1], 0), transpose=True, stream=stream)
        for lev in range(L - 1, -1, -1):
            h, w = spec.size(lev)
            c = spec.channels(lev)
            ea, eb = B[f"enc{lev}a"], B[f"enc{lev}b"]
            g_s = (ws.g_cat[lev], 0) if lev < L - 1 else (ws.g_d[lev], 0)
            if weights:
                self._wgrad(eb, (ws.a[lev], 0), g_s, n, h, w, stream)
            self._conv(eb, g_s, n, h, w, (ws.g_a[lev], 0), mask=(ws.a[lev], 0), transpose=True,
                       stream=stream)
            if weights:
                self._wgrad(ea, (ws.x[lev], 0), (ws.g_a[lev], 0), n, h, w, stream)
            if lev > 0:
                self._conv(ea, (ws.g_a[lev], 0), n, h, w, (ws.g_x[lev], 0),
                           mask=(ws.x[lev], 0), transpose=True, stream=stream)
                hu, wu = spec.size(lev - 1)
                cu = spec.channels(lev - 1)
                _native.check(lib.gdn_sur_maxpool2_grad_acc(
                    ws.g_x[lev].data_ptr(), ws.arg[lev - 1].data_ptr(), n, hu, wu, cu,
                    ws.g_cat[lev - 1].data_ptr(), 2 * cu, 0, stream))
            elif input_grad:
                self._conv(ea, (ws.g_a[0], 0), n, h, w, None, out32=ws.g_in32, transpose=True,
                           stream=stream)

    def _load_input(self, x) -> _Ws:
        x = torch.as_tensor(x)
        if x.ndim != 3 or tuple(x.shape[1:]) != self.spec.size(0):
            raise ValueError(f"densities must be (N, {self.spec.height}, {self.spec.width})")
        ws = self.workspace(int(x.shape[0]))
        ws.x32.copy_(x, non_blocking=True)
        return ws

    def forward(self, x):
        """Head output (N, H, W, C) float32 and predicted power (N,)."""
        with torch.cuda.device(self.dev):
            ws = self._load_input(x)
            s = self._s()
            self._forward(ws, s)
            out = ws.out32.clone()
        return out, out[..., 2].mean(dim=(1, 2))

    def train_step(self, x, target_field, target_power, *, field_weight: float = 1.0,
                   power_weight: float = 1.0, grad_hook=None):
        """One Adam step on the loss
        field_weight * mean (out[..., :2] - target_field)^2
        + power_weight * mean_n (mean_hw out[..., 2] - target_power)^2.
        Returns the loss before the step as a device scalar (no host sync).
        ``grad_hook(grad)`` runs between the backward pass and Adam on the
        flat FP32 gradient (in place): data-parallel training passes the
        all-reduce mean over the ranks there (``allreduce_mean``)."""
        with torch.cuda.device(self.dev):
            ws = self._load_input(x)
            tf = torch.as_tensor(target_field, dtype=torch.float32, device=self.dev).contiguous()
            tp = torch.as_tensor(target_power, dtype=torch.float32, device=self.dev).contiguous()
            if tuple(tf.shape) != tuple(ws.out32.shape[:3]) + (2,) or tp.shape != (ws.n,):
                raise ValueError("target shapes must be (N, H, W, 2) and (N,)")
            s = self._s()
            self._forward(ws, s)
            ws.loss.zero_()
            self.grad.zero_()
            h, w = self.spec.size(0)
            _native.check(self.lib.gdn_sur_head_grad(
                ws.out32.data_ptr(), ws.n, h * w, self.spec.out_channels, tf.data_ptr(),
                tp.data_ptr(), None, float(field_weight), float(power_weight),
                ws.mean.data_ptr(), ws.g_out.data_ptr(), ws.loss.data_ptr(), s))
            self._backward(ws, s, weights=True, input_grad=False)
            if grad_hook is not None:
                grad_hook(self.grad)
            _native.check(self.lib.gdn_sur_adam(
                self.theta.data_ptr(), self.grad.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
                self.theta16.data_ptr(), self.n_params, self.hyper.data_ptr(), self.betas[0],
                self.betas[1], self.eps, s))
            self._flipped = False
            self._kmajor = False
            return ws.loss.clone()[0]

    def gradients(self, x, target_field, target_power, *, field_weight: float = 1.0,
                  power_weight: float = 1.0):
        """(loss, dL/dtheta, dL/dx) of the train_step loss without updating
        the parameters (for checks against an autograd reference)."""
        with torch.cuda.device(self.dev):
            ws = self._load_input(x)
            tf = torch.as_tensor(target_field, dtype=torch.float32, device=self.dev).contiguous()
            tp = torch.as_tensor(target_power, dtype=torch.float32, device=self.dev).contiguous()
            s = self._s()
            self._forward(ws, s)
            ws.loss.zero_()
            self.grad.zero_()
            h, w = self.spec.size(0)
            _native.check(self.lib.gdn_sur_head_grad(
                ws.out32.data_ptr(), ws.n, h * w, self.spec.out_channels, tf.data_ptr(),
                tp.data_ptr(), None, float(field_weight), float(power_weight),
                ws.mean.data_ptr(), ws.g_out.data_ptr(), ws.loss.data_ptr(), s))
            self._backward(ws, s, weights=True, input_grad=True)
            return ws.loss.clone()[0], self.grad.clone(), ws.g_in32[..., 0].clone()

    def power_grad(self, x, weight=None):
        """Predicted power (N,) and d(sum_n weight_n * power_n)/dx (N, H, W)."""
        with torch.cuda.device(self.dev):
            ws = self._load_input(x)
            s = self._s()
            self._forward(ws, s)
            pw = None
            if weight is not None:
                pw = torch.as_tensor(weight, dtype=torch.float32, device=self.dev).contiguous()
            h, w = self.spec.size(0)
            _native.check(self.lib.gdn_sur_head_grad(
                ws.out32.data_ptr(), ws.n, h * w, self.spec.out_channels, None, None,
                _native.ptr(pw), 0.0, 0.0, ws.mean.data_ptr(), ws.g_out.data_ptr(), None, s))
            self._backward(ws, s, weights=False, input_grad=True)
            return ws.mean.clone(), ws.g_in32[..., 0].clone()
