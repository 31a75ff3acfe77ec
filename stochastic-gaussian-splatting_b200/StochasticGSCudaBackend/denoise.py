"""Learned resolve: a small convolutional denoiser that maps a few samples to the converged image.

The reference resolves only by progressive averaging (resolve.cu, Static mode), which stays the
fallback and the yardstick its output is measured against. This module adds, on the same render path:

* `render_features(...)`: renders n samples (Reset mode, one frame index each) and builds the
  8-channel FP16 input per pixel: mean premultiplied rgb, mean alpha, mean depth x depth_scale,
  the standard error of the mean luminance, the fraction of consecutive samples whose winner
  changed, and a zero channel (csrc/denoise.cu, features_*).
* `Denoiser`: 6 layers of 3x3 convolutions (8 -> 32 -> 32 -> 32 -> 32 -> 32 -> 3, ReLU between,
  the last layer adds the mean colour back), FP32 master weights, BF16 tensor-core kernels with
  FP32 accumulation for inference (`Denoiser.__call__`, one C-ABI call `sgs_denoise`) and for
  training (`denoise_train`, a torch.autograd.Function whose backward runs the data-gradient and
  weight-gradient kernels).

Weights W[co][ci][dy][dx] follow torch's conv2d (cross-correlation, zero padding 1).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _abi, _C
from .render import Settings

_lib = _abi.load()

# (input channels, output channels) of the model and as the kernels stage them
LAYERS = ((7, 32), (32, 32), (32, 32), (32, 32), (32, 32), (32, 3))
ABI_IN = (8, 32, 32, 32, 32, 32)
STAGED_IN = (16, 32, 32, 32, 32, 32)
STAGED_OUT = (32, 32, 32, 32, 32, 16)
FEATURES = 8
WIDTH = 32


def _check(status: int, what: str) -> None:
    if status != _abi.SGS_OK:
        raise RuntimeError(f"{what} failed ({status}): {_abi.last_error(_lib)}")


def _stream(device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def pack_forward(w: torch.Tensor, staged_in: int, staged_out: int) -> torch.Tensor:
    """W[co][ci][3][3] -> BF16 [tap][ci / 8][co][ci % 8], zero-padded to the staged channel counts."""
    co, ci = w.shape[:2]
    wp = torch.zeros((staged_out, staged_in, 3, 3), dtype=torch.float32, device=w.device)
    wp[:co, :ci] = w
    t = wp.permute(2, 3, 1, 0).reshape(9, staged_in // 8, 8, staged_out).permute(0, 1, 3, 2)
    return t.contiguous().to(torch.bfloat16).reshape(-1)


def pack_dgrad(w: torch.Tensor, staged_in: int, staged_out: int) -> torch.Tensor:
    """Data-gradient weights of a layer: W'[tap][n = ci][k = co] = W[co][ci][2 - dy][2 - dx], as
    BF16 [tap][co / 8][ci][co % 8]."""
    co, ci = w.shape[:2]
    wp = torch.zeros((staged_out, staged_in, 3, 3), dtype=torch.float32, device=w.device)
    wp[:co, :ci] = w
    t = wp.flip(2, 3).permute(2, 3, 0, 1).reshape(9, staged_out // 8, 8, staged_in).permute(0, 1, 3, 2)
    return t.contiguous().to(torch.bfloat16).reshape(-1)


def unpack_wgrad(g: torch.Tensor, layer: int) -> torch.Tensor:
    """[9][staged_out][staged_in] FP32 gradient -> [co][ci][3][3]."""
    ci, co = LAYERS[layer]
    g = g.view(3, 3, STAGED_OUT[layer], STAGED_IN[layer]).permute(2, 3, 0, 1)
    return g[:co, :ci].contiguous()


def init_params(seed: int = 0, device="cuda") -> list[torch.Tensor]:
    """He-initialised weights and zero biases, [W1, b1, ..., W6, b6]; the last layer starts at zero
    so that the untrained denoiser returns the plain average."""
    g = torch.Generator().manual_seed(seed)
    out = []
    for i, (ci, co) in enumerate(LAYERS):
        std = (2.0 / (9 * ci)) ** 0.5
        w = torch.randn((co, ci, 3, 3), generator=g) * std
        if i == len(LAYERS) - 1:
            w.zero_()
        out += [w.to(device), torch.zeros(co, device=device)]
    return out


def _conv(inp, out, weights, bias, epilogue, in_ch, out_ch, shape, mask=None, residual=None):
    b, h, w = shape
    args = _abi.Conv3x3Args(inp.data_ptr(), out.data_ptr(), weights.data_ptr(),
                            None if bias is None else bias.data_ptr(), None if mask is None else mask.data_ptr(),
                            None if residual is None else residual.data_ptr(), b, h, w, in_ch, out_ch, epilogue)
    _check(_lib.sgs_conv3x3(ctypes.byref(args), _stream(inp.device)), "sgs_conv3x3")


def conv3x3(inp: torch.Tensor, weights: torch.Tensor, bias: torch.Tensor | None, in_channels: int, out_channels: int,
            epilogue: int, mask: torch.Tensor | None = None, residual: torch.Tensor | None = None) -> torch.Tensor:
    """One layer through the C ABI (sgs_conv3x3). inp is [B, H, W, C] FP16 features (in_channels 8)
    or BF16; returns BF16 [B, H, W, out_channels], or FP32 [B, H, W, 3] for the final epilogue."""
    b, h, w = inp.shape[:3]
    if epilogue == _abi.SGS_CONV_FINAL:
        out = torch.empty((b, h, w, 3), dtype=torch.float32, device=inp.device)
    else:
        out = torch.empty((b, h, w, out_channels), dtype=torch.bfloat16, device=inp.device)
    _conv(inp, out, weights, bias, epilogue, in_channels, out_channels, (b, h, w), mask, residual)
    return out


def conv3x3_wgrad(inp: torch.Tensor, in_channels: int, grad_out: torch.Tensor, out_channels: int):
    """Weight and bias gradients of one layer (sgs_conv3x3_wgrad): ([9][out][16 or 32], [out]) FP32."""
    b, h, w = inp.shape[:3]
    staged_in = 16 if in_channels == 8 else in_channels
    gw = torch.zeros((9, out_channels, staged_in), dtype=torch.float32, device=inp.device)
    gb = torch.zeros(out_channels, dtype=torch.float32, device=inp.device)
    _check(_lib.sgs_conv3x3_wgrad(ctypes.c_void_p(inp.data_ptr()), in_channels, ctypes.c_void_p(grad_out.data_ptr()),
                                  out_channels, b, h, w, ctypes.c_void_p(gw.data_ptr()), ctypes.c_void_p(gb.data_ptr()),
                                  _stream(inp.device)), "sgs_conv3x3_wgrad")
    return gw, gb


def status(device=None) -> None:
    """Synchronises the current stream and raises if a denoiser kernel gave up a bounded wait."""
    _check(_lib.sgs_denoise_status(_stream(device)), "denoiser")


def _padded_bias(b: torch.Tensor, n: int) -> torch.Tensor:
    out = torch.zeros(n, dtype=torch.float32, device=b.device)
    out[:b.shape[0]] = b
    return out


class _DenoiseTrain(torch.autograd.Function):
    @staticmethod
    def forward(ctx, features, *params):
        ws = [pack_forward(params[2 * l].detach(), STAGED_IN[l], STAGED_OUT[l]) for l in range(6)]
        bs = [_padded_bias(params[2 * l + 1].detach(), STAGED_OUT[l]) for l in range(6)]
        acts = [features]
        x = features
        for l in range(5):
            x = conv3x3(x, ws[l], bs[l], ABI_IN[l], STAGED_OUT[l], _abi.SGS_CONV_RELU)
            acts.append(x)
        out = conv3x3(x, ws[5], bs[5], ABI_IN[5], STAGED_OUT[5], _abi.SGS_CONV_FINAL, residual=features)
        ctx.acts = acts
        ctx.save_for_backward(*[p.detach() for p in params[0::2]])
        return out

    @staticmethod
    def backward(ctx, g_out):
        weights = ctx.saved_tensors
        acts = ctx.acts
        b, h, w = g_out.shape[:3]
        gz = torch.zeros((b, h, w, STAGED_OUT[5]), dtype=torch.bfloat16, device=g_out.device)
        gz[..., :3] = g_out
        grads = [None] * 12
        for l in range(5, -1, -1):
            gw, gb = conv3x3_wgrad(acts[l], ABI_IN[l], gz, STAGED_OUT[l])
            grads[2 * l] = unpack_wgrad(gw, l)
            grads[2 * l + 1] = gb[:LAYERS[l][1]].clone()
            if l > 0:
                wd = pack_dgrad(weights[l], STAGED_IN[l], STAGED_OUT[l])
                gz = conv3x3(gz, wd, None, STAGED_OUT[l], STAGED_IN[l], _abi.SGS_CONV_MASK, mask=acts[l])
        ctx.acts = None
        # the residual path gives the features a gradient too; the input is data, not trained
        return (None, *grads)


def denoise_train(features: torch.Tensor, params: list[torch.Tensor]) -> torch.Tensor:
    """Differentiable denoiser forward on BF16 tensor cores: features FP16 [B, H, W, 8] -> FP32
    [B, H, W, 3]; gradients flow to the 12 parameters [W1, b1, ..., W6, b6]."""
    return _DenoiseTrain.apply(features, *params)


class Denoiser:
    """Inference wrapper: packed BF16 weights for `sgs_denoise` and FP32 masters for saving."""

    def __init__(self, params: list[torch.Tensor] | None = None, device="cuda", seed: int = 0):
        self.params = [p.detach().to(device).float() for p in (params or init_params(seed, device))]
        self.device = torch.device(device)
        self.refresh()

    def refresh(self) -> None:
        """Repacks the BF16 weights after the FP32 parameters changed."""
        self.weights = torch.cat([pack_forward(self.params[2 * l], STAGED_IN[l], STAGED_OUT[l]) for l in range(6)])
        self.biases = torch.cat([_padded_bias(self.params[2 * l + 1], STAGED_OUT[l]) for l in range(6)])
        assert self.weights.numel() * 2 == _lib.sgs_denoise_weights_size()

    def __call__(self, features: torch.Tensor, out: torch.Tensor | None = None,
                 scratch: torch.Tensor | None = None) -> torch.Tensor:
        squeeze = features.dim() == 3
        if squeeze:
            features = features[None]
        b, h, w = features.shape[:3]
        if out is None:
            out = torch.empty((b, h, w, 3), dtype=torch.float32, device=features.device)
        need = _lib.sgs_denoise_scratch_size(b, h, w)
        if scratch is None or scratch.numel() < need:
            scratch = torch.empty(need, dtype=torch.uint8, device=features.device)
        _check(_lib.sgs_denoise(ctypes.c_void_p(features.data_ptr()), b, h, w, ctypes.c_void_p(self.weights.data_ptr()),
                                ctypes.c_void_p(self.biases.data_ptr()), ctypes.c_void_p(scratch.data_ptr()),
                                scratch.numel(), ctypes.c_void_p(out.data_ptr()), _stream(features.device)),
               "sgs_denoise")
        return out[0] if squeeze else out

    def state(self) -> dict[str, np.ndarray]:
        return {f"p{i}": p.cpu().numpy() for i, p in enumerate(self.params)}

    @classmethod
    def from_state(cls, state, device="cuda") -> "Denoiser":
        return cls([torch.from_numpy(np.asarray(state[f"p{i}"])) for i in range(12)], device=device)


class FeatureAccumulator:
    """Per-pixel running sums of samples (sgs_denoise_features_accumulate / _finalize)."""

    def __init__(self, height: int, width: int, device="cuda"):
        self.n_px = height * width
        self.shape = (height, width)
        self.accum = torch.empty((self.n_px, 8), dtype=torch.float32, device=device)
        self.n = 0

    def add(self, image: torch.Tensor, alpha: torch.Tensor, depth: torch.Tensor,
            framebuffer: torch.Tensor | None = None, first: bool | None = None) -> None:
        dev = self.accum.device
        first = self.n == 0 if first is None else first
        _check(_lib.sgs_denoise_features_accumulate(
            ctypes.c_void_p(image.data_ptr()), ctypes.c_void_p(alpha.data_ptr()), ctypes.c_void_p(depth.data_ptr()),
            None if framebuffer is None else ctypes.c_void_p(framebuffer.data_ptr()),
            ctypes.c_void_p(self.accum.data_ptr()), self.n_px, int(first), _stream(dev)),
            "sgs_denoise_features_accumulate")
        self.n = 1 if first else self.n + 1

    def finalize(self, depth_scale: float, out: torch.Tensor | None = None) -> torch.Tensor:
        if out is None:
            out = torch.empty((*self.shape, FEATURES), dtype=torch.float16, device=self.accum.device)
        _check(_lib.sgs_denoise_features_finalize(ctypes.c_void_p(self.accum.data_ptr()), self.n_px, self.n,
                                                  ctypes.c_float(depth_scale), ctypes.c_void_p(out.data_ptr()),
                                                  _stream(self.accum.device)), "sgs_denoise_features_finalize")
        return out


def render_features(tensors, settings: Settings, n_samples: int, first_frame: int, depth_scale: float,
                    accumulator: FeatureAccumulator | None = None, checkpoints=()):
    """Renders n_samples Reset-mode samples at frames first_frame.. and returns their features
    (FP16 [H, W, 8]); with `checkpoints` (sample counts), returns {count: features} instead."""
    dev = tensors[0].device
    h, w = settings.height, settings.width
    n_fb = w * h * max(1, settings.supersampling_factor) ** 2
    acc = accumulator or FeatureAccumulator(h, w, dev)
    acc.n = 0
    e = torch.empty(0)
    kb = (torch.empty((0, n_fb, 2), dtype=torch.int32, device=dev), torch.empty((0, n_fb, 4), device=dev))
    eye = torch.eye(4, device=dev)
    bn = torch.empty(0, dtype=torch.uint8, device=dev)
    marks = {}
    for s in range(n_samples):
        _C.set_frame_index(first_frame + s)
        outs, ws, layout = _C.render_with_workspace(*tensors, *settings.as_tuple(), bn, *kb, e, e, e, e, eye, 0)
        fb = None
        if max(1, settings.supersampling_factor) == 1:
            fb = _C.workspace_views(ws, layout, n_fb, False)["framebuffer"]
        acc.add(outs[0], outs[2], outs[1], fb)
        if s + 1 in checkpoints:
            marks[s + 1] = acc.finalize(depth_scale)
    if checkpoints:
        return marks
    return acc.finalize(depth_scale)


class CapturedFeatures:
    """`render_features` with each sample after the first replayed from a CUDA graph.

    One graph holds a Reset-mode render (frame index from a device counter, advanced on the GPU)
    and its feature accumulation, so the host issues one replay per sample. The scene tensors, the
    camera pose (`w2c`, `position`) and the accumulator are captured by address: `set_scene` and
    `set_pose` copy new values into them; the resolution and intrinsics stay those of `settings`.
    Frames first_frame .. first_frame + n - 1 give the same features as `render_features`.
    """

    def __init__(self, tensors, settings: Settings, depth_scale: float):
        self.device = tensors[0].device
        self.tensors = tuple(t.clone() for t in tensors)
        self.settings = settings._replace(w2c=settings.w2c.clone().contiguous(),
                                          cam_position=settings.cam_position.clone().contiguous())
        self.depth_scale = depth_scale
        h, w = settings.height, settings.width
        self.ss = max(1, settings.supersampling_factor)
        self.n_fb = w * h * self.ss ** 2
        self.acc = FeatureAccumulator(h, w, self.device)
        self.counter = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.kb = (torch.empty((0, self.n_fb, 2), dtype=torch.int32, device=self.device),
                   torch.empty((0, self.n_fb, 4), device=self.device))
        self.eye = torch.eye(4, device=self.device)
        self.blue = torch.empty(0, dtype=torch.uint8, device=self.device)
        self.graph = None

    def _step(self, first: bool):
        e = torch.empty(0)
        outs, ws, layout = _C.render_with_workspace(*self.tensors, *self.settings.as_tuple(), self.blue, *self.kb,
                                                    e, e, e, e, self.eye, 0)
        fb = _C.workspace_views(ws, layout, self.n_fb, False)["framebuffer"] if self.ss == 1 else None
        self.acc.add(outs[0], outs[2], outs[1], fb, first=first)
        return outs, ws

    def capture(self) -> "CapturedFeatures":
        _C.set_device_frame_counter(self.counter)
        try:
            stream = torch.cuda.Stream(self.device)
            stream.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(stream):
                self._step(first=True)
            torch.cuda.current_stream(self.device).wait_stream(stream)
            torch.cuda.synchronize(self.device)
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self._kept = self._step(first=False)
        finally:
            _C.set_device_frame_counter(None, self.device)
        return self

    def set_scene(self, tensors) -> None:
        for d, s in zip(self.tensors, tensors):
            d.copy_(s)

    def set_pose(self, w2c: torch.Tensor, position: torch.Tensor) -> None:
        self.settings.w2c.copy_(w2c)
        self.settings.cam_position.copy_(position)

    def run(self, n_samples: int, first_frame: int, checkpoints=()):
        """Features of n_samples samples (FP16 [H, W, 8]), or {count: features} at `checkpoints`."""
        if self.graph is None:
            self.capture()
        self.counter.fill_(first_frame)
        _C.set_device_frame_counter(self.counter)
        try:
            self._step(first=True)
        finally:
            _C.set_device_frame_counter(None, self.device)
        marks = {}
        if 1 in checkpoints:
            marks[1] = self.acc.finalize(self.depth_scale)
        for s in range(1, n_samples):
            self.graph.replay()
            self.acc.n = s + 1
            if s + 1 in checkpoints:
                marks[s + 1] = self.acc.finalize(self.depth_scale)
        if checkpoints:
            return marks
        return self.acc.finalize(self.depth_scale)
