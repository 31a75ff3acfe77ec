"""Drop-in replacement of the reference extension module `StochasticGSCudaBackend._C`.

`render(...)` takes the same 29 positional arguments as the reference binding
(StochasticGSCudaBackend/render.cu:16-45, bound at render.cu:162-165) and returns the same tuple of
four freshly allocated CUDA tensors (image, depth, alpha, weight_mass). It validates the inputs,
allocates the outputs and a scratch workspace through PyTorch's caching allocator on the inputs'
device, and calls the C ABI (include/sgs_b200.h) on the current PyTorch stream. All compute runs in
the CUDA kernels of libsgs_b200.so; there is no CPU path.

Extras beyond the reference module: `get_frame_index` / `set_frame_index` expose the process-wide
frame counter that seeds the random numbers (a hidden static in render.cu:56-57), and
`render_with_workspace` additionally returns the scratch workspace and its layout so callers can
inspect the winner framebuffer and the samples.
"""
from __future__ import annotations

import ctypes

import torch

from . import _abi

_lib = _abi.load()

k_buffer_size: int = int(_lib.sgs_k_buffer_size())

_VALID_SH_BASES = (1, 4, 9, 16)


def get_frame_index() -> int:
    return int(_lib.sgs_get_frame_index())


def set_frame_index(frame_index: int) -> None:
    _lib.sgs_set_frame_index(int(frame_index) & 0xFFFFFFFF)


_device_frame_counters: dict = {}


def set_device_frame_counter(counter: torch.Tensor | None, device=None) -> None:
    """Keeps the frame index of subsequent calls on `counter`'s device in that one-element int32 CUDA
    tensor: each call reads it as its frame index and advances it on the GPU, so render calls
    captured in a CUDA graph draw new random numbers on every replay. None returns that device to
    the process-wide counter (`get_frame_index`). The tensor must stay alive while it is in use."""
    if counter is None:
        _device_frame_counters.pop(_device_key(device), None)
        return
    _check(counter.is_cuda and counter.dtype == torch.int32 and counter.numel() == 1 and counter.is_contiguous(),
           "the frame counter must be a contiguous one-element int32 CUDA tensor")
    _device_frame_counters[_device_key(counter.device)] = counter


def _device_key(device) -> int:
    """CUDA device ordinal of `device` (None, "cuda", "cuda:1", torch.device or int)."""
    if device is None:
        return torch.cuda.current_device()
    if isinstance(device, int):
        return device
    d = torch.device(device)
    return d.index if d.index is not None else torch.cuda.current_device()


def _device_frame_pointer(device: torch.device) -> int | None:
    t = _device_frame_counters.get(_device_key(device))
    return None if t is None else t.data_ptr()


def set_stage_events(start=None, end=None) -> None:
    """Records `start`/`end` (cudaEvent_t handles as int or c_void_p) around the accumulate stage of
    this thread's next render calls; None disables. Timing aid (no counterpart in the reference module)."""
    _lib.sgs_set_stage_events(start, end)


def set_queue_limit(max_entries: int = 0) -> None:
    """Caps the large-Gaussian work queue of stochastic transparency (0: default); a testing aid for
    the in-place path taken by Gaussians that find the queue full."""
    _lib.sgs_set_queue_limit(int(max_entries))


def preactivate(scales: torch.Tensor, rotations: torch.Tensor, opacities: torch.Tensor) -> torch.Tensor:
    """The preactivated layout of these Gaussians (sgs_preactivate): an (N, 8) float32 tensor holding,
    per Gaussian, the 3-D covariance's upper triangle (c11, c12, c13, c22, c23, c33), the opacity
    sigmoid and 1 (0 for a degenerate quaternion). Compute it once per model and pass it as
    `preactivated=` to the render calls; recompute it whenever the parameters change."""
    device = scales.device
    scales = _cuda_f32(scales, "scales", device)
    rotations = _cuda_f32(rotations, "rotations", device)
    opacities = _cuda_f32(opacities, "opacities", device)
    n = scales.shape[0]
    _check(tuple(scales.shape) == (n, 3) and tuple(rotations.shape) == (n, 4) and opacities.numel() == n,
           "scales (N, 3), rotations (N, 4) and opacities (N) must describe the same Gaussians")
    out = torch.empty((n, 8), dtype=torch.float32, device=device)
    g = _abi.Gaussians(None, _ptr(scales), _ptr(rotations), _ptr(opacities), None, n, 1, None)
    with torch.cuda.device(device):
        stream = torch.cuda.current_stream(device).cuda_stream
        status = _lib.sgs_preactivate(ctypes.byref(g), ctypes.c_void_p(out.data_ptr()) if n else None,
                                      ctypes.c_void_p(stream))
    if status != _abi.SGS_OK:
        raise RuntimeError(f"sgs_preactivate failed ({status}): {_abi.last_error(_lib)}")
    return out


class Quantized(tuple):
    """The quantised layout of a model (`quantize`): (records (N, 4) int32, chunks (C, 8) float32,
    sh_half (N, B, 3) float16)."""

    __slots__ = ()

    def __new__(cls, records, chunks, sh_half):
        return super().__new__(cls, (records, chunks, sh_half))

    records = property(lambda self: self[0])
    chunks = property(lambda self: self[1])
    sh_half = property(lambda self: self[2])

    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in self)


def quantize(means: torch.Tensor, scales: torch.Tensor, rotations: torch.Tensor, opacities: torch.Tensor,
             sh_coefficients: torch.Tensor) -> Quantized:
    """The quantised layout of these Gaussians (sgs_quantize): 16 bytes per Gaussian for positions (11-10-11
    bits inside the box of each chunk of 256 consecutive Gaussians), rotations (three smallest quaternion
    components, 10 bits each), log-scales and opacity logits (half), plus half-precision SH. Pass it as
    `quantized=` to the render calls; the images then differ from the float32 ones by the quantisation.
    Recompute it whenever the parameters change."""
    device = means.device
    means = _cuda_f32(means, "means", device)
    scales = _cuda_f32(scales, "scales", device)
    rotations = _cuda_f32(rotations, "rotations", device)
    opacities = _cuda_f32(opacities, "opacities", device)
    sh_coefficients = _cuda_f32(sh_coefficients, "sh_coefficients", device)
    n = means.shape[0]
    bases = sh_coefficients.shape[1]
    _check(tuple(means.shape) == (n, 3) and tuple(scales.shape) == (n, 3) and tuple(rotations.shape) == (n, 4)
           and opacities.numel() == n and tuple(sh_coefficients.shape) == (n, bases, 3) and bases in _VALID_SH_BASES,
           "means (N, 3), scales (N, 3), rotations (N, 4), opacities (N) and sh_coefficients (N, B, 3)")
    records = torch.empty((n, 4), dtype=torch.int32, device=device)
    chunks = torch.empty((int(_lib.sgs_quantized_chunks(n)), 8), dtype=torch.float32, device=device)
    sh_half = torch.empty((n, bases, 3), dtype=torch.float16, device=device)
    g = _abi.Gaussians(_ptr(means), _ptr(scales), _ptr(rotations), _ptr(opacities), _ptr(sh_coefficients), n, bases)
    with torch.cuda.device(device):
        stream = torch.cuda.current_stream(device).cuda_stream
        status = _lib.sgs_quantize(ctypes.byref(g), _ptr(records), _ptr(chunks), _ptr(sh_half),
                                   ctypes.c_void_p(stream))
    if status != _abi.SGS_OK:
        raise RuntimeError(f"sgs_quantize failed ({status}): {_abi.last_error(_lib)}")
    return Quantized(records, chunks, sh_half)


def probe_atomic_min(slots: torch.Tensor, ops_per_thread: int, blocks: int, pattern: int = 0, seed: int = 0) -> int:
    """Launches the red.min.u64 throughput probe (sgs_probe_atomic_min) on the current stream into
    `slots` (a contiguous int64 CUDA tensor of power-of-two length); returns the number of
    reductions issued. Measurement aid (no counterpart in the reference module)."""
    _check(slots.is_cuda and slots.dtype == torch.int64 and slots.is_contiguous(),
           "slots must be a contiguous int64 CUDA tensor")
    stream = torch.cuda.current_stream(slots.device).cuda_stream
    status = _lib.sgs_probe_atomic_min(ctypes.c_void_p(slots.data_ptr()), slots.numel(), int(ops_per_thread),
                                       int(blocks), int(pattern), int(seed) & 0xFFFFFFFF, ctypes.c_void_p(stream))
    if status != _abi.SGS_OK:
        raise RuntimeError(f"sgs_probe_atomic_min failed ({status}): {_abi.last_error(_lib)}")
    return int(blocks) * 256 * int(ops_per_thread)


def composite(image: torch.Tensor, depth: torch.Tensor, alpha: torch.Tensor, background: torch.Tensor,
              out: tuple | None = None):
    """The renderer plugin's frame compositing (Renderer.py:91-97) as one kernel (sgs_composite) on the
    current stream: returns (rgb, depth, alpha) = (clamp(image + (1 - a) * background, 0, 1),
    depth / max(a, 1e-8), a) with a = clamp(alpha, 0, 1), bit for bit the values of those tensor
    operations. `background` is a (3,) float32 CUDA tensor; `out` optionally three caller-owned tensors
    of the result shapes (nothing is allocated then, so the call can sit in a CUDA graph)."""
    device = image.device
    image = _cuda_f32(image, "image", device)
    depth = _cuda_f32(depth, "depth", device)
    alpha = _cuda_f32(alpha, "alpha", device)
    background = _cuda_f32(background, "background", device)
    n = alpha.numel()
    _check(image.numel() == 3 * n and depth.numel() == n and background.numel() == 3,
           "image (H, W, 3), depth and alpha (H, W, 1) and a background of 3 values")
    if out is None:
        out = (torch.empty_like(image), torch.empty_like(depth), torch.empty_like(alpha))
    for t, ref in zip(out, (image, depth, alpha)):
        _check(t.is_cuda and t.device == device and t.dtype == torch.float32 and t.is_contiguous()
               and t.numel() == ref.numel(), "outputs must be contiguous float32 tensors of the inputs' sizes")
    stream = torch.cuda.current_stream(device).cuda_stream
    status = _lib.sgs_composite(image.data_ptr(), depth.data_ptr(), alpha.data_ptr(), background.data_ptr(), n,
                                out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), ctypes.c_void_p(stream))
    if status != _abi.SGS_OK:
        raise RuntimeError(f"sgs_composite failed ({status}): {_abi.last_error(_lib)}")
    return out


def _check(cond: bool, msg: str) -> None:
    if not cond:
        raise RuntimeError(msg)


def _cuda_f32(t: torch.Tensor, name: str, device: torch.device) -> torch.Tensor:
    _check(isinstance(t, torch.Tensor), f"{name} must be a tensor")
    _check(t.is_cuda and t.device == device, f"{name} must be a CUDA tensor on {device}")
    _check(t.dtype == torch.float32, f"{name} must be float32")
    return t.contiguous()


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None or t.numel() == 0 else t.data_ptr()


def _prepare(means, scales, rotations, opacities, sh_coefficients, w2c, cam_position, width, height, focal_x, focal_y,
             center_x, center_y, near_plane, far_plane, proper_antialiasing, supersampling_factor_raw, use_gps,
             hybrid_scheduling, spatial_reuse, blue_noise, k_buffer_primitives, k_buffer_occlusion, history_image,
             history_depth, history_alpha, history_weight_mass, view_to_previous_view, temporal_mode, preactivated=None,
             max_fragments=0, max_binned=0, quantized=None):
    _check(isinstance(means, torch.Tensor) and means.is_cuda, "means must be a CUDA tensor")
    device = means.device
    means = _cuda_f32(means, "means", device)
    n = means.shape[0]
    _check(means.dim() == 2 and means.shape[1] == 3, "means must have shape (N, 3)")
    scales = _cuda_f32(scales, "scales", device)
    _check(tuple(scales.shape) == (n, 3), "scales must have shape (N, 3)")
    rotations = _cuda_f32(rotations, "rotations", device)
    _check(tuple(rotations.shape) == (n, 4), "rotations must have shape (N, 4)")
    opacities = _cuda_f32(opacities, "opacities", device)
    _check(opacities.numel() == n, "opacities must hold N values")
    sh_coefficients = _cuda_f32(sh_coefficients, "sh_coefficients", device)
    _check(sh_coefficients.dim() == 3 and sh_coefficients.shape[0] == n and sh_coefficients.shape[2] == 3,
           "sh_coefficients must have shape (N, B, 3)")
    sh_bases = sh_coefficients.shape[1]
    _check(sh_bases in _VALID_SH_BASES, f"sh_coefficients must have 1, 4, 9 or 16 bases, got {sh_bases}")
    w2c = _cuda_f32(w2c, "w2c", device)
    _check(w2c.numel() >= 12 and w2c.shape[-1] == 4, "w2c must hold at least 3 rows of 4 floats")
    cam_position = _cuda_f32(cam_position, "cam_position", device)
    _check(cam_position.numel() == 3, "cam_position must hold 3 floats")
    width, height = int(width), int(height)
    _check(0 < width < 2 ** 32 and 0 < height < 2 ** 32, "width and height must be positive")
    ss = max(1, int(supersampling_factor_raw))
    n_fb = width * height * ss * ss
    n_px = width * height
    mode = int(temporal_mode)
    _check(mode in (0, 1, 2), f"invalid temporal mode {mode}")

    if blue_noise is not None and blue_noise.numel() > 0:
        _check(blue_noise.is_cuda and blue_noise.device == device and blue_noise.dtype == torch.uint8
               and blue_noise.numel() == 64 * 128 * 128, "blue_noise must be a (64, 128, 128) uint8 CUDA tensor")
        blue_noise = blue_noise.contiguous()
    else:
        blue_noise = None

    if spatial_reuse:
        k = k_buffer_size
        _check(k_buffer_primitives.is_cuda and k_buffer_primitives.device == device
               and k_buffer_primitives.dtype == torch.int32 and tuple(k_buffer_primitives.shape) == (k, n_fb, 2)
               and k_buffer_primitives.is_contiguous(), f"k_buffer_primitives must be a contiguous ({k}, {n_fb}, 2) int32 CUDA tensor")
        _check(k_buffer_occlusion.is_cuda and k_buffer_occlusion.device == device
               and k_buffer_occlusion.dtype == torch.float32 and tuple(k_buffer_occlusion.shape) == (k, n_fb, 4)
               and k_buffer_occlusion.is_contiguous(), f"k_buffer_occlusion must be a contiguous ({k}, {n_fb}, 4) float32 CUDA tensor")

    if mode != 0:
        for name, t, ch in (("history_image", history_image, 3), ("history_depth", history_depth, 1),
                            ("history_alpha", history_alpha, 1), ("history_weight_mass", history_weight_mass, 1)):
            _check(isinstance(t, torch.Tensor) and t.is_cuda and t.device == device and t.dtype == torch.float32
                   and t.numel() == n_px * ch and t.is_contiguous(),
                   f"{name} must be a contiguous ({height}, {width}, {ch}) float32 CUDA tensor in temporal mode {mode}")
    if mode == 2:
        view_to_previous_view = _cuda_f32(view_to_previous_view, "view_to_previous_view", device)
        _check(view_to_previous_view.numel() >= 12, "view_to_previous_view must be a 4x4 matrix")
    else:
        view_to_previous_view = None

    if preactivated is not None:
        _check(isinstance(preactivated, torch.Tensor) and preactivated.is_cuda and preactivated.device == device
               and preactivated.dtype == torch.float32 and tuple(preactivated.shape) == (n, 8)
               and preactivated.is_contiguous() and preactivated.data_ptr() % 16 == 0,
               "preactivated must be the contiguous (N, 8) float32 CUDA tensor of preactivate()")
    max_fragments, max_binned = int(max_fragments or 0), int(max_binned or 0)
    _check(0 <= max_fragments < 2 ** 32 and 0 <= max_binned < 2 ** 32,
           "max_fragments and max_binned must be non-negative 32-bit counts (0 = the reference's default)")
    if quantized is not None:
        _check(isinstance(quantized, Quantized) and preactivated is None,
               "quantized must be the result of quantize(), without preactivated=")
        rec, chunks, sh_half = quantized
        _check(rec.is_cuda and rec.device == device and tuple(rec.shape) == (n, 4) and rec.dtype == torch.int32
               and tuple(sh_half.shape) == (n, sh_bases, 3) and sh_half.dtype == torch.float16
               and chunks.shape[0] == int(_lib.sgs_quantized_chunks(n)),
               "quantized does not describe these Gaussians")
    g = _abi.Gaussians(_ptr(means), _ptr(scales), _ptr(rotations), _ptr(opacities), _ptr(sh_coefficients), n, sh_bases,
                       _ptr(preactivated), *((_ptr(t) for t in quantized) if quantized is not None else (None,) * 3))
    c = _abi.Camera(w2c.data_ptr(), cam_position.data_ptr(), width, height, float(focal_x), float(focal_y),
                    float(center_x), float(center_y), float(near_plane), float(far_plane))
    s = _abi.SettingsC(int(bool(proper_antialiasing)), ss, int(bool(use_gps)), int(bool(hybrid_scheduling)),
                       int(bool(spatial_reuse)), mode, _ptr(blue_noise), _ptr(view_to_previous_view), max_fragments,
                       max_binned, _device_frame_pointer(device))
    h = _abi.HistoryC(
        _ptr(history_image) if mode else None, _ptr(history_depth) if mode else None,
        _ptr(history_alpha) if mode else None, _ptr(history_weight_mass) if mode else None,
        _ptr(k_buffer_primitives) if spatial_reuse else None, _ptr(k_buffer_occlusion) if spatial_reuse else None)
    # keep the contiguous copies alive for the duration of the call
    keep = (means, scales, rotations, opacities, sh_coefficients, w2c, cam_position, blue_noise, view_to_previous_view,
            preactivated, *(quantized or ()))
    return device, g, c, s, h, (width, height), keep


def _render_impl(args, want_workspace: bool, streams=None, preactivated=None, caps=None):
    device, g, c, s, h, (width, height), keep = _prepare(*args, preactivated=preactivated, **(caps or {}))
    with torch.cuda.device(device):
        opts = dict(dtype=torch.float32, device=device)
        image = torch.empty((height, width, 3), **opts)
        depth = torch.empty((height, width, 1), **opts)
        alpha = torch.empty((height, width, 1), **opts)
        weight_mass = torch.empty((height, width, 1), **opts)
        o = _abi.Outputs(image.data_ptr(), depth.data_ptr(), alpha.data_ptr(), weight_mass.data_ptr())
        ws_bytes = int(_lib.sgs_workspace_size(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s)))
        if ws_bytes == 0:
            raise RuntimeError(_abi.last_error(_lib) or "invalid render arguments")
        workspace = torch.empty((ws_bytes,), dtype=torch.uint8, device=device)
        if streams is None:
            stream = torch.cuda.current_stream(device).cuda_stream
            status = _lib.sgs_render(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.byref(h),
                                     ctypes.byref(o), ctypes.c_void_p(workspace.data_ptr()), ctypes.c_size_t(ws_bytes),
                                     ctypes.c_void_p(stream))
        else:
            acc, res = streams
            status = _lib.sgs_render_split(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.byref(h),
                                           ctypes.byref(o), ctypes.c_void_p(workspace.data_ptr()),
                                           ctypes.c_size_t(ws_bytes), ctypes.c_void_p(acc.cuda_stream),
                                           ctypes.c_void_p(res.cuda_stream))
            # the caching allocator must not hand these blocks out again before the streams are done
            for t in (image, depth, alpha, weight_mass):
                t.record_stream(res)
            workspace.record_stream(acc)
            workspace.record_stream(res)
            for t in keep:
                if t is not None:
                    t.record_stream(acc)
                    t.record_stream(res)
        if status != _abi.SGS_OK:
            raise RuntimeError(f"sgs_render failed ({status}): {_abi.last_error(_lib)}")
        del keep
        if not want_workspace:
            return image, depth, alpha, weight_mass
        layout = _abi.WorkspaceLayout()
        _lib.sgs_get_workspace_layout(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.byref(layout))
        return (image, depth, alpha, weight_mass), workspace, layout


def render(*args, preactivated=None, max_fragments=0, max_binned=0, quantized=None):
    """`_C.render` with the reference's 29 positional arguments; returns (image, depth, alpha, weight_mass).

    Keyword-only extras (not in the reference's binding):
      preactivated   the (N, 8) tensor of `preactivate()` for these Gaussians; the accumulate pass then
                     reads covariance and opacity from it (same bits);
      max_fragments  GPS points per Gaussian cap of hybrid scheduling (0: the reference's
                     round(W_fb * H_fb / (2 ss^2)), accumulate_hybrid_gps.cu:86);
      max_binned     capacity of the hybrid work queue in Gaussians (0: the reference's min(N, 2^20),
                     accumulate_hybrid_gps.cu:22 and accumulate_hybrid.cu:27). Gaussians beyond it are
                     rendered in place, as in the reference;
      quantized      the `quantize()` layout of these Gaussians, read by every pass in place of the
                     float32 arrays (the images differ by the quantisation)."""
    if len(args) != 29:
        raise TypeError(f"render() takes 29 positional arguments ({len(args)} given)")
    return _render_impl(args, want_workspace=False, preactivated=preactivated,
                        caps=dict(max_fragments=max_fragments, max_binned=max_binned, quantized=quantized))


def render_split(accumulate_stream: torch.cuda.Stream, resolve_stream: torch.cuda.Stream, *args, preactivated=None,
                 max_fragments=0, max_binned=0):
    """As `render` (the same 29 arguments after the two streams), with the clear and accumulate passes
    enqueued on `accumulate_stream` and the sample and resolve passes on `resolve_stream` (the C ABI's
    sgs_render_split): a following call can accumulate while this one resolves. The outputs are
    complete on `resolve_stream`; the caller orders its other streams against the two."""
    if len(args) != 29:
        raise TypeError(f"render_split() takes 2 streams and 29 positional arguments ({len(args)} given)")
    return _render_impl(args, want_workspace=False, streams=(accumulate_stream, resolve_stream),
                        preactivated=preactivated, caps=dict(max_fragments=max_fragments, max_binned=max_binned))


def render_samples(n_samples: int, *args, preactivated=None, **caps):
    """`n_samples` samples in one call (the C ABI's sgs_render_samples): the same 29 arguments as
    `render`, frames f .. f + n_samples - 1 merged in order (the first in the given temporal mode, the
    rest Static); returns the final (image, depth, alpha, weight_mass), equal bit for bit to
    `n_samples` `render` calls (the k-buffer too, with spatial reuse). Keyword extras as `render`."""
    return _render_samples(n_samples, args, want_workspace=False, preactivated=preactivated, caps=caps)


def render_samples_with_workspace(n_samples: int, *args, preactivated=None, **caps):
    """As `render_samples`, plus the workspace (its framebuffer section holds the n_samples winner
    framebuffers back to back; with spatial reuse or a Reproject first sample, only the last sample's
    framebuffer, in the first slot) and its layout."""
    return _render_samples(n_samples, args, want_workspace=True, preactivated=preactivated, caps=caps)


def _render_samples(n_samples: int, args, want_workspace: bool, preactivated=None, caps=None):
    if len(args) != 29:
        raise TypeError(f"render_samples() takes n_samples and 29 render arguments ({len(args)} given)")
    n = int(n_samples)
    _check(1 <= n <= 1024, f"n_samples must be between 1 and 1024, got {n}")
    caps = dict(caps or {})
    _check(set(caps) <= {"max_fragments", "max_binned", "quantized"}, f"unexpected keyword arguments {sorted(caps)}")
    device = args[0].device if isinstance(args[0], torch.Tensor) else None
    if device is not None and device.type == "cuda" and device.index != torch.cuda.current_device():
        with torch.cuda.device(device):
            return _render_samples_impl(n, args, want_workspace, preactivated, caps)
    return _render_samples_impl(n, args, want_workspace, preactivated, caps)


def _render_samples_impl(n: int, args, want_workspace: bool, preactivated=None, caps=None):
    device, g, c, s, h, (width, height), keep = _prepare(*args, preactivated=preactivated, **(caps or {}))
    opts = dict(dtype=torch.float32, device=device)
    outs = (torch.empty((height, width, 3), **opts), torch.empty((height, width, 1), **opts),
            torch.empty((height, width, 1), **opts), torch.empty((height, width, 1), **opts))
    o = _abi.Outputs(*(t.data_ptr() for t in outs))
    ws_bytes = int(_lib.sgs_samples_workspace_size(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), n))
    if ws_bytes == 0:
        raise RuntimeError(_abi.last_error(_lib) or "invalid render arguments")
    workspace = torch.empty((ws_bytes,), dtype=torch.uint8, device=device)
    stream = torch.cuda.current_stream(device).cuda_stream
    status = _lib.sgs_render_samples(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.byref(h),
                                     ctypes.byref(o), n, ctypes.c_void_p(workspace.data_ptr()),
                                     ctypes.c_size_t(ws_bytes), ctypes.c_void_p(stream))
    if status != _abi.SGS_OK:
        raise RuntimeError(f"sgs_render_samples failed ({status}): {_abi.last_error(_lib)}")
    del keep
    if not want_workspace:
        return outs
    layout = _abi.WorkspaceLayout()
    _lib.sgs_get_workspace_layout(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.byref(layout))
    return outs, workspace, layout


def workspace_size(*args, max_fragments=0, max_binned=0) -> int:
    """Bytes of scratch a render with these 29 `render` arguments needs (sgs_workspace_size)."""
    _, g, c, s, _, _, _ = _prepare(*args, max_fragments=max_fragments, max_binned=max_binned)
    n = int(_lib.sgs_workspace_size(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s)))
    if n == 0:
        raise RuntimeError(_abi.last_error(_lib) or "invalid render arguments")
    return n


def render_into(outputs, workspace: torch.Tensor, streams, *args, preactivated=None, max_fragments=0,
                max_binned=0) -> None:
    """Renders like `render` into caller-owned buffers: `outputs` = (image (H, W, 3), depth, alpha,
    weight_mass (H, W, 1)) float32 CUDA tensors, `workspace` a uint8 CUDA tensor of at least
    `workspace_size(*args)` bytes (256-byte aligned), `streams` = None (current stream) or
    (accumulate stream, resolve stream) as in `render_split`. Nothing is allocated, so the call can
    be captured in a CUDA graph with fixed buffers (for example ping-ponged histories)."""
    if len(args) != 29:
        raise TypeError(f"render_into() takes outputs, workspace, streams and 29 render arguments ({len(args)} given)")
    device, g, c, s, h, (width, height), keep = _prepare(*args, preactivated=preactivated, max_fragments=max_fragments,
                                                         max_binned=max_binned)
    shapes = ((height, width, 3), (height, width, 1), (height, width, 1), (height, width, 1))
    for name, t, shape in zip(("image", "depth", "alpha", "weight_mass"), outputs, shapes):
        _check(isinstance(t, torch.Tensor) and t.is_cuda and t.device == device and t.dtype == torch.float32
               and tuple(t.shape) == shape and t.is_contiguous(),
               f"output {name} must be a contiguous {shape} float32 CUDA tensor on {device}")
    ws_bytes = int(_lib.sgs_workspace_size(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s)))
    _check(ws_bytes > 0, _abi.last_error(_lib) or "invalid render arguments")
    _check(workspace.is_cuda and workspace.device == device and workspace.dtype == torch.uint8
           and workspace.numel() >= ws_bytes and workspace.data_ptr() % 256 == 0,
           f"workspace must be a 256-byte aligned uint8 CUDA tensor of at least {ws_bytes} bytes")
    o = _abi.Outputs(*(t.data_ptr() for t in outputs))
    if streams is None:
        acc = res = torch.cuda.current_stream(device)
    else:
        acc, res = streams
    status = _lib.sgs_render_split(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.byref(h), ctypes.byref(o),
                                   ctypes.c_void_p(workspace.data_ptr()), ctypes.c_size_t(workspace.numel()),
                                   ctypes.c_void_p(acc.cuda_stream), ctypes.c_void_p(res.cuda_stream))
    if status != _abi.SGS_OK:
        raise RuntimeError(f"sgs_render_split failed ({status}): {_abi.last_error(_lib)}")
    del keep


def render_samples_into(outputs, workspace: torch.Tensor, n_samples: int, *args, preactivated=None, max_fragments=0,
                        max_binned=0, quantized=None) -> None:
    """`render_samples` into caller-owned buffers: `outputs` = (image (H, W, 3), depth, alpha,
    weight_mass (H, W, 1)) float32 CUDA tensors, not the history; `workspace` a uint8 CUDA tensor of
    at least `samples_workspace_size(n_samples, *args)` bytes, 256-byte aligned. Nothing is allocated,
    so the call can be captured in a CUDA graph."""
    if len(args) != 29:
        raise TypeError(f"render_samples_into() takes outputs, workspace, n_samples and 29 render arguments "
                        f"({len(args)} given)")
    n = int(n_samples)
    _check(1 <= n <= 1024, f"n_samples must be between 1 and 1024, got {n}")
    device, g, c, s, h, (width, height), keep = _prepare(*args, preactivated=preactivated, max_fragments=max_fragments,
                                                         max_binned=max_binned, quantized=quantized)
    shapes = ((height, width, 3), (height, width, 1), (height, width, 1), (height, width, 1))
    for name, t, shape in zip(("image", "depth", "alpha", "weight_mass"), outputs, shapes):
        _check(isinstance(t, torch.Tensor) and t.is_cuda and t.device == device and t.dtype == torch.float32
               and tuple(t.shape) == shape and t.is_contiguous(),
               f"output {name} must be a contiguous {shape} float32 CUDA tensor on {device}")
    ws_bytes = int(_lib.sgs_samples_workspace_size(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), n))
    _check(ws_bytes > 0, _abi.last_error(_lib) or "invalid render arguments")
    _check(workspace.is_cuda and workspace.device == device and workspace.dtype == torch.uint8
           and workspace.numel() >= ws_bytes and workspace.data_ptr() % 256 == 0,
           f"workspace must be a 256-byte aligned uint8 CUDA tensor of at least {ws_bytes} bytes")
    o = _abi.Outputs(*(t.data_ptr() for t in outputs))
    stream = torch.cuda.current_stream(device).cuda_stream
    status = _lib.sgs_render_samples(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.byref(h),
                                     ctypes.byref(o), n, ctypes.c_void_p(workspace.data_ptr()),
                                     ctypes.c_size_t(workspace.numel()), ctypes.c_void_p(stream))
    if status != _abi.SGS_OK:
        raise RuntimeError(f"sgs_render_samples failed ({status}): {_abi.last_error(_lib)}")
    del keep


def samples_workspace_size(n_samples: int, *args, max_fragments=0, max_binned=0) -> int:
    """Bytes of scratch `render_samples` with these 29 arguments needs (sgs_samples_workspace_size)."""
    _, g, c, s, _, _, _ = _prepare(*args, max_fragments=max_fragments, max_binned=max_binned)
    n = int(_lib.sgs_samples_workspace_size(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), int(n_samples)))
    if n == 0:
        raise RuntimeError(_abi.last_error(_lib) or "invalid render arguments")
    return n


def render_with_workspace(*args, preactivated=None, max_fragments=0, max_binned=0, quantized=None):
    """As `render`, plus the workspace tensor and its layout (winner framebuffer, samples, reuse weights)."""
    if len(args) != 29:
        raise TypeError(f"render_with_workspace() takes 29 positional arguments ({len(args)} given)")
    return _render_impl(args, want_workspace=True, preactivated=preactivated,
                        caps=dict(max_fragments=max_fragments, max_binned=max_binned, quantized=quantized))


def workspace_views(workspace: torch.Tensor, layout, n_fb: int, spatial_reuse: bool) -> dict[str, torch.Tensor]:
    """Typed views of a workspace returned by `render_with_workspace`."""
    fb = workspace[layout.framebuffer:layout.framebuffer + 8 * n_fb].view(torch.int64)
    samples = workspace[layout.samples:layout.samples + 16 * n_fb].view(torch.float32).view(n_fb, 4)
    out = {"framebuffer": fb, "samples": samples}
    if spatial_reuse:
        out["reuse_weights"] = workspace[layout.reuse_weights:layout.reuse_weights + 16 * n_fb].view(torch.float32).view(n_fb, 4)
    return out
