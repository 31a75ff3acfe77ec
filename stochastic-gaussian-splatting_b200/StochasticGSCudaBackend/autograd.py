"""Differentiable rendering: gradients of the progressively averaged image w.r.t. the Gaussians.

`render_samples(means, scales, rotations, opacities, sh, settings, n_samples)` renders n_samples
samples (Reset, then Static: their plain average, as Renderer.py's SAMPLES_PER_PIXEL loop produces
it) with stochastic transparency or Gaussian point splatting (`settings.use_gps`, scatter or hybrid
scheduling) and returns (image, depth, alpha) like `History`, with a backward pass to all five
parameter tensors (the reference renders only; it has no backward).

The backward is an unbiased estimator of the gradient of the expected image (see
csrc/backward_st.cu): each sample's winners give a one-sample estimate, averaged over the samples.
For GPS a fragment's alpha is replaced by the probability that the Gaussian puts a point into the
(sub)pixel, from the law of the point count the render draws and a quadrature of the point density
over the pixel.
The forward renders all samples in one call (`_C.render_samples`: one fragment walk, the samples'
winner framebuffers side by side in its workspace, outputs bit-identical to one call per sample).
Winners are either kept from the forward pass (`store_winners=True`, 8 bytes per framebuffer pixel
and sample) or recomputed in backward by rendering the same frame indices again
(`store_winners=False`: one more multi-sample render, nothing kept between the passes). The backward
tabulates every sample's winner and colour term (12 bytes per framebuffer pixel and sample, 8 more
per pixel) and walks the Gaussians' fragments once for all samples
(sgs_backward_accumulate_framebuffers).
"""
from __future__ import annotations

import ctypes

import torch

from . import _abi, _C
from .render import Settings

_lib = _abi.load()


def _structs(means, scales, rotations, opacities, sh, settings: Settings):
    g = _abi.Gaussians(means.data_ptr(), scales.data_ptr(), rotations.data_ptr(), opacities.data_ptr(), sh.data_ptr(),
                       means.shape[0], sh.shape[1])
    c = _abi.Camera(settings.w2c.data_ptr(), settings.cam_position.data_ptr(), settings.width, settings.height,
                    float(settings.focal_x), float(settings.focal_y), float(settings.center_x),
                    float(settings.center_y), float(settings.near_plane), float(settings.far_plane))
    s = _abi.SettingsC(int(settings.proper_antialiasing), max(1, int(settings.supersampling_factor)),
                       int(settings.use_gps), int(settings.hybrid_scheduling), int(settings.spatial_reuse), 1, None,
                       None, 0, 0, None)
    return g, c, s


def _render_one(tensors, settings: Settings, hist, mode: int, frame: int):
    _C.set_frame_index(frame)
    n_fb = settings.width * settings.height * max(1, settings.supersampling_factor) ** 2
    dev = tensors[0].device
    kb = (torch.empty((0, n_fb, 2), dtype=torch.int32, device=dev), torch.empty((0, n_fb, 4), device=dev))
    return _C.render_with_workspace(*tensors, *settings.as_tuple(), torch.empty(0, dtype=torch.uint8, device=dev),
                                    *kb, *hist, torch.eye(4, device=dev), mode)


def _render_all(tensors, settings: Settings, n_samples: int, first_frame: int):
    """n_samples samples (Reset, then Static) in one call; returns (outputs, workspace, layout) and
    leaves the process-wide frame index where it was."""
    saved = _C.get_frame_index()
    _C.set_frame_index(first_frame)
    try:
        n_fb = settings.width * settings.height * max(1, settings.supersampling_factor) ** 2
        dev = tensors[0].device
        kb = (torch.empty((0, n_fb, 2), dtype=torch.int32, device=dev), torch.empty((0, n_fb, 4), device=dev))
        e = torch.empty(0)
        return _C.render_samples_with_workspace(n_samples, *tensors, *settings.as_tuple(),
                                                torch.empty(0, dtype=torch.uint8, device=dev), *kb, e, e, e, e,
                                                torch.eye(4, device=dev), 0)
    finally:
        _C.set_frame_index(saved)


class _RenderSamples(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means, scales, rotations, opacities, sh, settings, n_samples, first_frame, store_winners):
        if settings.spatial_reuse:
            raise RuntimeError("render_samples does not differentiate spatial reuse")
        tensors = tuple(t.detach().contiguous() for t in (means, scales, rotations, opacities, sh))
        (image, depth, alpha, _), ws, layout = _render_all(tensors, settings, n_samples, first_frame)
        ctx.save_for_backward(*tensors)
        ctx.settings = settings
        ctx.n_samples = n_samples
        ctx.first_frame = first_frame
        ctx.winners = (ws, layout.framebuffer) if store_winners else None
        return image, depth, alpha

    @staticmethod
    def backward(ctx, g_image, g_depth, g_alpha):
        tensors = ctx.saved_tensors
        settings = ctx.settings
        dev = tensors[0].device
        g, c, s = _structs(*tensors, settings)
        grads_in = [None if t is None else t.contiguous() for t in (g_image, g_alpha, g_depth)]
        if grads_in[0] is None:
            grads_in[0] = torch.zeros((settings.height, settings.width, 3), device=dev)
        bw = torch.empty(_lib.sgs_backward_workspace_size(tensors[0].shape[0]) // 4 + 4, dtype=torch.float32,
                         device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        weight = 1.0 / ctx.n_samples
        n = ctx.n_samples
        if ctx.winners is not None:
            ws, fb_offset = ctx.winners
        else:
            _, ws, layout = _render_all(tensors, settings, n, ctx.first_frame)
            fb_offset = layout.framebuffer
        scratch = torch.empty(_lib.sgs_backward_samples_scratch_size(ctypes.byref(c), ctypes.byref(s), n),
                              dtype=torch.uint8, device=dev)
        gptr = [None if t is None else ctypes.c_void_p(t.data_ptr()) for t in grads_in]
        st = _lib.sgs_backward_accumulate_framebuffers(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s),
                                                       ctypes.c_void_p(ws.data_ptr() + fb_offset), n, gptr[0],
                                                       gptr[1], gptr[2], ctypes.c_float(weight), 1,
                                                       ctypes.c_void_p(scratch.data_ptr()),
                                                       ctypes.c_void_p(bw.data_ptr()), ctypes.c_void_p(stream))
        if st != _abi.SGS_OK:
            raise RuntimeError(f"sgs_backward_accumulate_framebuffers failed ({st}): {_abi.last_error(_lib)}")
        outs = [torch.empty_like(t) for t in tensors]
        st = _lib.sgs_backward_finish(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.c_void_p(bw.data_ptr()),
                                      *(ctypes.c_void_p(t.data_ptr()) for t in outs), ctypes.c_void_p(stream))
        if st != _abi.SGS_OK:
            raise RuntimeError(f"sgs_backward_finish failed ({st}): {_abi.last_error(_lib)}")
        ctx.winners = None
        return (*outs, None, None, None, None)


def render_samples(means, scales, rotations, opacities, sh_coefficients, settings: Settings, n_samples: int = 1,
                   first_frame: int | None = None, store_winners: bool = True):
    """Differentiable average of `n_samples` samples (stochastic transparency or, with
    `settings.use_gps`, Gaussian point splatting): (image, depth, alpha), premultiplied by alpha like
    `History`. Frames first_frame .. first_frame + n_samples - 1 (default:
    the process-wide frame index, which advances by n_samples)."""
    if first_frame is None:
        first_frame = _C.get_frame_index()
    out = _RenderSamples.apply(means, scales, rotations, opacities, sh_coefficients, settings, int(n_samples),
                               int(first_frame), bool(store_winners))
    _C.set_frame_index(first_frame + n_samples)
    return out
