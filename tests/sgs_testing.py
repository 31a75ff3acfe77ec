"""Helpers shared by the GPU parity tests: one call of the B200 render path with its intermediates."""
from __future__ import annotations

import numpy as np
import torch


def render_once(scene: dict, cam: dict, flags: dict, frame_idx: int, *, blue_noise=None, temporal_mode: int = 0,
                history=None, k_buffer=None, v2pv=None, spatial_reuse: bool = False, device="cuda",
                preactivate: bool = False) -> dict:
    """Renders one sample-frame through `_C.render_with_workspace` with the frame index pinned.

    `scene` holds numpy or torch arrays (means, scales, rotations, opacities, sh_coefficients), `cam` the
    camera dict of the golden manifest, `flags` aa/ss/gps/hybrid. Returns numpy copies of the winner
    framebuffer, the samples (and reuse weights), the four outputs and the torch outputs for chaining.
    `preactivate` renders with the preactivated layout of the same Gaussians.
    """
    from StochasticGSCudaBackend import _C

    dev = torch.device(device)

    def t(x):
        return x.to(dev) if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(x)).to(dev)

    tensors = [t(scene[k]) for k in ("means", "scales", "rotations", "opacities", "sh_coefficients")]
    w2c = t(np.asarray(cam["w2c"], dtype=np.float32))
    pos = t(np.asarray(cam["position"], dtype=np.float32))
    ss = flags["ss"]
    n_fb = cam["width"] * cam["height"] * ss * ss
    if k_buffer is None:
        k = _C.k_buffer_size if spatial_reuse else 0
        k_buffer = (torch.full((k, n_fb, 2), -1, dtype=torch.int32, device=dev),
                    torch.full((k, n_fb, 4), 0.5, dtype=torch.float32, device=dev))
    if history is None:
        history = tuple(torch.empty(0) for _ in range(4))
    if v2pv is None:
        v2pv = torch.eye(4, device=dev)
    bn = t(blue_noise) if blue_noise is not None else torch.empty(0, dtype=torch.uint8, device=dev)
    _C.set_frame_index(frame_idx)
    outs, ws, layout = _C.render_with_workspace(
        *tensors, w2c, pos, cam["width"], cam["height"], cam["focal_x"], cam["focal_y"], cam["center_x"],
        cam["center_y"], cam["near_plane"], cam["far_plane"], flags["aa"], ss, flags["gps"], flags["hybrid"],
        spatial_reuse, bn, k_buffer[0], k_buffer[1], *history, t(v2pv), temporal_mode,
        preactivated=_C.preactivate(tensors[1], tensors[2], tensors[3]) if preactivate else None)
    views = _C.workspace_views(ws, layout, n_fb, spatial_reuse)
    torch.cuda.synchronize()
    res = {
        "fb": views["framebuffer"].cpu().numpy(),
        "samples": views["samples"].cpu().numpy(),
        "image": outs[0].cpu().numpy(),
        "depth": outs[1].cpu().numpy(),
        "alpha": outs[2].cpu().numpy(),
        "weight_mass": outs[3].cpu().numpy(),
        "outputs": outs,
        "k_buffer": k_buffer,
    }
    if spatial_reuse:
        res["reuse"] = views["reuse_weights"].cpu().numpy()
    return res


def mismatch_report(name: str, got: np.ndarray, want: np.ndarray) -> str:
    got = np.asarray(got)
    want = np.asarray(want)
    if got.shape != want.shape:
        return f"{name}: shape {got.shape} != {want.shape}"
    if got.dtype.kind == "f":
        bad = ~((got == want) | (np.isnan(got) & np.isnan(want)))
    else:
        bad = got != want
    n = int(bad.sum())
    if n == 0:
        return ""
    idx = np.argwhere(bad)[:5].tolist()
    return f"{name}: {n} of {bad.size} differ, first at {idx}"


def assert_bitwise(name: str, got, want):
    msg = mismatch_report(name, got, want)
    assert msg == "", msg


# The reference binding seeds every render with a process-global counter (render.cu:56-57) that
# starts at 0 in each loaded copy of the extension and advances by one per call. Tests that call a
# reference module's `render` go through this helper so that they all know the frame it used.
_reference_calls: dict[str, int] = {}


def reference_render(module, *args):
    """Calls `module.render(*args)` (a reference extension); returns (frame index it used, outputs)."""
    frame = _reference_calls.get(module.__name__, 0)
    out = module.render(*args)
    _reference_calls[module.__name__] = frame + 1
    return frame, out
