"""Python API of the render path, identical to the reference's StochasticGSCudaBackend/render.py.

`Settings`, `TemporalMode`, `History`, `blue_noise()`, `create_k_buffer()` and `render()` keep the
reference's names, fields, order and semantics (render.py:8-96), so callers such as the NeRFICG
renderer (Renderer.py:41-103) use this package unchanged.
"""
from enum import IntEnum
from functools import cache
from pathlib import Path
from typing import NamedTuple

import torch

from StochasticGSCudaBackend import _C  # noqa


class Settings(NamedTuple):
    w2c: torch.Tensor  # world-to-camera matrix, rows of 4 floats (OpenCV axes: x right, y down, z forward)
    cam_position: torch.Tensor  # (3,) eye point in world coordinates, the origin of the SH view direction
    width: int  # output image columns
    height: int  # output image rows
    focal_x: float  # horizontal focal length, in pixels
    focal_y: float  # vertical focal length, in pixels
    center_x: float  # principal point column, in pixels from the left edge
    center_y: float  # principal point row, in pixels from the top edge
    near_plane: float  # Gaussians closer than this view depth are culled
    far_plane: float  # Gaussians beyond this view depth are culled; background depth for reprojection
    proper_antialiasing: bool  # smaller screen-space dilation with opacity compensation
    supersampling_factor: int  # s: each output pixel averages s x s framebuffer subpixels
    use_gps: bool  # splat Poisson-distributed points instead of stochastic transparency
    hybrid_scheduling: bool  # hand large footprints to a load-balanced work queue
    spatial_reuse: bool  # also resample each subpixel's four neighbours through the k-buffer

    def as_tuple(self) -> tuple:
        return (
            self.w2c,
            self.cam_position,
            self.width,
            self.height,
            self.focal_x,
            self.focal_y,
            self.center_x,
            self.center_y,
            self.near_plane,
            self.far_plane,
            self.proper_antialiasing,
            self.supersampling_factor,
            self.use_gps,
            self.hybrid_scheduling,
            self.spatial_reuse,
        )


class TemporalMode(IntEnum):
    RESET = 0  # start over: the history is not read
    STATIC = 1  # unchanged camera: running average weighted by weight_mass
    REPROJECT = 2  # camera moved: history warped by view_to_previous_view, rejected where it disagrees


class History(NamedTuple):
    image: torch.Tensor  # (H, W, 3) premultiplied RGB (multiplied by alpha)
    depth: torch.Tensor  # (H, W, 1) premultiplied view depth
    alpha: torch.Tensor  # (H, W, 1) coverage
    weight_mass: torch.Tensor  # (H, W, 1) total sample weight merged into this pixel so far


BLUE_NOISE_FILE = "stbn_scalar_128x128x64.bin"


@cache
def blue_noise() -> torch.Tensor:
    """The (64, 128, 128) uint8 spatio-temporal blue-noise volume if its file sits next to `_C`; otherwise an
    empty tensor, which selects hashed white-noise thresholds."""
    path = Path(_C.__file__).parent / BLUE_NOISE_FILE
    if not path.is_file():
        return torch.empty(0, dtype=torch.uint8, device='cuda')
    return torch.frombuffer(bytearray(path.read_bytes()), dtype=torch.uint8).view(64, 128, 128).cuda()


def create_k_buffer(settings: Settings) -> tuple[torch.Tensor, torch.Tensor]:
    """Fresh k-buffer state for `settings`: (K, P_fb, 2) int32 entries of (Gaussian index, depth bits), all -1,
    and (K, P_fb, 4) float32 occlusion ratios towards the four neighbours; K = 0 without spatial reuse."""
    n_entries = (_C.k_buffer_size if settings.spatial_reuse else 0,
                 settings.width * settings.height * settings.supersampling_factor ** 2)
    return (
        torch.full((*n_entries, 2), -1, dtype=torch.int32, device='cuda'),
        torch.empty((*n_entries, 4), dtype=torch.float32, device='cuda'),
    )


def render(
    means: torch.Tensor,
    scales: torch.Tensor,
    rotations: torch.Tensor,
    opacities: torch.Tensor,
    sh_coefficients: torch.Tensor,
    settings: Settings,
    k_buffer: tuple[torch.Tensor, torch.Tensor],
    history: History,
    view_to_previous_view: torch.Tensor,
    temporal_mode: TemporalMode,
    *,
    preactivated: torch.Tensor | None = None,
    max_fragments: int = 0,
    max_binned: int = 0,
    quantized=None,
) -> History:
    """One sample-frame (render.py:72-96 of the reference). Keyword-only additions: `preactivated`, the
    `_C.preactivate(scales, rotations, opacities)` tensor of these Gaussians, read by the accumulate
    pass in place of the per-sample covariance and sigmoid (same bits); `max_fragments` and
    `max_binned`, the GPS point cap and the hybrid queue capacity (0 keeps the reference's values);
    `quantized`, the `_C.quantize(...)` layout of these Gaussians (16 bytes each, half SH), read in place
    of the float32 arrays (the images differ by the quantisation)."""
    return History(*_C.render(
        means,
        scales,
        rotations,
        opacities,
        sh_coefficients,
        *settings.as_tuple(),
        blue_noise(),
        *k_buffer,
        *history,
        view_to_previous_view,
        int(temporal_mode),
        preactivated=preactivated,
        max_fragments=max_fragments,
        max_binned=max_binned,
        quantized=quantized,
    ))
