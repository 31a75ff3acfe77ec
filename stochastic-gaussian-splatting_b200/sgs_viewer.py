"""The caller side of the render path without NeRFICG: frame logic, camera paths, FPS harness, images.

The reference's method plugin drives `render()` from NeRFICG (Renderer.py, Trainer.py), which is not
available here. This module restates what those callers do, on this library:

* `ProgressiveRenderer.render_image(view)` is `StochasticGSRenderer.render_image` (Renderer.py:48-103):
  the settings of the view; a new k-buffer and an empty history (RESET) when any setting other than
  the pose changed or progressive rendering is disabled; STATIC when the pose is unchanged; otherwise
  REPROJECT with temporal reuse, else RESET; SAMPLES_PER_PIXEL samples, the first in that mode and
  the rest STATIC; then the background composite and the depth normalisation. The sample loop runs
  as one `_C.render_samples` call where that path applies (no spatial reuse, first mode RESET or
  STATIC, GPS only with scatter scheduling), which renders the same bits as the loop.
* `load_camera_path(path)` reads the camera-path .json of Trainer.py:28-65 (per frame: `rotation`
  3x3 and `position` of camera-to-world, `fx`, `fy`, `width`, `height`, `id`).
* `benchmark_camera_path(renderer, views)` is the FPS measurement of Trainer.py:79-120: one warm-up
  pass over the views, then passes with a device synchronisation around every frame, average FPS
  and per-frame milliseconds.
* `write_png(path, image)` stores an (H, W, 3) image in [0, 1] as an 8-bit PNG (the headless
  replacement of the GUI and of Datasets.utils.save_image).

Cameras follow the renderer's convention (x right, y down, z forward; StochasticGSCudaBackend
render.py:15-16): `c2w` is camera-to-world and `w2c` its inverse.
"""
from __future__ import annotations

import json
import struct
import time
import zlib
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch

from StochasticGSCudaBackend import History, Settings, TemporalMode, _C, create_k_buffer, render


@dataclass
class View:
    """One frame's camera: pose (camera-to-world, float64), pinhole intrinsics and background."""

    c2w: np.ndarray
    width: int
    height: int
    focal_x: float
    focal_y: float
    center_x: float
    center_y: float
    near_plane: float = 0.2
    far_plane: float = 10000.0
    background_color: tuple = (0.0, 0.0, 0.0)
    frame_idx: int = 0
    _device_pose: dict = field(default_factory=dict, repr=False)

    @property
    def w2c_numpy(self) -> np.ndarray:
        return np.linalg.inv(self.c2w)

    def pose(self, device) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        """(w2c, position, c2w) as float32 tensors on `device` (cached per device)."""
        key = str(device)
        if key not in self._device_pose:
            w2c = torch.as_tensor(self.w2c_numpy, dtype=torch.float32).to(device).contiguous()
            pos = torch.as_tensor(self.c2w[:3, 3], dtype=torch.float32).to(device).contiguous()
            c2w = torch.as_tensor(self.c2w, dtype=torch.float32).to(device).contiguous()
            self._device_pose[key] = (w2c, pos, c2w)
        return self._device_pose[key]

    @staticmethod
    def from_camera(cam, background_color=(0.0, 0.0, 0.0), frame_idx: int = 0) -> "View":
        """A View of an `sgs_scenes.Camera`."""
        c2w = np.linalg.inv(cam.w2c.double().numpy())
        return View(c2w, cam.width, cam.height, cam.focal_x, cam.focal_y, cam.center_x, cam.center_y,
                    cam.near_plane, cam.far_plane, background_color, frame_idx)


class ProgressiveRenderer:
    """Renders views of one Gaussian model with the frame logic of Renderer.py:48-103."""

    def __init__(self, means, scales, rotations, opacities, sh_coefficients, *, proper_antialiasing: bool = False,
                 use_gps: bool = False, hybrid_scheduling: bool = False, supersampling_factor: int = 1,
                 samples_per_pixel: int = 1, disable_progressive_rendering: bool = False,
                 spatial_reuse: bool = False, temporal_reuse: bool = False, preactivate: bool = False):
        self.model = (means, scales, rotations, opacities, sh_coefficients)
        # covariance and opacity sigmoid once per model (README.md:139-142); the images are the same bits
        self.preactivated = _C.preactivate(scales, rotations, opacities) if preactivate else None
        self.device = means.device
        self.proper_antialiasing = proper_antialiasing
        self.use_gps = use_gps
        self.hybrid_scheduling = hybrid_scheduling
        self.supersampling_factor = supersampling_factor
        self.samples_per_pixel = samples_per_pixel
        self.disable_progressive_rendering = disable_progressive_rendering
        self.spatial_reuse = spatial_reuse
        self.temporal_reuse = temporal_reuse
        self.settings = None
        self.k_buffer = None
        self.history = None
        self.history_c2w = None
        self.history_w2c = None

    def _settings(self, view: View) -> Settings:
        w2c, pos, _ = view.pose(self.device)
        return Settings(w2c, pos, view.width, view.height, view.focal_x, view.focal_y, view.center_x, view.center_y,
                        view.near_plane, view.far_plane, self.proper_antialiasing, self.supersampling_factor,
                        self.use_gps, self.hybrid_scheduling, self.spatial_reuse)

    @staticmethod
    def _same_settings(a: Settings, b: Settings) -> bool:
        """Every setting but the pose (Renderer.py:75 compares as_tuple()[2:])."""
        return a.as_tuple()[2:] == b.as_tuple()[2:]

    def _samples(self, settings: Settings, v2pv: torch.Tensor, mode: TemporalMode, n: int) -> None:
        """n samples merged into the history, the first in `mode`, the rest STATIC."""
        one_call = (not (settings.use_gps and settings.hybrid_scheduling) and not settings.spatial_reuse
                    and mode in (TemporalMode.RESET, TemporalMode.STATIC) and n > 1)
        if one_call:
            self.history = History(*_C.render_samples(
                n, *self.model, *settings.as_tuple(), _blue_noise(self.device), *self.k_buffer, *self.history, v2pv,
                int(mode), preactivated=self.preactivated))
            return
        for _ in range(n):
            self.history = render(*self.model, settings, self.k_buffer, self.history, v2pv, mode,
                                  preactivated=self.preactivated)
            mode = TemporalMode.STATIC

    @torch.inference_mode()
    def render_image(self, view: View, to_chw: bool = False, benchmark: bool = False) -> dict[str, torch.Tensor]:
        settings = self._settings(view)
        reset = self.disable_progressive_rendering and not benchmark
        if reset or self.settings is None or not self._same_settings(settings, self.settings):
            self.settings = settings
            self.k_buffer = create_k_buffer(settings)
            self.history = History(*(torch.empty(0) for _ in range(4)))
            mode = TemporalMode.RESET
        elif (self.history_c2w == view.c2w).all():
            mode = TemporalMode.STATIC
        else:
            mode = TemporalMode.REPROJECT if self.temporal_reuse else TemporalMode.RESET
        _, _, c2w = view.pose(self.device)
        v2pv = self.history_w2c @ c2w if mode == TemporalMode.REPROJECT else c2w
        n = max(self.samples_per_pixel, 1)
        if mode == TemporalMode.REPROJECT:
            self._samples(settings, v2pv, mode, 1)
            n -= 1
            mode = TemporalMode.STATIC
        if n > 0:
            self._samples(settings, v2pv, mode, n)
        self.history_c2w = view.c2w.copy()
        self.history_w2c = view.pose(self.device)[0]

        # the history is premultiplied by alpha and must not be modified in place
        image, depth, alpha, _ = self.history
        alpha = alpha.clamp(0.0, 1.0)
        bg = torch.as_tensor(view.background_color, dtype=torch.float32, device=image.device)
        image = (image + (1.0 - alpha) * bg).clamp(0.0, 1.0)
        if benchmark:
            return {"rgb": image}
        depth = depth / alpha.clamp_min(1.0e-8)
        if to_chw:
            image, depth, alpha = image.permute(2, 0, 1), depth.permute(2, 0, 1), alpha.permute(2, 0, 1)
        return {"rgb": image, "depth": depth, "alpha": alpha}


def _blue_noise(device) -> torch.Tensor:
    """The blue-noise volume `render()` passes (StochasticGSCudaBackend.render.blue_noise)."""
    from StochasticGSCudaBackend.render import blue_noise

    return blue_noise().to(device)


def load_camera_path(path, camera: View | None = None, width: int = 1920, height: int = 1080,
                     near_plane: float = 0.2, far_plane: float = 10000.0,
                     background_color=(0.0, 0.0, 0.0)) -> list[View]:
    """Views of a camera-path .json (Trainer.py:38-63). With `camera`, every frame uses its intrinsics
    (the dataset camera); otherwise a width x height pinhole with the frame's focal lengths scaled from
    its own width and height, principal point at the image centre."""
    with open(path, "r") as f:
        frames = json.load(f)
    views = []
    for frame in frames:
        c2w = np.eye(4, dtype=np.float64)
        c2w[:3, :3] = np.asarray(frame["rotation"], dtype=np.float64)
        c2w[:3, 3] = np.asarray(frame["position"], dtype=np.float64)
        if camera is not None:
            views.append(View(c2w, camera.width, camera.height, camera.focal_x, camera.focal_y, camera.center_x,
                              camera.center_y, camera.near_plane, camera.far_plane, camera.background_color,
                              int(frame["id"])))
        else:
            views.append(View(c2w, width, height, float(frame["fx"]) * (width / float(frame["width"])),
                              float(frame["fy"]) * (height / float(frame["height"])), width / 2.0, height / 2.0,
                              near_plane, far_plane, background_color, int(frame["id"])))
    return views


def save_camera_path(path, views: list[View]) -> None:
    """Writes views in the camera-path .json format (the inverse of `load_camera_path`)."""
    frames = [{"rotation": v.c2w[:3, :3].tolist(), "position": v.c2w[:3, 3].tolist(), "fx": v.focal_x,
               "fy": v.focal_y, "width": v.width, "height": v.height, "id": v.frame_idx} for v in views]
    with open(path, "w") as f:
        json.dump(frames, f)


def benchmark_camera_path(renderer: ProgressiveRenderer, views: list[View], iterations: int = 10,
                          per_frame_timings: bool = True) -> dict:
    """Average FPS over `iterations` passes of the views after one warm-up pass (Trainer.py:79-120)."""
    for view in views:
        renderer.render_image(view, benchmark=True)
    torch.cuda.synchronize()
    per_frame = np.zeros(len(views), dtype=np.float64)
    start = time.perf_counter()
    for _ in range(iterations):
        for i, view in enumerate(views):
            if per_frame_timings:
                torch.cuda.synchronize()
                t = time.perf_counter()
                renderer.render_image(view, benchmark=True)
                torch.cuda.synchronize()
                per_frame[i] += (time.perf_counter() - t) * 1000.0
            else:
                renderer.render_image(view, benchmark=True)
    torch.cuda.synchronize()
    total = time.perf_counter() - start
    n = len(views) * iterations
    out = {"frames": len(views), "iterations": iterations, "avg_fps": n / total, "avg_ms": total * 1000.0 / n}
    if per_frame_timings:
        out["per_frame_ms"] = (per_frame / iterations).tolist()
    return out


def write_png(path, image) -> None:
    """Stores an (H, W, 3) (or CHW) image in [0, 1] (tensor or array) as an 8-bit RGB PNG."""
    a = image.detach().float().cpu().numpy() if isinstance(image, torch.Tensor) else np.asarray(image, np.float32)
    if a.ndim == 3 and a.shape[0] == 3 and a.shape[2] != 3:
        a = np.transpose(a, (1, 2, 0))
    if a.ndim != 3 or a.shape[2] != 3:
        raise ValueError(f"expected an (H, W, 3) image, got shape {a.shape}")
    px = (np.clip(a, 0.0, 1.0) * 255.0 + 0.5).astype(np.uint8)
    h, w = px.shape[:2]
    raw = b"".join(b"\x00" + px[y].tobytes() for y in range(h))

    def chunk(tag: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    png = (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)) +
           chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))
    Path(path).write_bytes(png)


def read_png(path) -> np.ndarray:
    """Reads an 8-bit RGB PNG written by `write_png` (no filtering) as an (H, W, 3) uint8 array."""
    data = Path(path).read_bytes()
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG file")
    pos, w, h, idat = 8, 0, 0, b""
    while pos < len(data):
        (length,) = struct.unpack(">I", data[pos:pos + 4])
        tag = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + length]
        if tag == b"IHDR":
            w, h, depth, color = struct.unpack(">IIBB", body[:10])
            if depth != 8 or color != 2:
                raise ValueError("only 8-bit RGB PNGs are supported")
        elif tag == b"IDAT":
            idat += body
        pos += 12 + length
    raw = zlib.decompress(idat)
    rows = np.frombuffer(raw, dtype=np.uint8).reshape(h, 1 + 3 * w)
    if (rows[:, 0] != 0).any():
        raise ValueError("filtered scanlines are not supported")
    return rows[:, 1:].reshape(h, w, 3).copy()
