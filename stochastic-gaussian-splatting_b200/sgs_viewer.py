"""The caller side of the render path without NeRFICG: frame logic, camera paths, FPS harness, images.

The reference's method plugin drives `render()` from NeRFICG (Renderer.py, Trainer.py), which is not
available here. This module restates what those callers do, on this library:

* `ProgressiveRenderer.render_image(view)` is `StochasticGSRenderer.render_image` (Renderer.py:48-103):
  the settings of the view; a new k-buffer and an empty history (RESET) when any setting other than
  the pose changed or progressive rendering is disabled; STATIC when the pose is unchanged; otherwise
  REPROJECT with temporal reuse, else RESET; SAMPLES_PER_PIXEL samples, the first in that mode and
  the rest STATIC; then the background composite and the depth normalisation. The sample loop runs
  as one `_C.render_samples` call, which renders the same bits as the loop in every mode. With
  `graphs=True` every frame is one CUDA graph launch: the pose, background and frame index are copied
  in from pinned host memory, the samples rendered and the frame composited (`_C.composite`) by the
  replayed graph of the frame's temporal mode, with the same bits as the eager frame.
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
import weakref
import zlib
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch

from StochasticGSCudaBackend import History, Settings, TemporalMode, _C, create_k_buffer, render
from sgs_batch import graph_capture


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
                 spatial_reuse: bool = False, temporal_reuse: bool = False, preactivate: bool = False,
                 graphs: bool = False):
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
        self.graphs = graphs
        self._frames = None  # _FrameGraphs of the current settings (graphs=True)

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
        """n samples merged into the history, the first in `mode`, the rest STATIC (one call)."""
        self.history = History(*_C.render_samples(
            n, *self.model, *settings.as_tuple(), _blue_noise(self.device), *self.k_buffer, *self.history, v2pv,
            int(mode), preactivated=self.preactivated))

    def _frame_mode(self, view: View, settings: Settings, benchmark: bool) -> TemporalMode:
        """The temporal mode of the frame's first sample (Renderer.py:73-84); a new k-buffer and an empty
        history when any setting but the pose changed."""
        reset = self.disable_progressive_rendering and not benchmark
        changed = self.settings is None or not self._same_settings(settings, self.settings)
        if reset or changed:
            self.settings = settings
            if changed or not self.graphs:
                self.k_buffer = create_k_buffer(settings)
                self._frames = None
            else:
                # the captured graphs keep this k-buffer: emptied in place (entries -1, as created)
                self.k_buffer[0].fill_(-1)
            self.history = History(*(torch.empty(0) for _ in range(4)))
            return TemporalMode.RESET
        if (self.history_c2w == view.c2w).all():
            return TemporalMode.STATIC
        return TemporalMode.REPROJECT if self.temporal_reuse else TemporalMode.RESET

    @torch.inference_mode()
    def render_image(self, view: View, to_chw: bool = False, benchmark: bool = False) -> dict[str, torch.Tensor]:
        settings = self._settings(view)
        mode = self._frame_mode(view, settings, benchmark)
        n = max(self.samples_per_pixel, 1)
        if self.graphs:
            if self._frames is None:
                self._frames = _FrameGraphs(self, settings, n)
            image, depth, alpha = self._frames.frame(view, self.history_c2w, mode)
            self.history = self._frames.history()
        else:
            _, _, c2w = view.pose(self.device)
            v2pv = self.history_w2c @ c2w if mode == TemporalMode.REPROJECT else c2w
            self._samples(settings, v2pv, mode, n)
        self.history_c2w = view.c2w.copy()
        self.history_w2c = view.pose(self.device)[0]
        if self.graphs:
            if benchmark:
                return {"rgb": image}
            if to_chw:
                image, depth, alpha = image.permute(2, 0, 1), depth.permute(2, 0, 1), alpha.permute(2, 0, 1)
            return {"rgb": image, "depth": depth, "alpha": alpha}

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


class _FrameGraphs:
    """One CUDA graph per (temporal mode of the first sample, parity) for the frames of fixed settings.

    A replayed graph copies the frame's parameters (w2c, camera position, the previous view's w2c, the
    camera-to-world matrix, background, frame index) from a pinned host staging buffer into device
    buffers, forms view-to-previous-view as the eager frame does (a float32 product on the GPU),
    renders the frame's samples with `_C.render_samples_into` (frame index read from device memory)
    from history buffer `parity` into history buffer 1 - parity, and composites the result into fixed
    output buffers (`_C.composite`). Staging buffers alternate with the parity; a frame waits for the
    replay two frames back (the same staging buffer) before writing its parameters. The output tensors
    are overwritten by the next frame.
    """

    # w2c 16, position 3 (+1), previous w2c 16, c2w 16, background 3 (+1)
    _W2C, _POS, _PREV, _C2W, _BG, _PARAMS = 0, 16, 20, 36, 52, 56

    def __init__(self, renderer: "ProgressiveRenderer", settings: Settings, n_samples: int):
        dev = renderer.device
        # a weak reference: the renderer owns these graphs, and without a cycle between the two they
        # are released as soon as the renderer is, never later by the cyclic garbage collector (which
        # may run while another renderer is capturing a graph)
        self.r = weakref.proxy(renderer)
        self.n = n_samples
        self.settings = settings
        h, w = settings.height, settings.width
        opts = dict(dtype=torch.float32, device=dev)
        self.params = torch.zeros(self._PARAMS, **opts)
        self.v2pv = torch.zeros((4, 4), **opts)
        self.counter = torch.zeros(1, dtype=torch.int32, device=dev)
        self.staging = [torch.zeros(self._PARAMS, dtype=torch.float32).pin_memory() for _ in range(2)]
        self.staging_frame = [torch.zeros(1, dtype=torch.int32).pin_memory() for _ in range(2)]
        self.done = [torch.cuda.Event() for _ in range(2)]
        self.used = [False, False]
        self.hist = [tuple(torch.zeros(shape, **opts) for shape in ((h, w, 3), (h, w, 1), (h, w, 1), (h, w, 1)))
                     for _ in range(2)]
        self.out = (torch.empty((h, w, 3), **opts), torch.empty((h, w, 1), **opts), torch.empty((h, w, 1), **opts))
        self.parity = 0
        self.graphs = {}
        self.workspace = None

    def _param(self, at: int, n: int) -> torch.Tensor:
        return self.params[at:at + n]

    def _args(self, mode: TemporalMode, history, k_buffer):
        s = self.settings
        w2c = self._param(self._W2C, 16).view(4, 4)
        pos = self._param(self._POS, 3)
        e = torch.empty(0)
        hist = history if mode != TemporalMode.RESET else (e, e, e, e)
        v2pv = self.v2pv if mode == TemporalMode.REPROJECT else self._param(self._C2W, 16).view(4, 4)
        return (*self.r.model, w2c, pos, *s.as_tuple()[2:], _blue_noise(self.r.device), *k_buffer, *hist, v2pv,
                int(mode))

    def _body(self, mode: TemporalMode, parity: int, k_buffer):
        src, dst = self.hist[parity], self.hist[1 - parity]
        if mode == TemporalMode.REPROJECT:
            torch.matmul(self._param(self._PREV, 16).view(4, 4), self._param(self._C2W, 16).view(4, 4), out=self.v2pv)
        _C.render_samples_into(dst, self.workspace, self.n, *self._args(mode, src, k_buffer),
                               preactivated=self.r.preactivated)
        _C.composite(dst[0], dst[1], dst[2], self._param(self._BG, 3), out=self.out)

    def _capture(self, mode: TemporalMode, parity: int):
        k_buffer = self.r.k_buffer
        if self.workspace is None:
            size = _C.samples_workspace_size(self.n, *self._args(mode, self.hist[parity], k_buffer))
            raw = torch.empty(size + 256, dtype=torch.uint8, device=self.r.device)
            off = (-raw.data_ptr()) % 256
            self.workspace = raw[off:off + size]
        _C.set_device_frame_counter(self.counter)
        try:
            # one uncaptured run of the same launches first (its scratch k-buffer keeps the real one intact;
            # the staging copy at every replay restores the parameters and the frame index)
            self.params.copy_(self.staging[parity])
            scratch = tuple(t.clone() for t in k_buffer)
            self._body(mode, parity, scratch)
            torch.cuda.synchronize(self.r.device)
            graph = torch.cuda.CUDAGraph()
            with graph_capture(graph):
                self.params.copy_(self.staging[parity], non_blocking=True)
                self.counter.copy_(self.staging_frame[parity], non_blocking=True)
                self._body(mode, parity, k_buffer)
        finally:
            _C.set_device_frame_counter(None, self.r.device)
        return graph

    def frame(self, view: View, previous_c2w, mode: TemporalMode):
        p = self.parity
        if self.used[p]:
            self.done[p].synchronize()
        st = self.staging[p].numpy()
        st[self._W2C:self._W2C + 16] = view.w2c_numpy.astype(np.float32).reshape(-1)
        st[self._POS:self._POS + 3] = view.c2w[:3, 3].astype(np.float32)
        if previous_c2w is not None:
            st[self._PREV:self._PREV + 16] = np.linalg.inv(previous_c2w).astype(np.float32).reshape(-1)
        st[self._C2W:self._C2W + 16] = view.c2w.astype(np.float32).reshape(-1)
        st[self._BG:self._BG + 3] = np.asarray(view.background_color, dtype=np.float32)
        frame = _C.get_frame_index()
        self.staging_frame[p].numpy()[0] = np.uint32(frame).view(np.int32)
        key = (int(mode), p)
        if key not in self.graphs:
            self.graphs[key] = self._capture(mode, p)
        self.graphs[key].replay()
        self.done[p].record()
        self.used[p] = True
        _C.set_frame_index(frame + self.n)
        self.parity = 1 - p
        return self.out

    def history(self) -> History:
        """The history the last frame wrote (the next frame's input)."""
        return History(*self.hist[self.parity])


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
