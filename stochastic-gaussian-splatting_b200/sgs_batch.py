"""Many views, one CUDA graph: batched sample-frames through the drop-in `_C.render`.

`CapturedViews` records one `_C.render` call per view (each with its own resolution and history)
into a single CUDA graph. The frame index lives in device memory (`_C.set_device_frame_counter`), so
every replay renders the next sample of every view with new random numbers, exactly the frames that
the same calls made eagerly would render. Nothing in a render call synchronises the host, hybrid
scheduling included, which is what makes the capture possible.
"""
from __future__ import annotations

import torch

from StochasticGSCudaBackend import _C


class CapturedViews:
    """One graph rendering one sample of each view; `replay()` advances every view by one sample.

    views: list of dicts with keys w2c (4x4), position (3), width, height, focal_x, focal_y, center_x,
    center_y, near_plane, far_plane (the camera of `Settings`). `flags`: aa, ss, gps, hybrid.
    The first replay resets each view's history (TemporalMode.RESET is recorded in a warm-up call
    outside the graph), later replays merge progressively (STATIC).
    """

    def __init__(self, scene_tensors, views, flags, first_frame: int = 0, device=None):
        self.device = torch.device(device or "cuda")
        self.scene = tuple(t.to(self.device) for t in scene_tensors)
        self.flags = flags
        self.counter = torch.tensor([first_frame], dtype=torch.int32, device=self.device)
        self.views = []
        for v in views:
            ss = flags["ss"]
            n_fb = v["width"] * v["height"] * ss * ss
            self.views.append(dict(
                v, w2c=torch.as_tensor(v["w2c"], dtype=torch.float32).to(self.device).contiguous(),
                position=torch.as_tensor(v["position"], dtype=torch.float32).to(self.device).contiguous(),
                kb=(torch.empty((0, n_fb, 2), dtype=torch.int32, device=self.device),
                    torch.empty((0, n_fb, 4), device=self.device))))
        self.eye = torch.eye(4, device=self.device)
        self.blue = torch.empty(0, dtype=torch.uint8, device=self.device)
        self.graph = None
        self.histories = None

    def _call(self, v, hist, mode):
        f = self.flags
        return _C.render(*self.scene, v["w2c"], v["position"], v["width"], v["height"], v["focal_x"], v["focal_y"],
                         v["center_x"], v["center_y"], v["near_plane"], v["far_plane"], f["aa"], f["ss"], f["gps"],
                         f["hybrid"], False, self.blue, *v["kb"], *hist, self.eye, mode)

    def _render_all(self, histories, mode):
        return [self._call(v, h, mode) for v, h in zip(self.views, histories)]

    def capture(self):
        """Renders the first sample of every view eagerly (Reset), then captures the Static step."""
        _C.set_device_frame_counter(self.counter)
        try:
            e = torch.empty(0)
            self.histories = self._render_all([(e, e, e, e)] * len(self.views), 0)
            static_in = [tuple(h) for h in self.histories]
            stream = torch.cuda.Stream(self.device)
            stream.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(stream):
                # one uncaptured pass so that every allocation of the step exists before capture
                saved = self.counter.clone()
                self._render_all(static_in, 1)
                self.counter.copy_(saved)
            torch.cuda.current_stream(self.device).wait_stream(stream)
            torch.cuda.synchronize(self.device)
            self.static_in = static_in
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self.static_out = self._render_all(static_in, 1)
                # the next replay merges into this one's outputs
                for dst, src in zip(static_in, self.static_out):
                    for d, s in zip(dst, src):
                        d.copy_(s)
        finally:
            _C.set_device_frame_counter(None, self.device)
        return self

    def replay(self):
        """One more sample of every view; returns the views' histories (image, depth, alpha, weight mass)."""
        self.graph.replay()
        return self.static_out


def batch_views(n_views: int, radius: float, resolutions, fov_y_deg: float = 60.0):
    """Views on an orbit around the origin cycling through `resolutions` [(width, height), ...]."""
    import sgs_scenes

    views = []
    for i in range(n_views):
        w, h = resolutions[i % len(resolutions)]
        cam = sgs_scenes.orbit_cameras(n_views, radius, w, h, fov_y_deg)[i]
        views.append(dict(w2c=cam.w2c, position=cam.position, width=w, height=h, focal_x=cam.focal_x,
                          focal_y=cam.focal_y, center_x=cam.center_x, center_y=cam.center_y,
                          near_plane=cam.near_plane, far_plane=cam.far_plane))
    return views
