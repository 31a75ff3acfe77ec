"""Many views, one CUDA graph: batched sample-frames through the render path.

`CapturedViews` records one render per view (each with its own resolution and history) into a CUDA
graph. The frame index lives in device memory (`_C.set_device_frame_counter`), so every replay
renders the next sample of every view with new random numbers, exactly the frames that the same
`_C.render` calls made eagerly would render. Nothing in a render call synchronises the host, hybrid
scheduling included, which is what makes the capture possible.

Each render is split over two streams (`_C.render_into` with sgs_render_split): the clear and
accumulate passes of view j + 1 run on one stream while view j samples and resolves on the other,
so the memory-bound resolve overlaps the issue-bound accumulation. Histories are ping-ponged between
two caller-owned buffers per view (one graph renders A -> B, a second B -> A; replays alternate), so
no copy merges a replay's outputs into the next replay's inputs.
"""
from __future__ import annotations

import contextlib
import gc

import torch

from StochasticGSCudaBackend import _C


@contextlib.contextmanager
def graph_capture(graph: torch.cuda.CUDAGraph, **kwargs):
    """`torch.cuda.graph(graph)` with Python's cyclic garbage collector kept out of the capture.

    Garbage left to the collector (a dropped renderer's graphs, pinned buffers, events) is finalised
    before the capture begins; during it the collector is off, so no finaliser releases CUDA
    resources inside the capture, which would invalidate it or abort the process."""
    gc.collect()
    enabled = gc.isenabled()
    gc.disable()
    try:
        with torch.cuda.graph(graph, **kwargs):
            yield
    finally:
        if enabled:
            gc.enable()


class CapturedViews:
    """Graphs rendering one sample of each view; `replay()` advances every view by one sample.

    views: list of dicts with keys w2c (4x4), position (3), width, height, focal_x, focal_y, center_x,
    center_y, near_plane, far_plane (the camera of `Settings`). `flags`: aa, ss, gps, hybrid.
    The first sample of each view is rendered eagerly in TemporalMode.RESET by `capture()`; replays
    merge progressively (STATIC).
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
        self.graphs = None
        self.parity = 0

    def _args(self, v, hist, mode):
        f = self.flags
        return (*self.scene, v["w2c"], v["position"], v["width"], v["height"], v["focal_x"], v["focal_y"],
                v["center_x"], v["center_y"], v["near_plane"], v["far_plane"], f["aa"], f["ss"], f["gps"],
                f["hybrid"], False, self.blue, *v["kb"], *hist, self.eye, mode)

    def _alloc(self):
        e = torch.empty(0)
        bufs, wss = [], []
        for v in self.views:
            h, w = v["height"], v["width"]
            bufs.append(tuple(torch.empty((h, w, ch), dtype=torch.float32, device=self.device) for ch in (3, 1, 1, 1)))
            n = _C.workspace_size(*self._args(v, (e, e, e, e), 0))
            wss.append(torch.empty((n,), dtype=torch.uint8, device=self.device))
        return bufs, wss

    def _render_all_into(self, src, dst, mode, wss, streams):
        for v, h, o, ws in zip(self.views, src, dst, wss):
            _C.render_into(o, ws, streams, *self._args(v, h, mode))

    def _step_on_streams(self, src, dst):
        cur = torch.cuda.current_stream(self.device)
        self.acc.wait_stream(cur)
        self.res.wait_stream(cur)
        self._render_all_into(self.buf[src], self.buf[dst], 1, self.ws[dst], (self.acc, self.res))
        cur.wait_stream(self.acc)
        cur.wait_stream(self.res)

    def capture(self):
        """Renders the first sample of every view eagerly (Reset), then captures the Static steps."""
        _C.set_device_frame_counter(self.counter)
        try:
            e = torch.empty(0)
            b0, w0 = self._alloc()
            b1, w1 = self._alloc()
            self.buf, self.ws = (b0, b1), (w0, w1)
            self._render_all_into([(e, e, e, e)] * len(self.views), self.buf[0], 0, self.ws[0], None)
            self.acc = torch.cuda.Stream(self.device)
            self.res = torch.cuda.Stream(self.device)
            # one uncaptured step: the library creates its stream-split event outside the capture
            saved = self.counter.clone()
            self._step_on_streams(0, 1)
            self.counter.copy_(saved)
            torch.cuda.synchronize(self.device)
            self.graphs = []
            for src, dst in ((0, 1), (1, 0)):
                graph = torch.cuda.CUDAGraph()
                with graph_capture(graph):
                    self._step_on_streams(src, dst)
                self.graphs.append(graph)
            self.parity = 0
        finally:
            _C.set_device_frame_counter(None, self.device)
        return self

    def replay(self):
        """One more sample of every view; returns the views' histories (image, depth, alpha, weight mass),
        valid until the replay after next."""
        self.graphs[self.parity].replay()
        out = self.buf[1 - self.parity]
        self.parity ^= 1
        return out

    def eager_step(self):
        """The same step without the graphs (one sample of every view, split streams)."""
        _C.set_device_frame_counter(self.counter)
        try:
            self._step_on_streams(self.parity, 1 - self.parity)
        finally:
            _C.set_device_frame_counter(None, self.device)
        out = self.buf[1 - self.parity]
        self.parity ^= 1
        return out


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
