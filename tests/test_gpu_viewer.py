"""The progressive renderer (sgs_viewer) against the frame logic of Renderer.py:48-103 written as a
loop of single-sample `render()` calls (GPU): same images, depths and alphas bit for bit, through
RESET, STATIC, REPROJECT and setting changes (also with the preactivated layout on the renderer side
only); the camera-path benchmark and the PNG output run."""
import numpy as np
import pytest
import torch

import sgs_scenes
from StochasticGSCudaBackend import History, Settings, TemporalMode, _C, create_k_buffer, render

pytestmark = pytest.mark.gpu


class LoopRenderer:
    """Renderer.py:48-103 with one render() call per sample."""

    def __init__(self, model, spp, **flags):
        self.model, self.spp, self.f = model, spp, flags
        self.settings = self.k_buffer = self.history = self.history_c2w = self.history_w2c = None

    def render_image(self, view):
        w2c, pos, c2w = view.pose("cuda")
        f = self.f
        settings = Settings(w2c, pos, view.width, view.height, view.focal_x, view.focal_y, view.center_x,
                            view.center_y, view.near_plane, view.far_plane, f.get("proper_antialiasing", False),
                            f.get("supersampling_factor", 1), f.get("use_gps", False),
                            f.get("hybrid_scheduling", False), f.get("spatial_reuse", False))
        if self.settings is None or settings.as_tuple()[2:] != self.settings.as_tuple()[2:]:
            self.settings = settings
            self.k_buffer = create_k_buffer(settings)
            self.history = History(*(torch.empty(0) for _ in range(4)))
            mode = TemporalMode.RESET
        elif (self.history_c2w == view.c2w).all():
            mode = TemporalMode.STATIC
        else:
            mode = TemporalMode.REPROJECT if f.get("temporal_reuse", False) else TemporalMode.RESET
        v2pv = self.history_w2c @ c2w if mode == TemporalMode.REPROJECT else c2w
        for _ in range(max(self.spp, 1)):
            self.history = render(*self.model, settings, self.k_buffer, self.history, v2pv, mode)
            mode = TemporalMode.STATIC
        self.history_c2w = view.c2w.copy()
        self.history_w2c = w2c
        image, depth, alpha, _ = self.history
        alpha = alpha.clamp(0.0, 1.0)
        bg = torch.as_tensor(view.background_color, dtype=torch.float32, device=image.device)
        image = (image + (1.0 - alpha) * bg).clamp(0.0, 1.0)
        return {"rgb": image, "depth": depth / alpha.clamp_min(1.0e-8), "alpha": alpha}


def _views(sgs_viewer):
    cams = sgs_scenes.orbit_cameras(8, 4.0, 160, 120, step_deg=3.0)
    v = [sgs_viewer.View.from_camera(c, background_color=(0.2, 0.3, 0.4)) for c in cams]
    wide = sgs_scenes.orbit_cameras(8, 4.0, 200, 120, step_deg=3.0)
    # static, static, moving, moving, static, new resolution, moving
    return [v[0], v[0], v[1], v[2], v[2], sgs_viewer.View.from_camera(wide[2]), sgs_viewer.View.from_camera(wide[3])]


@pytest.mark.parametrize("flags", [dict(), dict(temporal_reuse=True), dict(temporal_reuse=True, spatial_reuse=True),
                                   dict(supersampling_factor=2, hybrid_scheduling=True),
                                   dict(use_gps=True, temporal_reuse=True), dict(preactivate=True),
                                   dict(use_gps=True, temporal_reuse=True, spatial_reuse=True, preactivate=True),
                                   dict(use_gps=True, hybrid_scheduling=True, supersampling_factor=2,
                                        temporal_reuse=True, spatial_reuse=True)])
@pytest.mark.parametrize("spp", [1, 4])
@pytest.mark.parametrize("graphs", [False, True])
def test_progressive_renderer_equals_the_sample_loop(flags, spp, graphs, cuda_device):
    """Eager frames (one render_samples call each) and replayed CUDA graphs (one launch per frame)."""
    import sgs_viewer

    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=20_000, log_scale_mean=-3.5), seed=9)
    model = tuple(t.cuda() for t in scene.tensors())
    ours = sgs_viewer.ProgressiveRenderer(*model, samples_per_pixel=spp, graphs=graphs, **flags)
    ref = LoopRenderer(model, spp, **flags)
    _C.set_frame_index(1000)
    # graph frames are written into fixed buffers that the next frame overwrites
    a = [{k: t.clone() for k, t in ours.render_image(v).items()} for v in _views(sgs_viewer)]
    _C.set_frame_index(1000)
    b = [ref.render_image(v) for v in _views(sgs_viewer)]
    for i, (x, y) in enumerate(zip(a, b)):
        for k in ("rgb", "depth", "alpha"):
            assert torch.equal(x[k], y[k]), f"frame {i} {k}"


def test_dropped_renderer_releases_its_graphs_at_once(cuda_device):
    """The frame graphs hold their renderer weakly: with the cyclic collector off, dropping a renderer
    releases its captured graphs immediately (none is left for a collection that might run while
    another renderer captures), and the next renderer's captures and frames work."""
    import gc
    import weakref

    import sgs_viewer

    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=5_000, log_scale_mean=-3.5), seed=12)
    model = tuple(t.cuda() for t in scene.tensors())
    views = _views(sgs_viewer)
    enabled = gc.isenabled()
    gc.collect()
    gc.disable()
    try:
        first = sgs_viewer.ProgressiveRenderer(*model, samples_per_pixel=1, graphs=True, temporal_reuse=True)
        for v in views[:3]:
            first.render_image(v)
        frames = weakref.ref(first._frames)
        assert len(first._frames.graphs) == 3
        del first
        assert frames() is None
        second = sgs_viewer.ProgressiveRenderer(*model, samples_per_pixel=1, graphs=True, temporal_reuse=True)
        got = [second.render_image(v)["alpha"].clone() for v in views[:3]]
    finally:
        if enabled:
            gc.enable()
    assert all(bool(torch.isfinite(a).all()) for a in got) and float(got[-1].mean()) > 0.0


def test_composite_equals_the_tensor_operations(cuda_device):
    """_C.composite (one kernel) against the plugin's tensor operations (Renderer.py:91-97), bit for bit,
    with alphas below 0, above 1 and at 0."""
    g = torch.Generator(device="cuda").manual_seed(4)
    h, w = 37, 53
    image = torch.rand((h, w, 3), device="cuda", generator=g) * 1.3 - 0.1
    depth = torch.rand((h, w, 1), device="cuda", generator=g) * 20.0
    alpha = torch.rand((h, w, 1), device="cuda", generator=g) * 1.4 - 0.2
    alpha[0, :5] = 0.0
    bg = torch.tensor([0.2, 0.7, 1.0], device="cuda")
    rgb, d, a = _C.composite(image, depth, alpha, bg)
    a_want = alpha.clamp(0.0, 1.0)
    assert torch.equal(a, a_want)
    assert torch.equal(rgb, (image + (1.0 - a_want) * bg).clamp(0.0, 1.0))
    assert torch.equal(d, depth / a_want.clamp_min(1.0e-8))


def test_camera_path_benchmark_and_png(tmp_path, cuda_device):
    import sgs_viewer

    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=5_000), seed=10)
    model = tuple(t.cuda() for t in scene.tensors())
    views = [sgs_viewer.View.from_camera(c, frame_idx=i) for i, c in enumerate(sgs_scenes.orbit_cameras(4, 4.0, 96, 72))]
    sgs_viewer.save_camera_path(tmp_path / "p.json", views)
    views = sgs_viewer.load_camera_path(tmp_path / "p.json", camera=views[0])
    r = sgs_viewer.ProgressiveRenderer(*model, samples_per_pixel=2)
    res = sgs_viewer.benchmark_camera_path(r, views, iterations=2)
    assert res["frames"] == 4 and res["avg_fps"] > 0 and len(res["per_frame_ms"]) == 4
    img = r.render_image(views[0])["rgb"]
    sgs_viewer.write_png(tmp_path / "f.png", img)
    back = sgs_viewer.read_png(tmp_path / "f.png")
    want = (img.clamp(0, 1).cpu().numpy() * 255 + 0.5).astype(np.uint8)
    assert (back == want).all()
