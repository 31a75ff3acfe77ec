"""Device-resident frame index and CUDA-graph capture of a batch of views (GPU).

A graph of render calls with the frame index in device memory must render, replay after replay,
exactly the frames the same calls render eagerly with the process-wide index pinned to the same
values; the device index advances once per call.
"""
import pytest
import torch

import sgs_batch
import sgs_scenes
from StochasticGSCudaBackend import _C

pytestmark = pytest.mark.gpu


def _eager(scene, views, flags, first_frame, n_samples):
    """The same sequence eagerly: Reset at frame f0 + i, then Static, view after view."""
    outs = []
    frame = first_frame
    e = torch.empty(0)
    hist = [(e, e, e, e)] * len(views)
    for s in range(n_samples):
        step = []
        for vi, v in enumerate(views):
            ss = flags["ss"]
            kb = (torch.empty((0, v["width"] * v["height"] * ss * ss, 2), dtype=torch.int32, device="cuda"),
                  torch.empty((0, v["width"] * v["height"] * ss * ss, 4), device="cuda"))
            _C.set_frame_index(frame)
            frame += 1
            h = _C.render(*scene, v["w2c"].cuda(), v["position"].cuda(), v["width"], v["height"], v["focal_x"],
                          v["focal_y"], v["center_x"], v["center_y"], v["near_plane"], v["far_plane"], flags["aa"],
                          ss, flags["gps"], flags["hybrid"], False, torch.empty(0, dtype=torch.uint8, device="cuda"),
                          *kb, *hist[vi], torch.eye(4, device="cuda"), 0 if s == 0 else 1)
            step.append(h)
        hist = step
        outs.append(step)
    return outs


@pytest.mark.parametrize("flags", [dict(aa=False, ss=1, gps=False, hybrid=False),
                                   dict(aa=False, ss=1, gps=True, hybrid=True)])
def test_graph_replays_equal_eager_frames(flags, cuda_device):
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=200_000, means="uniform", means_scale=10.0,
                                                       log_scale_mean=-3.5, log_scale_std=0.8), seed=2)
    tensors = tuple(t.cuda() for t in scene.tensors())
    views = sgs_batch.batch_views(6, 25.0, [(320, 180), (480, 270), (640, 360)])
    batch = sgs_batch.CapturedViews(tensors, views, flags, first_frame=100).capture()
    assert int(batch.counter.item()) == 100 + len(views)
    replays = [[tuple(t.clone() for t in h) for h in batch.replay()] for _ in range(2)]
    assert int(batch.counter.item()) == 100 + 3 * len(views)
    eager = _eager(tensors, views, flags, 100, 3)
    for r in range(2):
        for vi in range(len(views)):
            for name, a, b in zip(("image", "depth", "alpha", "weight_mass"), replays[r][vi], eager[r + 1][vi]):
                assert torch.equal(a, b), f"replay {r} view {vi} {name}"
    assert not torch.equal(replays[0][0][0], replays[1][0][0])


def test_device_counter_does_not_touch_the_process_counter(cuda_device):
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=1000), seed=3)
    tensors = tuple(t.cuda() for t in scene.tensors())
    cam = sgs_scenes.front_camera(64, 48)
    counter = torch.tensor([7], dtype=torch.int32, device="cuda")
    _C.set_frame_index(55)
    e = torch.empty(0)
    kb = (torch.empty((0, 64 * 48, 2), dtype=torch.int32, device="cuda"), torch.empty((0, 64 * 48, 4), device="cuda"))
    args = (*tensors, cam.w2c.cuda(), cam.position.cuda(), 64, 48, cam.focal_x, cam.focal_y, 32.0, 24.0, 0.2, 1e4,
            False, 1, False, False, False, torch.empty(0, dtype=torch.uint8, device="cuda"), *kb, e, e, e, e,
            torch.eye(4, device="cuda"), 0)
    _C.set_device_frame_counter(counter)
    try:
        a = _C.render(*args)
        b = _C.render(*args)
    finally:
        _C.set_device_frame_counter(None)
    assert int(counter.item()) == 9 and _C.get_frame_index() == 55
    _C.set_frame_index(7)
    c = _C.render(*args)
    _C.set_frame_index(8)
    d = _C.render(*args)
    assert torch.equal(a[0], c[0]) and torch.equal(b[0], d[0]) and not torch.equal(a[0], b[0])


@pytest.mark.parametrize("flags", [dict(aa=False, ss=1, gps=False, hybrid=False),
                                   dict(aa=True, ss=2, gps=False, hybrid=True),
                                   dict(aa=False, ss=1, gps=True, hybrid=True)])
def test_split_streams_and_caller_buffers_equal_render(flags, cuda_device):
    """render_split (accumulate and resolve on two streams) and render_into (caller buffers) give the
    outputs of render, frame for frame, in Reset and Static mode."""
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=50_000, log_scale_mean=-3.0, log_scale_std=0.8), seed=4)
    tensors = tuple(t.cuda() for t in scene.tensors())
    cam = sgs_scenes.front_camera(160, 120)
    ss = flags["ss"]
    n_fb = 160 * 120 * ss * ss
    kb = (torch.empty((0, n_fb, 2), dtype=torch.int32, device="cuda"), torch.empty((0, n_fb, 4), device="cuda"))
    e = torch.empty(0)

    def args(hist, mode):
        return (*tensors, cam.w2c.cuda(), cam.position.cuda(), 160, 120, cam.focal_x, cam.focal_y, cam.center_x,
                cam.center_y, cam.near_plane, cam.far_plane, flags["aa"], ss, flags["gps"], flags["hybrid"], False,
                torch.empty(0, dtype=torch.uint8, device="cuda"), *kb, *hist, torch.eye(4, device="cuda"), mode)

    acc, res = torch.cuda.Stream(), torch.cuda.Stream()
    cur = torch.cuda.current_stream()
    h_ref = h_split = h_into = (e, e, e, e)
    outs = tuple(torch.empty((120, 160, ch), device="cuda") for ch in (3, 1, 1, 1))
    outs2 = tuple(torch.empty_like(t) for t in outs)
    ws = torch.empty(_C.workspace_size(*args((e, e, e, e), 0)), dtype=torch.uint8, device="cuda")
    for k in range(3):
        mode = 0 if k == 0 else 1
        _C.set_frame_index(40 + k)
        h_ref = _C.render(*args(h_ref, mode))
        _C.set_frame_index(40 + k)
        acc.wait_stream(cur)
        res.wait_stream(cur)
        h_split = _C.render_split(acc, res, *args(h_split, mode))
        cur.wait_stream(res)
        _C.set_frame_index(40 + k)
        dst = outs if k % 2 == 0 else outs2
        acc.wait_stream(cur)
        res.wait_stream(cur)
        _C.render_into(dst, ws, (acc, res), *args(h_into, mode))
        cur.wait_stream(res)
        cur.wait_stream(acc)
        h_into = dst
        for name, a, b, c in zip(("image", "depth", "alpha", "weight_mass"), h_ref, h_split, h_into):
            assert torch.equal(a, b), f"render_split, frame {k}, {name}"
            assert torch.equal(a, c), f"render_into, frame {k}, {name}"
    with pytest.raises(RuntimeError, match="workspace"):
        _C.render_into(outs, ws[:64], None, *args((e, e, e, e), 0))
