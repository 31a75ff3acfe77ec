"""Several samples in one call (sgs_render_samples) against one render call per sample (GPU).

The multi-sample path walks each fragment once for all samples (stochastic transparency) or projects
once and draws each frame's points (GPS), and merges the samples into the history in one resolve
pass; its outputs must equal those of the same number of `_C.render` calls
(first call in the given temporal mode, the rest Static) bit for bit, and the frame index must
advance by the number of samples.
"""
import pytest
import torch

import sgs_scenes
from StochasticGSCudaBackend import _C

pytestmark = pytest.mark.gpu


def _args(tensors, cam, flags, hist, mode, blue=None):
    ss = flags["ss"]
    n_fb = cam.width * cam.height * ss * ss
    kb = (torch.empty((0, n_fb, 2), dtype=torch.int32, device="cuda"), torch.empty((0, n_fb, 4), device="cuda"))
    bn = blue if blue is not None else torch.empty(0, dtype=torch.uint8, device="cuda")
    return (*tensors, cam.w2c.cuda(), cam.position.cuda(), cam.width, cam.height, cam.focal_x, cam.focal_y,
            cam.center_x, cam.center_y, cam.near_plane, cam.far_plane, flags["aa"], ss, flags["gps"], flags["hybrid"],
            False, bn, *kb, *hist, torch.eye(4, device="cuda"), mode)


CASES = [
    (dict(aa=False, ss=1, gps=False, hybrid=False), False, 0, 8),
    (dict(aa=False, ss=1, gps=False, hybrid=False), False, 1, 5),
    (dict(aa=True, ss=2, gps=False, hybrid=True), False, 0, 3),
    (dict(aa=False, ss=3, gps=False, hybrid=False), True, 1, 4),
    (dict(aa=False, ss=1, gps=False, hybrid=True), True, 0, 2),
    (dict(aa=False, ss=1, gps=False, hybrid=False), False, 0, 1),
    (dict(aa=False, ss=1, gps=True, hybrid=False), False, 0, 6),
    (dict(aa=True, ss=2, gps=True, hybrid=False), False, 1, 3),
]


@pytest.mark.parametrize("flags,blue,first_mode,n", CASES)
def test_samples_in_one_call_equal_one_call_per_sample(flags, blue, first_mode, n, cuda_device):
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=40_000, log_scale_mean=-3.0, log_scale_std=1.0), seed=6)
    tensors = tuple(t.cuda() for t in scene.tensors())
    cam = sgs_scenes.front_camera(192, 144)
    bn = sgs_scenes.synthetic_blue_noise(2).cuda() if blue else None
    e = torch.empty(0)
    # a history to merge into (Static first) from two earlier samples
    _C.set_frame_index(500)
    hist = _C.render(*_args(tensors, cam, flags, (e, e, e, e), 0, bn))
    hist = _C.render(*_args(tensors, cam, flags, hist, 1, bn))
    start = hist if first_mode == 1 else (e, e, e, e)
    _C.set_frame_index(600)
    ref = start
    for k in range(n):
        ref = _C.render(*_args(tensors, cam, flags, ref, first_mode if k == 0 else 1, bn))
    assert _C.get_frame_index() == 600 + n
    _C.set_frame_index(600)
    got = _C.render_samples(n, *_args(tensors, cam, flags, start, first_mode, bn))
    assert _C.get_frame_index() == 600 + n
    for name, a, b in zip(("image", "depth", "alpha", "weight_mass"), got, ref):
        assert torch.equal(a, b), f"{name} differs after {n} samples"


def test_samples_in_one_call_with_device_frame_counter(cuda_device):
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=5_000), seed=7)
    tensors = tuple(t.cuda() for t in scene.tensors())
    cam = sgs_scenes.front_camera(96, 72)
    flags = dict(aa=False, ss=1, gps=False, hybrid=False)
    e = torch.empty(0)
    counter = torch.tensor([40], dtype=torch.int32, device="cuda")
    _C.set_device_frame_counter(counter)
    try:
        got = _C.render_samples(6, *_args(tensors, cam, flags, (e, e, e, e), 0))
    finally:
        _C.set_device_frame_counter(None)
    assert int(counter.item()) == 46
    _C.set_frame_index(40)
    ref = (e, e, e, e)
    for k in range(6):
        ref = _C.render(*_args(tensors, cam, flags, ref, 0 if k == 0 else 1))
    assert all(torch.equal(a, b) for a, b in zip(got, ref))


@pytest.mark.parametrize("change", ["gps_hybrid", "reuse", "reproject", "zero"])
def test_samples_in_one_call_rejects_unsupported_settings(change, cuda_device):
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=1_000), seed=8)
    tensors = tuple(t.cuda() for t in scene.tensors())
    cam = sgs_scenes.front_camera(64, 48)
    e = torch.empty(0)
    flags = dict(aa=False, ss=1, gps=change == "gps_hybrid", hybrid=change == "gps_hybrid")
    args = list(_args(tensors, cam, flags, (e, e, e, e), 0))
    n = 0 if change == "zero" else 3
    if change == "reuse":
        k = _C.k_buffer_size
        args[19] = True
        args[21] = torch.full((k, 64 * 48, 2), -1, dtype=torch.int32, device="cuda")
        args[22] = torch.zeros((k, 64 * 48, 4), device="cuda")
    if change == "reproject":
        hist = _C.render(*_args(tensors, cam, flags, (e, e, e, e), 0))
        args[23:27] = hist
        args[28] = 2
    with pytest.raises(RuntimeError):
        _C.render_samples(n, *args)
