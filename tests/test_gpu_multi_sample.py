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


def _full_args(tensors, cam, flags, hist, mode, kb, v2pv, reuse):
    args = list(_args(tensors, cam, flags, hist, mode))
    args[19] = reuse
    args[21], args[22] = kb
    args[27] = v2pv
    return args


WIDE_CASES = [
    # (flags, spatial reuse, first mode, samples, caps)
    (dict(aa=False, ss=1, gps=True, hybrid=True), False, 0, 5, {}),
    (dict(aa=False, ss=2, gps=True, hybrid=True), False, 1, 4, dict(max_fragments=1024, max_binned=65536)),
    (dict(aa=False, ss=1, gps=False, hybrid=False), True, 0, 4, {}),
    (dict(aa=False, ss=2, gps=True, hybrid=True), True, 2, 4, dict(max_fragments=1024, max_binned=65536)),
    (dict(aa=False, ss=1, gps=False, hybrid=True), True, 1, 3, {}),
    (dict(aa=True, ss=2, gps=False, hybrid=False), False, 2, 3, {}),
    (dict(aa=False, ss=3, gps=True, hybrid=False), True, 2, 2, {}),
]


@pytest.mark.parametrize("flags,reuse,first_mode,n,caps", WIDE_CASES)
def test_hybrid_gps_reuse_and_reproject_in_one_call(flags, reuse, first_mode, n, caps, cuda_device):
    """GPS with hybrid scheduling (each frame's queue pass into its own framebuffer), spatial reuse (the
    k-buffer updated sample by sample) and a Reproject first sample: the outputs and the k-buffer of one
    render_samples call equal those of n render calls."""
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=40_000, log_scale_mean=-3.0, log_scale_std=1.0), seed=6)
    tensors = tuple(t.cuda() for t in scene.tensors())
    cams = sgs_scenes.orbit_cameras(16, 4.0, 128, 96, step_deg=4.0)
    ss = flags["ss"]
    n_fb = 128 * 96 * ss * ss
    k = _C.k_buffer_size if reuse else 0
    kb0 = (torch.full((k, n_fb, 2), -1, dtype=torch.int32, device="cuda"), torch.zeros((k, n_fb, 4), device="cuda"))
    e = torch.empty(0)
    eye = torch.eye(4, device="cuda")
    # a history (and k-buffer) from two samples of the previous view
    _C.set_frame_index(300)
    hist = _C.render(*_full_args(tensors, cams[0], flags, (e, e, e, e), 0, kb0, eye, reuse), **caps)
    hist = _C.render(*_full_args(tensors, cams[0], flags, hist, 1, kb0, eye, reuse), **caps)
    cam = cams[1] if first_mode == 2 else cams[0]
    v2pv = (cams[0].w2c.double() @ torch.linalg.inv(cam.w2c.double())).float().cuda() if first_mode == 2 else eye
    start = hist if first_mode != 0 else (e, e, e, e)
    kb_ref = (kb0[0].clone(), kb0[1].clone())
    kb_got = (kb0[0].clone(), kb0[1].clone())
    _C.set_frame_index(700)
    ref = start
    for i in range(n):
        ref = _C.render(*_full_args(tensors, cam, flags, ref, first_mode if i == 0 else 1, kb_ref, v2pv, reuse),
                        **caps)
    _C.set_frame_index(700)
    got = _C.render_samples(n, *_full_args(tensors, cam, flags, start, first_mode, kb_got, v2pv, reuse), **caps)
    assert _C.get_frame_index() == 700 + n
    for name, a, b in zip(("image", "depth", "alpha", "weight_mass"), got, ref):
        assert torch.equal(a, b), f"{name} differs after {n} samples"
    if reuse:
        assert torch.equal(kb_got[0], kb_ref[0]) and torch.equal(kb_got[1], kb_ref[1])
    assert float(got[2].mean()) > 0.2


@pytest.mark.parametrize("reuse", [False, True])
def test_hybrid_gps_and_reuse_samples_with_device_frame_counter(reuse, cuda_device):
    """The per-sample frame offsets of the hybrid-GPS and per-sample paths with the frame index in device
    memory: the counter advances by n and the frames are those of n render calls."""
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=20_000, log_scale_mean=-3.0, log_scale_std=1.0), seed=5)
    tensors = tuple(t.cuda() for t in scene.tensors())
    cam = sgs_scenes.front_camera(96, 72)
    flags = dict(aa=False, ss=1, gps=True, hybrid=True)
    k = _C.k_buffer_size if reuse else 0
    kb_got = (torch.full((k, 96 * 72, 2), -1, dtype=torch.int32, device="cuda"),
              torch.zeros((k, 96 * 72, 4), device="cuda"))
    kb_ref = (kb_got[0].clone(), kb_got[1].clone())
    e = torch.empty(0)
    eye = torch.eye(4, device="cuda")
    counter = torch.tensor([77], dtype=torch.int32, device="cuda")
    _C.set_device_frame_counter(counter)
    try:
        got = _C.render_samples(5, *_full_args(tensors, cam, flags, (e, e, e, e), 0, kb_got, eye, reuse))
    finally:
        _C.set_device_frame_counter(None)
    assert int(counter.item()) == 82
    _C.set_frame_index(77)
    ref = (e, e, e, e)
    for i in range(5):
        ref = _C.render(*_full_args(tensors, cam, flags, ref, 0 if i == 0 else 1, kb_ref, eye, reuse))
    assert all(torch.equal(a, b) for a, b in zip(got, ref))


def test_samples_in_one_call_rejects_zero_samples(cuda_device):
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=1_000), seed=8)
    tensors = tuple(t.cuda() for t in scene.tensors())
    cam = sgs_scenes.front_camera(64, 48)
    e = torch.empty(0)
    flags = dict(aa=False, ss=1, gps=False, hybrid=False)
    with pytest.raises(RuntimeError):
        _C.render_samples(0, *_args(tensors, cam, flags, (e, e, e, e), 0))
