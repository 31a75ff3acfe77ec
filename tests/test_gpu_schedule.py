"""The winner framebuffer does not depend on how the accumulate pass splits its work.

Stochastic transparency draws every threshold from (frame, Gaussian, pixel) and merges with a
minimum, so the queue of large Gaussians, the in-place path taken when that queue is full, and the
row segmentation of wide footprints must all give the same bits. Each case renders with the default
queue and with small queue caps (sgs_set_queue_limit), compares the framebuffers bit for bit, and
checks them against the CPU restatement (>= 99.99 % identical winners, the restatement's float
tolerance).
"""
import numpy as np
import pytest
import torch

import sgs_scenes
from oracle import cpu
from sgs_testing import assert_bitwise, render_once

pytestmark = pytest.mark.gpu

KEYS = ("means", "scales", "rotations", "opacities", "sh_coefficients")


def cam_dict(cam):
    return dict(width=cam.width, height=cam.height, focal_x=cam.focal_x, focal_y=cam.focal_y, center_x=cam.center_x,
                center_y=cam.center_y, near_plane=cam.near_plane, far_plane=cam.far_plane, w2c=cam.w2c.numpy(),
                position=cam.position.numpy())


def heavy_scene(n: int, seed: int = 3) -> sgs_scenes.Scene:
    """Heavy-tailed footprints (log-scales N(-3, 1)): many AABBs above the queue threshold."""
    return sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=n, log_scale_mean=-3.0, log_scale_std=1.0), seed=seed)


def wide_scene(n: int, seed: int = 5) -> sgs_scenes.Scene:
    """Axis-aligned needles, long in x and thin in y and z: wide, flat AABBs whose chunks have few
    rows, so each row is walked by several lanes."""
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=n, log_scale_mean=-5.5, log_scale_std=0.3), seed=seed)
    g = torch.Generator().manual_seed(seed + 1)
    scales = scene.scales.clone()
    scales[:, 0] = -1.0 + 0.5 * torch.rand(n, generator=g)
    rotations = torch.zeros_like(scene.rotations)
    rotations[:, 0] = 1.0
    return sgs_scenes.Scene(scene.means, scales, rotations, scene.opacities, scene.sh_coefficients)


CASES = [
    ("heavy", 20_000, sgs_scenes.front_camera(320, 180), dict(aa=False, ss=2, gps=False, hybrid=False)),
    ("heavy", 20_000, sgs_scenes.front_camera(320, 180), dict(aa=True, ss=1, gps=False, hybrid=True)),
    ("wide", 4_000, sgs_scenes.front_camera(640, 360), dict(aa=False, ss=1, gps=False, hybrid=False)),
    ("wide", 4_000, sgs_scenes.front_camera(320, 180), dict(aa=False, ss=3, gps=False, hybrid=True)),
]


@pytest.mark.parametrize("kind,n,cam,flags", CASES)
def test_queue_caps_and_segments_do_not_change_winners(kind, n, cam, flags, cuda_device):
    from StochasticGSCudaBackend import _C

    scene = heavy_scene(n) if kind == "heavy" else wide_scene(n)
    cd = cam_dict(cam)
    dev_scene = {k: t.to(cuda_device) for k, t in zip(KEYS, scene.tensors())}
    sc = {k: t.numpy() for k, t in zip(KEYS, scene.tensors())}
    blue = sgs_scenes.synthetic_blue_noise(1).numpy() if flags["hybrid"] else None
    for frame in (2, 65):
        _C.set_queue_limit(0)
        try:
            want = render_once(dev_scene, cd, flags, frame, blue_noise=blue)
            for cap in (1, 7, 300):
                _C.set_queue_limit(cap)
                got = render_once(dev_scene, cd, flags, frame, blue_noise=blue)
                assert_bitwise(f"framebuffer, queue cap {cap}, frame {frame}", got["fb"], want["fb"])
                assert_bitwise(f"image, queue cap {cap}, frame {frame}", got["image"], want["image"])
        finally:
            _C.set_queue_limit(0)
        ref = cpu.accumulate(sc, cd, flags, frame, blue_noise=blue)
        assert (ref != -1).sum() > 1000
        agree = float((want["fb"] == ref).mean())
        assert agree >= 0.9999, f"frame {frame}: winners agree with the CPU restatement on {agree:.6f}"


def test_queue_cap_restores_default_workspace(cuda_device):
    """The cap enters the workspace size and is undone by a cap of 0."""
    from StochasticGSCudaBackend import _C, _abi

    lib = _abi.load()
    scene = heavy_scene(1000)
    cam = sgs_scenes.front_camera(160, 90)
    g = _abi.Gaussians(0, 0, 0, 0, 0, 1000, 16)
    c = _abi.Camera(0, 0, cam.width, cam.height, cam.focal_x, cam.focal_y, cam.center_x, cam.center_y,
                    cam.near_plane, cam.far_plane)
    s = _abi.SettingsC(0, 1, 0, 0, 0, 0, None, None, 0, 0, None)
    import ctypes

    default = lib.sgs_workspace_size(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s))
    _C.set_queue_limit(4)
    try:
        capped = lib.sgs_workspace_size(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s))
    finally:
        _C.set_queue_limit(0)
    assert capped < default
    assert lib.sgs_workspace_size(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s)) == default
    del scene
