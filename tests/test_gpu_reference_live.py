"""Live bit-exact parity with the reference CUDA backend at workload scale.

The reference is compiled from its own sources into oracle/_ref/ (oracle/build_ref.py) and runs on
the same GPU in the same process. Its winner framebuffer (through the test harness, frame index
explicit) and its `_C.render` outputs (through its unmodified binding, process-global frame counter)
are compared with the B200 path bit for bit.
"""
import pytest
import torch

import sgs_scenes
from oracle import build_ref
from sgs_testing import assert_bitwise, reference_render, render_once

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not build_ref.available(), reason="reference oracle not built (oracle/build_ref.py)")]


@pytest.fixture(scope="module")
def ref():
    return build_ref.load()


def cam_dict(cam: sgs_scenes.Camera) -> dict:
    return dict(width=cam.width, height=cam.height, focal_x=cam.focal_x, focal_y=cam.focal_y, center_x=cam.center_x,
                center_y=cam.center_y, near_plane=cam.near_plane, far_plane=cam.far_plane, w2c=cam.w2c.tolist(),
                position=cam.position.tolist())


def ref_framebuffer(harness, scene, cam, flags, frame, blue=None):
    dev = scene.means.device
    bn = blue.to(dev) if blue is not None else torch.empty(0, dtype=torch.uint8, device=dev)
    fb = harness.accumulate(scene.means, scene.scales, scene.rotations, scene.opacities, cam.w2c.to(dev), cam.width,
                            cam.height, cam.focal_x, cam.focal_y, cam.center_x, cam.center_y, cam.near_plane,
                            cam.far_plane, flags["aa"], flags["ss"], flags["gps"], flags["hybrid"], bn, frame)
    torch.cuda.synchronize()
    return fb.cpu().numpy()


WORKLOADS = {
    # 100k Gaussians, 640x480 (the plain stochastic-transparency workload)
    "st_100k_640": (sgs_scenes.SCENES["st_100k"], 0, lambda: sgs_scenes.front_camera(640, 480)),
    # 1M heavy-tailed footprints at 1280x720 (the GPS hybrid workload), on a smaller budget
    "gps_1m_320ss2": (sgs_scenes.SceneSpec(n=250_000, log_scale_mean=-3.0, log_scale_std=1.0), 0,
                      lambda: sgs_scenes.orbit_cameras(16, 4.0, 320, 180)[3]),
    # uniform cube seen from radius 25 (the batched 6M-Gaussian scene, 1M of it)
    "cube_1m_1080": (sgs_scenes.SceneSpec(n=1_000_000, means="uniform", means_scale=10.0, log_scale_mean=-4.5,
                                          log_scale_std=0.8, opacity_logit_std=2.0), 0,
                     lambda: sgs_scenes.orbit_cameras(1, 25.0, 1920, 1080)[0]),
}

FLAGS = {
    "st": dict(aa=False, ss=1, gps=False, hybrid=False),
    "st_ss2_aa": dict(aa=True, ss=2, gps=False, hybrid=False),
    "st_hybrid": dict(aa=False, ss=1, gps=False, hybrid=True),
    "gps": dict(aa=False, ss=1, gps=True, hybrid=False),
    "gps_hybrid": dict(aa=False, ss=1, gps=True, hybrid=True),
    "gps_hybrid_ss2": dict(aa=False, ss=2, gps=True, hybrid=True),
}

CASES = [
    ("st_100k_640", "st", 0), ("st_100k_640", "st", 1), ("st_100k_640", "st_ss2_aa", 5),
    ("st_100k_640", "gps", 3), ("st_100k_640", "st_hybrid", 4), ("st_100k_640", "gps_hybrid", 9),
    ("gps_1m_320ss2", "gps_hybrid_ss2", 2), ("gps_1m_320ss2", "gps", 7), ("gps_1m_320ss2", "st", 8),
    ("gps_1m_320ss2", "st_ss2_aa", 11),
    ("cube_1m_1080", "st", 0), ("cube_1m_1080", "gps", 1), ("cube_1m_1080", "gps_hybrid", 2),
]

_scene_cache = {}


def get_scene(name):
    if name not in _scene_cache:
        spec, seed, _ = WORKLOADS[name]
        _scene_cache.clear()
        _scene_cache[name] = sgs_scenes.make_scene(spec, seed).to("cuda")
    return _scene_cache[name]


@pytest.mark.parametrize("workload,flags,frame", CASES)
def test_winners_bitwise_live(ref, workload, flags, frame, cuda_device):
    _, harness = ref
    scene = get_scene(workload)
    cam = WORKLOADS[workload][2]()
    fl = FLAGS[flags]
    want = ref_framebuffer(harness, scene, cam, fl, frame)
    got = render_once({k: v for k, v in zip(("means", "scales", "rotations", "opacities", "sh_coefficients"),
                                           scene.tensors())}, cam_dict(cam), fl, frame)
    assert (want != -1).any()
    assert_bitwise("framebuffer", got["fb"], want)


def test_blue_noise_winners_live(ref, cuda_device):
    _, harness = ref
    scene = get_scene("st_100k_640")
    cam = sgs_scenes.front_camera(640, 480)
    blue = sgs_scenes.synthetic_blue_noise(3)
    for frame in (0, 63, 64, 200):
        fl = FLAGS["st"]
        want = ref_framebuffer(harness, scene, cam, fl, frame, blue)
        got = render_once({k: v for k, v in zip(("means", "scales", "rotations", "opacities", "sh_coefficients"),
                                               scene.tensors())}, cam_dict(cam), fl, frame, blue_noise=blue)
        assert_bitwise(f"framebuffer frame {frame}", got["fb"], want)


def test_render_binding_progressive_live(ref, cuda_device):
    """The reference's own `_C.render` against ours over a progressive, moving, reusing sequence."""
    ref_C, _ = ref
    from StochasticGSCudaBackend import _C

    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=60_000, log_scale_mean=-3.2, log_scale_std=0.6), 5).to("cuda")
    cams = sgs_scenes.orbit_cameras(24, 4.0, 320, 240, step_deg=2.0)
    dev = torch.device("cuda")
    e = torch.empty(0)
    for gps, reuse, ss in ((False, True, 1), (True, False, 2), (True, True, 1)):
        n_fb = 320 * 240 * ss * ss
        k = 4 if reuse else 0
        kb_ref = (torch.full((k, n_fb, 2), -1, dtype=torch.int32, device=dev), torch.zeros((k, n_fb, 4), device=dev))
        kb_our = (kb_ref[0].clone(), kb_ref[1].clone())
        h_ref = h_our = (e, e, e, e)
        prev = None
        for i, mode in enumerate([0, 1, 1, 2, 1, 2, 2]):
            cam = cams[i]
            v2pv = (prev.w2c.double() @ torch.linalg.inv(cam.w2c.double())).float() if mode == 2 else torch.eye(4)
            args = lambda kb, h: (*scene.tensors(), cam.w2c.to(dev), cam.position.to(dev), cam.width, cam.height,
                                  cam.focal_x, cam.focal_y, cam.center_x, cam.center_y, cam.near_plane, cam.far_plane,
                                  False, ss, gps, False, reuse, torch.empty(0, dtype=torch.uint8, device=dev), *kb, *h,
                                  v2pv.to(dev), mode)
            frame, h_ref = reference_render(ref_C, *args(kb_ref, h_ref))
            _C.set_frame_index(frame)
            h_our = _C.render(*args(kb_our, h_our))
            torch.cuda.synchronize()
            for name, a, b in zip(("image", "depth", "alpha", "weight_mass"), h_our, h_ref):
                assert_bitwise(f"gps={gps} reuse={reuse} step {i} {name}", a.cpu().numpy(), b.cpu().numpy())
            if reuse:
                assert_bitwise("k-buffer primitives", kb_our[0].cpu().numpy(), kb_ref[0].cpu().numpy())
            prev = cam

