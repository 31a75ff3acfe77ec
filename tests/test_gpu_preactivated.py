"""The preactivated layout (sgs_preactivate; the reference README's first listed improvement,
README.md:139-142): its values against a float64 restatement, and renders that read it equal bit
for bit to renders that rebuild covariance and opacity per sample."""
import numpy as np
import pytest
import torch

import sgs_scenes
from sgs_testing import assert_bitwise, render_once

pytestmark = pytest.mark.gpu

KEYS = ("means", "scales", "rotations", "opacities", "sh_coefficients")


def scene_with_edge_cases(n: int, seed: int) -> dict:
    """Heavy-tailed footprints plus degenerate quaternions and opacities below 1/255."""
    s = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=n, log_scale_mean=-3.0, log_scale_std=1.0), seed=seed)
    rot = s.rotations.clone()
    rot[::97] = 0.0
    rot[1::89] = rot[1::89] * 1e-5
    op = s.opacities.clone()
    op[::53] = -7.0
    return dict(zip(KEYS, (s.means, s.scales, rot, op, s.sh_coefficients)))


def cam_dict(cam):
    return dict(width=cam.width, height=cam.height, focal_x=cam.focal_x, focal_y=cam.focal_y, center_x=cam.center_x,
                center_y=cam.center_y, near_plane=cam.near_plane, far_plane=cam.far_plane, w2c=cam.w2c.numpy(),
                position=cam.position.numpy())


def test_preactivated_values_match_float64(cuda_device):
    from StochasticGSCudaBackend import _C

    sc = scene_with_edge_cases(4096, 1)
    pre = _C.preactivate(*(sc[k].to(cuda_device) for k in ("scales", "rotations", "opacities"))).cpu().double()
    q = sc["rotations"].double()
    nq = (q * q).sum(1)
    valid = nq >= 1e-8
    assert torch.equal(pre[:, 7] == 1.0, valid) and bool(((pre[:, 7] == 0.0) | (pre[:, 7] == 1.0)).all())
    qn = q[valid] / nq[valid].sqrt()[:, None]
    r, i, j, k = qn.unbind(1)
    R = torch.stack([1 - 2 * (j * j + k * k), 2 * (i * j - r * k), 2 * (i * k + r * j),
                     2 * (i * j + r * k), 1 - 2 * (i * i + k * k), 2 * (j * k - r * i),
                     2 * (i * k - r * j), 2 * (j * k + r * i), 1 - 2 * (i * i + j * j)], 1).view(-1, 3, 3)
    var = torch.exp(2 * sc["scales"].double()[valid])
    cov = R @ torch.diag_embed(var) @ R.transpose(1, 2)
    want = torch.stack([cov[:, 0, 0], cov[:, 0, 1], cov[:, 0, 2], cov[:, 1, 1], cov[:, 1, 2], cov[:, 2, 2]], 1)
    scale = var.max(1).values[:, None]
    err = ((pre[valid][:, :6] - want).abs() / scale).max().item()
    assert err < 2e-5, f"covariance relative to the largest variance off by {err}"
    sig = torch.sigmoid(sc["opacities"].double())
    assert torch.allclose(pre[:, 6], sig, rtol=2e-6, atol=1e-7)


CASES = [
    ("st", dict(aa=False, ss=1, gps=False, hybrid=False), False),
    ("st blue", dict(aa=False, ss=1, gps=False, hybrid=False), True),
    ("st hybrid aa", dict(aa=True, ss=1, gps=False, hybrid=True), False),
    ("st ss2", dict(aa=False, ss=2, gps=False, hybrid=False), False),
    ("gps", dict(aa=False, ss=1, gps=True, hybrid=False), False),
    ("gps hybrid ss2", dict(aa=False, ss=2, gps=True, hybrid=True), False),
]


@pytest.mark.parametrize("name,flags,blue", CASES, ids=[c[0] for c in CASES])
def test_preactivated_render_is_bit_identical(name, flags, blue, cuda_device):
    sc = scene_with_edge_cases(30_000, 2)
    cam = cam_dict(sgs_scenes.front_camera(320, 180))
    bn = sgs_scenes.synthetic_blue_noise(3).numpy() if blue else None
    for frame in (0, 17):
        want = render_once(sc, cam, flags, frame, blue_noise=bn)
        got = render_once(sc, cam, flags, frame, blue_noise=bn, preactivate=True)
        assert (want["fb"] != -1).sum() > 1000
        assert_bitwise(f"{name} framebuffer, frame {frame}", got["fb"], want["fb"])
        for key in ("image", "depth", "alpha", "weight_mass"):
            assert_bitwise(f"{name} {key}, frame {frame}", got[key], want[key])


@pytest.mark.parametrize("gps", [False, True])
def test_preactivated_samples_per_call(gps, cuda_device):
    from StochasticGSCudaBackend import _C

    sc = {k: v.to(cuda_device) for k, v in scene_with_edge_cases(20_000, 3).items()}
    cam = sgs_scenes.front_camera(256, 144)
    e = torch.empty(0)
    kb = (torch.empty((0, 256 * 144, 2), dtype=torch.int32, device=cuda_device),
          torch.empty((0, 256 * 144, 4), device=cuda_device))
    args = (*(sc[k] for k in KEYS), cam.w2c.to(cuda_device), cam.position.to(cuda_device), cam.width, cam.height,
            cam.focal_x, cam.focal_y, cam.center_x, cam.center_y, cam.near_plane, cam.far_plane, False, 1, gps, False,
            False, torch.empty(0, dtype=torch.uint8, device=cuda_device), *kb, e, e, e, e,
            torch.eye(4, device=cuda_device), 0)
    pre = _C.preactivate(sc["scales"], sc["rotations"], sc["opacities"])
    _C.set_frame_index(5)
    want = _C.render_samples(6, *args)
    _C.set_frame_index(5)
    got = _C.render_samples(6, *args, preactivated=pre)
    for a, b, key in zip(got, want, ("image", "depth", "alpha", "weight_mass")):
        assert_bitwise(f"{key}, 6 samples, gps={gps}", a.cpu().numpy(), b.cpu().numpy())


def test_preactivated_shape_is_checked(cuda_device):
    from StochasticGSCudaBackend import _C

    sc = {k: v.to(cuda_device) for k, v in scene_with_edge_cases(100, 4).items()}
    cam = sgs_scenes.front_camera(64, 48)
    e = torch.empty(0)
    kb = (torch.empty((0, 64 * 48, 2), dtype=torch.int32, device=cuda_device),
          torch.empty((0, 64 * 48, 4), device=cuda_device))
    args = (*(sc[k] for k in KEYS), cam.w2c.to(cuda_device), cam.position.to(cuda_device), 64, 48, cam.focal_x,
            cam.focal_y, cam.center_x, cam.center_y, cam.near_plane, cam.far_plane, False, 1, False, False, False,
            torch.empty(0, dtype=torch.uint8, device=cuda_device), *kb, e, e, e, e, torch.eye(4, device=cuda_device), 0)
    with pytest.raises(RuntimeError, match="preactivated"):
        _C.render(*args, preactivated=torch.zeros((99, 8), device=cuda_device))
    assert _C.preactivate(sc["scales"][:0], sc["rotations"][:0], sc["opacities"][:0]).shape == (0, 8)
