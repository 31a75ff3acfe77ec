"""Synthetic workload generators: determinism, layouts and camera conventions (CPU)."""
import math

import numpy as np
import torch

import sgs_scenes


def test_scene_is_deterministic_and_shaped():
    spec = sgs_scenes.SceneSpec(n=5000)
    a = sgs_scenes.make_scene(spec, seed=3)
    b = sgs_scenes.make_scene(spec, seed=3)
    for x, y in zip(a.tensors(), b.tensors()):
        assert torch.equal(x, y)
    assert a.means.shape == (5000, 3) and a.scales.shape == (5000, 3) and a.rotations.shape == (5000, 4)
    assert a.opacities.shape == (5000,) and a.sh_coefficients.shape == (5000, 16, 3)
    assert torch.allclose(a.rotations.norm(dim=1), torch.ones(5000), atol=1e-5)
    c = sgs_scenes.make_scene(spec, seed=4)
    assert not torch.equal(a.means, c.means)


def test_distributions_follow_the_spec():
    spec = sgs_scenes.SCENES["batch_6m"]
    small = sgs_scenes.SceneSpec(**{**spec.__dict__, "n": 200_000})
    s = sgs_scenes.make_scene(small, seed=0, morton=False)
    assert s.means.abs().max() <= 10.0 and abs(float(s.means.mean())) < 0.1
    assert abs(float(s.scales.mean()) + 4.5) < 0.01 and abs(float(s.scales.std()) - 0.8) < 0.01
    assert abs(float(s.opacities.std()) - 2.0) < 0.02
    assert abs(float(s.sh_coefficients[:, 0].std()) - 0.5) < 0.01
    assert abs(float(s.sh_coefficients[:, 1:].std()) - 0.05) < 0.001


def test_morton_order_is_a_permutation_with_spatial_locality():
    spec = sgs_scenes.SceneSpec(n=20_000)
    raw = sgs_scenes.make_scene(spec, seed=1, morton=False)
    srt = sgs_scenes.make_scene(spec, seed=1, morton=True)
    a = raw.means.numpy()[np.lexsort(raw.means.numpy().T)]
    b = srt.means.numpy()[np.lexsort(srt.means.numpy().T)]
    assert np.array_equal(a, b)
    codes = sgs_scenes.morton_codes(srt.means)
    assert bool((codes[1:] >= codes[:-1]).all())
    assert float((srt.means[1:] - srt.means[:-1]).norm(dim=1).mean()) < 0.5 * float((raw.means[1:] - raw.means[:-1]).norm(dim=1).mean())


def test_camera_conventions():
    cam = sgs_scenes.front_camera(640, 480)
    expect = torch.eye(4)
    expect[2, 3] = 4.0
    assert torch.allclose(cam.w2c, expect, atol=1e-6)
    assert math.isclose(cam.focal_y, 480 / (2 * math.tan(math.radians(30))), rel_tol=1e-6)
    for c in sgs_scenes.orbit_cameras(8, 25.0, 1920, 1080):
        origin_view = c.w2c @ torch.tensor([0.0, 0.0, 0.0, 1.0])
        assert abs(float(origin_view[0])) < 1e-4 and abs(float(origin_view[1])) < 1e-4
        assert abs(float(origin_view[2]) - 25.0) < 1e-3
        assert torch.allclose(c.w2c[:3, :3] @ c.w2c[:3, :3].T, torch.eye(3), atol=1e-5)


def test_blue_noise_volume_is_fixed():
    v = sgs_scenes.synthetic_blue_noise(0)
    assert v.shape == (64, 128, 128) and v.dtype == torch.uint8
    assert torch.equal(v, sgs_scenes.synthetic_blue_noise(0))
    counts = torch.bincount(v.flatten().long(), minlength=256).float()
    assert float(counts.std() / counts.mean()) < 0.05
