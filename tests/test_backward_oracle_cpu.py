"""The analytic gradient of the expected image (the backward's checker) against central finite
differences (eps 1e-3) on 64 sampled parameters (CPU)."""
import numpy as np
import pytest

import sgs_scenes
from oracle import cpu

KEYS = ("means", "scales", "rotations", "opacities", "sh_coefficients")


def _setup(ss=1):
    spec = sgs_scenes.SceneSpec(n=120, log_scale_mean=-2.3, log_scale_std=0.4, opacity_logit_std=1.0)
    scene = {k: t.numpy() for k, t in zip(KEYS, sgs_scenes.make_scene(spec, seed=5, morton=False).tensors())}
    cam = sgs_scenes.pinhole((0.3, -0.2, -4.0), 48, 36, 60.0)
    cd = dict(width=48, height=36, focal_x=cam.focal_x, focal_y=cam.focal_y, center_x=cam.center_x,
              center_y=cam.center_y, near_plane=cam.near_plane, far_plane=cam.far_plane, w2c=cam.w2c.numpy(),
              position=cam.position.numpy())
    rng = np.random.default_rng(0)
    gi = rng.normal(size=(36, 48, 3))
    ga = rng.normal(size=(36, 48, 1))
    gd = rng.normal(size=(36, 48, 1)) * 0.1
    return scene, cd, gi, ga, gd


def test_expected_image_matches_the_monte_carlo_mean_of_the_oracle():
    """The frozen-support expected image equals the average of many single samples (same support)."""
    scene, cd, *_ = _setup()
    exp = cpu.expected_image(scene, cd)
    flags = dict(aa=False, ss=1, gps=False, hybrid=False)
    acc = np.zeros((36, 48, 3))
    n = 600
    for f in range(n):
        fb = cpu.accumulate(scene, cd, flags, f, threads=2)
        acc += cpu.sample_resolve(scene, cd, flags, fb, threads=2)["image"]
    err = np.abs(acc / n - exp["image"])
    assert err.mean() < 0.01 and np.percentile(err, 99) < 0.08


def test_expected_image_matches_the_monte_carlo_mean_with_antialiasing():
    """The same check with proper antialiasing (opacity scaled by sqrt(det / det dilated))."""
    scene, cd, *_ = _setup()
    exp = cpu.expected_image(scene, cd, aa=True)
    flags = dict(aa=True, ss=1, gps=False, hybrid=False)
    acc = np.zeros((36, 48, 3))
    n = 600
    for f in range(n):
        fb = cpu.accumulate(scene, cd, flags, f, threads=2)
        acc += cpu.sample_resolve(scene, cd, flags, fb, threads=2)["image"]
    err = np.abs(acc / n - exp["image"])
    assert err.mean() < 0.01 and np.percentile(err, 99) < 0.08


@pytest.mark.parametrize("aa", [False, True])
def test_analytic_gradient_matches_central_differences(aa):
    scene, cd, gi, ga, gd = _setup()
    base = {k: v.copy() for k, v in scene.items()}
    res = cpu.expected_image(scene, cd, base=base, g_image=gi, g_alpha=ga, g_depth=gd, grad=True, aa=aa)
    rng = np.random.default_rng(1)
    eps = 1e-3
    checked = 0
    worst = []
    for k in KEYS:
        flat = scene[k].reshape(-1)
        for idx in rng.choice(flat.size, size=13, replace=False):
            plus = {kk: vv.astype(np.float64).copy() for kk, vv in scene.items()}
            minus = {kk: vv.astype(np.float64).copy() for kk, vv in scene.items()}
            plus[k].reshape(-1)[idx] += eps
            minus[k].reshape(-1)[idx] -= eps
            lp = cpu.expected_image(plus, cd, base=base, g_image=gi, g_alpha=ga, g_depth=gd, aa=aa)["loss"]
            lm = cpu.expected_image(minus, cd, base=base, g_image=gi, g_alpha=ga, g_depth=gd, aa=aa)["loss"]
            fd = (lp - lm) / (2 * eps)
            an = res["grad"][k].reshape(-1)[idx]
            worst.append((abs(fd - an) / max(1e-3, abs(fd)), k, idx, fd, an))
            checked += 1
    worst.sort(reverse=True)
    assert checked >= 64
    assert worst[0][0] < 2e-3, worst[:5]
