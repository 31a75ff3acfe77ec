"""The B200 backward pass: unbiased gradient estimates of the expected image (GPU).

The estimator (csrc/backward_st.cu) averaged over many samples must agree with the exact gradient of
the expected image computed in double precision by the CPU restatement (oracle: expected_image),
which tests/test_backward_oracle_cpu.py pins to central finite differences. The samples are split
into independent batches: every parameter's mean estimate must lie within 6 standard errors of the
exact value, and the relative L2 error of each parameter group must be small.
"""
import numpy as np
import pytest
import torch

import sgs_scenes
from oracle import cpu
from StochasticGSCudaBackend import Settings
from StochasticGSCudaBackend.autograd import render_samples

pytestmark = pytest.mark.gpu

KEYS = ("means", "scales", "rotations", "opacities", "sh_coefficients")
W, H = 48, 36


def _problem(ss=1, sh_bases=16):
    spec = sgs_scenes.SceneSpec(n=120, log_scale_mean=-2.3, log_scale_std=0.4, opacity_logit_std=1.0,
                                sh_bases=sh_bases)
    scene = sgs_scenes.make_scene(spec, seed=5, morton=False)
    cam = sgs_scenes.pinhole((0.3, -0.2, -4.0), W, H, 60.0)
    rng = np.random.default_rng(0)
    gi = rng.normal(size=(H, W, 3))
    ga = rng.normal(size=(H, W, 1))
    gd = rng.normal(size=(H, W, 1)) * 0.1
    return scene, cam, gi, ga, gd


def _settings(cam, ss):
    return Settings(cam.w2c.cuda(), cam.position.cuda(), W, H, cam.focal_x, cam.focal_y, cam.center_x, cam.center_y,
                    cam.near_plane, cam.far_plane, False, ss, False, False, False)


@pytest.mark.parametrize("ss,hybrid,store", [(1, False, True), (2, False, False), (1, True, True)])
def test_estimator_matches_exact_gradient(ss, hybrid, store, cuda_device):
    scene, cam, gi, ga, gd = _problem(ss)
    sc = {k: t.numpy() for k, t in zip(KEYS, scene.tensors())}
    cd = dict(width=W, height=H, focal_x=cam.focal_x, focal_y=cam.focal_y, center_x=cam.center_x,
              center_y=cam.center_y, near_plane=cam.near_plane, far_plane=cam.far_plane, w2c=cam.w2c.numpy(),
              position=cam.position.numpy())
    exact = cpu.expected_image(sc, cd, ss=ss, g_image=gi, g_alpha=ga, g_depth=gd, grad=True)["grad"]
    settings = _settings(cam, ss)._replace(hybrid_scheduling=hybrid)
    gi_t = torch.tensor(gi, dtype=torch.float32, device="cuda")
    ga_t = torch.tensor(ga, dtype=torch.float32, device="cuda")
    gd_t = torch.tensor(gd, dtype=torch.float32, device="cuda")
    batches, per_batch = 16, 512
    est = {k: [] for k in KEYS}
    for bi in range(batches):
        params = [t.cuda().requires_grad_(True) for t in scene.tensors()]
        image, depth, alpha = render_samples(*params, settings, n_samples=per_batch, first_frame=1000 + bi * per_batch,
                                             store_winners=store)
        loss = (image * gi_t).sum() + (alpha * ga_t).sum() + (depth * gd_t).sum()
        loss.backward()
        for k, p in zip(KEYS, params):
            est[k].append(p.grad.detach().cpu().numpy().astype(np.float64))
    for k in KEYS:
        e = np.stack(est[k])
        mean = e.mean(0)
        se = e.std(0, ddof=1) / np.sqrt(batches)
        ex = exact[k]
        rel = np.linalg.norm(mean - ex) / np.linalg.norm(ex)
        z = np.abs(mean - ex) / np.maximum(se, 1e-6 * np.abs(ex).max())
        assert rel < 0.06, f"{k}: relative L2 error {rel:.4f}"
        assert np.percentile(z, 99.5) < 6.0, f"{k}: z-scores {np.sort(z.ravel())[-5:]}"


def test_backward_rejects_unsupported_modes(cuda_device):
    scene, cam, *_ = _problem()
    params = [t.cuda().requires_grad_(True) for t in scene.tensors()]
    with pytest.raises(RuntimeError, match="stochastic transparency"):
        render_samples(*params, _settings(cam, 1)._replace(use_gps=True), n_samples=2)
