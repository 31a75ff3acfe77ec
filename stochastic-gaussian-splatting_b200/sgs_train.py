"""Differentiable training step on the render path: L1 + 0.2 (1 - SSIM) of the averaged samples.

The training workload: 500k Gaussians drawn like the plain 100k scene with log-scales N(-3.5, 0.7^2),
views on an orbit at 800x800, targets rendered by the same path from a perturbed copy of the scene
(means + N(0, 0.02^2), SH + N(0, 0.1^2)); each step renders 8 samples of one view, compares them with
the target and back-propagates through the hand-written backward
(StochasticGSCudaBackend.autograd.render_samples).
"""
from __future__ import annotations

import dataclasses

import torch
import torch.nn.functional as F

import sgs_scenes
from StochasticGSCudaBackend import Settings, _C
from StochasticGSCudaBackend.autograd import render_samples


def _gaussian_window(size: int = 11, sigma: float = 1.5, device=None) -> torch.Tensor:
    x = torch.arange(size, dtype=torch.float32, device=device) - size // 2
    g = torch.exp(-(x * x) / (2 * sigma * sigma))
    g = g / g.sum()
    return (g[:, None] * g[None, :]).expand(3, 1, size, size).contiguous()


def ssim(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """Mean SSIM of two (H, W, 3) images in [0, 1] (11x11 Gaussian window, sigma 1.5)."""
    x = a.permute(2, 0, 1)[None]
    y = b.permute(2, 0, 1)[None]
    w = _gaussian_window(device=a.device)
    mu_x = F.conv2d(x, w, padding=5, groups=3)
    mu_y = F.conv2d(y, w, padding=5, groups=3)
    sxx = F.conv2d(x * x, w, padding=5, groups=3) - mu_x * mu_x
    syy = F.conv2d(y * y, w, padding=5, groups=3) - mu_y * mu_y
    sxy = F.conv2d(x * y, w, padding=5, groups=3) - mu_x * mu_y
    c1, c2 = 0.01 ** 2, 0.03 ** 2
    s = ((2 * mu_x * mu_y + c1) * (2 * sxy + c2)) / ((mu_x * mu_x + mu_y * mu_y + c1) * (sxx + syy + c2))
    return s.mean()


def loss_fn(image: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
    return (image - target).abs().mean() + 0.2 * (1.0 - ssim(image, target))


def view_settings(cam: sgs_scenes.Camera, device) -> Settings:
    return Settings(cam.w2c.to(device), cam.position.to(device), cam.width, cam.height, cam.focal_x, cam.focal_y,
                    cam.center_x, cam.center_y, cam.near_plane, cam.far_plane, False, 1, False, False, False)


@torch.no_grad()
def render_target(tensors, settings: Settings, spp: int, first_frame: int, samples_per_call: int = 64) -> torch.Tensor:
    """The plain progressive average of `spp` samples (frames first_frame .. first_frame + spp - 1), rendered
    `samples_per_call` at a time (the same bits as one `_C.render` call per sample)."""
    e = torch.empty(0)
    hist = (e, e, e, e)
    dev = tensors[0].device
    n_fb = settings.width * settings.height
    kb = (torch.empty((0, n_fb, 2), dtype=torch.int32, device=dev), torch.empty((0, n_fb, 4), device=dev))
    _C.set_frame_index(first_frame)
    done = 0
    while done < spp:
        n = min(samples_per_call, spp - done)
        hist = _C.render_samples(n, *tensors, *settings.as_tuple(), torch.empty(0, dtype=torch.uint8, device=dev),
                                 *kb, *hist, torch.eye(4, device=dev), 0 if done == 0 else 1)
        done += n
    return hist[0]


def make_problem(n: int = 500_000, views: int = 24, resolution: int = 800, target_spp: int = 1024, seed: int = 0,
                 device="cuda"):
    spec = dataclasses.replace(sgs_scenes.SCENES["train_500k"], n=n)
    scene = sgs_scenes.make_scene(spec, seed=seed)
    g = torch.Generator().manual_seed(seed + 1)
    perturbed = sgs_scenes.Scene(scene.means + torch.randn(scene.means.shape, generator=g) * 0.02, scene.scales,
                                 scene.rotations, scene.opacities,
                                 scene.sh_coefficients + torch.randn(scene.sh_coefficients.shape, generator=g) * 0.1)
    cams = sgs_scenes.orbit_cameras(views, 4.0, resolution, resolution)
    target_tensors = tuple(t.to(device) for t in perturbed.tensors())
    targets = [render_target(target_tensors, view_settings(c, device), target_spp, first_frame=(1 << 24) + 4096 * i)
               for i, c in enumerate(cams)]
    return scene, cams, targets


def train_step(params, settings: Settings, target: torch.Tensor, spp: int = 8, first_frame: int | None = None):
    image, depth, alpha = render_samples(*params, settings, n_samples=spp, first_frame=first_frame)
    loss = loss_fn(image, target)
    loss.backward()
    return loss.detach()
