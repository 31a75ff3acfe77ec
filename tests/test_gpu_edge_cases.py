"""Edge cases of the render path on the GPU, against the reference built here (oracle/_ref).

* Ragged image sizes (not multiples of the 32 x 8-pixel resolve tiles, supersampling 1-3) through a
  progressive sequence with spatial reuse and Reproject between views, in ST, GPS and GPS hybrid: the
  four outputs and the k-buffer bitwise equal to the reference's own `_C.render` after every sample.
* The empty scene in every mode (scatter, hybrid, ST, GPS, spatial reuse, Reproject, several samples
  per call): background everywhere, the k-buffer untouched.
* The frame indices just below the 32-bit wrap (the seeds multiply and add the index modulo 2^32):
  winner framebuffers bitwise equal to the reference harness's, white and blue noise, ST and GPS.
"""
import numpy as np
import pytest
import torch

import sgs_scenes
from oracle import build_ref
from sgs_testing import assert_bitwise, reference_render

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    return build_ref.load()


# (width, height, supersampling, use_gps, hybrid_scheduling), spatial reuse on
RAGGED = [(97, 61, 1, False, False), (45, 23, 2, True, True), (33, 17, 3, False, False), (129, 9, 2, True, False),
          (61, 37, 2, False, True)]


@pytest.mark.parametrize("width,height,ss,gps,hybrid", RAGGED)
def test_ragged_sizes_progressive_bitwise(ref, width, height, ss, gps, hybrid, cuda_device):
    from StochasticGSCudaBackend import _C

    ref_C, _ = ref
    dev = cuda_device
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=20_000, log_scale_mean=-3.0, log_scale_std=0.8), 11).to(dev)
    cams = sgs_scenes.orbit_cameras(8, 4.0, width, height, step_deg=3.0)
    n_fb = width * height * ss * ss
    kb_ref = (torch.full((4, n_fb, 2), -1, dtype=torch.int32, device=dev), torch.zeros((4, n_fb, 4), device=dev))
    kb_our = (kb_ref[0].clone(), kb_ref[1].clone())
    e = torch.empty(0)
    h_ref = h_our = (e, e, e, e)
    prev = None
    step = 0
    for v, cam in enumerate(cams[:3]):
        for s in range(3):
            mode = (0 if prev is None else 2) if s == 0 else 1
            v2pv = (prev.w2c.double() @ torch.linalg.inv(cam.w2c.double())).float() if mode == 2 else torch.eye(4)

            def args(kb, h):
                return (*scene.tensors(), cam.w2c.to(dev), cam.position.to(dev), width, height, cam.focal_x,
                        cam.focal_y, cam.center_x, cam.center_y, cam.near_plane, cam.far_plane, False, ss, gps, hybrid,
                        True, torch.empty(0, dtype=torch.uint8, device=dev), *kb, *h, v2pv.to(dev), mode)

            frame, h_ref = reference_render(ref_C, *args(kb_ref, h_ref))
            _C.set_frame_index(frame)
            h_our = _C.render(*args(kb_our, h_our))
            torch.cuda.synchronize()
            tag = f"{width}x{height} ss {ss} gps {gps} hybrid {hybrid} step {step} (mode {mode})"
            for name, a, b in zip(("image", "depth", "alpha", "weight_mass"), h_our, h_ref):
                assert_bitwise(f"{tag} {name}", a.cpu().numpy(), b.cpu().numpy())
            assert_bitwise(f"{tag} k-buffer entries", kb_our[0].cpu().numpy(), kb_ref[0].cpu().numpy())
            assert_bitwise(f"{tag} k-buffer occlusion", kb_our[1].cpu().numpy(), kb_ref[1].cpu().numpy())
            step += 1
        prev = cam
    assert float(h_our[2].mean()) > 0.05


def test_empty_scene_in_every_mode(cuda_device):
    """N = 0: every mode renders the background (image 0, alpha 0, depth 0) and leaves the k-buffer as it
    was; several samples per call too."""
    from StochasticGSCudaBackend import _C

    dev = cuda_device
    e = torch.empty(0)
    zero = (torch.zeros((0, 3), device=dev), torch.zeros((0, 3), device=dev), torch.zeros((0, 4), device=dev),
            torch.zeros((0,), device=dev), torch.zeros((0, 16, 3), device=dev))
    width, height = 45, 23
    cams = sgs_scenes.orbit_cameras(4, 4.0, width, height, step_deg=5.0)
    for gps in (False, True):
        for hybrid in (False, True):
            for reuse in (False, True):
                for ss in (1, 2):
                    n_fb = width * height * ss * ss
                    k = 4 if reuse else 0
                    kb = (torch.full((k, n_fb, 2), -1, dtype=torch.int32, device=dev),
                          torch.zeros((k, n_fb, 4), device=dev))
                    hist = (e, e, e, e)
                    prev = None
                    for i, mode in enumerate((0, 1, 2, 1)):
                        cam = cams[i]
                        v2pv = ((prev.w2c.double() @ torch.linalg.inv(cam.w2c.double())).float() if mode == 2
                                else torch.eye(4))
                        args = (*zero, cam.w2c.to(dev), cam.position.to(dev), width, height, cam.focal_x, cam.focal_y,
                                cam.center_x, cam.center_y, cam.near_plane, cam.far_plane, False, ss, gps, hybrid,
                                reuse, torch.empty(0, dtype=torch.uint8, device=dev), *kb, *hist, v2pv.to(dev), mode)
                        hist = _C.render_samples(3, *args) if i == 3 else _C.render(*args)
                        prev = cam
                    torch.cuda.synchronize()
                    img, depth, alpha, wm = hist
                    tag = f"gps {gps} hybrid {hybrid} reuse {reuse} ss {ss}"
                    assert float(img.abs().sum()) == 0.0 and float(alpha.abs().sum()) == 0.0, tag
                    assert float(depth.abs().sum()) == 0.0, tag
                    assert bool(torch.isfinite(wm).all()) and float(wm.min()) > 0.0, tag
                    if reuse:
                        assert bool((kb[0] == -1).all()) and float(kb[1].abs().sum()) == 0.0, tag


@pytest.mark.parametrize("frame", [0xFFFFFFFE, 0xFFFFFFFF])
def test_frames_at_the_32_bit_wrap(ref, frame, cuda_device):
    """The seeds of every mode combine the frame index modulo 2^32; the last two indices before the wrap
    give the reference harness's winners (white and blue noise, ST scatter and hybrid, GPS scatter and
    hybrid)."""
    from sgs_testing import render_once

    _, harness = ref
    dev = cuda_device
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=30_000, log_scale_mean=-3.0, log_scale_std=0.8), 4)
    sd = scene.to(dev)
    cam = sgs_scenes.orbit_cameras(1, 4.0, 160, 96)[0]
    cd = dict(width=cam.width, height=cam.height, focal_x=cam.focal_x, focal_y=cam.focal_y, center_x=cam.center_x,
              center_y=cam.center_y, near_plane=cam.near_plane, far_plane=cam.far_plane, w2c=cam.w2c.tolist(),
              position=cam.position.tolist())
    sc = {k: t for k, t in zip(("means", "scales", "rotations", "opacities", "sh_coefficients"), sd.tensors())}
    blue = sgs_scenes.synthetic_blue_noise(3)
    for gps, hybrid, use_blue in ((False, False, False), (False, False, True), (False, True, False),
                                  (True, False, False), (True, True, False)):
        flags = dict(aa=False, ss=2, gps=gps, hybrid=hybrid)
        bn = blue.to(dev) if use_blue else torch.empty(0, dtype=torch.uint8, device=dev)
        want = harness.accumulate(sd.means, sd.scales, sd.rotations, sd.opacities, cam.w2c.to(dev), cam.width,
                                  cam.height, cam.focal_x, cam.focal_y, cam.center_x, cam.center_y, cam.near_plane,
                                  cam.far_plane, False, 2, gps, hybrid, bn, frame)
        torch.cuda.synchronize()
        want = want.cpu().numpy()
        got = render_once(sc, cd, flags, frame, blue_noise=blue if use_blue else None)["fb"]
        assert (want != -1).any()
        assert_bitwise(f"frame {frame:#x} gps {gps} hybrid {hybrid} blue {use_blue}", got, want)


def _extreme_scene(dev):
    """Duplicated Gaussians (equal depth keys, the index decides) and extreme parameters: opacity logits
    of +-12, log-scales from -7 (sub-pixel) to +1 (covering the image), means straddling the near plane."""
    base = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=3000, log_scale_mean=-2.5, log_scale_std=1.5), 21)
    g = torch.Generator().manual_seed(22)
    m, s, r, o, sh = (t.clone() for t in base.tensors())
    o[:300] = 12.0
    o[300:600] = -12.0
    s[600:700] = -7.0
    s[700:720] = 1.0
    m[720:800, 2] = -4.0 + 0.2 + torch.rand(80, generator=g) * 0.01  # near the camera's near plane (z = -4 + 0.2)
    dup = slice(800, 1400)
    m2, s2, r2, o2, sh2 = (torch.cat([t, t[dup]]) for t in (m, s, r, o, sh))
    return sgs_scenes.Scene(m2, s2, r2, o2, sh2).to(dev)


@pytest.mark.parametrize("gps,hybrid", [(False, False), (False, True), (True, False), (True, True)])
def test_collisions_and_extreme_parameters_bitwise(ref, gps, hybrid, cuda_device):
    """Equal depth keys resolve to the lower index and extreme opacities, scales and near-plane means are
    culled, clamped and binned as the reference does: outputs and k-buffer bitwise over Reset, Static and
    Reproject with spatial reuse (supersampling 2)."""
    from StochasticGSCudaBackend import _C

    ref_C, _ = ref
    dev = cuda_device
    scene = _extreme_scene(dev)
    width, height, ss = 96, 64, 2
    cams = sgs_scenes.orbit_cameras(8, 4.0, width, height, step_deg=4.0)
    n_fb = width * height * ss * ss
    kb_ref = (torch.full((4, n_fb, 2), -1, dtype=torch.int32, device=dev), torch.zeros((4, n_fb, 4), device=dev))
    kb_our = (kb_ref[0].clone(), kb_ref[1].clone())
    e = torch.empty(0)
    h_ref = h_our = (e, e, e, e)
    prev = cams[0]
    for i, mode in enumerate((0, 1, 2, 1)):
        cam = cams[1] if i >= 2 else cams[0]
        v2pv = (prev.w2c.double() @ torch.linalg.inv(cam.w2c.double())).float() if mode == 2 else torch.eye(4)

        def args(kb, h):
            return (*scene.tensors(), cam.w2c.to(dev), cam.position.to(dev), width, height, cam.focal_x, cam.focal_y,
                    cam.center_x, cam.center_y, cam.near_plane, cam.far_plane, False, ss, gps, hybrid, True,
                    torch.empty(0, dtype=torch.uint8, device=dev), *kb, *h, v2pv.to(dev), mode)

        frame, h_ref = reference_render(ref_C, *args(kb_ref, h_ref))
        _C.set_frame_index(frame)
        h_our = _C.render(*args(kb_our, h_our))
        torch.cuda.synchronize()
        tag = f"gps {gps} hybrid {hybrid} step {i}"
        for name, a, b in zip(("image", "depth", "alpha", "weight_mass"), h_our, h_ref):
            assert_bitwise(f"{tag} {name}", a.cpu().numpy(), b.cpu().numpy())
        assert_bitwise(f"{tag} k-buffer entries", kb_our[0].cpu().numpy(), kb_ref[0].cpu().numpy())
        prev = cam
    assert float(h_our[2].mean()) > 0.05
