"""Generates the golden fixtures under tests/golden/ by running the REFERENCE CUDA backend.

Runs on a B200 with the reference built into oracle/_ref/ (oracle/build_ref.py). For every case
it records the reference's own intermediate and final buffers:
  fb          int64 (P_fb,)   packed (depth_bits << 32 | index) winner per (sub)pixel
  samples     f32 (P_fb, 4)   sample_cu's (rgb, depth) per (sub)pixel
  reuse       f32 (P_fb, 4)   spatial-reuse weights (spatial_reuse cases)
  image/depth/alpha/weight_mass   resolve_cu's outputs
  kbuf_prims/kbuf_occl            the k-buffer after the call (spatial_reuse cases)
plus the per-Gaussian projection dump of gs_utils.h:38-193.

Inputs are stored beside the outputs (scene_<name>.npz) so the fixtures do not depend on the
torch RNG of the machine that reads them. Usage:
    python tests/golden/make_golden.py --out <directory>   (then copy the files into tests/golden/)
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "stochastic-gaussian-splatting_b200"))
sys.path.insert(0, str(ROOT))

import sgs_scenes  # noqa: E402
from oracle import build_ref  # noqa: E402

# small scenes: ragged sizes (not multiples of 32 or 256), mixed footprints so that both the
# sequential and the warp-cooperative scatter paths and the hybrid binning all occur
GOLDEN_SCENES = {
    "mixed": (sgs_scenes.SceneSpec(n=1537, log_scale_mean=-2.0, log_scale_std=0.7), 11),
    "large": (sgs_scenes.SceneSpec(n=421, log_scale_mean=-1.3, log_scale_std=0.5, opacity_logit_std=2.0), 12),
    "sh1": (sgs_scenes.SceneSpec(n=777, log_scale_mean=-2.2, log_scale_std=0.6, sh_bases=1), 13),
    "sh4": (sgs_scenes.SceneSpec(n=650, log_scale_mean=-2.2, log_scale_std=0.6, sh_bases=4), 14),
    "sh9": (sgs_scenes.SceneSpec(n=650, log_scale_mean=-2.2, log_scale_std=0.6, sh_bases=9), 15),
}


def golden_camera(width=80, height=60, position=(0.0, 0.0, -4.0)):
    return sgs_scenes.pinhole(position, width, height, 60.0)


def camera_dict(cam: sgs_scenes.Camera) -> dict:
    return dict(width=cam.width, height=cam.height, focal_x=cam.focal_x, focal_y=cam.focal_y,
                center_x=cam.center_x, center_y=cam.center_y, near_plane=cam.near_plane, far_plane=cam.far_plane,
                w2c=cam.w2c.tolist(), position=cam.position.tolist())


# name -> (scene, camera kwargs, flags, frame_idx, use blue noise)
# flags: proper_antialiasing, supersampling_factor, use_gps, hybrid_scheduling
CASES = {
    "st": ("mixed", {}, dict(aa=False, ss=1, gps=False, hybrid=False), 0, False),
    "st_f7": ("mixed", {}, dict(aa=False, ss=1, gps=False, hybrid=False), 7, False),
    "st_aa": ("mixed", {}, dict(aa=True, ss=1, gps=False, hybrid=False), 3, False),
    "st_ss2": ("mixed", {}, dict(aa=False, ss=2, gps=False, hybrid=False), 5, False),
    "st_ss3_odd": ("mixed", dict(width=37, height=23), dict(aa=False, ss=3, gps=False, hybrid=False), 2, False),
    "st_blue": ("mixed", {}, dict(aa=False, ss=1, gps=False, hybrid=False), 70, True),
    "st_large": ("large", {}, dict(aa=False, ss=1, gps=False, hybrid=False), 1, False),
    "st_hybrid": ("large", {}, dict(aa=False, ss=1, gps=False, hybrid=True), 1, False),
    "st_hybrid_ss2_blue": ("large", {}, dict(aa=False, ss=2, gps=False, hybrid=True), 131, True),
    "gps": ("mixed", {}, dict(aa=False, ss=1, gps=True, hybrid=False), 0, False),
    "gps_f9_aa": ("mixed", {}, dict(aa=True, ss=1, gps=True, hybrid=False), 9, False),
    "gps_ss2": ("mixed", {}, dict(aa=False, ss=2, gps=True, hybrid=False), 4, False),
    "gps_large": ("large", {}, dict(aa=False, ss=1, gps=True, hybrid=False), 2, False),
    "gps_hybrid": ("large", {}, dict(aa=False, ss=1, gps=True, hybrid=True), 2, False),
    "gps_hybrid_ss2": ("large", {}, dict(aa=False, ss=2, gps=True, hybrid=True), 6, False),
    "st_sh1": ("sh1", {}, dict(aa=False, ss=1, gps=False, hybrid=False), 0, False),
    "st_sh4": ("sh4", {}, dict(aa=False, ss=1, gps=False, hybrid=False), 0, False),
    "st_sh9": ("sh9", {}, dict(aa=False, ss=1, gps=False, hybrid=False), 0, False),
    "st_offcenter": ("mixed", dict(position=(1.5, -0.7, -3.0)), dict(aa=False, ss=1, gps=False, hybrid=False), 12, False),
}

# progressive sequences: (scene, camera kwargs, flags, spatial_reuse, [(frame_idx, temporal_mode, camera kwargs)])
SEQUENCES = {
    "seq_static_reuse": ("mixed", dict(width=48, height=36), dict(aa=False, ss=1, gps=False, hybrid=False), True,
                         [(20, 0, {}), (21, 1, {}), (22, 1, {}), (23, 2, dict(position=(0.15, 0.0, -4.0)))]),
    "seq_static_plain_ss2": ("mixed", dict(width=40, height=30), dict(aa=False, ss=2, gps=False, hybrid=False), False,
                             [(30, 0, {}), (31, 1, {}), (32, 1, {})]),
    "seq_reproject": ("mixed", dict(width=48, height=36), dict(aa=False, ss=1, gps=True, hybrid=False), False,
                      [(40, 0, {}), (41, 2, dict(position=(0.1, 0.05, -4.0))), (42, 2, dict(position=(0.2, 0.1, -3.9)))]),
    "seq_reuse_ss2_gps": ("large", dict(width=32, height=24), dict(aa=True, ss=2, gps=True, hybrid=True), True,
                          [(50, 0, {}), (51, 1, {}), (52, 2, dict(position=(0.1, 0.0, -4.0)))]),
}


def to_np(t: torch.Tensor) -> np.ndarray:
    return t.detach().cpu().numpy()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory for the new fixtures")
    args = ap.parse_args()
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    _, harness = build_ref.load()
    dev = torch.device("cuda")
    blue = sgs_scenes.synthetic_blue_noise(0)
    blue_d = blue.to(dev)
    empty_u8 = torch.empty(0, dtype=torch.uint8, device=dev)
    scenes = {}
    for name, (spec, seed) in GOLDEN_SCENES.items():
        sc = sgs_scenes.make_scene(spec, seed=seed, morton=False)
        scenes[name] = sc.to(dev)
        np.savez_compressed(out / f"scene_{name}.npz", means=sc.means.numpy(), scales=sc.scales.numpy(),
                            rotations=sc.rotations.numpy(), opacities=sc.opacities.numpy(),
                            sh_coefficients=sc.sh_coefficients.numpy())
    manifest = {"cases": {}, "sequences": {}}

    def cam_args(cam):
        return (cam.width, cam.height, cam.focal_x, cam.focal_y, cam.center_x, cam.center_y, cam.near_plane,
                cam.far_plane)

    for name, (scene_name, cam_kw, fl, frame, use_blue) in CASES.items():
        sc = scenes[scene_name]
        cam = golden_camera(**cam_kw)
        w2c = cam.w2c.to(dev)
        fb = harness.accumulate(sc.means, sc.scales, sc.rotations, sc.opacities, w2c, *cam_args(cam), fl["aa"],
                                fl["ss"], fl["gps"], fl["hybrid"], blue_d if use_blue else empty_u8, frame)
        proj = harness.project(sc.means, sc.scales, sc.rotations, sc.opacities, w2c, *cam_args(cam), fl["aa"], fl["ss"])
        n_fb = fb.numel()
        kp = torch.full((0, n_fb, 2), -1, dtype=torch.int32, device=dev)
        ko = torch.empty((0, n_fb, 4), dtype=torch.float32, device=dev)
        e = torch.empty(0, device=dev)
        samples, reuse, image, depth, alpha, wm = harness.sample_resolve(
            sc.means, sc.scales, sc.rotations, sc.opacities, sc.sh_coefficients, w2c, cam.position.to(dev),
            *cam_args(cam), fl["aa"], fl["ss"], False, fb, kp, ko, e, e, e, e, torch.eye(4, device=dev), 0)
        torch.cuda.synchronize()
        np.savez_compressed(out / f"case_{name}.npz", fb=to_np(fb), samples=to_np(samples), image=to_np(image),
                            depth=to_np(depth), alpha=to_np(alpha), weight_mass=to_np(wm), projection=to_np(proj))
        manifest["cases"][name] = dict(scene=scene_name, camera=camera_dict(cam), flags=fl, frame_idx=frame,
                                       blue_noise=use_blue)
        print("case", name, "winners", int((fb != -1).sum()), "of", n_fb, flush=True)

    for name, (scene_name, cam_kw, fl, reuse_on, steps) in SEQUENCES.items():
        sc = scenes[scene_name]
        cam0 = golden_camera(**cam_kw)
        n_fb = cam0.width * cam0.height * fl["ss"] ** 2
        k = 4 if reuse_on else 0
        kp = torch.full((k, n_fb, 2), -1, dtype=torch.int32, device=dev)
        ko = torch.empty((k, n_fb, 4), dtype=torch.float32, device=dev)
        if reuse_on:
            # deterministic content for the never-read occlusion slots of empty entries
            ko.fill_(0.5)
        hist = [torch.empty(0, device=dev)] * 4
        prev_w2c = cam0.w2c
        rec = {}
        step_meta = []
        for si, (frame, mode, kw) in enumerate(steps):
            cam = golden_camera(**{**cam_kw, **kw})
            w2c = cam.w2c.to(dev)
            v2pv = (prev_w2c.double() @ torch.linalg.inv(cam.w2c.double())).float() if mode == 2 else cam.c2w
            fb = harness.accumulate(sc.means, sc.scales, sc.rotations, sc.opacities, w2c, *cam_args(cam), fl["aa"],
                                    fl["ss"], fl["gps"], fl["hybrid"], empty_u8, frame)
            samples, reuse, image, depth, alpha, wm = harness.sample_resolve(
                sc.means, sc.scales, sc.rotations, sc.opacities, sc.sh_coefficients, w2c, cam.position.to(dev),
                *cam_args(cam), fl["aa"], fl["ss"], reuse_on, fb, kp, ko, *hist, v2pv.to(dev), mode)
            torch.cuda.synchronize()
            rec.update({f"s{si}_fb": to_np(fb), f"s{si}_samples": to_np(samples), f"s{si}_reuse": to_np(reuse),
                        f"s{si}_image": to_np(image), f"s{si}_depth": to_np(depth), f"s{si}_alpha": to_np(alpha),
                        f"s{si}_weight_mass": to_np(wm), f"s{si}_v2pv": to_np(v2pv)})
            step_meta.append(dict(frame_idx=frame, temporal_mode=mode, camera=camera_dict(cam)))
            hist = [image, depth, alpha, wm]
            prev_w2c = cam.w2c
        rec.update({"kbuf_prims": to_np(kp), "kbuf_occl": to_np(ko)})
        np.savez_compressed(out / f"seq_{name}.npz", **rec)
        manifest["sequences"][name] = dict(scene=scene_name, flags=fl, spatial_reuse=reuse_on, steps=step_meta,
                                           kbuf_occl_fill=0.5)
        print("sequence", name, "done", flush=True)

    (out / "manifest.json").write_text(json.dumps(manifest, indent=1))
    print("golden fixtures written to", out)


if __name__ == "__main__":
    main()
