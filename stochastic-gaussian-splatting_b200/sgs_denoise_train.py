"""Learned-resolve workload: training pairs rendered by the plain path, training and evaluation.

Training data: 2000 pairs at 512 x 512 from 6M-Gaussian scenes drawn like the batched-throughput
scene (means U[-10, 10]^3, log-scales N(-4.5, 0.8^2), opacity logits N(0, 2^2), SH degree 3) with
seeds 1..50, 40 random views each (camera 14..30 units from a point within 3 units of the origin,
with the focal length in pixels of the 60-degree 1080p evaluation camera, a 30.6-degree field of
view at 512 x 512, so that Gaussians cover as many pixels as in the evaluated frames). Each pair holds the features of the first 4, 16, 64 and 256 stochastic-
transparency samples and the 1024-sample average as the target. The denoiser trains on random
128 x 128 crops with an MSE loss (Adam), through the BF16 tensor-core kernels; each crop's input
sample count is drawn from the four.

Evaluation: the seed-0 scene at 1920 x 1080 from views on the radius-25 orbit. The ground truth is
the 4096-sample average (frames disjoint from the evaluated ones); plain = the progressive average
of k samples, learned = the denoiser applied to the features of the same k samples, for k in 4, 16,
32, 64, 128, 256. PSNR (peak 1) and SSIM on premultiplied RGB. Equal-PSNR time: the smallest k at which the
learned resolve reaches the PSNR of the plain 256-sample average, and its render + denoise time
against 256 plain samples.

    python stochastic-gaussian-splatting_b200/sgs_denoise_train.py --out weights.npz [--pairs 2000]
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import threading
import time

import numpy as np
import torch
import torch.nn.functional as F

import sgs_scenes
from sgs_train import ssim
from StochasticGSCudaBackend import Settings, _C
from StochasticGSCudaBackend import denoise as dn

SCENE = sgs_scenes.SCENES["batch_6m"]
TRAIN_RES = 512
INPUT_SPP = (4, 16, 64, 256)
TARGET_SPP = 1024
DEPTH_SCALE = 1.0 / 32.0
EVAL_SPP = (4, 16, 32, 64, 128, 256)
# training views use the focal length (in pixels) of the 60-degree 1080p evaluation camera, so that
# Gaussians cover as many pixels in the crops as in the evaluated frames
EVAL_FOCAL = 540.0 / math.tan(math.radians(30.0))
GT_SPP = 4096


def settings_for(cam: sgs_scenes.Camera, device) -> Settings:
    return Settings(cam.w2c.to(device), cam.position.to(device), cam.width, cam.height, cam.focal_x, cam.focal_y,
                    cam.center_x, cam.center_y, cam.near_plane, cam.far_plane, False, 1, False, False, False)


def random_view(gen: torch.Generator, res: int) -> sgs_scenes.Camera:
    d = torch.randn(3, generator=gen, dtype=torch.float64)
    d = d / d.norm()
    radius = 14.0 + 16.0 * float(torch.rand(1, generator=gen, dtype=torch.float64))
    target = (torch.rand(3, generator=gen, dtype=torch.float64) * 6.0 - 3.0)
    pos = target + radius * d
    fov = math.degrees(2.0 * math.atan(0.5 * res / EVAL_FOCAL))
    return sgs_scenes.pinhole(tuple(float(v) for v in pos), res, res, fov, target=tuple(float(v) for v in target))


class _Prefetch:
    """Draws the next scene on the host while the GPU renders the current one."""

    def __init__(self, seeds, n: int | None):
        self.seeds = list(seeds)
        self.n = n
        self.result = None
        self.thread = None

    def _make(self, seed):
        spec = SCENE if self.n is None else dataclasses.replace(SCENE, n=self.n)
        self.result = sgs_scenes.make_scene(spec, seed=seed)

    def start(self, i):
        if i < len(self.seeds):
            self.thread = threading.Thread(target=self._make, args=(self.seeds[i],))
            self.thread.start()

    def get(self):
        self.thread.join()
        return self.result


def make_pairs(n_pairs: int = 2000, seeds=range(1, 51), res: int = TRAIN_RES, input_spp=INPUT_SPP,
               target_spp: int = TARGET_SPP, n_gaussians: int | None = None, device="cuda", log=print):
    """Renders the training pairs: {"features": FP16 [levels, P, H, W, 8], "levels": input_spp,
    "target": FP32 [P, H, W, 3]}."""
    seeds = list(seeds)
    per_scene = [n_pairs // len(seeds) + (1 if i < n_pairs % len(seeds) else 0) for i in range(len(seeds))]
    feats = torch.empty((len(input_spp), n_pairs, res, res, dn.FEATURES), dtype=torch.float16, device=device)
    target = torch.empty((n_pairs, res, res, 3), dtype=torch.float32, device=device)
    pre = _Prefetch(seeds, n_gaussians)
    pre.start(0)
    sampler = None
    p = 0
    t0 = time.time()
    for si, seed in enumerate(seeds):
        scene = pre.get()
        pre.start(si + 1)
        tensors = tuple(t.to(device) for t in scene.tensors())
        gen = torch.Generator().manual_seed(1000 + seed)
        for v in range(per_scene[si]):
            cam = random_view(gen, res)
            if sampler is None:
                sampler = dn.CapturedFeatures(tensors, settings_for(cam, device), DEPTH_SCALE).capture()
            elif v == 0:
                sampler.set_scene(tensors)
            sampler.set_pose(cam.w2c.to(device), cam.position.to(device))
            marks = sampler.run(target_spp, first_frame=(seed * 64 + v) * 2048, checkpoints=tuple(input_spp))
            for li, k in enumerate(input_spp):
                feats[li, p] = marks[k]
            target[p] = sampler.acc.accum[:, :3].view(res, res, 3) / target_spp
            p += 1
        del tensors
        if log:
            torch.cuda.synchronize()
            log(f"scene {seed}: {p} pairs, {time.time() - t0:.1f} s")
    return {"features": feats, "levels": tuple(input_spp), "target": target}


def train(data, iters: int = 4000, batch: int = 16, crop: int = 128, lr: float = 2e-3, seed: int = 0,
          device="cuda", log=print):
    """Adam on the MSE of random crops; the input sample count is drawn per crop from the pairs'."""
    params = [p.requires_grad_(True) for p in dn.init_params(seed, device)]
    opt = torch.optim.Adam(params, lr=lr)
    sched = torch.optim.lr_scheduler.LambdaLR(opt, lambda i: 0.5 * (1 + math.cos(math.pi * min(i, iters) / iters)))
    feats, target = data["features"], data["target"]
    n_levels = feats.shape[0]
    n, res = target.shape[0], target.shape[1]
    gen = torch.Generator(device=device).manual_seed(seed)
    history = []
    t0 = time.time()
    for it in range(iters):
        idx = torch.randint(0, n, (batch,), generator=gen, device=device)
        lvl = torch.randint(0, n_levels, (batch,), generator=gen, device=device)
        ys = torch.randint(0, res - crop + 1, (batch,), generator=gen, device=device)
        xs = torch.randint(0, res - crop + 1, (batch,), generator=gen, device=device)
        rows = (ys[:, None] + torch.arange(crop, device=device))[:, :, None]
        cols = (xs[:, None] + torch.arange(crop, device=device))[:, None, :]
        x = feats[lvl[:, None, None], idx[:, None, None], rows, cols]
        y = target[idx[:, None, None], rows, cols]
        out = dn.denoise_train(x.contiguous(), params)
        loss = F.mse_loss(out, y)
        opt.zero_grad(set_to_none=True)
        loss.backward()
        opt.step()
        sched.step()
        if it % 100 == 0 or it == iters - 1:
            history.append((it, float(loss)))
            if log:
                log(f"iter {it}: loss {float(loss):.6f} ({time.time() - t0:.1f} s)")
    dn.status()
    return [p.detach() for p in params], history


def psnr(a: torch.Tensor, b: torch.Tensor) -> float:
    mse = float(((a.float() - b.float()) ** 2).mean())
    return 10.0 * math.log10(1.0 / mse) if mse > 0 else float("inf")


def _events():
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def time_denoise(model: dn.Denoiser, width: int = 1920, height: int = 1080, reps: int = 20, device="cuda"):
    """Mean ms of one sgs_denoise call on a full frame (inputs resident, after warm-up)."""
    feats = torch.rand((1, height, width, dn.FEATURES), device=device).half()
    out = torch.empty((1, height, width, 3), device=device)
    scratch = torch.empty(dn._lib.sgs_denoise_scratch_size(1, height, width), dtype=torch.uint8, device=device)
    for _ in range(3):
        model(feats, out, scratch)
    s, e = _events()
    torch.cuda.synchronize()
    s.record()
    for _ in range(reps):
        model(feats, out, scratch)
    e.record()
    torch.cuda.synchronize()
    dn.status()
    return s.elapsed_time(e) / reps




def evaluate(model: dn.Denoiser, views: int = 2, width: int = 1920, height: int = 1080, spps=EVAL_SPP,
             gt_spp: int = GT_SPP, n_gaussians: int | None = None, device="cuda", log=print):
    spec = SCENE if n_gaussians is None else dataclasses.replace(SCENE, n=n_gaussians)
    scene = sgs_scenes.make_scene(spec, seed=0)
    tensors = tuple(t.to(device) for t in scene.tensors())
    cams = sgs_scenes.orbit_cameras(views, 25.0, width, height, step_deg=45.0)
    sampler = dn.CapturedFeatures(tensors, settings_for(cams[0], device), DEPTH_SCALE).capture()
    rows = {k: {"plain_psnr": [], "learned_psnr": [], "plain_ssim": [], "learned_ssim": []} for k in spps}
    for vi, cam in enumerate(cams):
        sampler.set_pose(cam.w2c.to(device), cam.position.to(device))
        sampler.run(gt_spp, (1 << 30) + vi * 65536)
        gt = (sampler.acc.accum[:, :3].view(height, width, 3) / gt_spp).clone()
        marks = sampler.run(max(spps), first_frame=(1 << 29) + vi * 65536, checkpoints=tuple(spps))
        for k in spps:
            plain = marks[k][..., :3].float()
            learned = model(marks[k])
            rows[k]["plain_psnr"].append(psnr(plain, gt))
            rows[k]["learned_psnr"].append(psnr(learned, gt))
            rows[k]["plain_ssim"].append(float(ssim(plain, gt)))
            rows[k]["learned_ssim"].append(float(ssim(learned, gt)))
        if log:
            log(f"view {vi}: " + ", ".join(f"{k} spp {rows[k]['plain_psnr'][-1]:.2f}/{rows[k]['learned_psnr'][-1]:.2f} dB"
                                          for k in spps))
    table = {k: {m: float(np.mean(v)) for m, v in r.items()} for k, r in rows.items()}

    # times at this resolution: plain progressive samples (Static), feature samples (Reset +
    # accumulate) and the denoiser
    st = settings_for(cams[0], device)
    e = torch.empty(0)
    n_fb = width * height
    kb = (torch.empty((0, n_fb, 2), dtype=torch.int32, device=device), torch.empty((0, n_fb, 4), device=device))
    bn = torch.empty(0, dtype=torch.uint8, device=device)
    eye = torch.eye(4, device=device)
    hist = (e, e, e, e)
    for i in range(4):
        hist = _C.render(*tensors, *st.as_tuple(), bn, *kb, *hist, eye, 0 if i == 0 else 1)
    s, en = _events()
    torch.cuda.synchronize()
    s.record()
    reps = 64
    for i in range(reps):
        hist = _C.render(*tensors, *st.as_tuple(), bn, *kb, *hist, eye, 1)
    en.record()
    torch.cuda.synchronize()
    plain_ms = s.elapsed_time(en) / reps
    sampler.set_pose(cams[0].w2c.to(device), cams[0].position.to(device))
    s, en = _events()
    s.record()
    sampler.run(reps, first_frame=123456)
    en.record()
    torch.cuda.synchronize()
    feature_ms = s.elapsed_time(en) / reps
    denoise_ms = time_denoise(model, width, height, device=device)

    target_psnr = table[max(spps)]["plain_psnr"]
    reached = [k for k in spps if table[k]["learned_psnr"] >= target_psnr]
    plain_time = max(spps) * plain_ms
    equal = None
    if reached:
        k = min(reached)
        t = k * feature_ms + denoise_ms
        equal = {"spp": k, "ms": t, "plain_ms": plain_time, "fraction": t / plain_time}
    return {"table": table, "plain_ms_per_sample": plain_ms, "feature_ms_per_sample": feature_ms,
            "denoise_ms": denoise_ms, "target_psnr": target_psnr, "equal_psnr": equal,
            "views": views, "width": width, "height": height, "gt_spp": gt_spp}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=2000)
    ap.add_argument("--scenes", type=int, default=50)
    ap.add_argument("--iters", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--target-spp", type=int, default=TARGET_SPP)
    ap.add_argument("--gaussians", type=int, default=None, help="override N (smoke runs)")
    ap.add_argument("--res", type=int, default=TRAIN_RES)
    ap.add_argument("--eval-views", type=int, default=2)
    ap.add_argument("--gt-spp", type=int, default=GT_SPP)
    ap.add_argument("--out", default=None, help="weights .npz")
    ap.add_argument("--report", default=None, help="evaluation .json")
    args = ap.parse_args()
    t0 = time.time()
    data = make_pairs(args.pairs, range(1, args.scenes + 1), res=args.res, target_spp=args.target_spp,
                      n_gaussians=args.gaussians)
    t_data = time.time() - t0
    params, history = train(data, iters=args.iters, batch=args.batch, lr=args.lr)
    t_train = time.time() - t0 - t_data
    del data
    torch.cuda.empty_cache()
    model = dn.Denoiser(params)
    if args.out:
        np.savez(args.out, **model.state())
    report = evaluate(model, views=args.eval_views, gt_spp=args.gt_spp, n_gaussians=args.gaussians)
    report.update({"pairs": args.pairs, "scenes": args.scenes, "iters": args.iters, "batch": args.batch,
                   "target_spp": args.target_spp, "data_s": t_data, "train_s": t_train, "loss": history})
    print(json.dumps({k: v for k, v in report.items() if k != "loss"}, indent=1))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
