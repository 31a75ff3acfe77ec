"""Benchmark of the per-sample stochastic render path: sample-frames/s at 1080p on 6M Gaussians.

One step is one `_C.render` call (one stochastic sample merged progressively, Static resolve) of the
synthetic 6M-Gaussian scene at 1920x1080: stochastic transparency, scatter scheduling, no
supersampling. Inputs are resident in HBM; their 1.43 GB exceed the 126 MB L2, so no flush is done
between steps. Prints one JSON line (see the keys below).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

--impl reference times the reference semantics on the host cores (the C++ restatement in oracle/,
the reference having no CPU path) on the same workload. Multi-GPU runs are independent replicas, one
per rank (the north-star path is single-GPU), timed on the device and reported as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "stochastic-gaussian-splatting_b200"))
sys.path.insert(0, str(ROOT))

import torch  # noqa: E402

import sgs_scenes  # noqa: E402

METRIC = "sample-frames/s at 1080p, 6M Gaussians"


def metric_name(workload: str) -> str:
    """The headline metric for the default workload; the other workloads name their own size."""
    if workload == DEFAULT_WORKLOAD:
        return METRIC
    scene, width, height, _, fl = WORKLOADS[workload]
    return f"sample-frames/s at {width}x{height}{' ss ' + str(fl['ss']) if fl['ss'] > 1 else ''}, {scene} scene"


UNIT = "sample-frames/s"

# name -> (scene, width, height, orbit radius, flags)
WORKLOADS = {
    "batch_6m_1080_st": ("batch_6m", 1920, 1080, 25.0, dict(aa=False, ss=1, gps=False, hybrid=False)),
    "batch_6m_1080_gps": ("batch_6m", 1920, 1080, 25.0, dict(aa=False, ss=1, gps=True, hybrid=False)),
    "batch_6m_4k_st": ("batch_6m", 3840, 2160, 25.0, dict(aa=False, ss=1, gps=False, hybrid=False)),
    "st_100k_640_st": ("st_100k", 640, 480, 4.0, dict(aa=False, ss=1, gps=False, hybrid=False)),
    "gps_1m_720ss2_hybrid": ("gps_1m", 1280, 720, 4.0, dict(aa=False, ss=2, gps=True, hybrid=True)),
}
DEFAULT_WORKLOAD = "batch_6m_1080_st"

# One `ncu --set full` capture of st_scatter_kernel on the default workload: DRAM bytes (read + write)
# and warp instructions of one launch, with the digest of the kernel sources the capture ran. When
# those sources change, the figures no longer describe the kernel: bench then reports them as null
# ("stale") until a new capture replaces them.
SCATTER_SOURCES = ("accumulate_st.cu", "sgs_rows.cuh", "sgs_project.cuh", "sgs_common.cuh", "sgs_internal.h")
NCU_CAPTURE = {
    "batch_6m_1080_st": {"sources_digest": "181952a8e319cca7", "dram_bytes": 278.77e6 + 15.54e6,
                         "warp_instructions": 469.53e6},
}
CSRC = ROOT / "stochastic-gaussian-splatting_b200" / "csrc"


def scatter_sources_digest() -> str:
    import hashlib

    h = hashlib.sha256()
    for name in SCATTER_SOURCES:
        h.update((CSRC / name).read_bytes())
    return h.hexdigest()[:16]


def ncu_capture(workload: str) -> dict | None:
    """The capture's figures for `workload` if they were measured on the current kernel sources."""
    cap = NCU_CAPTURE.get(workload)
    if cap is None or cap["sources_digest"] != scatter_sources_digest():
        return None
    return cap


# measured copy bandwidth and bf16 GEMM rate of this pool's B200s when MEASURED_PEAKS.json is absent
FALLBACK_HBM_GBS = 6650.0
FALLBACK_BF16_TFLOPS = 1590.0

DENOISER_WEIGHTS = ROOT / "stochastic-gaussian-splatting_b200" / "StochasticGSCudaBackend" / "denoiser_c2.npz"


def bf16_peak() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.is_file():
        try:
            return float(json.loads(path.read_text())["bf16_tflops"]), "measured"
        except (KeyError, ValueError):
            pass
    return FALLBACK_BF16_TFLOPS, "fallback"


def hbm_peak() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.is_file():
        try:
            return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region (200 ms period)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        try:
            for line in Path(self.path).read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        finally:
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


class RawEvents:
    """cudaEvent_t handles from the CUDA runtime already loaded by torch, for events that the render
    library records itself (torch only times events it recorded)."""

    def __init__(self):
        import ctypes

        self.ct = ctypes
        self.rt = ctypes.CDLL("libcudart.so.12")
        self.rt.cudaEventCreate.argtypes = [ctypes.POINTER(ctypes.c_void_p)]
        self.rt.cudaEventElapsedTime.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_void_p, ctypes.c_void_p]
        self.rt.cudaEventDestroy.argtypes = [ctypes.c_void_p]
        self.rt.cudaEventRecord.argtypes = [ctypes.c_void_p, ctypes.c_void_p]

    def create(self):
        ev = self.ct.c_void_p()
        if self.rt.cudaEventCreate(self.ct.byref(ev)) != 0:
            raise RuntimeError("cudaEventCreate failed")
        return ev

    def record(self, ev, stream_handle: int):
        if self.rt.cudaEventRecord(ev, self.ct.c_void_p(stream_handle)) != 0:
            raise RuntimeError("cudaEventRecord failed")

    def elapsed_ms(self, start, end) -> float:
        ms = self.ct.c_float()
        if self.rt.cudaEventElapsedTime(self.ct.byref(ms), start, end) != 0:
            raise RuntimeError("cudaEventElapsedTime failed")
        return ms.value

    def destroy(self, ev):
        self.rt.cudaEventDestroy(ev)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    return world, rank, local


def max_over_ranks(value: float, world: int) -> float:
    """The largest of the ranks' values (device time of the slowest replica)."""
    if world == 1:
        return value
    import torch.distributed as dist

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(steps_per_rank: int, world: int, max_elapsed_ms: float) -> float:
    """Whole-job sample-frames/s of `world` independent replicas timed by the slowest one."""
    return world * steps_per_rank / (max_elapsed_ms * 1e-3)


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def make_inputs(name: str):
    scene_name, width, height, radius, flags = WORKLOADS[name]
    scene = sgs_scenes.make_scene(sgs_scenes.SCENES[scene_name], seed=0)
    cam = sgs_scenes.orbit_cameras(1, radius, width, height)[0] if radius != 4.0 else sgs_scenes.front_camera(width, height)
    return scene, cam, flags


def algorithmic_bytes(n: int, n_fb: int, n_px: int, unique_winners: int) -> dict:
    """Bytes a sample-frame must move at least (plain path, Static resolve): Gaussian parameters read
    once (44 B each), framebuffer clear + read (16 B per subpixel), samples written and read (32 B per
    subpixel), history read and outputs written (48 B per pixel), winner means and SH gathered (204 B
    per distinct winner)."""
    accumulate = 44 * n + 8 * n_fb
    frame = 44 * n + 48 * n_fb + 48 * n_px + 204 * unique_winners
    return {"accumulate": accumulate, "frame": frame}


def issue_roofline(workload: str, acc_ms: float, sms: int, max_mhz: float | None) -> dict | None:
    """Warp instructions issued per second by the accumulate stage against the SMs' issue limit (4 warp
    instructions per clock per SM at the maximum SM clock). The count is the scatter kernel's from ncu
    (the queue kernel's few instructions are left out), the time the stage's live CUDA-event time."""
    cap = ncu_capture(workload)
    if cap is None or not max_mhz:
        return None
    instructions = cap["warp_instructions"]
    peak = sms * 4 * max_mhz * 1e6
    achieved = instructions / (acc_ms * 1e-3)
    return {"bound": "issue", "warp_instructions_per_launch": instructions, "achieved": round(achieved / 1e9, 1),
            "peak": round(peak / 1e9, 1), "unit": "G warp instructions/s", "frac": round(achieved / peak, 4),
            "source": "ncu smsp__inst_executed.sum of st_scatter_kernel on the current sources"}


def workload_config(workload: str, n: int, width: int, height: int, fl: dict, world: int, scene_bytes: int) -> dict:
    """The `config` object of both arms' lines: the same keys and values for the same workload."""
    return {
        "workload": f"{workload}: {n} Gaussians, {width}x{height}, supersampling {fl['ss']}, "
                    f"{'GPS' if fl['gps'] else 'stochastic transparency'}, "
                    f"{'hybrid' if fl['hybrid'] else 'scatter'} scheduling, 1 spp per step, Static resolve",
        "gaussians": n, "width": width, "height": height, "supersampling": fl["ss"], "use_gps": fl["gps"],
        "hybrid_scheduling": fl["hybrid"], "spatial_reuse": False, "parallelism": f"replicas x{world}",
        "l2": (f"inputs ({scene_bytes / 1e9:.2f} GB) larger than L2 (126 MB), no flush" if scene_bytes > 126e6
               else f"inputs ({scene_bytes / 1e6:.1f} MB) fit in L2 (126 MB), not flushed"),
    }


def run_ours(args, world, rank, local) -> dict | None:
    from StochasticGSCudaBackend import History, Settings, TemporalMode, _C, render

    dev = torch.device("cuda", local)
    scene_cpu, cam, fl = make_inputs(args.workload)
    scene = scene_cpu.to(dev)
    n = scene.means.shape[0]
    W, H, ss = cam.width, cam.height, fl["ss"]
    n_fb, n_px = W * H * ss * ss, W * H
    w2c = cam.w2c.to(dev)
    pos = cam.position.to(dev)
    empty = torch.empty(0)
    eye = torch.eye(4, device=dev)
    blue = torch.empty(0, dtype=torch.uint8, device=dev)
    kb = (torch.empty((0, n_fb, 2), dtype=torch.int32, device=dev), torch.empty((0, n_fb, 4), device=dev))
    cam_args = (W, H, cam.focal_x, cam.focal_y, cam.center_x, cam.center_y, cam.near_plane, cam.far_plane)
    flag_args = (fl["aa"], ss, fl["gps"], fl["hybrid"], False)

    def step(hist, mode):
        return _C.render(*scene.tensors(), w2c, pos, *cam_args, *flag_args, blue, *kb, *hist, eye, mode)

    stream = torch.cuda.current_stream(dev)
    hist = step((empty,) * 4, 0)
    for _ in range(max(args.warmup, 3)):
        hist = step(hist, 1)
    torch.cuda.synchronize(dev)

    # device-timed region: K steps, accumulate stage bracketed by events on the launching stream
    raw = RawEvents()
    starts = [raw.create() for _ in range(args.steps)]
    ends = [raw.create() for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    props = torch.cuda.get_device_properties(dev)
    clocks = ClockSampler(f"GPU-{props.uuid}" if getattr(props, "uuid", None) else str(local))
    barrier(world)
    torch.cuda.synchronize(dev)
    clocks.start()
    time.sleep(0.3)
    t0.record(stream)
    for k in range(args.steps):
        _C.set_stage_events(starts[k], ends[k])
        hist = step(hist, 1)
    t1.record(stream)
    _C.set_stage_events(None, None)
    torch.cuda.synchronize(dev)
    clock_info = clocks.stop()
    barrier(world)
    elapsed_ms = t0.elapsed_time(t1)
    acc_ms = sum(raw.elapsed_ms(s, e) for s, e in zip(starts, ends)) / args.steps
    for ev in starts + ends:
        raw.destroy(ev)
    elapsed_ms = max_over_ranks(elapsed_ms, world)
    acc_ms = max_over_ranks(acc_ms, world)

    # one more sample for the algorithmic-byte count (distinct winners) and the launch count
    _C.set_frame_index(_C.get_frame_index())
    (_, _, _, _), ws, layout = _C.render_with_workspace(*scene.tensors(), w2c, pos, *cam_args, *flag_args, blue, *kb,
                                                       *hist, eye, 1)
    fb = _C.workspace_views(ws, layout, n_fb, False)["framebuffer"]
    winners = fb[fb != -1]
    unique = int(torch.unique(winners & 0xFFFFFFFF).numel())
    alg = algorithmic_bytes(n, n_fb, n_px, unique)
    launches_per_step = 2 + (2 if not fl["gps"] else (2 if fl["hybrid"] else 1))

    # end to end through the public API: each step copies the camera in from pinned host memory,
    # renders, and reads the image back into pinned host memory; the read-back runs on a second
    # stream so that it overlaps the next step's render (as a streaming viewer would), and the timed
    # region ends only when the last image has arrived in host memory
    settings_host = (cam.w2c.pin_memory(), cam.position.pin_memory())
    w2c_e = torch.empty_like(w2c)
    pos_e = torch.empty_like(pos)
    image_host = [torch.empty((H, W, 3), dtype=torch.float32).pin_memory() for _ in range(2)]
    copy_stream = torch.cuda.Stream(dev)
    k_buffer = kb
    hist_e = History(*hist)

    def e2e_step(k):
        nonlocal hist_e
        w2c_e.copy_(settings_host[0], non_blocking=True)
        pos_e.copy_(settings_host[1], non_blocking=True)
        settings = Settings(w2c_e, pos_e, W, H, cam.focal_x, cam.focal_y, cam.center_x, cam.center_y,
                            cam.near_plane, cam.far_plane, fl["aa"], ss, fl["gps"], fl["hybrid"], False)
        hist_e = render(*scene.tensors(), settings, k_buffer, hist_e, eye, TemporalMode.STATIC)
        copy_stream.wait_stream(stream)
        with torch.cuda.stream(copy_stream):
            image_host[k % 2].copy_(hist_e.image, non_blocking=True)
        hist_e.image.record_stream(copy_stream)

    for i in range(3):
        e2e_step(i)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    for k in range(args.steps):
        e2e_step(k)
    stream.wait_stream(copy_stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
    h2d = w2c.numel() * 4 + pos.numel() * 4
    d2h = H * W * 3 * 4

    # opt-in preactivated layout (covariance and opacity sigmoid once per model; the same bits)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    pre = _C.preactivate(scene.scales, scene.rotations, scene.opacities)
    p1.record(stream)
    for _ in range(3):
        hist = _C.render(*scene.tensors(), w2c, pos, *cam_args, *flag_args, blue, *kb, *hist, eye, 1, preactivated=pre)
    torch.cuda.synchronize(dev)
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    for _ in range(args.steps):
        hist = _C.render(*scene.tensors(), w2c, pos, *cam_args, *flag_args, blue, *kb, *hist, eye, 1, preactivated=pre)
    q1.record(stream)
    torch.cuda.synchronize(dev)
    pre_ms = q0.elapsed_time(q1) / args.steps
    preactivated = {"ms_per_sample": round(pre_ms, 5), "sample_frames_per_s": round(1000.0 / pre_ms, 2),
                    "preactivate_ms_once": round(p0.elapsed_time(p1), 4), "bytes": pre.numel() * 4}
    del pre

    # opt-in quantised layout (16-byte records and half SH; the images differ by the quantisation)
    qz = _C.quantize(*scene.tensors())
    for _ in range(3):
        hist = _C.render(*scene.tensors(), w2c, pos, *cam_args, *flag_args, blue, *kb, *hist, eye, 1, quantized=qz)
    torch.cuda.synchronize(dev)
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    for _ in range(args.steps):
        hist = _C.render(*scene.tensors(), w2c, pos, *cam_args, *flag_args, blue, *kb, *hist, eye, 1, quantized=qz)
    q1.record(stream)
    torch.cuda.synchronize(dev)
    q_ms = q0.elapsed_time(q1) / args.steps
    quantized = {"ms_per_sample": round(q_ms, 5), "sample_frames_per_s": round(1000.0 / q_ms, 2),
                 "layout_bytes": qz.nbytes(), "float32_bytes": scene_cpu.nbytes(),
                 "accumulate_algorithmic_bytes_per_launch": 16 * n + qz.chunks.numel() * 4 + 8 * n_fb,
                 "note": "records of 16 B per Gaussian and half SH; statistical parity with float32 "
                         "(tests/test_gpu_quantized.py)"}
    del qz

    if rank != 0:
        return None
    peak, peak_kind = hbm_peak()
    scene_bytes = scene_cpu.nbytes()
    achieved = alg["accumulate"] / (acc_ms * 1e-3) / 1e9
    capture = ncu_capture(args.workload)
    traffic = capture["dram_bytes"] if capture else None
    ms_per_step = elapsed_ms / args.steps
    value = replica_throughput(args.steps, world, elapsed_ms)
    line = {
        "metric": metric_name(args.workload),
        "value": round(value, 2),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": f"synthetic (seeded {n}-Gaussian scene drawn as the {args.workload} workload; no dataset)",
        "config": workload_config(args.workload, n, W, H, fl, world, scene_bytes),
        "roofline": {
            "bound": "hbm",
            "kernel": "accumulate stage (st_scatter_kernel + st_queue_kernel)" if not fl["gps"] else "accumulate stage (gps kernels)",
            "achieved": round(achieved, 1),
            "peak": peak,
            "peak_source": f"{peak_kind} hbm_gbs",
            "unit": "GB/s",
            "frac": round(achieved / peak, 4),
            "traffic": traffic,
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of st_scatter_kernel, one launch, "
                               "captured on the current sources") if capture else
                              "no capture of the current kernel sources (stale figures are not reported)",
            "algorithmic_bytes_per_launch": alg["accumulate"],
            "accumulate_ms": round(acc_ms, 5),
            "issue": issue_roofline(args.workload, acc_ms, torch.cuda.get_device_properties(dev).multi_processor_count,
                                    clock_info.get("sm_max_mhz")),
            "frame": {"algorithmic_bytes": alg["frame"], "achieved_gbs": round(alg["frame"] / (ms_per_step * 1e-3) / 1e9, 1),
                      "frac": round(alg["frame"] / (ms_per_step * 1e-3) / 1e9 / peak, 4),
                      "unique_winners": unique},
        },
        "e2e": {"value": round(replica_throughput(args.steps, world, e2e_ms), 2), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clock_info,
    }
    line["preactivated"] = preactivated
    line["quantized"] = quantized
    if not fl["gps"]:
        line["samples_per_call"] = samples_per_call(scene, cam, fl, dev, n_samples=8, calls=max(4, args.steps // 8))
    if not args.no_batch and args.workload.startswith("batch_6m"):
        line["camera_path"] = camera_path_fps(scene, fl, dev, spp=8)
    if not args.no_batch and args.workload.startswith("batch_6m"):
        line["batch32_graph"] = {
            "stochastic_transparency": batch_graph(scene, dict(fl, gps=False), dev, steps=max(4, args.steps // 8)),
            "gps": batch_graph(scene, dict(fl, gps=True), dev, steps=max(4, args.steps // 8)),
        }
    if not args.no_reference_cuda and args.workload.startswith("batch_6m"):
        # the reference's own CUDA backend on this scene and camera, in this process (a baseline leg)
        line["reference_cuda"] = {
            "stochastic_transparency": reference_cuda_baseline(scene, cam, dict(fl, gps=False), dev),
            "gps": reference_cuda_baseline(scene, cam, dict(fl, gps=True), dev),
        }
        # the small-scene configuration (100k Gaussians at 640x480), where the per-call host work of
        # the bindings weighs as much as the kernels
        s_c0, cam_c0, fl_c0 = make_inputs("st_100k_640_st")
        line["reference_cuda"]["c0_st_100k_640"] = reference_cuda_baseline(s_c0.to(dev), cam_c0, fl_c0, dev, calls=64)
        del s_c0
    if not (args.no_train and args.no_learned) and args.workload.startswith("batch_6m"):
        del scene
        torch.cuda.empty_cache()
    if not args.no_learned and args.workload == "batch_6m_1080_st":
        line["learned_resolve"] = learned_resolve_measure(dev)
        torch.cuda.empty_cache()
    if not args.no_train and args.workload.startswith("batch_6m"):
        line["train_step"] = train_measure(dev)
    if not args.no_progressive and args.workload.startswith("batch_6m"):
        line["progressive_gps_hybrid"] = progressive_measure(dev, reference=not args.no_reference_cuda)
        torch.cuda.empty_cache()
    probe = atomic_probe(dev)
    line["atomics"] = {"probe": probe}
    if not args.no_cpu_baseline:
        line["cpu_baseline"], counts = cpu_baseline(scene_cpu, cam, fl, args.cpu_frames, args.workload)
        # fragments evaluated (the reference's clipped-AABB count for stochastic transparency, points
        # for GPS) and atomics issued per sample-frame, counted by the CPU restatement over the
        # baseline's frames (other frame indices than the timed ones: the same expectation)
        acc_s = acc_ms * 1e-3
        line["atomics"].update({
            "fragments_per_sample_frame": round(counts["fragments"]),
            "issued_per_sample_frame": round(counts["accepted"]),
            "fragments_per_s": round(counts["fragments"] / acc_s, 0),
            "issued_per_s": round(counts["accepted"] / acc_s, 0),
            "frac_of_probe_rows": round(counts["accepted"] / acc_s / probe["rows_per_s"], 4),
            "counts_source": f"CPU restatement, mean of {args.cpu_frames} frames; rates over the accumulate stage",
        })
    return line


def learned_resolve_measure(dev) -> dict:
    """The learned resolve on the 6M scene at 1920x1080 with the committed weights: one sgs_denoise
    call timed with CUDA events (six tensor-core conv launches) against the bf16 tensor peak and
    HBM; PSNR / SSIM of learned and plain resolves at 4, 16, 64 and 256 samples against a
    4096-sample ground truth (one orbit view); the equal-PSNR time against 256 plain samples."""
    import numpy as np

    import sgs_denoise_train
    from StochasticGSCudaBackend import denoise as dn

    trained = DENOISER_WEIGHTS.is_file()
    model = dn.Denoiser.from_state(np.load(DENOISER_WEIGHTS), device=dev) if trained else dn.Denoiser(device=dev)
    rep = sgs_denoise_train.evaluate(model, views=1, log=None, device=dev)
    px = 1920 * 1080
    flops = 2 * 9 * sum(ci * co for ci, co in dn.LAYERS) * px
    # per pixel: features read twice (layer 1, residual) 32 B, five activations written and read
    # back 5 x 128 B, RGB out 12 B
    hbm_bytes = (32 + 5 * 128 + 12) * px
    ms = rep["denoise_ms"]
    peak, src = bf16_peak()
    hpeak, _ = hbm_peak()
    tflops = flops / (ms * 1e-3) / 1e12
    gbs = hbm_bytes / (ms * 1e-3) / 1e9
    return {
        "weights": "trained (denoiser_c2.npz)" if trained else "untrained (plain average)",
        "denoise_ms_1080p": round(ms, 4),
        "roofline": {"bound": "hbm", "kernels": "conv3x3_tma_kernel x5 + conv3x3_kernel (layer 1)",
                     "achieved": round(gbs, 1), "peak": hpeak, "unit": "GB/s", "frac": round(gbs / hpeak, 4),
                     "algorithmic_bytes_per_call": hbm_bytes,
                     "tensor": {"achieved_tflops": round(tflops, 1), "peak_tflops": peak, "peak_source": src,
                                "frac": round(tflops / peak, 4), "flops_per_call": flops}},
        "psnr_db": {k: {"plain": round(v["plain_psnr"], 3), "learned": round(v["learned_psnr"], 3)}
                    for k, v in rep["table"].items()},
        "ssim": {k: {"plain": round(v["plain_ssim"], 4), "learned": round(v["learned_ssim"], 4)}
                 for k, v in rep["table"].items()},
        "plain_ms_per_sample": round(rep["plain_ms_per_sample"], 4),
        "feature_ms_per_sample": round(rep["feature_ms_per_sample"], 4),
        "equal_psnr": rep["equal_psnr"],
        "ground_truth_spp": rep["gt_spp"],
    }


def train_measure(dev, views: int = 24, target_spp: int = 1024, steps_per_view: int = 2) -> dict:
    """Differentiable training step of the 500k-Gaussian 800x800 workload: 24 orbit views whose targets
    are 1024-sample renders of a perturbed copy of the scene; per step 8 samples forward, L1 + 0.2
    (1 - SSIM), hand-written backward to all parameters, Adam update."""
    import sgs_train

    t_targets = time.perf_counter()
    scene, cams, targets = sgs_train.make_problem(views=views, target_spp=target_spp, device=dev)
    torch.cuda.synchronize(dev)
    t_targets = time.perf_counter() - t_targets
    params = [t.to(dev).requires_grad_(True) for t in scene.tensors()]
    opt = torch.optim.Adam(params, lr=1e-3)
    settings = [sgs_train.view_settings(c, dev) for c in cams]
    losses = []
    # warm-up (allocations, autotuning of torch's conv) then timed steps
    for i in range(views):
        opt.zero_grad(set_to_none=True)
        losses.append(float(sgs_train.train_step(params, settings[i], targets[i])))
        opt.step()
    torch.cuda.synchronize(dev)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = views * steps_per_view
    t0.record()
    last = []
    for k in range(n):
        opt.zero_grad(set_to_none=True)
        last.append(sgs_train.train_step(params, settings[k % views], targets[k % views]))
        opt.step()
    t1.record()
    torch.cuda.synchronize(dev)
    ms = t0.elapsed_time(t1) / n
    return {"gaussians": int(scene.means.shape[0]), "resolution": "800x800", "spp_per_step": 8,
            "views": views, "target_spp": target_spp, "target_render_s": round(t_targets, 2),
            "ms_per_step": round(ms, 3), "steps_per_s": round(1000.0 / ms, 2),
            "loss_first_epoch": round(sum(losses) / len(losses), 5),
            "loss_last_epoch": round(float(sum(last[-views:]) / views), 5)}


def samples_per_call(scene, cam, fl, dev, n_samples: int, calls: int) -> dict:
    """The same workload with `n_samples` samples per call (`_C.render_samples`: one fragment walk and
    one resolve pass for all of them, outputs equal to one call per sample), Static mode."""
    from StochasticGSCudaBackend import _C

    W, H, ss = cam.width, cam.height, fl["ss"]
    n_fb = W * H * ss * ss
    kb = (torch.empty((0, n_fb, 2), dtype=torch.int32, device=dev), torch.empty((0, n_fb, 4), device=dev))
    e = torch.empty(0)
    args = lambda hist, mode: (*scene.tensors(), cam.w2c.to(dev), cam.position.to(dev), W, H, cam.focal_x,
                               cam.focal_y, cam.center_x, cam.center_y, cam.near_plane, cam.far_plane, fl["aa"], ss,
                               fl["gps"], fl["hybrid"], False, torch.empty(0, dtype=torch.uint8, device=dev), *kb,
                               *hist, torch.eye(4, device=dev), mode)
    hist = _C.render_samples(n_samples, *args((e, e, e, e), 0))
    for _ in range(2):
        hist = _C.render_samples(n_samples, *args(hist, 1))
    stream = torch.cuda.current_stream(dev)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    t0.record(stream)
    for _ in range(calls):
        hist = _C.render_samples(n_samples, *args(hist, 1))
    t1.record(stream)
    torch.cuda.synchronize(dev)
    ms = t0.elapsed_time(t1) / (calls * n_samples)
    return {"samples_per_call": n_samples, "ms_per_sample": round(ms, 5),
            "sample_frames_per_s": round(1000.0 / ms, 1)}


def camera_path_fps(scene, fl, dev, spp: int, n_views: int = 16, iterations: int = 3) -> dict:
    """The reference's FPS harness (Trainer.py:79-120: warm-up pass, then passes with a device
    synchronisation around every frame) over 16 orbit views at 1920x1080, each frame `spp` samples
    with the frame logic of Renderer.py:48-103 (sgs_viewer.ProgressiveRenderer; moving views reset)."""
    import sgs_viewer

    views = [sgs_viewer.View.from_camera(c, frame_idx=i)
             for i, c in enumerate(sgs_scenes.orbit_cameras(n_views, 25.0, 1920, 1080))]
    out = {"views": n_views, "resolution": "1920x1080", "samples_per_pixel": spp, "iterations": iterations,
           "timing": "perf_counter with a device synchronisation around every frame (Trainer.py:97-106)"}
    for graphs in (False, True):
        r = sgs_viewer.ProgressiveRenderer(*scene.tensors(), supersampling_factor=fl["ss"], use_gps=fl["gps"],
                                           hybrid_scheduling=fl["hybrid"], samples_per_pixel=spp, graphs=graphs)
        res = sgs_viewer.benchmark_camera_path(r, views, iterations=iterations)
        out["graphs" if graphs else "eager"] = {"avg_fps": round(res["avg_fps"], 2), "avg_ms": round(res["avg_ms"], 4)}
        del r
    # the reference-facing figures: eager frames, as the plugin renders them
    out["avg_fps"], out["avg_ms"] = out["eager"]["avg_fps"], out["eager"]["avg_ms"]
    return out


def batch_graph(scene, fl, dev, steps: int) -> dict:
    """32 views cycling 720p, 1080p, 1440p and 4K on the orbit, one sample each, captured in CUDA
    graphs (the batched-throughput workload; each render split over an accumulate and a resolve
    stream, histories ping-ponged); also the same step without the graphs."""
    import sgs_batch

    res = [(1280, 720), (1920, 1080), (2560, 1440), (3840, 2160)]
    views = sgs_batch.batch_views(32, 25.0, res)
    batch = sgs_batch.CapturedViews(scene.tensors(), views, fl, first_frame=1 << 20, device=dev).capture()
    for _ in range(2):
        batch.replay()
    stream = torch.cuda.current_stream(dev)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    t0.record(stream)
    for _ in range(steps):
        batch.replay()
    t1.record(stream)
    torch.cuda.synchronize(dev)
    graph_ms = t0.elapsed_time(t1) / steps
    for _ in range(2):
        batch.eager_step()
    torch.cuda.synchronize(dev)
    t0.record(stream)
    for _ in range(steps):
        batch.eager_step()
    t1.record(stream)
    torch.cuda.synchronize(dev)
    eager_ms = t0.elapsed_time(t1) / steps
    pixels = sum(w * h for w, h in res) * 8
    del batch
    torch.cuda.empty_cache()
    return {"views": 32, "resolutions": "1280x720, 1920x1080, 2560x1440, 3840x2160 (8 each)",
            "ms_per_batch_graph": round(graph_ms, 4), "ms_per_batch_eager": round(eager_ms, 4),
            "sample_frames_per_s_graph": round(32 / (graph_ms * 1e-3), 1),
            "megapixels_per_s_graph": round(pixels / (graph_ms * 1e-3) / 1e6, 1)}


def reference_cuda_baseline(scene, cam, fl, dev, calls: int = 32, rounds: int = 2) -> dict:
    """The reference's own CUDA backend, its unmodified `_C.render` built from its sources into
    oracle/_ref/C, on the same scene, camera, flags and Static loop as this library's `_C.render`, in
    this process on this GPU. A baseline leg like `cpu_baseline`: the measured path never touches it.
    CUDA events around `calls` calls after 4 warm-up calls; the two implementations alternate for
    `rounds` rounds and each keeps its fastest round."""
    from oracle import build_ref

    if not build_ref.available():
        return {"unavailable": "the reference extension was not built under oracle/_ref (oracle/build_ref.py)"}
    from StochasticGSCudaBackend import _C

    ref_C, _ = build_ref.load()
    W, H, ss = cam.width, cam.height, fl["ss"]
    n_fb = W * H * ss * ss
    kb = (torch.empty((0, n_fb, 2), dtype=torch.int32, device=dev), torch.empty((0, n_fb, 4), device=dev))
    e = torch.empty(0)
    w2c, pos, eye = cam.w2c.to(dev), cam.position.to(dev), torch.eye(4, device=dev)
    blue = torch.empty(0, dtype=torch.uint8, device=dev)

    def args(hist, mode):
        return (*scene.tensors(), w2c, pos, W, H, cam.focal_x, cam.focal_y, cam.center_x, cam.center_y,
                cam.near_plane, cam.far_plane, fl["aa"], ss, fl["gps"], fl["hybrid"], False, blue, *kb, *hist, eye,
                mode)

    stream = torch.cuda.current_stream(dev)

    def timed(render) -> float:
        hist = render(*args((e, e, e, e), 0))
        for _ in range(4):
            hist = render(*args(hist, 1))
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        t0.record(stream)
        for _ in range(calls):
            hist = render(*args(hist, 1))
        t1.record(stream)
        torch.cuda.synchronize(dev)
        return t0.elapsed_time(t1) / calls

    ref_ms, our_ms = [], []
    for _ in range(rounds):
        ref_ms.append(timed(ref_C.render))
        our_ms.append(timed(_C.render))
    r, o = min(ref_ms), min(our_ms)
    return {"implementation": "reference _C.render built from its sources (oracle/_ref/C), same process and GPU",
            "workload": f"{scene.means.shape[0]} Gaussians, {W}x{H}, ss {ss}, {'GPS' if fl['gps'] else 'ST'}, "
                        f"{'hybrid' if fl['hybrid'] else 'scatter'}, Static",
            "calls": calls, "rounds": rounds, "reference_ms_per_sample": round(r, 5), "ours_ms_per_sample": round(o, 5),
            "reference_sample_frames_per_s": round(1000.0 / r, 2), "ours_sample_frames_per_s": round(1000.0 / o, 2),
            "ratio": round(r / o, 3), "same_box": True}


def progressive_measure(dev, views: int = 16, spp: int = 16, reference: bool = True) -> dict:
    """The GPS-hybrid progressive workload: 1M Gaussians with heavy-tailed footprints (log-scales
    N(-3, 1^2)), 1280x720 with supersampling 2, GPS with hybrid scheduling capped at 1024 points per
    Gaussian and 65,536 queued Gaussians, 16 orbit views at radius 4, 16 samples per view: the first
    sample of a view in Reproject (Reset for the first view), the others Static, spatial reuse on
    (Renderer.py:74-97). One untimed pass over the first view, then all 256 samples timed with CUDA
    events per call; the sample/resolve passes of each Reproject sample timed from the event the
    library records after its accumulate stage. The reference arm runs the same loop on the
    reference extension built with those two caps (oracle/build_ref.py)."""
    from StochasticGSCudaBackend import _C

    W, H, ss = 1280, 720, 2
    max_fragments, max_binned = 1024, 65536
    scene = sgs_scenes.make_scene(sgs_scenes.SCENES["gps_1m"], seed=0).to(dev)
    cams = sgs_scenes.orbit_cameras(views, 4.0, W, H)
    n_fb, n_px = W * H * ss * ss, W * H
    e = torch.empty(0)
    blue = torch.empty(0, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    cam_t = [(c.w2c.to(dev), c.position.to(dev)) for c in cams]
    v2pv = [torch.eye(4, device=dev)] + [
        (cams[i - 1].w2c.double() @ torch.linalg.inv(cams[i].w2c.double())).float().to(dev) for i in range(1, views)]

    def args(v, kb, hist, mode):
        c = cams[v]
        return (*scene.tensors(), *cam_t[v], W, H, c.focal_x, c.focal_y, c.center_x, c.center_y, c.near_plane,
                c.far_plane, False, ss, True, True, True, blue, *kb, *hist, v2pv[v], mode)

    raw = RawEvents()

    def run(render, kwargs, timed: bool, n_views: int, stage_events: bool):
        kb = (torch.full((4, n_fb, 2), -1, dtype=torch.int32, device=dev), torch.zeros((4, n_fb, 4), device=dev))
        hist = (e, e, e, e)
        marks = []
        for v in range(n_views):
            for s in range(spp):
                mode = (0 if v == 0 else 2) if s == 0 else 1
                if timed:
                    ev = [raw.create() for _ in range(4)]  # call start, accumulate start/end, call end
                    if stage_events:
                        _C.set_stage_events(ev[1], ev[2])
                    raw.record(ev[0], stream.cuda_stream)
                hist = render(*args(v, kb, hist, mode), **kwargs)
                if timed:
                    raw.record(ev[3], stream.cuda_stream)
                    marks.append((mode, ev))
        _C.set_stage_events(None, None)
        torch.cuda.synchronize(dev)
        if not timed:
            return None
        mean = lambda xs: sum(xs) / len(xs)
        rep = [ev for mode, ev in marks if mode == 2]
        out = {"ms_per_sample": mean([raw.elapsed_ms(ev[0], ev[3]) for _, ev in marks]),
               "reproject_ms_per_sample": mean([raw.elapsed_ms(ev[0], ev[3]) for ev in rep])}
        if stage_events:
            out["accumulate_ms"] = mean([raw.elapsed_ms(ev[1], ev[2]) for _, ev in marks])
            out["reproject_resolve_ms"] = mean([raw.elapsed_ms(ev[2], ev[3]) for ev in rep])
            out["static_resolve_ms"] = mean([raw.elapsed_ms(ev[2], ev[3]) for mode, ev in marks if mode == 1])
        for _, ev in marks:
            for x in ev:
                raw.destroy(x)
        return out

    kwargs = dict(max_fragments=max_fragments, max_binned=max_binned)
    run(_C.render, kwargs, timed=False, n_views=1, stage_events=False)
    ours = run(_C.render, kwargs, timed=True, n_views=views, stage_events=True)
    # distinct winners of one sample of the second view, for the algorithmic bytes of the sample and
    # resolve passes: per framebuffer subpixel the winner key 8, samples written and read 32, reuse
    # weights written and read 32, the k-buffer (4 entries of 24 B) read and rewritten 192; per pixel
    # the Reproject history read 20 and the outputs written 24; per distinct winner its geometry
    # re-projected 44 and its mean and SH 204 (the means counted once: 236)
    kb = (torch.full((4, n_fb, 2), -1, dtype=torch.int32, device=dev), torch.zeros((4, n_fb, 4), device=dev))
    _, ws, layout = _C.render_with_workspace(*args(1, kb, (e, e, e, e), 0), **kwargs)
    fb = _C.workspace_views(ws, layout, n_fb, True)["framebuffer"]
    unique = int(torch.unique(fb[fb != -1] & 0xFFFFFFFF).numel())
    del ws, fb, kb
    resolve_bytes = 264 * n_fb + 44 * n_px + 236 * unique
    peak, peak_kind = hbm_peak()
    gbs = resolve_bytes / (ours["reproject_resolve_ms"] * 1e-3) / 1e9
    result = {
        "workload": f"1M heavy-tailed Gaussians, {W}x{H} ss {ss}, GPS hybrid (max_fragments {max_fragments}, "
                    f"max_binned {max_binned}), spatial reuse, {views} orbit views x {spp} samples, Reproject "
                    f"between views, Static within a view",
        "ms_per_sample": round(ours["ms_per_sample"], 4),
        "sample_frames_per_s": round(1000.0 / ours["ms_per_sample"], 2),
        "reproject_ms_per_sample": round(ours["reproject_ms_per_sample"], 4),
        "accumulate_ms": round(ours["accumulate_ms"], 4),
        "static_resolve_ms": round(ours["static_resolve_ms"], 4),
        "reproject_resolve": {"ms": round(ours["reproject_resolve_ms"], 4), "algorithmic_bytes": resolve_bytes,
                              "unique_winners": unique, "achieved_gbs": round(gbs, 1), "peak": peak,
                              "peak_source": f"{peak_kind} hbm_gbs", "frac": round(gbs / peak, 4)},
    }
    if reference:
        from oracle import build_ref

        if build_ref.available():
            ref_c1 = build_ref.load_c1()
            run(ref_c1.render, {}, timed=False, n_views=1, stage_events=False)
            theirs = run(ref_c1.render, {}, timed=True, n_views=views, stage_events=False)
            result["reference_cuda"] = {
                "implementation": "reference _C.render built from its sources with the workload's two caps "
                                  "(oracle/_ref/c1), same process and GPU",
                "ms_per_sample": round(theirs["ms_per_sample"], 4),
                "reproject_ms_per_sample": round(theirs["reproject_ms_per_sample"], 4),
                "ratio": round(theirs["ms_per_sample"] / ours["ms_per_sample"], 3), "same_box": True}
        else:
            result["reference_cuda"] = {"unavailable": "the reference extension was not built under oracle/_ref"}
    del scene
    return result


def cpu_baseline(scene_cpu, cam, fl, frames: int, workload: str) -> tuple[dict, dict]:
    """The C++ restatement of the reference path (oracle/) on all host cores, a bounded sample."""
    from oracle import cpu

    threads = len(os.sched_getaffinity(0))
    sc = {k: t.numpy() for k, t in zip(("means", "scales", "rotations", "opacities", "sh_coefficients"),
                                       scene_cpu.tensors())}
    cd = dict(width=cam.width, height=cam.height, focal_x=cam.focal_x, focal_y=cam.focal_y, center_x=cam.center_x,
              center_y=cam.center_y, near_plane=cam.near_plane, far_plane=cam.far_plane, w2c=cam.w2c.numpy(),
              position=cam.position.numpy())
    hist = None
    fb = cpu.accumulate(sc, cd, fl, 0, threads=threads)  # warm-up (page-in, thread pool)
    counts = {"fragments": 0, "accepted": 0}
    t = time.perf_counter()
    for f in range(frames):
        fb, st = cpu.accumulate(sc, cd, fl, f + 1, threads=threads, return_stats=True)
        out = cpu.sample_resolve(sc, cd, fl, fb, history=hist, temporal_mode=1 if hist else 0, threads=threads)
        hist = (out["image"], out["depth"], out["alpha"], out["weight_mass"])
        counts["fragments"] += st["fragments"]
        counts["accepted"] += st["accepted"]
    dt = time.perf_counter() - t
    line = {"value": round(frames / dt, 4), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{frames} sample-frames of {workload} (accumulate + sample + resolve), {dt:.1f} s"}
    per_frame = {k: v / max(frames, 1) for k, v in counts.items()}
    return line, per_frame


def atomic_probe(dev, slots_log2: int = 21, ops: int = 256, launches: int = 5) -> dict:
    """red.min.u64 reductions per second of the library's probe kernel (sgs_probe_atomic_min) into
    2^21 u64 slots (16.8 MB, L2-resident like the 1080p framebuffer), 8 blocks of 256 threads per SM,
    for both access patterns; CUDA events around `launches` launches after two warm-up launches."""
    from StochasticGSCudaBackend import _C

    slots = torch.full((1 << slots_log2,), -1, dtype=torch.int64, device=dev)
    blocks = torch.cuda.get_device_properties(dev).multi_processor_count * 8
    stream = torch.cuda.current_stream(dev)
    out = {"slots": 1 << slots_log2, "blocks": blocks, "threads_per_block": 256, "ops_per_thread": ops}
    for name, pattern in (("random", 0), ("rows", 1)):
        for _ in range(2):
            _C.probe_atomic_min(slots, ops, blocks, pattern, seed=7)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        t0.record(stream)
        issued = sum(_C.probe_atomic_min(slots, ops, blocks, pattern, seed=k) for k in range(launches))
        t1.record(stream)
        torch.cuda.synchronize(dev)
        out[f"{name}_per_s"] = round(issued / (t0.elapsed_time(t1) * 1e-3), 0)
    return out


def run_reference(args, world, rank) -> dict | None:
    if rank != 0:
        return None
    scene_cpu, cam, fl = make_inputs(args.workload)
    from oracle import cpu

    threads = len(os.sched_getaffinity(0))
    sc = {k: t.numpy() for k, t in zip(("means", "scales", "rotations", "opacities", "sh_coefficients"),
                                       scene_cpu.tensors())}
    cd = dict(width=cam.width, height=cam.height, focal_x=cam.focal_x, focal_y=cam.focal_y, center_x=cam.center_x,
              center_y=cam.center_y, near_plane=cam.near_plane, far_plane=cam.far_plane, w2c=cam.w2c.numpy(),
              position=cam.position.numpy())
    hist = None
    frame = 0

    def one():
        nonlocal hist, frame
        fb = cpu.accumulate(sc, cd, fl, frame, threads=threads)
        out = cpu.sample_resolve(sc, cd, fl, fb, history=hist, temporal_mode=1 if hist else 0, threads=threads)
        hist = (out["image"], out["depth"], out["alpha"], out["weight_mass"])
        frame += 1

    for _ in range(max(args.warmup, 1)):
        one()
    t = time.perf_counter()
    for _ in range(args.steps):
        one()
    dt = time.perf_counter() - t
    value = args.steps / dt
    return {
        "metric": metric_name(args.workload), "value": round(value, 4), "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": f"synthetic (seeded {int(scene_cpu.means.shape[0])}-Gaussian scene drawn as the {args.workload} "
                "workload; no dataset)",
        "config": workload_config(args.workload, int(scene_cpu.means.shape[0]), cam.width, cam.height, fl, world,
                                  scene_cpu.nbytes()),
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full sample-frames of {args.workload}: the C++ restatement of the "
                                   f"reference kernels (the reference has no CPU path)"},
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def ncu_case(name: str) -> dict:
    """Short fixed sequences for one-GPU ncu captures of kernels the default line does not reach in a
    few launches. c1_progressive: 1M heavy-tailed Gaussians at 1280x720 ss 2, GPS hybrid with the
    workload's caps, spatial reuse, 2 orbit views x 3 samples (Reset, Static, Static, Reproject,
    Static, Static); launches per sample: clear, gps_scatter, gps_queue, reuse_sample, tile_resolve.
    denoise_1080: 4 calls of the 6-layer denoiser on one 1920x1080 feature image (6 conv launches
    each)."""
    from StochasticGSCudaBackend import _C

    dev = torch.device("cuda", 0)
    if name == "denoise_1080":
        from StochasticGSCudaBackend import denoise

        g = torch.Generator(device="cpu").manual_seed(0)
        feat = (torch.rand((1, 1080, 1920, 8), generator=g) * 0.8).to(torch.float16).to(dev)
        dn = denoise.Denoiser(device=dev, seed=0)
        out = None
        for _ in range(4):
            out = dn(feat, out=out)
        torch.cuda.synchronize()
        denoise.status(dev)
        return {"ncu_case": name, "mean": round(float(out.mean()), 6)}
    w, h, ss = 1280, 720, 2
    scene = sgs_scenes.make_scene(sgs_scenes.SCENES["gps_1m"], seed=0).to(dev)
    cams = sgs_scenes.orbit_cameras(16, 4.0, w, h)
    n_fb = w * h * ss * ss
    kb = (torch.full((4, n_fb, 2), -1, dtype=torch.int32, device=dev), torch.zeros((4, n_fb, 4), device=dev))
    e = torch.empty(0)
    hist = (e, e, e, e)
    blue = torch.empty(0, dtype=torch.uint8, device=dev)
    for v in range(2):
        c = cams[v]
        v2pv = ((cams[v - 1].w2c.double() @ torch.linalg.inv(c.w2c.double())).float().to(dev) if v
                else torch.eye(4, device=dev))
        for sm in range(3):
            mode = (0 if v == 0 else 2) if sm == 0 else 1
            hist = _C.render(*scene.tensors(), c.w2c.to(dev), c.position.to(dev), w, h, c.focal_x, c.focal_y,
                             c.center_x, c.center_y, c.near_plane, c.far_plane, False, ss, True, True, True, blue,
                             *kb, *hist, v2pv, mode, max_fragments=1024, max_binned=65536)
    torch.cuda.synchronize()
    return {"ncu_case": name, "alpha_mean": round(float(hist[2].mean()), 6)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--cpu-frames", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 32-view CUDA-graph measurement")
    ap.add_argument("--no-train", action="store_true", help="skip the differentiable training-step measurement")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-resolve measurement")
    ap.add_argument("--no-progressive", action="store_true",
                    help="skip the GPS-hybrid progressive workload (16 views x 16 samples, reuse, Reproject)")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip the timing of the reference's own CUDA backend in this process")
    ap.add_argument("--ncu-case", choices=["c1_progressive", "denoise_1080"],
                    help="run one short fixed sequence for an ncu capture and exit")
    args = ap.parse_args()
    if args.ncu_case:
        print(json.dumps(ncu_case(args.ncu_case)), flush=True)
        return
    if args.impl == "reference":
        # reference semantics on the host cores; no GPU work, no process group needed
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        line = run_reference(args, world, rank)
    else:
        world, rank, local = dist_setup()
        line = run_ours(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
