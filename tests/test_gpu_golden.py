"""Bit-exact parity of the B200 kernels with the reference CUDA backend's golden outputs.

Every case and sequence in tests/golden/ was produced by the reference's own kernels on a B200
(tests/golden/make_golden.py). The B200 path must reproduce the packed winner framebuffer, the
samples, the reuse weights, the k-buffer and all four outputs bit for bit: same inputs, same
frame index, same intrinsics under -use_fast_math.
"""
import numpy as np
import pytest

import golden_data as gd
from sgs_testing import assert_bitwise, mismatch_report, render_once

pytestmark = pytest.mark.gpu

CASES = sorted(gd.manifest()["cases"])
SEQUENCES = sorted(gd.manifest()["sequences"])


@pytest.mark.parametrize("name", CASES)
def test_case_bitwise(name, cuda_device):
    meta = gd.manifest()["cases"][name]
    want = gd.case(name)
    got = render_once(gd.scene(meta["scene"]), meta["camera"], meta["flags"], meta["frame_idx"],
                      blue_noise=gd.blue_noise() if meta["blue_noise"] else None)
    reports = [mismatch_report(k, got[k], want[k])
               for k in ("fb", "samples", "image", "depth", "alpha", "weight_mass")]
    reports = [r for r in reports if r]
    assert not reports, f"{name}: " + "; ".join(reports)


@pytest.mark.parametrize("name", SEQUENCES)
def test_sequence_bitwise(name, cuda_device):
    import torch

    meta = gd.manifest()["sequences"][name]
    want = gd.sequence(name)
    scene = gd.scene(meta["scene"])
    reuse = meta["spatial_reuse"]
    history = None
    k_buffer = None
    for si, step in enumerate(meta["steps"]):
        got = render_once(scene, step["camera"], meta["flags"], step["frame_idx"], temporal_mode=step["temporal_mode"],
                          history=history, k_buffer=k_buffer, v2pv=want[f"s{si}_v2pv"], spatial_reuse=reuse)
        keys = ["fb", "samples", "image", "depth", "alpha", "weight_mass"] + (["reuse"] if reuse else [])
        reports = [mismatch_report(f"step{si}.{k}", got[k], want[f"s{si}_{k}"]) for k in keys]
        reports = [r for r in reports if r]
        assert not reports, f"{name}: " + "; ".join(reports)
        history = got["outputs"]
        k_buffer = got["k_buffer"]
    if reuse:
        assert_bitwise("kbuf_prims", k_buffer[0].cpu().numpy(), want["kbuf_prims"])
        assert_bitwise("kbuf_occl", k_buffer[1].cpu().numpy(), want["kbuf_occl"])
    torch.cuda.synchronize()


def test_projection_matches_winner_depths(cuda_device):
    """Winner keys carry the reference projection's depth bits: decode and cross-check."""
    meta = gd.manifest()["cases"]["st"]
    want = gd.case("st")
    fb = want["fb"]
    proj = want["projection"]
    hit = fb != -1
    idx = (fb[hit] & 0xFFFFFFFF).astype(np.int64)
    depth_bits = (fb[hit] >> 32).astype(np.uint32)
    assert np.array_equal(proj[idx, 1].view(np.uint32), depth_bits)
    got = render_once(gd.scene(meta["scene"]), meta["camera"], meta["flags"], meta["frame_idx"])
    assert_bitwise("fb", got["fb"], fb)
