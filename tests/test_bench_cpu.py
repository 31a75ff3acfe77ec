"""bench.py's bookkeeping on the CPU: the algorithmic-byte model, whole-job throughput, the workload
table and the argument defaults the driver relies on (no GPU work)."""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["bench_under_test"] = mod
    spec.loader.exec_module(mod)
    return mod


def test_algorithmic_bytes_of_the_headline(bench):
    # 6M Gaussians at 1920x1080, no supersampling: 44 B per Gaussian + 8 B per framebuffer pixel for the
    # accumulate stage; the frame adds the samples, history, outputs and the winners' SH
    n, n_fb, n_px, u = 6_000_000, 1920 * 1080, 1920 * 1080, 442_933
    alg = bench.algorithmic_bytes(n, n_fb, n_px, u)
    assert alg["accumulate"] == 280_588_800
    assert alg["frame"] == 44 * n + 48 * n_fb + 48 * n_px + 204 * u == 553_423_932


def test_replica_throughput_counts_every_rank(bench):
    assert bench.replica_throughput(64, 1, 37.76) == pytest.approx(64 / 0.03776)
    assert bench.replica_throughput(64, 8, 37.76) == pytest.approx(8 * 64 / 0.03776)


def test_workloads_and_defaults(bench):
    assert bench.DEFAULT_WORKLOAD == "batch_6m_1080_st"
    for name, (scene, w, h, radius, flags) in bench.WORKLOADS.items():
        assert scene in __import__("sgs_scenes").SCENES
        assert w > 0 and h > 0 and radius > 0
        assert set(flags) == {"aa", "ss", "gps", "hybrid"}
    assert bench.WORKLOADS["batch_6m_1080_st"][1:3] == (1920, 1080)


def test_peaks_fall_back_without_the_measured_file(bench, tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.hbm_peak() == (bench.FALLBACK_HBM_GBS, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text('{"hbm_gbs": 6541.5, "bf16_tflops": 1657.2}')
    assert bench.hbm_peak() == (6541.5, "measured")
    assert bench.bf16_peak() == (1657.2, "measured")


def test_issue_roofline(bench, monkeypatch):
    monkeypatch.setitem(bench.NCU_CAPTURE, "batch_6m_1080_st",
                        {"sources_digest": bench.scatter_sources_digest(), "dram_bytes": 1.0,
                         "warp_instructions": 467.5e6})
    r = bench.issue_roofline("batch_6m_1080_st", 0.512, 148, 1965.0)
    assert r["bound"] == "issue" and r["peak"] == pytest.approx(148 * 4 * 1.965, rel=1e-3)
    assert r["frac"] == pytest.approx(467.5e6 / 0.512e-3 / (148 * 4 * 1965e6), rel=1e-3)
    assert bench.issue_roofline("batch_6m_1080_st", 0.512, 148, None) is None
    assert bench.issue_roofline("st_100k_640_st", 0.1, 148, 1965.0) is None


def test_capture_of_other_kernel_sources_is_not_reported(bench, monkeypatch):
    """ncu figures measured on other scatter-kernel sources are stale: bench reports none of them."""
    monkeypatch.setitem(bench.NCU_CAPTURE, "batch_6m_1080_st",
                        {"sources_digest": "0" * 16, "dram_bytes": 1.0, "warp_instructions": 1.0})
    assert bench.ncu_capture("batch_6m_1080_st") is None
    assert bench.issue_roofline("batch_6m_1080_st", 0.512, 148, 1965.0) is None


def test_both_arms_describe_the_workload_alike(bench):
    """The ours and reference lines build `config` from the same function and arguments."""
    import inspect

    src = inspect.getsource(bench.run_ours) + inspect.getsource(bench.run_reference)
    assert src.count("workload_config(") == 2
    fl = bench.WORKLOADS["batch_6m_1080_st"][4]
    cfg = bench.workload_config("batch_6m_1080_st", 6_000_000, 1920, 1080, fl, 1, 1_440_000_000)
    assert cfg["supersampling"] == 1 and cfg["use_gps"] is False and cfg["hybrid_scheduling"] is False
    assert "larger than L2" in cfg["l2"]
