"""Builds the reference CUDA backend from its own sources into oracle/_ref/ (test infrastructure).

This is ORACLE infrastructure, never product code. It compiles, for sm_100a and with the
reference's own nvcc flags (StochasticGSCudaBackend/setup.py:79-86: -O3 -use_fast_math, C++17):

  oracle/_ref/C/_C.so                 the reference extension itself: every *.cu of
                                      StochasticGSCudaBackend/StochasticGSCudaBackend/ (setup.py:89-94),
                                      exposing the unmodified `_C.render` and `_C.k_buffer_size`
  oracle/_ref/harness/sgs_ref_harness.so
                                      oracle/ref_harness.cu linked with the reference's kernel files,
                                      exposing the winner framebuffer, the samples and the per-Gaussian
                                      projection that `_C.render` keeps internal
  oracle/_ref/c1/sgs_ref_c1.so        the reference extension with the two caps of the GPS-hybrid
                                      progressive workload changed: max_fragments = 1024 points per
                                      Gaussian (accumulate_hybrid_gps.cu:86 computes W*H/(2 ss^2)) and
                                      max_binned_gaussians = 65536 (accumulate_hybrid_gps.cu:22 holds
                                      2^20). Only those two lines of a build copy of that one file,
                                      written to oracle/_ref/c1/src/, differ; its `render` is otherwise
                                      the unmodified `_C.render`

The reference's own build system (setup.py, which also downloads blue noise) is not run: this
script hands the reference's source files to torch's extension builder directly. The sources are
read in place under /root/reference and nothing is copied into the repository. The build needs
no GPU; the result runs on the B200 as the bit-exact GPU oracle. When the reference tree is absent
(as on a GPU box) the prebuilt files are used as they are.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

REFERENCE_ROOT = Path(os.environ.get("SGS_REFERENCE_ROOT", "/root/reference"))
SOURCE_DIR = REFERENCE_ROOT / "StochasticGSCudaBackend" / "StochasticGSCudaBackend"
ORACLE_DIR = Path(__file__).resolve().parent
OUT_DIR = ORACLE_DIR / "_ref"
KERNEL_FILES = ["accumulate_scatter.cu", "accumulate_hybrid.cu", "accumulate_hybrid_gps.cu", "resolve.cu"]
NVCC_FLAGS = ["-O3", "-use_fast_math", "-std=c++17", "-gencode=arch=compute_100a,code=sm_100a"]
CXX_FLAGS = ["-O3", "-std=c++17"]


# the two lines of accumulate_hybrid_gps.cu that hold the caps, and their values in the c1 build
C1_PATCHES = (
    ("inline constexpr uint32_t max_binned_gaussians = 1u << 20;",
     "inline constexpr uint32_t max_binned_gaussians = 65536u;"),
    ("const uint32_t max_fragments = __float2uint_rn(width * height / (2.0f * supersampling_factor * supersampling_factor));",
     "const uint32_t max_fragments = 1024u;"),
)
C1_MAX_FRAGMENTS = 1024
C1_MAX_BINNED = 65536


def built_paths() -> dict[str, Path]:
    return {"C": OUT_DIR / "C" / "_C.so", "harness": OUT_DIR / "harness" / "sgs_ref_harness.so",
            "c1": OUT_DIR / "c1" / "sgs_ref_c1.so"}


def patched_c1_source() -> Path:
    """Writes the build copy of accumulate_hybrid_gps.cu with the c1 caps to oracle/_ref/c1/src/."""
    text = (SOURCE_DIR / "accumulate_hybrid_gps.cu").read_text()
    for old, new in C1_PATCHES:
        if text.count(old) != 1:
            raise RuntimeError(f"reference line not found exactly once: {old}")
        text = text.replace(old, new)
    out = OUT_DIR / "c1" / "src" / "accumulate_hybrid_gps.cu"
    out.parent.mkdir(parents=True, exist_ok=True)
    if not out.is_file() or out.read_text() != text:
        out.write_text(text)
    return out


def available() -> bool:
    return all(p.is_file() for p in built_paths().values())


def _newest_source_mtime() -> float:
    files = [SOURCE_DIR / f for f in os.listdir(SOURCE_DIR)] + [ORACLE_DIR / "ref_harness.cu", Path(__file__)]
    return max(f.stat().st_mtime for f in files if f.is_file())


def build(verbose: bool = False) -> bool:
    """Compiles both modules when the reference tree is present; returns True when both exist."""
    if not SOURCE_DIR.is_dir():
        return available()
    paths = built_paths()
    if available() and min(p.stat().st_mtime for p in paths.values()) >= _newest_source_mtime():
        return True
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0a")
    os.environ.setdefault("MAX_JOBS", str(os.cpu_count() or 4))
    from torch.utils import cpp_extension

    ref_sources = sorted(str(p) for p in SOURCE_DIR.glob("*.cu"))
    common = dict(
        extra_cflags=CXX_FLAGS,
        extra_cuda_cflags=NVCC_FLAGS,
        extra_include_paths=[str(SOURCE_DIR)],
        verbose=verbose,
        is_python_module=True,
    )
    for sub in ("C", "harness", "c1"):
        (OUT_DIR / sub).mkdir(parents=True, exist_ok=True)
    cpp_extension.load(name="_C", sources=ref_sources, build_directory=str(OUT_DIR / "C"), **common)
    harness_sources = [str(ORACLE_DIR / "ref_harness.cu")] + [str(SOURCE_DIR / f) for f in KERNEL_FILES]
    cpp_extension.load(name="sgs_ref_harness", sources=harness_sources, build_directory=str(OUT_DIR / "harness"), **common)
    c1_sources = [p for p in ref_sources if not p.endswith("accumulate_hybrid_gps.cu")] + [str(patched_c1_source())]
    cpp_extension.load(name="sgs_ref_c1", sources=c1_sources, build_directory=str(OUT_DIR / "c1"), **common)
    return available()


def load():
    """Imports the prebuilt reference modules; returns (reference _C module, harness module)."""
    import torch  # noqa: F401  (the modules link against torch's libraries)

    if not available():
        raise FileNotFoundError(f"reference oracle not built under {OUT_DIR}")
    mods = []
    for name, path in (("sgs_reference._C", built_paths()["C"]), ("sgs_ref_harness", built_paths()["harness"])):
        mods.append(_load_module(name, path))
    return tuple(mods)


def load_c1():
    """Imports the prebuilt reference extension with the GPS-hybrid caps of the progressive workload
    (max_fragments = C1_MAX_FRAGMENTS, max_binned = C1_MAX_BINNED); its `render` is `_C.render`."""
    import torch  # noqa: F401

    if not available():
        raise FileNotFoundError(f"reference oracle not built under {OUT_DIR}")
    return _load_module("sgs_ref_c1", built_paths()["c1"])


def _load_module(name: str, path: Path):
    import importlib.machinery
    import importlib.util

    if name in sys.modules:
        return sys.modules[name]
    loader = importlib.machinery.ExtensionFileLoader(name, str(path))
    spec = importlib.util.spec_from_file_location(name, str(path), loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    sys.modules[name] = mod
    return mod


if __name__ == "__main__":
    ok = build(verbose="-v" in sys.argv)
    print("reference oracle built:" if ok else "reference oracle missing:", OUT_DIR)
    sys.exit(0 if ok else 1)
