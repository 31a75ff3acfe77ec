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


def built_paths() -> dict[str, Path]:
    return {"C": OUT_DIR / "C" / "_C.so", "harness": OUT_DIR / "harness" / "sgs_ref_harness.so"}


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
    for sub in ("C", "harness"):
        (OUT_DIR / sub).mkdir(parents=True, exist_ok=True)
    cpp_extension.load(name="_C", sources=ref_sources, build_directory=str(OUT_DIR / "C"), **common)
    harness_sources = [str(ORACLE_DIR / "ref_harness.cu")] + [str(SOURCE_DIR / f) for f in KERNEL_FILES]
    cpp_extension.load(name="sgs_ref_harness", sources=harness_sources, build_directory=str(OUT_DIR / "harness"), **common)
    return available()


def load():
    """Imports the prebuilt reference modules; returns (reference _C module, harness module)."""
    import importlib.machinery
    import importlib.util

    import torch  # noqa: F401  (the modules link against torch's libraries)

    if not available():
        raise FileNotFoundError(f"reference oracle not built under {OUT_DIR}")
    mods = []
    for name, path in (("sgs_reference._C", built_paths()["C"]), ("sgs_ref_harness", built_paths()["harness"])):
        if name in sys.modules:
            mods.append(sys.modules[name])
            continue
        loader = importlib.machinery.ExtensionFileLoader(name, str(path))
        spec = importlib.util.spec_from_file_location(name, str(path), loader=loader)
        mod = importlib.util.module_from_spec(spec)
        loader.exec_module(mod)
        sys.modules[name] = mod
        mods.append(mod)
    return tuple(mods)


if __name__ == "__main__":
    ok = build(verbose="-v" in sys.argv)
    print("reference oracle built:" if ok else "reference oracle missing:", OUT_DIR)
    sys.exit(0 if ok else 1)
