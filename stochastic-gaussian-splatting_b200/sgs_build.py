"""Builds the render path's shared library for sm_100a: StochasticGSCudaBackend/libsgs_b200.so.

Each csrc/*.cu is compiled by nvcc with the reference's numerics flags (-O3 -use_fast_math, which
the bit-exact parity of the winners relies on) plus -lineinfo for profiling, then linked into one
C-ABI shared library (include/sgs_b200.h) with the CUDA runtime linked statically. Objects go to
_build/; the library is written in-tree so that it ships with the package.

    python stochastic-gaussian-splatting_b200/sgs_build.py [-v] [--ptxas-info]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG_ROOT = Path(__file__).resolve().parent
CSRC = PKG_ROOT / "csrc"
BUILD_DIR = PKG_ROOT / "_build"
LIB_PATH = PKG_ROOT / "StochasticGSCudaBackend" / "libsgs_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-use_fast_math", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr"]


def nvcc() -> str:
    found = shutil.which("nvcc")
    if found:
        return found
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    return str(Path(cuda_home) / "bin" / "nvcc")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [
        PKG_ROOT.parent / "include" / "sgs_b200.h", Path(__file__)]


def up_to_date() -> bool:
    if not LIB_PATH.is_file():
        return False
    lib_time = LIB_PATH.stat().st_mtime
    return all(p.stat().st_mtime <= lib_time for p in _deps() if p.is_file())


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> Path:
    if not force and up_to_date():
        return LIB_PATH
    BUILD_DIR.mkdir(exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []

    def compile_one(src: Path) -> tuple[Path, str]:
        obj = BUILD_DIR / (src.stem + ".o")
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-I", str(CSRC), "-I", str(PKG_ROOT.parent / "include"), "-c",
               str(src), "-o", str(obj)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
        return obj, res.stdout + res.stderr

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        results = list(ex.map(compile_one, sources()))
    for _, log in results:
        if verbose and log.strip():
            print(log)
    tmp = LIB_PATH.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(tmp), *(str(o) for o, _ in results)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    path = build(verbose="-v" in sys.argv, ptxas_info="--ptxas-info" in sys.argv, force="--force" in sys.argv)
    print("built", path)
