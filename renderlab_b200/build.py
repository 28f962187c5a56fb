"""Build the engine's shared library, ``renderlab_b200/_lib/librt_trace.so``.

CUDA translation units compile for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
the host builders compile with g++ and ``-ffp-contract=off`` (their f32 arithmetic must round
exactly as the reference writes it). The CUDA runtime is linked statically so the library loads
with nothing but the driver. Objects are rebuilt when a source or header is newer.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "librt_trace.so"
OBJ = PKG / "_build"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
              "--expt-relaxed-constexpr", "-I", str(ROOT / "include")] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-Wextra",
             "-Wno-unused-parameter", "-I", str(ROOT / "include")]

CU_SOURCES = ["rt_api.cu", "kernels_plain.cu", "kernels_fast.cu", "kernels_wide8.cu", "kernels_order.cu", "batches.cu", "serve.cu", "refit.cu", "kernels_cells.cu", "trace_static.cu", "move.cu", "blas_build.cu", "tlas_build.cu", "diag.cu"]
CPP_SOURCES = ["host/blas.cpp", "host/tlas.cpp", "host/pack.cpp", "host/validate.cpp", "host/wide8.cpp", "host/cooked.cpp", "host/wide8_check.cpp"]


def _headers():
    return [p for p in CSRC.rglob("*") if p.suffix in (".h", ".hpp", ".cuh")] + [ROOT / "include" / "rt_trace.h"]


def _stale(obj: Path, src: Path, headers) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in headers)


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(verbose: bool = False, extra_nvcc=()) -> Path:
    OBJ.mkdir(exist_ok=True)
    OUT_DIR.mkdir(exist_ok=True)
    headers = _headers()
    jobs, objs = [], []
    for s in CU_SOURCES:
        src, obj = CSRC / s, OBJ / (Path(s).stem + ".cu.o")
        objs.append(obj)
        if _stale(obj, src, headers):
            jobs.append([NVCC, *NVCC_FLAGS, *extra_nvcc, "-c", str(src), "-o", str(obj)])
    for s in CPP_SOURCES:
        src, obj = CSRC / s, OBJ / (Path(s).stem + ".cpp.o")
        objs.append(obj)
        if _stale(obj, src, headers):
            jobs.append([CXX, *CXX_FLAGS, "-c", str(src), "-o", str(obj)])
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for log in ex.map(_compile, jobs):
            if verbose and log:
                print(log, file=sys.stderr)
    if jobs or not LIB.exists():
        _compile([NVCC, "-shared", *ARCH, "-cudart", "static", "-o", str(LIB), *map(str, objs), "-lpthread"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
