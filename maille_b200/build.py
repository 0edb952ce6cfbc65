"""Build recipe of the CUDA library libmaille_gpu.so (sm_100a), in-tree next to this file.

    python -m maille_b200.build          # or: from maille_b200.build import build; build()

nvcc compiles for sm_100a only (-gencode arch=compute_100a,code=sm_100a) with -lineinfo; the
CUDA runtime is linked statically so the library needs nothing but the driver at run time.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = [os.path.join(HERE, "csrc", f) for f in ("setup.cpp", "kernels.cu", "sparse.cu", "persist.cu", "solver.cu", "noalloc.cu",
                                                        "batch_kernels.cu", "batch.cu", "large_strain.cu", "analysis.cu", "memory.cu", "thermal.cu", "ordering.cu")]
HDR = [os.path.join(HERE, "csrc", f) for f in ("common.hpp", "kernels.cuh", "sparse.cuh", "reduce.cuh",
                                                         "cuda_host.hpp", "batch.cuh", "handle.hpp", "analysis.cuh", "tet.cuh", "ordering.cuh")] + [
    os.path.join(HERE, "..", "include", "maille_gpu.h")]
LIB = os.path.join(HERE, "libmaille_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-Xcompiler", "-fPIC,-O2", "-shared", "--expt-relaxed-constexpr"]


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in SRC + HDR)


OBJ_DIR = os.path.join(HERE, "..", "_build", "obj")


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
    cmd = [NVCC, *[f for f in FLAGS if f != "-shared"], "-c", "-o", obj, src]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n" + r.stdout + r.stderr)
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every translation unit (in parallel, one nvcc per file) and links the library."""
    if force or stale():
        from concurrent.futures import ThreadPoolExecutor
        os.makedirs(OBJ_DIR, exist_ok=True)
        with ThreadPoolExecutor(max_workers=min(len(SRC), os.cpu_count() or 1)) as pool:
            objs = list(pool.map(lambda f: _compile(f, verbose), SRC))
        r = subprocess.run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB, *objs],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
