"""Build recipe for libgpufft_b200.so (nvcc, sm_100a, in-tree).

``python -m gpu_fft_b200.build`` compiles every CUDA source of the library
into ``gpu_fft_b200/libgpufft_b200.so``.  nvcc cross-compiles for sm_100a
without a GPU present, so this runs on build hosts too.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgpufft_b200.so")

SOURCES = ["gpufft.cu", "fast_f32.cu", "fast_f64.cu", "noalloc.cu", "batch.cu", "s16.cu", "serve.cu", "dist.cu", "fast_f32_3s.cu", "hostpipe.cu", "fast_queue.cu"]
HEADERS = ["fft_kernels.cuh", "fft_radix.cuh", "fft_fast.cuh", "fft_s16.cuh", "fft_queue.cuh", "fast_registry.h", "fast_entries.h", "gpufft_internal.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _inputs() -> list[str]:
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files.append(os.path.join(ROOT, "include", "gpufft_b200.h"))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile each source to an object in parallel, then link the library."""
    if not force and up_to_date():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    procs, objs = [], []
    for f in SOURCES:
        obj = os.path.join(objdir, f.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [nvcc(), *ARCH, *FLAGS, "-c", "-o", obj, os.path.join(CSRC, f)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        procs.append((f, subprocess.Popen(cmd)))
    failed = [f for f, p in procs if p.wait() != 0]
    if failed:
        raise RuntimeError(f"nvcc failed on {failed}")
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart", "-ldl"], check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
