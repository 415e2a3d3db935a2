"""Builds the sm_100a dense library (libdense_b200.so) in-tree with nvcc.

The library is the product's only compute path; it is compiled for
sm_100a (B200) and loaded through ctypes by ``opensfm_b200._lib``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "_build", "libdense_b200.so")
SOURCES = ["kernels.cu", "cleanprune.cu", "learned.cu", "api.cu", "noalloc.cu", "lz4io.cu",
           "fuser.cu", "svo.cu", "acmmp.cu"]
# Per-file flags: the live-path estimator fixes its arithmetic without FMA
# contraction (every operation rounded by itself, as its C oracle, apart
# from the fused multiply-adds its source writes out).
FILE_FLAGS = {"acmmp.cu": ["--fmad=false"]}
HEADERS = ["common.cuh", "kernels.h", "learned.h", "device_guard.h", "cleanprune.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
         "--expt-relaxed-constexpr", "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    """Compiles the sources whose object is older than the source or any
    shared header (all of them in parallel), then links the library."""
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(ROOT, "include", "dense_b200.h")]
    if not force and not _stale(LIB, srcs + headers):
        return LIB
    objs = [os.path.join(os.path.dirname(LIB), os.path.basename(s) + ".o") for s in srcs]

    def compile_one(so):
        s, o = so
        if not force and not _stale(o, [s] + headers):
            return
        cmd = [NVCC, *ARCH, *FLAGS, *FILE_FLAGS.get(os.path.basename(s), []), "-c", s, "-o", o]
        if ptxas_v:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)

    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        list(ex.map(compile_one, zip(srcs, objs)))
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_v="-v" in sys.argv)
    print(LIB)
