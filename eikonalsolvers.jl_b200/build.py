"""Builds libeikcuda.so (sm_100a) in-tree: eikonalsolvers.jl_b200/lib/libeikcuda.so.

The traveltime kernels are compiled with --fmad=false so that every floating-point
operation of the reference's local solver is rounded exactly as in the reference (Julia
contracts no multiply-add unless asked to).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libeikcuda.so")
SOURCES = ["api.cu", "fine.cu", "coarse.cu", "cluster.cu", "adjoint.cu", "noalloc.cu", "smooth.cu", "plan.cu", "rays.cu"]
HEADERS = ["common.cuh", "stencil.cuh", "kernels.cuh", "runtime.hpp", "rounds.cuh", "rays.cuh", "node.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "--fmad=false",
         "-std=c++17", "-Xcompiler", "-fPIC", "--cudart=static", "-Xptxas", "-v"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "eikcuda.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objs = [os.path.join(LIBDIR, src.replace(".cu", ".o")) for src in SOURCES]

    def compile_one(src, obj):
        cmd = [NVCC, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        return src, subprocess.run(cmd, capture_output=True, text=True)

    # the translation units compile independently: one nvcc process each
    with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda so: compile_one(*so), zip(SOURCES, objs)))
    for src, r in results:
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src}")
        if verbose:
            sys.stderr.write(r.stderr)
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "--cudart=static", "-shared",
           "-o", LIB, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link of libeikcuda.so failed")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
