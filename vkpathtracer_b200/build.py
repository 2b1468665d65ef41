"""Builds libvkpt_cuda.so in-tree for sm_100a with nvcc (no JIT, no torch extension).

Every translation unit is compiled with -fmad=false and IEEE division and
square root: the render path reproduces the reference CPU tracer's float
results, which an x86-64 build computes without fused multiply-adds.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "libvkpt_cuda.so")
SOURCES = ["kernels.cu", "batch.cu", "batch_loop.cu", "adjoint.cu", "context.cu", "bvh_build.cu", "bvh_host.cpp"]
HEADERS = ["bvh_layout.h", "common.cuh", "traverse.cuh", "kernels.cuh", "integrator.cuh", "batch.cuh", "bvh_host.h", "adjoint.cuh",
           "adjoint_launch.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-Xcompiler", "-fPIC,-O2",
         "-Xptxas", "-v"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "vkptc.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(LIB_DIR, os.path.splitext(src)[0] + ".o")
        cmd = [NVCC] + FLAGS + ["-I", os.path.join(HERE, "..", "include"), "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cpp"):
            cmd = [NVCC, "-x", "cu"] + cmd[1:]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed for {src}")
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    tmp = LIB + ".tmp"
    # --no-undefined: a symbol no object defines fails the build instead of the first dlopen
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xlinker", "--no-undefined", "-o", tmp] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link failed")
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
