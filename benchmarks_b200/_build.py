"""Builds libd3d_b200.so in-tree with nvcc for sm_100a.

    python -m benchmarks_b200._build [--force] [--ptxas-v]

Objects go to benchmarks_b200/_build/, the library to
benchmarks_b200/libd3d_b200.so (both git-ignored; the .so ships with the
source tree to wherever it runs).  The CUDA runtime is linked statically, so
the library loads without a GPU or driver present (it resolves the driver
entry points it needs at run time).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libd3d_b200.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# The host compiler must carry the C++ runtime; prefer the system one.
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17",
    # No multiply-add contraction anywhere: the stencil must round every
    # product and sum like the reference's CPU build.
    "-fmad=false",
    "-Xcompiler", "-fPIC,-O3,-Wall",
    "-ccbin", HOST_CXX,
    "-I" + INCLUDE, "-I" + CSRC,
]

SOURCES = ["d3d_step.cu", "d3d_step2d.cu", "d3d_tb.cu", "d3d_tb2.cu",
           "d3d_norm.cu",
           "d3d_batch.cu", "d3d_pitched.cu", "d3d_resident.cu", "d3d_serve.cu", "d3d_io.cu", "d3d_slab.cu", "d3d_api.cu"]
HEADERS = ["d3d_common.cuh", "d3d_kernels.h", "d3d_march.cuh"]


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else -1.0


def _compile(src, obj, extra):
    cmd = [NVCC] + NVCC_FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, r.stdout + r.stderr


def build(force: bool = False, ptxas_verbose: bool = False,
          quiet: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, h) for h in HEADERS]
    deps.append(os.path.join(INCLUDE, "d3d_b200.h"))
    dep_time = max(_mtime(d) for d in deps)
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    jobs = []
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s.replace(".cu", ".o"))
        objs.append(obj)
        if force or ptxas_verbose or _mtime(obj) < max(_mtime(src), dep_time):
            jobs.append((src, obj))
    logs = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for src, rc, out in ex.map(lambda j: _compile(*j, extra), jobs):
                logs.append(out)
                if rc != 0:
                    raise RuntimeError("nvcc failed on %s:\n%s" % (src, out))
    if jobs or force or _mtime(LIB) < max(_mtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static",
                               "-ccbin", HOST_CXX, "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    if not quiet or ptxas_verbose:
        sys.stdout.write("".join(logs))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, ptxas_verbose="--ptxas-v" in sys.argv,
          quiet=False)
    print(LIB)
