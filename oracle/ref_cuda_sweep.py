"""Test infrastructure only: times the reference's own CUDA variants on this
GPU, next to this repository's drop-in drivers.

    make -C oracle refcuda refcuda_diffusion   # the reference's kernels, sm_100a
    make -C benchmarks_b200/plugin             # our two drivers
    python oracle/ref_cuda_sweep.py [--sizes 256:1000,512:200]
    python oracle/ref_cuda_sweep.py --surface diffusion \
        [--configs 2:8192:1000,2:16384:200,3:256:1000]

Each executable is the reference's own driver (src/diffusion3d/main.cc or
src/diffusion/main.cc) built with one variant macro, so the numbers are
what it prints itself: the "Kernel-only performance" block of
DisplayResult (device time of the step loop, diffusion3d_cuda.cu:373-384,
diffusion_cuda.cu:163-174) and its Accuracy line.  One JSON line per
(variant, configuration) on stdout.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_CUDA = os.path.join(HERE, "_ref", "cuda")
REF_DIF_CUDA = os.path.join(HERE, "_ref", "difcuda")
OURS = os.path.join(ROOT, "benchmarks_b200", "plugin", "_build",
                    "d3d_b200_standalone.exe")
OURS_DIF = os.path.join(ROOT, "benchmarks_b200", "plugin", "_build",
                        "diffusion_b200_standalone.exe")

# variant name -> what the reference's Makefile calls it
VARIANTS = ["cuda", "zblock", "opt0", "opt1", "opt2", "opt3", "shared",
            "shared1", "shared3", "shared4", "shared5", "shared6", "xy",
            "temporal_blocking"]
# src/diffusion variants that compile with CUDA 12 (shfl1-3 use the
# pre-Volta __shfl intrinsics), and the dimensions each accepts.
DIF_VARIANTS = {"cuda": (2, 3), "restrict": (2, 3), "roc": (2, 3),
                "shared1": (2, 3), "shared2": (2, 3), "zblock": (3,),
                "opt1": (3,), "opt2": (3,), "shared3": (3,), "shared4": (3,),
                "shared5": (3,), "shared6": (3,)}


def parse(out: str) -> dict:
    """Elapsed / GFLOPS / GB/s of the whole RunKernel and of the kernel-only
    block, and the Accuracy line, as the driver printed them."""
    def grab(label, text):
        m = re.search(label + r"\s*:\s*([0-9.eE+-]+)", text)
        return float(m.group(1)) if m else None
    head, _, kern = out.partition("Kernel-only performance:")
    acc = re.search(r"Accuracy\s*:\s*(\S+)", out)
    return {"elapsed_s": grab("Elapsed time", head),
            "gbs": grab("Throughput", head),
            "kernel_elapsed_s": grab("Elapsed time", kern),
            "kernel_gflops": grab("FLOPS", kern),
            "kernel_gbs": grab("Throughput", kern),
            "accuracy": acc.group(1) if acc else None}


def run(exe, size, count, extra=(), nd=3):
    r = subprocess.run([exe, "--size", str(size), "--count", str(count)]
                       + list(extra), capture_output=True, text=True,
                       timeout=600)
    rec = {"exe": os.path.basename(exe), "nd": nd, "size": size,
           "count": count, "rc": r.returncode}
    if r.returncode == 0:
        rec.update(parse(r.stdout))
        if rec.get("kernel_elapsed_s"):
            rec["kernel_gpts"] = (float(size) ** nd * count
                                  / rec["kernel_elapsed_s"] / 1e9)
    else:
        rec["stderr_tail"] = r.stderr[-400:]
    return rec


def main_diffusion(configs):
    for nd, size, count in configs:
        for v, dims in DIF_VARIANTS.items():
            if nd not in dims:
                continue
            exe = os.path.join(REF_DIF_CUDA, "diffusion_cuda_%s.exe" % v)
            if not os.path.exists(exe):
                print(json.dumps({"exe": os.path.basename(exe),
                                  "missing": True}), flush=True)
                continue
            rec = run(exe, size, count, ["--nd", str(nd)], nd=nd)
            rec["impl"] = "reference:" + v
            print(json.dumps(rec), flush=True)
        for kernel in ("auto",) if nd == 2 else ("auto", "tb2"):
            rec = run(OURS_DIF, size, count,
                      ["--nd", str(nd), "--kernel", kernel], nd=nd)
            rec["impl"] = "b200:" + kernel
            print(json.dumps(rec), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--surface", default="diffusion3d",
                    choices=["diffusion3d", "diffusion"])
    ap.add_argument("--sizes", default="256:1000,512:200",
                    help="size:count list (diffusion3d)")
    ap.add_argument("--configs", default="2:8192:1000,2:16384:200,3:256:1000",
                    help="nd:size:count list (diffusion)")
    args = ap.parse_args()
    if args.surface == "diffusion":
        return main_diffusion([tuple(int(v) for v in c.split(":"))
                               for c in args.configs.split(",")])
    sizes = [tuple(int(v) for v in s.split(":"))
             for s in args.sizes.split(",")]
    for size, count in sizes:
        for v in VARIANTS:
            exe = os.path.join(REF_CUDA, "diffusion3d_cuda_%s.exe" % v)
            if not os.path.exists(exe):
                print(json.dumps({"exe": os.path.basename(exe),
                                  "missing": True}), flush=True)
                continue
            rec = run(exe, size, count)
            rec["impl"] = "reference:" + v
            print(json.dumps(rec), flush=True)
        for kernel in ("auto", "tb2"):
            rec = run(OURS, size, count, ["--kernel", kernel])
            rec["impl"] = "b200:" + kernel
            print(json.dumps(rec), flush=True)


if __name__ == "__main__":
    main()
