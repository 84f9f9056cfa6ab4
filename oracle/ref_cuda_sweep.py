"""Test infrastructure only: times the reference's own CUDA variants of
diffusion3d on this GPU, next to this repository's drop-in driver.

    make -C oracle refcuda                 # the reference's kernels, sm_100a
    make -C benchmarks_b200/plugin         # our Diffusion3DB200 driver
    python oracle/ref_cuda_sweep.py [--sizes 256:1000,512:200]

Each executable is the reference's own driver (src/diffusion3d/main.cc)
built with one variant macro, so the numbers are what it prints itself:
the "Kernel-only performance" block of Diffusion3DCUDA::DisplayResult
(device time of the step loop, diffusion3d_cuda.cu:373-384) and its
Accuracy line.  One JSON line per (variant, size) on stdout.
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
OURS = os.path.join(ROOT, "benchmarks_b200", "plugin", "_build",
                    "d3d_b200_standalone.exe")

# variant name -> what the reference's Makefile calls it
VARIANTS = ["cuda", "zblock", "opt0", "opt1", "opt2", "opt3", "shared",
            "shared1", "shared3", "shared4", "shared5", "shared6", "xy",
            "temporal_blocking"]


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


def run(exe, size, count, extra=()):
    r = subprocess.run([exe, "--size", str(size), "--count", str(count)]
                       + list(extra), capture_output=True, text=True,
                       timeout=600)
    rec = {"exe": os.path.basename(exe), "size": size, "count": count,
           "rc": r.returncode}
    if r.returncode == 0:
        rec.update(parse(r.stdout))
        if rec.get("kernel_elapsed_s"):
            rec["kernel_gpts"] = (float(size) ** 3 * count
                                  / rec["kernel_elapsed_s"] / 1e9)
    else:
        rec["stderr_tail"] = r.stderr[-400:]
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", default="256:1000,512:200")
    args = ap.parse_args()
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
