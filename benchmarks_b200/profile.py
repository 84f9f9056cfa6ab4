"""A small, fixed workload for profiling one kernel under ncu.

    python -m benchmarks_b200.profile --kernel tma --n 512 --steps 4
    python -m benchmarks_b200.profile --kernel step2d --n 16384 --steps 4

Runs `steps` time steps of one kernel on an n^3 FP32 (or FP64) field of
uniform random values through the C ABI and exits.  With n = 512 each FP32
buffer is 512 MiB (larger than the 126 MB L2), two buffers in all.
Kernels: tma, generic, tb2, tb3, tb4 (temporal blocking), step2d (an n^2
grid of the diffusion::Diffusion surface; n = 16384 gives 1 GiB buffers),
and the same names with an f64_ prefix.
"""
from __future__ import annotations

import argparse

import benchmarks_b200 as B

KERNELS = {
    "tma": (B.KERNEL_TMA, 1),
    "generic": (B.KERNEL_GENERIC, 1),
    "tb2": (B.KERNEL_TB, 2),
    "tb3": (B.KERNEL_TB, 3),
    "tb4": (B.KERNEL_TB, 4),
    "step2d": (B.KERNEL_AUTO, 1),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", default="tma")
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--variant", type=int, default=None)
    ap.add_argument("--zchunk", type=int, default=0)
    args = ap.parse_args()
    import torch
    name = args.kernel
    dtype = B.F32
    if name.startswith("f64_"):
        dtype = B.F64
        name = name[4:]
    kernel, tb = KERNELS[name]
    n = args.n
    if name == "step2d":
        plan = B.DiffusionPlan((n, n), dtype, kernel, zchunk=args.zchunk)
    else:
        plan = B.Plan(n, n, n, dtype, kernel, tb, variant=args.variant,
                      zchunk=args.zchunk)
    gen = torch.Generator(device="cuda").manual_seed(7)
    tdt = torch.float64 if dtype == B.F64 else torch.float32
    f1 = torch.rand(plan.shape, device="cuda", generator=gen, dtype=tdt)
    f2 = torch.empty_like(f1)
    plan.run(f1, f2, args.steps)
    torch.cuda.synchronize()
    flags = B.check_device_errors()
    print("profile case done: %s n=%d (%dD) x %d steps, %s, device flags %d"
          % (args.kernel, n, plan.ndim, args.steps,
             plan.info()["last_kernel"], flags))


if __name__ == "__main__":
    main()
