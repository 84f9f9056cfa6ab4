#!/usr/bin/env python
"""Benchmark: diffusion3d 7-point stencil, 512^3 FP32, 200 steps per step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One bench "step" is one RunKernel(200) of a 512^3 FP32 grid (the reference's
workload unit; 2.68e10 point-updates).  `value` is whole-job Gpoint-updates/s
with the field resident in HBM; `e2e` is the same metric through the
RunKernel-style C-ABI call (d3d_run_host) with pinned host buffers, so the
512 MiB host->device and device->host copies are inside its timed region.

N > 1 (torchrun, one rank per GPU): every rank advances its own 512^3 grid
(independent grids shard with no data-path collective: weak scaling); the
time is the max over ranks.

--impl reference times the reference's own Diffusion3DOpenMP::RunKernel
(oracle/_ref, compiled from the reference sources; the C restatement in
oracle/ when that is absent) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_SIDE = 512
COUNT = 200
METRIC = "Gpoint-updates/s (512^3 FP32, 200 steps per RunKernel)"
UNIT = "Gpt-updates/s"
BYTES_PER_UPDATE = 8  # FP32: one 4-byte read + one 4-byte write per point
PEAK_FALLBACK_GBS = 6650.0


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def measured_peak_gbs():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return PEAK_FALLBACK_GBS, "fallback"


def profile_traffic(name):
    """dram bytes per launch recorded in a committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled while the timed work runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu),
                 "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"),
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi"]}
        time.sleep(0.2)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        loaded = [s for s in sm if smax and s > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": smax, "samples": len(sm),
                "power_w_max": max(power) if power else None,
                "reasons": sorted(reasons)}


def cpu_reference_leg(n_side, repeats=2):
    """Times the reference's own Diffusion3DOpenMP::RunKernel(200) on the
    host (oracle/_ref), else the oracle port, on this workload's input:
    `repeats` whole RunKernel(200) calls on all host threads.  Returns a
    cpu_baseline dict."""
    import oracle as O
    from benchmarks_b200.workloads import field_noise
    threads = os.cpu_count() or 1
    kind = "reference" if O.ref_available() else "port"
    n = n_side
    O.set_threads(threads)
    c, _ = O.params(n, n, n)
    fin = O.initialize(n, n, n)
    fin += field_noise(fin.shape)
    t = 0.0
    for _ in range(repeats):
        if kind == "reference":
            _, _, secs = O.ref_run(n, n, n, COUNT, field=fin, coeff=c,
                                   want_time=True, want_field=False)
        else:
            t0 = time.perf_counter()
            O.run(fin, c, COUNT)
            secs = time.perf_counter() - t0
        t += secs
    rate = float(n) ** 3 * COUNT * repeats / t / 1e9
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": "%d^3 FP32, %d x RunKernel(%d) of Diffusion3DOpenMP "
                      "(%s) on this workload's input, %.2f s in all, setup "
                      "excluded" % (n, repeats, COUNT,
                                    "oracle/_ref" if kind == "reference"
                                    else "oracle port", t)}


def batched_leg(B, torch, n_grids=4096, plain_sample=64, kind=None):
    """Config: 4096 grids, sides U{16..96} per axis, kappa U[0.05,0.2],
    steps U{10..500}; one batched run (one CUDA graph) vs a plain per-solve
    loop (a plan, two device buffers and a RunKernel-style d3d_run per
    grid) on the first `plain_sample` grids, which also checks those grids'
    batched results bit for bit against their runs alone.  `kind` forces
    one kernel kind for every size class instead of the autotuner (for
    profiling: an autotuner timed under a profiler picks differently)."""
    from benchmarks_b200.workloads import batched_specs
    specs = batched_specs(n_grids)
    updates = sum(nx * ny * nz * s for nx, ny, nz, s, _ in specs)
    batch = B.Batch(specs)
    if kind is None:
        batch.autotune()
    else:
        batch.set_kind(kind)
    gen = torch.Generator(device="cuda").manual_seed(0xB47C)
    batch.arena.uniform_(0.0, 1.0, generator=gen)
    batch.run()  # capture + first replay
    runs = [batch.run() for _ in range(3)]
    ms = min(runs)
    info = batch.info()
    # A fresh seeded input, one more run, and the sampled grids' results.
    batch.arena.uniform_(0.0, 1.0, generator=gen)
    sample = specs[:plain_sample]
    inputs = [batch.input(i).clone() for i in range(len(sample))]
    batch.run()
    torch.cuda.synchronize()
    results = [batch.result(i).clone() for i in range(len(sample))]
    batch.close()
    del batch
    torch.cuda.empty_cache()
    upd_s = sum(nx * ny * nz * s for nx, ny, nz, s, _ in sample)
    torch.cuda.synchronize()
    alone = []
    t0 = time.perf_counter()
    for (nx, ny, nz, s, c), fin in zip(sample, inputs):
        p = B.Plan(nx, ny, nz)
        p.set_graphs(False)
        f1 = fin.clone()
        f2 = p.empty()
        res, _ = p.run(f1, f2, s, c)
        torch.cuda.synchronize()
        alone.append(res)
        p.close()
    t_plain = time.perf_counter() - t0
    mismatched = sum(1 for r, a in zip(results, alone)
                     if not torch.equal(r, a))
    plain_solves = len(sample) / t_plain
    solves = n_grids / (ms / 1e3)
    return {"grids": n_grids, "updates": updates, "ms": ms,
            "solves_per_s": solves, "value": updates / (ms / 1e3) / 1e9,
            "unit": UNIT, "launches_per_run": info["launches_per_run"],
            "class_kernels": [
                c["kernel"] + (" %dx%d" % tuple(c["tile"]) if "tile" in c
                               else " x%d" % c["segments_per_thread"]
                               if "segments_per_thread" in c else "")
                for c in info["classes"]],
            "info": info,
            "plain_loop": {"sample_grids": len(sample),
                           "solves_per_s": plain_solves,
                           "value": upd_s / t_plain / 1e9},
            "results_equal_alone": {"grids_checked": len(sample),
                                    "mismatched": mismatched},
            "speedup_solves": solves / plain_solves}


def serving_leg(B, torch, n_req=256, arena_gb=24.0, chunk=8, resident=None,
                compare=True, kernel=None):
    """Config: Poisson stream (mean 2000 req/s) of cubic FP32 solves, sides
    log-uniform in [32, 256], steps log-uniform in [10, 2000]; the
    continuous-batching server vs a plain per-request loop (allocate,
    RunKernel with host copies, free) over the same arrivals.  Latency is
    completion time minus scheduled arrival.  Every served result is
    compared bit for bit with the same request run alone (the plain loop)."""
    from benchmarks_b200.workloads import serving_requests
    reqs = serving_requests(n_req)
    sizes = [s ** 3 for _, s, _ in reqs]
    maxn = max(sizes)
    gen = torch.Generator().manual_seed(0x5E7F)
    pool_in = torch.rand(maxn, generator=gen).pin_memory().numpy()
    out_served = torch.empty(sum(sizes), pin_memory=True).numpy()
    out_other = torch.empty(sum(sizes), pin_memory=True).numpy()
    offs = np.cumsum([0] + sizes[:-1])
    coeff = {}
    for _, s, _ in reqs:
        if s not in coeff:
            coeff[s] = B.coefficients(s, s, s)[0]
    upd = sum(n * st for n, (_, _, st) in zip(sizes, reqs))

    def lat_stats(done_at):
        lat = np.array([done_at[i] - reqs[i][0] for i in range(n_req)])
        span = max(done_at) - reqs[0][0]
        return {"solves_per_s": n_req / span, "p50_ms": 1e3 * float(
            np.percentile(lat, 50)), "p99_ms": 1e3 * float(
            np.percentile(lat, 99)), "makespan_s": span,
            "value": upd / span / 1e9}

    def out_view(pool, i):
        s = reqs[i][1]
        return pool[offs[i]:offs[i] + s ** 3].reshape(s, s, s)

    def serve(out_pool, kernel=None, lanes=None):
        server = B.Server(int(arena_gb * 2 ** 30), chunk, kernel, lanes,
                          resident)
        done_at = [0.0] * n_req
        idmap = {}
        nxt = 0
        t0 = time.perf_counter()
        while len(idmap) < n_req or sum(server.pending()):
            now = time.perf_counter() - t0
            while nxt < n_req and reqs[nxt][0] <= now:
                _, s, st = reqs[nxt]
                hin = pool_in[:s ** 3].reshape(s, s, s)
                idmap[server.submit(hin, out_view(out_pool, nxt), st,
                                    coeff[s])] = nxt
                nxt += 1
            for rid in server.tick():
                done_at[idmap[rid]] = time.perf_counter() - t0
            if nxt < n_req and not sum(server.pending()):
                time.sleep(max(0.0, reqs[nxt][0] - (time.perf_counter() - t0)))
        out = lat_stats(done_at)
        out["stats"] = server.stats()
        server.close()
        return out

    def same_results(a_pool, b_pool):
        return sum(1 for i in range(n_req)
                   if not np.array_equal(out_view(a_pool, i).view(np.uint32),
                                         out_view(b_pool, i).view(np.uint32)))

    # served: the default server (pitched TMA step kernel, several
    # streams), then the same stream through the batch API's march kernel
    # on one stream for comparison
    served = serve(out_served, kernel=kernel)
    if not compare:
        return {"requests": n_req, "served": served}
    march = serve(out_other, kernel=-1, lanes=1)
    march_mismatched = same_results(out_served, out_other)
    # plain per-request loop
    import ctypes
    done_at = [0.0] * n_req
    t0 = time.perf_counter()
    for i, (arr, s, st) in enumerate(reqs):
        now = time.perf_counter() - t0
        if arr > now:
            time.sleep(arr - now)
        n = s ** 3
        p = B.Plan(s, s, s)
        p.set_graphs(False)
        d1, d2 = ctypes.c_void_p(), ctypes.c_void_p()
        B.check(B.lib().d3d_device_alloc(n * 4, ctypes.byref(d1)))
        B.check(B.lib().d3d_device_alloc(n * 4, ctypes.byref(d2)))
        host = out_other[offs[i]:offs[i] + n]
        host[:] = pool_in[:n]
        ms = ctypes.c_float()
        B.check(B.lib().d3d_run_host(p.handle, host.ctypes.data, d1, d2,
                                     coeff[s].ctypes.data, st, None,
                                     ctypes.byref(ms)))
        B.lib().d3d_device_free(d1)
        B.lib().d3d_device_free(d2)
        p.close()
        done_at[i] = time.perf_counter() - t0
    plain = lat_stats(done_at)
    return {"requests": n_req, "rate_per_s": 2000.0, "updates": upd,
            "unit": UNIT, "served": served,
            "served_march_one_stream": {
                k: march[k] for k in ("solves_per_s", "makespan_s", "value")},
            "plain_loop": plain,
            "results_equal_alone": {
                "requests_checked": n_req,
                "mismatched_vs_plain_loop": same_results(out_served,
                                                         out_other),
                "mismatched_vs_march_server": march_mismatched},
            "speedup_solves": served["solves_per_s"] / plain["solves_per_s"],
            "p99_ratio_plain_over_served": plain["p99_ms"] / served["p99_ms"]}


def slab_leg(B, torch, dist, side_n=1024, count=20):
    """One side_n^3 FP32 grid split into z slabs across the ranks, timed
    with two overlapped schedules: passes of 2 steps with 2 ghost planes
    (the 6-plane pieces around each rank boundary first, their exchange
    over NCCL while the owned planes run the pass as fused two-step
    kernels), and single steps with 1 ghost plane (boundary planes first
    through d3d_step_planes).  Gpt-updates/s of the whole grid, device time
    from CUDA events, max over ranks.  At one rank there is no exchange."""
    from benchmarks_b200.distributed import SingleProcess, SlabSolver
    group = dist if dist is not None else SingleProcess()
    c = B.coefficients(side_n, side_n, side_n)[0]
    two_pi = 2.0 * 3.141592653589793

    def timed(halo):
        solver = SlabSolver(group, side_n, side_n, side_n, c, halo=halo,
                            overlap=True)
        d = solver.dec
        # The analytic initial field on this rank's planes (ghosts included).
        dev = solver.f1.device

        def factor(lo, hi, n):
            i = torch.arange(lo, hi, device=dev, dtype=torch.float64)
            return 1.0 - torch.cos(two_pi * (i + 0.5) / n)
        f = (0.125 * factor(d.lo, d.hi, side_n)[:, None, None]
             * factor(0, side_n, side_n)[None, :, None]
             * factor(0, side_n, side_n)[None, None, :])
        solver.f1.copy_(f.float())
        del f
        solver.run(4)  # warm-up: both buffer parities (graph captures)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        solver.run(count)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist is not None:
            t = torch.tensor([ms], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        world = d.world
        solver.close()
        del solver
        torch.cuda.empty_cache()
        return ms, world

    ms, world = timed(2)
    ms1, _ = timed(1)
    rate = float(side_n) ** 3 * count / 1e9
    return {"grid": [side_n] * 3, "steps": count, "ranks": world,
            "schedule": "overlapped, halo 2: 2-step passes (boundary pieces "
                        "first, NCCL send/recv of 2 planes per neighbour "
                        "per pass, owned planes as fused two-step kernels)",
            "ms": ms, "value": rate / (ms / 1e3), "unit": UNIT,
            "scaling": "strong",
            "halo1_single_steps": {"ms": ms1, "value": rate / (ms1 / 1e3)}}


def diffusion2d_leg(B, torch, stream, side_n=16384, count=50, reps=4):
    """The second plugin surface's 2D 5-point grid (diffusion::Diffusion,
    nd = 2): device rate of the register-march kernel at side_n^2 (1 GiB
    per FP32 buffer, larger than L2), FP32 and FP64, with the FP64
    device accuracy report of a run from the analytic field."""
    peak, _ = measured_peak_gbs()
    out = {"grid": [side_n, side_n], "steps_per_run": count}
    for dtype, name, es in ((B.F32, "f32", 4), (B.F64, "f64", 8)):
        plan = B.DiffusionPlan((side_n, side_n), dtype)
        a, b = plan.empty(), plan.empty()
        plan.analytic(a, 0.0)
        c = plan.reference_coefficients()
        a, b = plan.run(a, b, count, c, stream)  # warm-up (graph capture)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            a, b = plan.run(a, b, count, c, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        rate = float(side_n) ** 2 * count * reps / t / 1e9
        acc = plan.accuracy(a, count * (reps + 1), stream)
        info = plan.info()
        out[name] = {"value": rate, "unit": UNIT,
                     "hbm_frac": rate * 2 * es / peak,
                     "rms_vs_analytic": acc[0],
                     "kernel": info["last_kernel"],
                     "variant": info["variant"],
                     "rows_per_task": info["launch_zchunk"]}
        del a, b
        plan.close()
        torch.cuda.empty_cache()
    return out


CONFIG = {"workload": "diffusion3d 512^3 FP32, 200 steps per RunKernel",
          "grid": [N_SIDE, N_SIDE, N_SIDE], "count": COUNT,
          "input": "analytic sinusoid (t=0) + seeded U[0,1e-3) noise",
          "l2": "inputs larger than L2 (512 MiB per buffer)"}


def run_reference_arm(args):
    """The reference's own Diffusion3DOpenMP::RunKernel(200) on the 512^3
    field (oracle/_ref, compiled from the reference sources; the C
    restatement when that is absent), every timed step one whole
    RunKernel(200), all host threads.  Rank 0 only."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    import oracle as O
    from benchmarks_b200.workloads import field_noise
    if not os.path.exists(O.LIB_PATH) or (
            not O.ref_available() and os.path.isdir(O.REF_SRC)):
        O.build()
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    kind = "reference" if O.ref_available() else "port"
    n = N_SIDE
    c, _ = O.params(n, n, n)
    fin = O.initialize(n, n, n)
    fin += field_noise(fin.shape)

    def one():
        if kind == "reference":
            # RunKernel(COUNT) alone, timed inside the probe (the
            # reference's InitializeBenchmark and the field copies excluded)
            _, _, secs = O.ref_run(n, n, n, COUNT, field=fin, coeff=c,
                                   want_time=True, want_field=False)
            return secs
        t0 = time.perf_counter()
        O.run(fin, c, COUNT)
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        one()
    times = [one() for _ in range(args.steps)]
    total = sum(times)
    value = float(n) ** 3 * COUNT * args.steps / total / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic: analytic sinusoid + seeded "
                                "U[0,1e-3) noise",
        "config": dict(CONFIG, parallelism="single GPU" if world == 1
                       else "independent grid per GPU"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                         "kind": kind,
                         "sample": "%d^3, RunKernel(%d) per timed step "
                                   "(Diffusion3DOpenMP%s), %d threads, "
                                   "%.2f s per step" % (
                                       n, COUNT, "" if kind == "reference"
                                       else ", oracle port", threads,
                                       total / args.steps)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_b200(args):
    import torch
    import benchmarks_b200 as B

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    n = N_SIDE
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    # The headline is the plain single-grid, single-step kernel (its %HBM
    # roofline is the target); the fused two-step rate that
    # D3D_KERNEL_AUTO picks at this size is reported separately (side.auto).
    plan = B.Plan(n, n, n, B.F32, B.KERNEL_TMA)
    coeff = plan.reference_coefficients()

    # Config: analytic sinusoid at t=0 plus seeded U[0, 1e-3) noise.
    from benchmarks_b200.workloads import field_noise
    f1 = plan.empty()
    f2 = plan.empty()
    plan.analytic(f1, 0.0)
    f1.add_(torch.from_numpy(field_noise(plan.shape, 0xD1FF + rank)).to(dev))
    init = f1.clone()

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def run_steps(p, a, b, k):
        for _ in range(k):
            a, b = p.run(a, b, COUNT, coeff, stream)
        return a, b

    # --- headline: plain TMA z-march kernel ---------------------------
    a, b = run_steps(plan, f1, f2, args.warmup)
    try:
        gpu_id = "GPU-%s" % torch.cuda.get_device_properties(local).uuid
    except Exception:
        gpu_id = str(local)
    sampler = ClockSampler(gpu_id)
    sampler.start()
    barrier()
    torch.cuda.synchronize()
    launches0 = B.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    a, b = run_steps(plan, a, b, args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    launches = B.launch_count() - launches0
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms)
    updates = float(n) ** 3 * COUNT * args.steps
    value = updates * world / (ms_max / 1e3) / 1e9
    info = plan.info()
    # The dominant kernel: AUTO runs this FP32 512^3 loop as fused two-step
    # passes (steps_tb2w: 2 updates per point per launch), otherwise one
    # single-step launch per step.  Algorithmic bytes are the reference's
    # 8 B per update (GetThroughput); the fused kernel moves about half of
    # that through DRAM (`traffic`, from its ncu summary).
    two_step = info["last_kernel"] == "steps_tb2w"
    updates_per_launch = 2 if two_step else 1
    per_launch_s = ms / 1e3 / (COUNT * args.steps / updates_per_launch)
    peak, peak_kind = measured_peak_gbs()
    algo_bytes = BYTES_PER_UPDATE * n ** 3 * updates_per_launch
    achieved = algo_bytes / per_launch_s / 1e9
    traffic = profile_traffic("steps_tb2w_512cube_f32.md" if two_step
                              else "step_tma_512cube_f32.md")
    traffic_from = ("dram__bytes_read.sum + dram__bytes_write.sum per launch "
                    "of one ncu capture of this kernel on this workload, read "
                    "from its committed profile summary (not measured in "
                    "this run)") if traffic else None

    # --- side measurements (not the headline) --------------------------
    def rate_of(p, a_, b_, steps):
        a_, b_ = run_steps(p, a_, b_, 1)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        a_, b_ = run_steps(p, a_, b_, steps)
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        return float(n) ** 3 * COUNT * steps / t / 1e9, p.info()

    side = {}
    # D3D_KERNEL_AUTO, the library default: fused two-step passes here.
    pauto = B.Plan(n, n, n, B.F32, B.KERNEL_AUTO)
    r, inf = rate_of(pauto, a, b, 3)
    side["auto"] = {
        "value": r, "unit": UNIT, "kernel": inf["last_kernel"],
        "effective_hbm_frac": r * 1e9 * BYTES_PER_UPDATE / (peak * 1e9),
        "note": "temporal-blocked effective rate: 8 B per update counted, "
                "about 3.9 B per update moved (ncu capture of the fused "
                "two-step kernel at 512^3)",
        "grid": inf["grid"], "zchunk": inf["launch_zchunk"]}
    pauto.close()
    for k in (2, 3, 4):
        ptb = B.Plan(n, n, n, B.F32, B.KERNEL_TB, k)
        ptb.autotune(a, b, steps=4 * k, coeff=coeff, stream=stream)
        r, _ = rate_of(ptb, a, b, 3)
        a, b = ptb.run(a, b, k, coeff, stream)  # one fused pass: its geometry
        inf = ptb.info()
        side["tb%d" % k] = {
            "value": r, "unit": UNIT,
            "effective_hbm_frac": r * 1e9 * BYTES_PER_UPDATE / (peak * 1e9),
            "kernel": inf["last_kernel"], "grid": inf["grid"],
            "zchunk": inf["launch_zchunk"], "smem": inf["smem"]}
        ptb.close()

    # --- HBM calibration: out = cc * in over the same 512^3 buffers (the
    # stencil's 8 B per point with no neighbours; d3d_copy_calibrate) ------
    B.copy_calibrate(a, b, passes=2, stream=stream)  # warm-up
    copy_ms, copy_gbs = B.copy_calibrate(a, b, passes=20, stream=stream)

    # --- correctness report: FP32 vs FP64 vs analytic, FP64 norms -------
    plan64 = B.Plan(n, n, n, B.F64, B.KERNEL_AUTO)
    c64 = plan64.reference_coefficients()
    g1 = init.double()
    g2 = torch.empty_like(g1)
    r64, o64 = plan64.run(g1, g2, COUNT, c64, stream)
    del o64
    x1 = init.clone()
    x2 = torch.empty_like(x1)
    r32, o32 = plan.run(x1, x2, COUNT, coeff, stream)
    del o32

    def norms(v, rel=True):
        d = {"rms": v[0], "max_abs": v[1]}
        if rel:
            d["max_rel"] = v[2]
        return d
    # Errors against the analytic decay: the closed form is evaluated per
    # point in FP64 on the device (d3d_accuracy); the input's noise is part
    # of that error, so only rms / max_abs are meaningful there.
    report = {
        "fp32_vs_fp64": norms(plan.compare(r32, r64, stream)),
        "fp32_vs_analytic": norms(plan.accuracy(r32, COUNT, stream), False),
        "fp64_vs_analytic": norms(plan64.accuracy(r64, COUNT, stream), False),
        "steps": COUNT, "input": "analytic(t=0) + U[0,1e-3) noise",
        "tolerance": "max_rel(fp32 vs fp64) <= 1e-5",
    }
    # FP64 throughput of the same workload (16 B per update).
    r64_rate, _ = rate_of(plan64, g1, g2, 2)
    side["fp64"] = {"value": r64_rate, "unit": UNIT,
                    "hbm_frac": r64_rate * 16 / peak}
    del g1, g2, r64, x1, x2, r32
    plan64.close()
    torch.cuda.synchronize()

    # --- e2e: RunKernel-style call with pinned host buffers -------------
    # The host field starts as this workload's input; every call copies it
    # in, runs RunKernel(200) and copies the result back over it, so after
    # E calls it must equal E * 200 device steps from the same input.
    host = B.pinned_empty((n, n, n), np.float32)
    host[...] = init.cpu().numpy()
    torch.cuda.synchronize()
    plan.run_host(host, a, b, COUNT, coeff, stream)  # warm-up (graph)
    e2e_steps = max(1, args.steps // 2)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        plan.run_host(host, a, b, COUNT, coeff, stream)
    t_e2e = time.perf_counter() - t0
    t_e2e = max_over_ranks(t_e2e)
    x1, x2 = init.clone(), torch.empty_like(init)
    for _ in range(e2e_steps + 1):
        x1, x2 = plan.run(x1, x2, COUNT, coeff, stream)
    torch.cuda.synchronize()
    e2e_equal = bool(np.array_equal(host.view(np.uint32),
                                    x1.cpu().numpy().view(np.uint32)))
    del x1, x2
    e2e = {"value": float(n) ** 3 * COUNT * e2e_steps * world / t_e2e / 1e9,
           "unit": UNIT, "h2d_bytes_per_step": n ** 3 * 4,
           "d2h_bytes_per_step": n ** 3 * 4,
           "calls": e2e_steps,
           "result_equals_device_run": e2e_equal}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: analytic sinusoid + seeded U[0,1e-3) noise",
        "config": dict(CONFIG, parallelism="independent grid per GPU"
                       if world > 1 else "single GPU"),
        "kernel": dict(info, what="fused two-step TMA passes" if two_step
                       else "plain single-step TMA z-march kernel (the "
                       "fused two-step rate is side.auto)"),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind,
                     "traffic": traffic,
                     "traffic_from": traffic_from,
                     "kernel": info["last_kernel"],
                     "updates_per_point_per_launch": updates_per_launch,
                     "algorithmic_bytes_per_launch": algo_bytes,
                     "copy_calibration": {
                         "gbs": copy_gbs, "frac_of_peak": copy_gbs / peak,
                         "kernel_frac_of_copy": achieved / copy_gbs,
                         "what": "20 ping-pong passes of f2 = cc*f1 over "
                                 "two 512 MiB buffers (d3d_copy_calibrate)"}},
        "clocks": clocks,
        "e2e": e2e,
        "gpu_launches": launches,
        "correctness": report,
        "side": side,
    }
    if not args.no_side:
        # Every rank takes part (the exchange is a collective step).  A
        # failure here is recorded in the line rather than losing the
        # headline measured above; the process group's timeout bounds a
        # rank left waiting for a failed peer.
        try:
            side["slab"] = slab_leg(B, torch, dist)
        except Exception as e:  # noqa: BLE001 -- reported, not hidden
            side["slab"] = {"error": "%s: %s" % (type(e).__name__, e)}
            torch.cuda.synchronize()
    if not args.no_side and world == 1:
        del a, b, f1, f2, host, init
        torch.cuda.empty_cache()
        side["batched"] = batched_leg(B, torch)
        torch.cuda.empty_cache()
        side["serving"] = serving_leg(B, torch)
        torch.cuda.empty_cache()
        side["diffusion2d"] = diffusion2d_leg(B, torch, stream)
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_reference_leg(n)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true",
                    help="skip the CPU baseline leg")
    ap.add_argument("--no-side", action="store_true",
                    help="skip the batched, serving and 2D legs")
    ap.add_argument("--only-leg", choices=["batched", "serving", "served",
                                           "diffusion2d", "slab"],
                    help="run one side leg alone on GPU 0 and print its "
                         "JSON (no headline line; for profiling)")
    ap.add_argument("--batch-kind", type=int, default=None,
                    help="with --only-leg batched: one kernel kind for "
                         "every size class instead of the autotuner")
    ap.add_argument("--only-kernel", default=None,
                    help="run `--count` steps of one single-grid kernel "
                         "(tma, generic, tb2, tb3, tb4, step2d; f64_ "
                         "prefix for FP64) on a --side^3 field (side^2 for "
                         "step2d) of seeded uniform values and exit: a "
                         "fixed small case to profile; `resident` runs a "
                         "batch of --grids such grids on the cluster-"
                         "resident kernel")
    ap.add_argument("--side", type=int, default=512)
    ap.add_argument("--grids", type=int, default=128,
                    help="with --only-kernel resident: grids in the batch")
    ap.add_argument("--count", type=int, default=4)
    ap.add_argument("--variant", type=int, default=None)
    ap.add_argument("--zchunk", type=int, default=0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.only_kernel:
        return run_one_kernel(args)
    if args.only_leg:
        return run_one_leg(args.only_leg, args.batch_kind)
    return run_b200(args)


def run_one_kernel(args):
    """`args.count` steps of one kernel on a seeded field, then exit."""
    import torch
    import benchmarks_b200 as B
    if args.only_kernel == "resident":
        return run_resident_case(args)
    kernels = {"tma": (B.KERNEL_TMA, 1), "generic": (B.KERNEL_GENERIC, 1),
               "tb2": (B.KERNEL_TB, 2), "tb3": (B.KERNEL_TB, 3),
               "tb4": (B.KERNEL_TB, 4), "step2d": (B.KERNEL_AUTO, 1)}
    torch.cuda.set_device(0)
    name, dtype = args.only_kernel, B.F32
    if name.startswith("f64_"):
        name, dtype = name[4:], B.F64
    kernel, tb = kernels[name]
    n = args.side
    if name == "step2d":
        plan = B.DiffusionPlan((n, n), dtype, kernel, zchunk=args.zchunk)
    else:
        plan = B.Plan(n, n, n, dtype, kernel, tb, variant=args.variant,
                      zchunk=args.zchunk)
    gen = torch.Generator(device="cuda").manual_seed(7)
    tdt = torch.float64 if dtype == B.F64 else torch.float32
    f1 = torch.rand(plan.shape, device="cuda", generator=gen, dtype=tdt)
    f2 = torch.empty_like(f1)
    plan.run(f1, f2, args.count)
    torch.cuda.synchronize()
    flags = B.check_device_errors()
    print("kernel case done: %s n=%d (%dD) x %d steps, %s, device flags %d"
          % (args.only_kernel, n, plan.ndim, args.count,
             plan.info()["last_kernel"], flags), flush=True)
    return 1 if flags else 0


def run_resident_case(args):
    """A batch of `args.grids` cubic grids of side `args.side`, `args.count`
    steps each, on the cluster-resident kernel (one class: one persistent
    launch per run), run twice; prints the device time of the second run."""
    import torch
    import benchmarks_b200 as B
    torch.cuda.set_device(0)
    n = args.side
    c = B.batch_coefficients(n, n, n, 0.1)
    batch = B.Batch([(n, n, n, args.count, c)] * args.grids)
    batch.set_kind(B.BATCH_KIND_RESIDENT)
    gen = torch.Generator(device="cuda").manual_seed(7)
    batch.arena.uniform_(0.0, 1.0, generator=gen)
    batch.run()
    ms = batch.run()
    info = batch.info()
    flags = B.check_device_errors()
    upd = float(n) ** 3 * args.count * args.grids
    print(json.dumps({"case": "resident", "grids": args.grids, "side": n,
                      "steps": args.count, "ms": ms,
                      "gpts": upd / (ms / 1e3) / 1e9,
                      "resident": info["resident"],
                      "launches_per_run": info["launches_per_run"],
                      "device_flags": flags}), flush=True)
    batch.close()
    return 1 if flags else 0


def run_one_leg(leg, batch_kind=None):
    import torch
    import benchmarks_b200 as B
    torch.cuda.set_device(0)
    if leg == "batched":
        out = batched_leg(B, torch, kind=batch_kind)
    elif leg == "serving":
        out = serving_leg(B, torch)
    elif leg == "served":  # the server alone: no march or plain-loop runs
        out = serving_leg(B, torch, compare=False)
    elif leg == "slab":
        out = slab_leg(B, torch, None)
    else:
        out = diffusion2d_leg(B, torch, torch.cuda.current_stream())
    print(json.dumps({"leg": leg, **out}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
