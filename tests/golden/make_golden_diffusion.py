"""Generates the diffusion::Diffusion fixtures in tests/golden/ from the
reference's own CPU objects and driver (src/diffusion).

Run in a container that has the reference tree (it builds oracle/_ref from
the reference sources in place, then runs them):

    python tests/golden/make_golden_diffusion.py

Outputs
  diffusion.json         known answers printed by the reference's own driver
                         (main.cc, `Accuracy : %e`) for its OpenMP and serial
                         builds, plus per probe case: nd, dims, steps,
                         coefficients, GetAccuracy, sha256 of the float32
                         output bytes and a strided sample of output values
  diffusion_fields.npz   full input and output fields of the small cases

The driver cases use the driver's own options (--nd, --size, --count).  The
probe cases run the reference's objects through oracle/ref_shim_diffusion.cc
on ragged 2D and 3D shapes, seeded noise and anisotropic coefficients, which
the driver cannot express.
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def sample(a: np.ndarray, k: int = 64) -> list:
    flat = a.reshape(-1)
    idx = np.linspace(0, flat.size - 1, num=min(k, flat.size)).astype(np.int64)
    return [[int(i), float(flat[i])] for i in idx]


def driver_kat(exe: str, nd: int, size: int, count: int) -> str:
    out = subprocess.run(
        [os.path.join(ROOT, "oracle", "_ref", exe), "--nd", str(nd),
         "--size", str(size), "--count", str(count)],
        check=True, capture_output=True, text=True).stdout
    m = re.search(r"Accuracy\s*:\s*(\S+)", out)
    assert m, out
    return m.group(1)


def main() -> None:
    O.build(with_ref=True)
    kats = []
    for exe, backend in (("diffusion_openmp.exe", "openmp"),
                         ("diffusion_baseline.exe", "baseline")):
        for nd, size, count in ((2, 256, 100), (2, 256, 1000),
                                (2, 1024, 100), (3, 64, 100),
                                (3, 128, 100)):
            if backend == "baseline" and size * (size if nd == 3 else 1) > 2 ** 14:
                continue  # the serial build is slow; OpenMP covers these
            acc = driver_kat(exe, nd, size, count)
            kats.append(dict(backend=backend, nd=nd, size=size, count=count,
                             accuracy=acc))
            print(backend, nd, size, count, acc, flush=True)

    cases = []
    fields = {}

    def add(name, nd, nx, ny, nz, count, noise_seed=None, coeff=None,
            backend=O.DIF_OPENMP, keep_field=False):
        init, _, _ = O.difref_run(nd, nx, ny, nz, count=0, backend=backend)
        fin = init
        if noise_seed is not None:
            fin = init + O.seeded_noise(init.shape, noise_seed)
        use_in = fin if noise_seed is not None else None
        _, out, acc = O.difref_run(nd, nx, ny, nz, count=count, field=use_in,
                                   coeff=coeff, backend=backend,
                                   want_accuracy=True)
        c_used = (np.asarray(coeff, np.float32) if coeff is not None
                  else O.difref_params(nd, nx, ny, nz)[0])
        case = dict(name=name, nd=nd, nx=nx, ny=ny,
                    nz=nz if nd == 3 else 1, count=count,
                    noise_seed=noise_seed, backend=backend,
                    coeff=[float(x) for x in c_used],
                    coeff_hex=[int(x) for x in c_used.view(np.uint32)],
                    accuracy=acc, sha256_in=sha(fin), sha256_out=sha(out),
                    sample_out=sample(out))
        cases.append(case)
        if keep_field:
            fields[name + "/in"] = fin
            fields[name + "/out"] = out
        print(name, acc, flush=True)

    aniso = np.array([0.11, 0.07, 0.09, 0.13, 0.05, 0.08, 0.47], np.float32)
    aniso2 = np.array([0.11, 0.07, 0.09, 0.13, 0.0, 0.0, 0.6], np.float32)
    # 2D, small and ragged (kept in full): nx odd, nx = 2 mod 4, one row,
    # one column, a row wider than one 128-column warp segment.
    add("d2_37x23_n7", 2, 37, 23, 1, 7, noise_seed=11, keep_field=True)
    add("d2_1x1_n3", 2, 1, 1, 1, 3, keep_field=True)
    add("d2_2x3_n4", 2, 2, 3, 1, 4, keep_field=True)
    add("d2_1x9_n5", 2, 1, 9, 1, 5, noise_seed=12, keep_field=True)
    add("d2_9x1_n5", 2, 9, 1, 1, 5, noise_seed=13, keep_field=True)
    add("d2_130x7_n9", 2, 130, 7, 1, 9, noise_seed=14, keep_field=True)
    add("d2_260x33_n6", 2, 260, 33, 1, 6, noise_seed=15, keep_field=True)
    add("d2_131x17_n8", 2, 131, 17, 1, 8, noise_seed=16, keep_field=True)
    add("d2_64x4_n0", 2, 64, 4, 1, 0, noise_seed=17, keep_field=True)
    add("d2_aniso12x10_n6", 2, 12, 10, 1, 6, noise_seed=18, coeff=aniso2,
        keep_field=True)
    add("d2_24x40_n50", 2, 24, 40, 1, 50, noise_seed=19, keep_field=True)
    add("d2_48x20_n11_serial", 2, 48, 20, 1, 11, noise_seed=20,
        backend=O.DIF_BASELINE, keep_field=True)
    # 3D through the same surface (y order s = y-1 first, cc as it sums).
    add("d3_17x23x5_n7", 3, 17, 23, 5, 7, noise_seed=21, keep_field=True)
    add("d3_aniso12x10x8_n6", 3, 12, 10, 8, 6, noise_seed=22, coeff=aniso,
        keep_field=True)
    add("d3_33x8x70_n9", 3, 33, 8, 70, 9, noise_seed=23, keep_field=True)
    add("d3_20x12x9_n5_serial", 3, 20, 12, 9, 5, noise_seed=24,
        backend=O.DIF_BASELINE, keep_field=True)
    # Larger cases (hash, samples and accuracy only).
    add("d2_1000x1000_n50_noise", 2, 1000, 1000, 1, 50, noise_seed=25)
    add("d2_4096x4096_n100", 2, 4096, 4096, 1, 100)
    add("d2_2048x512_n200_noise", 2, 2048, 512, 1, 200, noise_seed=26)
    add("d3_64_n100", 3, 64, 64, 64, 100)
    add("d3_64_n100_serial", 3, 64, 64, 64, 100, backend=O.DIF_BASELINE)
    add("d3_128_n100_noise", 3, 128, 128, 128, 100, noise_seed=27)

    gf2, gb2 = O.difref_rates(2, 4096, 4096, 1, 100, 1.0)
    gf3, gb3 = O.difref_rates(3, 256, 256, 256, 100, 1.0)
    meta = dict(
        generator="tests/golden/make_golden_diffusion.py",
        source="reference diffusion::DiffusionOpenMP / diffusion::Baseline "
               "(src/diffusion) compiled by oracle/Makefile; driver "
               "src/diffusion/main.cc for the known answers",
        noise="numpy default_rng(seed).random(shape) * 1e-3 as float32, "
              "added to the backend's InitializeInput field",
        rates=dict(nd2_4096_n100_t1=dict(gflops=gf2, gbs=gb2),
                   nd3_256_n100_t1=dict(gflops=gf3, gbs=gb3)),
        driver_kats=kats,
        cases=cases)
    with open(os.path.join(HERE, "diffusion.json"), "w") as f:
        json.dump(meta, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "diffusion_fields.npz"), **fields)


if __name__ == "__main__":
    main()
