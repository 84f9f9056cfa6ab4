"""Generates tests/golden/ from the reference's own CPU objects.

Run in a container that has the reference tree (it builds oracle/_ref from
the reference sources in place, then runs them):

    python tests/golden/make_golden.py

Outputs
  golden.json   per case: dims, steps, coefficients, the reference's
                GetAccuracy value, sha256 of the float32 output bytes and a
                strided sample of output values
  fields.npz    full input and output fields of the small cases

Cases follow the reference's own configurations (its 64^3/100 OpenMP run,
the 256^3/100 default of main.cc:65-66,131) plus small ragged shapes, custom
anisotropic coefficients and seeded noise, which the reference's driver cannot
express but its objects compute through the oracle/ref_shim.cc probe.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def sample(a: np.ndarray, k: int = 64) -> list:
    flat = a.reshape(-1)
    idx = np.linspace(0, flat.size - 1, num=min(k, flat.size)).astype(np.int64)
    return [[int(i), float(flat[i])] for i in idx]


def main() -> None:
    O.build(with_ref=True)
    cases = []
    fields = {}

    def add(name, nx, ny, nz, count, noise_seed=None, coeff=None,
            backend=O.REF_OPENMP, keep_field=False):
        fin = O.ref_initialize(nx, ny, nz)
        if noise_seed is not None:
            fin = fin + O.seeded_noise(fin.shape, noise_seed)
        use_in = fin if (noise_seed is not None) else None
        out, acc = O.ref_run(nx, ny, nz, count, field=use_in, coeff=coeff,
                             backend=backend, want_accuracy=True)
        c_used = (np.asarray(coeff, np.float32) if coeff is not None
                  else O.ref_params(nx, ny, nz)[0])
        case = dict(name=name, nx=nx, ny=ny, nz=nz, count=count,
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

    # Small and ragged shapes (kept in full).
    add("r17x23x5_n7", 17, 23, 5, 7, noise_seed=1, keep_field=True)
    add("r1x1x1_n3", 1, 1, 1, 3, keep_field=True)
    add("r2x3x1_n4", 2, 3, 1, 4, keep_field=True)
    add("r5x1x9_n5", 5, 1, 9, 5, noise_seed=2, keep_field=True)
    add("r33x8x70_n9", 33, 8, 70, 9, noise_seed=3, keep_field=True)
    add("r64x4x3_n0", 64, 4, 3, 0, noise_seed=4, keep_field=True)
    # Anisotropic custom coefficients (ce != cw != cn ...), stable.
    aniso = np.array([0.11, 0.07, 0.09, 0.13, 0.05, 0.08, 0.47], np.float32)
    add("aniso12x10x8_n6", 12, 10, 8, 6, noise_seed=5, coeff=aniso,
        keep_field=True)
    # Non-cubic grid with the reference constructor's own coefficients
    # (cn = 0.1*(ny/nx)^2, ct = 0.1*(nz/nx)^2; cc > 0, so stable).
    add("r24x40x16_n50", 24, 40, 16, 50, noise_seed=6, keep_field=True)
    # The reference's own configurations (hash + accuracy only).
    add("c64_n100", 64, 64, 64, 100)
    add("c64_n100_serial", 64, 64, 64, 100, backend=O.REF_BASELINE)
    add("c64_n100_omp_tb", 64, 64, 64, 100, backend=O.REF_OPENMP_TB)
    add("c128_n100", 128, 128, 128, 100)
    add("c256_n100", 256, 256, 256, 100)
    add("c128_n1000_noise", 128, 128, 128, 1000, noise_seed=7)

    gf, gb = O.ref_rates(256, 256, 256, 100, 1.0)
    meta = dict(
        generator="tests/golden/make_golden.py",
        source="reference Diffusion3DOpenMP / Baseline / "
               "Diffusion3DOpenMPTemporalBlocking compiled by oracle/Makefile",
        noise="numpy default_rng(seed).random(shape) * 1e-3 as float32, "
              "added to the reference's Initialize(t=0) field",
        rates_256_n100_t1=dict(gflops=gf, gbs=gb),
        cases=cases)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "fields.npz"), **fields)


if __name__ == "__main__":
    main()
