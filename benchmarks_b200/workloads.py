"""Seeded synthetic workloads for the batched and served solvers.

* ``batched_specs`` -- independent grids with sides drawn uniformly from
  {16..96} per axis (non-cubic), kappa uniform in [0.05, 0.2], step counts
  uniform in [10, 500]; coefficients from the stability policy
  (d3d_batch_coefficients).
* ``serving_requests`` -- a Poisson request stream (mean rate `rate`/s) of
  cubic grids with sides log-uniform in [32, 256] and step counts
  log-uniform in [10, 2000].
* ``field_noise`` -- the seeded U[0, 1e-3) noise added to the analytic
  initial field of the single-grid workload (512^3, 200 steps).

No public dataset is involved; the reference has none for this path.
"""
from __future__ import annotations

import math

import numpy as np

from . import batch_coefficients


def batched_specs(n=4096, seed=0xB47C, side=(16, 96), steps=(10, 500),
                  kappa=(0.05, 0.2)):
    rng = np.random.default_rng(seed)
    dims = rng.integers(side[0], side[1] + 1, size=(n, 3))
    st = rng.integers(steps[0], steps[1] + 1, size=n)
    ka = rng.uniform(kappa[0], kappa[1], size=n)
    out = []
    for (nx, ny, nz), s, k in zip(dims.tolist(), st.tolist(), ka.tolist()):
        out.append((nx, ny, nz, s, batch_coefficients(nx, ny, nz, k)))
    return out


def serving_requests(n=256, seed=0x5E7F, rate=2000.0, side=(32, 256),
                     steps=(10, 2000)):
    """[(arrival_s, side, steps)] sorted by arrival."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=n)
    t = np.cumsum(gaps) - gaps[0]
    sides = np.exp(rng.uniform(math.log(side[0]), math.log(side[1]), n))
    sts = np.exp(rng.uniform(math.log(steps[0]), math.log(steps[1]), n))
    return [(float(a), int(round(s)), int(round(k)))
            for a, s, k in zip(t, sides, sts)]


def field_noise(shape, seed=0xD1FF, amplitude=1e-3):
    """Seeded U[0, amplitude) FP32 noise of `shape` (numpy, host)."""
    rng = np.random.default_rng(seed)
    noise = rng.random(shape, dtype=np.float32)
    noise *= np.float32(amplitude)
    return noise
