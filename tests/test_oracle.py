"""Pins the oracle (oracle/d3d_oracle.c) before anything is checked with it.

* against the committed golden fixtures generated from the reference's own
  objects (tests/golden/make_golden.py) -- always;
* against the reference objects themselves (oracle/_ref) -- where they were
  built, i.e. where the reference tree was present at build time.
"""
import hashlib

import numpy as np
import pytest

import oracle as O


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _case_input(case, fields):
    key = case["name"] + "/in"
    if key in fields:
        return fields[key]
    f = O.initialize(case["nx"], case["ny"], case["nz"])
    if case["noise_seed"] is not None:
        f = f + O.seeded_noise(f.shape, case["noise_seed"])
    return f


def _coeff(case):
    return np.array(case["coeff_hex"], np.uint32).view(np.float32)


def test_params_match_reference_constructor(golden):
    meta, _ = golden
    for case in meta["cases"]:
        if case["name"].startswith("aniso"):
            continue  # custom coefficients, not the constructor's
        c, _ = O.params(case["nx"], case["ny"], case["nz"])
        assert (c.view(np.uint32) == np.array(case["coeff_hex"],
                                              np.uint32)).all(), case["name"]


def test_initialize_matches_reference_inputs(golden):
    meta, fields = golden
    for case in meta["cases"]:
        f = O.initialize(case["nx"], case["ny"], case["nz"])
        if case["noise_seed"] is not None:
            f = f + O.seeded_noise(f.shape, case["noise_seed"])
        assert _sha(f) == case["sha256_in"], case["name"]


@pytest.mark.parametrize("small", [True, False])
def test_run_bit_exact_vs_golden(golden, small):
    meta, fields = golden
    for case in meta["cases"]:
        n = case["nx"] * case["ny"] * case["nz"] * max(case["count"], 1)
        if small != (n < 5e6):
            continue
        fin = _case_input(case, fields)
        out = O.run(fin, _coeff(case), case["count"])
        assert _sha(out) == case["sha256_out"], case["name"]
        flat = out.reshape(-1)
        for i, v in case["sample_out"]:
            assert flat[i] == np.float32(v)
        if case["name"] + "/out" in fields:
            ref = fields[case["name"] + "/out"]
            assert (out.view(np.uint32) == ref.view(np.uint32)).all()


def test_accuracy_known_answers(golden):
    """GetAccuracy KATs: 64^3/100 -> 7.976817e-06, 128^3/100 -> 7.227031e-07,
    256^3/100 -> 4.336409e-07 (the reference's own non-FMA build)."""
    meta, fields = golden
    kat = {"c64_n100": "7.976817e-06", "c128_n100": "7.227031e-07",
           "c256_n100": "4.336409e-07"}
    by_name = {c["name"]: c for c in meta["cases"]}
    for name, printed in kat.items():
        case = by_name[name]
        assert "%e" % case["accuracy"] == printed
        if case["nx"] <= 128:
            out = O.run(_case_input(case, fields), _coeff(case), case["count"])
            acc = O.accuracy(out, case["count"])
            assert np.float32(acc) == np.float32(case["accuracy"])
    for case in meta["cases"]:
        key = case["name"] + "/out"
        if key in fields:
            acc = O.accuracy(fields[key], case["count"])
            assert np.float32(acc) == np.float32(case["accuracy"]), case["name"]


def test_temporal_blocking_reference_equals_plain(golden):
    """The reference's 2-step OpenMP temporal blocking computes the same
    bits as its plain loop (same per-point expression)."""
    meta, _ = golden
    by_name = {c["name"]: c for c in meta["cases"]}
    assert (by_name["c64_n100_omp_tb"]["sha256_out"]
            == by_name["c64_n100"]["sha256_out"]
            == by_name["c64_n100_serial"]["sha256_out"])


def test_fp64_restatement_close_to_fp32():
    nx, ny, nz = 20, 12, 9
    c32, _ = O.params(nx, ny, nz, np.float32)
    c64, _ = O.params(nx, ny, nz, np.float64)
    f32 = O.run(O.initialize(nx, ny, nz, dtype=np.float32), c32, 25)
    f64 = O.run(O.initialize(nx, ny, nz, dtype=np.float64), c64, 25)
    rms, mx, mr, _ = O.norms(f32, f64)
    assert mr < 1e-5
    acc64 = O.accuracy(f64, 25)
    acc32 = O.accuracy(f32, 25)
    assert abs(acc64 - acc32) < 1e-5


def test_norms_plant_a_mistake():
    a = np.linspace(1, 2, 1000).astype(np.float32)
    b = a.copy()
    assert O.norms(a, b)[1] == 0.0
    b[17] += np.float32(1e-3)
    rms, mx, mr, _ = O.norms(a, b)
    assert mx == pytest.approx(1e-3, rel=1e-3)
    assert rms == pytest.approx(1e-3 / np.sqrt(1000), rel=1e-3)


@pytest.mark.ref
@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("dims", [(17, 23, 5), (1, 1, 1), (40, 3, 2),
                                  (9, 31, 12)])
@pytest.mark.parametrize("count", [0, 1, 4])
def test_oracle_vs_reference_objects(dims, count):
    nx, ny, nz = dims
    c, g = O.params(nx, ny, nz)
    rc, rg = O.ref_params(nx, ny, nz)
    assert (c.view(np.uint32) == rc.view(np.uint32)).all()
    assert (g.view(np.uint32) == rg.view(np.uint32)).all()
    fin = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 11)
    for backend in (O.REF_OPENMP, O.REF_BASELINE):
        ref, acc = O.ref_run(nx, ny, nz, count, field=fin, backend=backend,
                             want_accuracy=True)
        mine = O.run(fin, c, count)
        assert (mine.view(np.uint32) == ref.view(np.uint32)).all()
        assert np.float32(O.accuracy(mine, count)) == np.float32(acc)
    t = O.initialize(nx, ny, nz, time=0.25)
    assert (t.view(np.uint32)
            == O.ref_initialize(nx, ny, nz, 0.25).view(np.uint32)).all()
