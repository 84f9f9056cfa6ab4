"""Pins the oracle's restatement of the reference's second plugin surface,
diffusion::Diffusion (src/diffusion; oracle/dif_oracle_impl.h), before any
2D or diffusion-surface GPU result is checked with it:

* against the committed fixtures tests/golden/make_golden_diffusion.py made
  from the reference's own objects and driver -- always;
* against the reference objects themselves (oracle/_ref/libdif_ref.so) --
  where they were built.
"""
import hashlib

import numpy as np
import pytest

import oracle as O


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _coeff(case):
    return np.array(case["coeff_hex"], np.uint32).view(np.float32)


def _case_input(case, fields):
    key = case["name"] + "/in"
    if key in fields:
        return fields[key]
    f = O.dif_initialize(case["nd"], case["nx"], case["ny"], case["nz"],
                         omp=case["backend"] == O.DIF_OPENMP)
    if case["noise_seed"] is not None:
        f = f + O.seeded_noise(f.shape, case["noise_seed"])
    return f


def _is_custom(case):
    return "aniso" in case["name"]


def test_params_match_reference_constructor(golden_diffusion):
    meta, _ = golden_diffusion
    for case in meta["cases"]:
        if _is_custom(case):
            continue
        c, _ = O.dif_params(case["nd"], case["nx"], case["ny"], case["nz"])
        assert (c.view(np.uint32) == _coeff(case).view(np.uint32)).all(), \
            case["name"]


def test_cc_differs_from_diffusion3d_where_the_sum_order_matters():
    """diffusion.h:107 adds (ct+cb) as a pair; diffusion3d.h:65 adds left to
    right.  Both restatements follow their own reference."""
    differs = 0
    for nx, ny, nz in ((17, 23, 5), (24, 40, 16), (33, 8, 70), (64, 64, 64)):
        a, _ = O.dif_params(3, nx, ny, nz)
        b, _ = O.params(nx, ny, nz)
        assert (a[:6] == b[:6]).all()
        differs += int(a[6] != b[6])
    assert differs >= 1


def test_initialize_matches_reference_inputs(golden_diffusion):
    meta, _ = golden_diffusion
    for case in meta["cases"]:
        f = O.dif_initialize(case["nd"], case["nx"], case["ny"], case["nz"],
                             omp=case["backend"] == O.DIF_OPENMP)
        if case["noise_seed"] is not None:
            f = f + O.seeded_noise(f.shape, case["noise_seed"])
        assert _sha(f) == case["sha256_in"], case["name"]


@pytest.mark.parametrize("small", [True, False])
def test_run_bit_exact_vs_golden(golden_diffusion, small):
    meta, fields = golden_diffusion
    for case in meta["cases"]:
        n = case["nx"] * case["ny"] * case["nz"] * max(case["count"], 1)
        if small != (n < 5e6):
            continue
        out = O.dif_run(_case_input(case, fields), _coeff(case),
                        case["count"])
        assert _sha(out) == case["sha256_out"], case["name"]
        flat = out.reshape(-1)
        for i, v in case["sample_out"]:
            assert flat[i] == np.float32(v)
        key = case["name"] + "/out"
        if key in fields:
            assert (out.view(np.uint32) == fields[key].view(np.uint32)).all()
        if not _is_custom(case):
            assert (np.float32(O.dif_accuracy(out, case["count"]))
                    == np.float32(case["accuracy"])), case["name"]


def test_driver_known_answers(golden_diffusion):
    """`Accuracy : %e` as the reference's own driver printed it, reproduced
    from the oracle's Initialize + run + GetAccuracy: 2D 256^2/100 ->
    4.972005e-07 (both builds); 3D 64^3/100 -> 7.976976e-06 (OpenMP, whose
    Initialize3D rounds once) and 7.976800e-06 (serial, header Initialize)."""
    meta, _ = golden_diffusion
    kats = {(k["backend"], k["nd"], k["size"], k["count"]): k["accuracy"]
            for k in meta["driver_kats"]}
    assert kats[("openmp", 2, 256, 100)] == "4.972005e-07"
    assert kats[("openmp", 3, 64, 100)] == "7.976976e-06"
    assert kats[("baseline", 3, 64, 100)] == "7.976800e-06"
    for (backend, nd, size, count), printed in kats.items():
        if size ** nd * count > 2e8:
            continue
        nz = size if nd == 3 else 1
        c, _ = O.dif_params(nd, size, size, nz)
        f = O.dif_initialize(nd, size, size, nz, omp=backend == "openmp")
        out = O.dif_run(f, c, count)
        assert "%e" % O.dif_accuracy(out, count) == printed, \
            (backend, nd, size, count)


def test_fp64_restatement_close_to_fp32():
    for nd, (nx, ny, nz) in ((2, (40, 28, 1)), (3, (20, 12, 9))):
        c32, _ = O.dif_params(nd, nx, ny, nz, np.float32)
        c64, _ = O.dif_params(nd, nx, ny, nz, np.float64)
        f32 = O.dif_run(O.dif_initialize(nd, nx, ny, nz), c32, 25)
        f64 = O.dif_run(O.dif_initialize(nd, nx, ny, nz, dtype=np.float64),
                        c64, 25)
        assert O.norms(f32, f64)[2] < 1e-5


@pytest.mark.ref
@pytest.mark.skipif(not O.dif_ref_available(),
                    reason="oracle/_ref/libdif_ref.so not built")
@pytest.mark.parametrize("nd,dims", [(2, (17, 23, 1)), (2, (1, 1, 1)),
                                     (2, (129, 3, 1)), (2, (6, 40, 1)),
                                     (3, (17, 23, 5)), (3, (40, 3, 2)),
                                     (3, (9, 31, 12))])
@pytest.mark.parametrize("count", [0, 1, 4])
def test_oracle_vs_reference_objects(nd, dims, count):
    nx, ny, nz = dims
    c, g = O.dif_params(nd, nx, ny, nz)
    rc, rg = O.difref_params(nd, nx, ny, nz)
    assert (c.view(np.uint32) == rc.view(np.uint32)).all()
    assert (g.view(np.uint32) == rg.view(np.uint32)).all()
    for backend in (O.DIF_OPENMP, O.DIF_BASELINE):
        omp = backend == O.DIF_OPENMP
        init, _, _ = O.difref_run(nd, nx, ny, nz, backend=backend)
        mine0 = O.dif_initialize(nd, nx, ny, nz, omp=omp)
        assert (mine0.view(np.uint32) == init.view(np.uint32)).all()
        fin = mine0 + O.seeded_noise(mine0.shape, 31)
        _, ref, acc = O.difref_run(nd, nx, ny, nz, count, field=fin,
                                   backend=backend, want_accuracy=True)
        mine = O.dif_run(fin, c, count)
        assert (mine.view(np.uint32) == ref.view(np.uint32)).all()
        assert np.float32(O.dif_accuracy(mine, count)) == np.float32(acc)
    t = O.dif_initialize(nd, nx, ny, nz, time=0.25)
    assert (t.view(np.uint32)
            == O.difref_initialize(nd, nx, ny, nz, 0.25).view(np.uint32)).all()
