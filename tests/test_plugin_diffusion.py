"""The DiffusionB200 plugin (the reference's second plugin surface,
diffusion::Diffusion, 2D and 3D) and its driver (benchmarks_b200/plugin).

CPU: the restated surface (plugin/mirror/diffusion) computes the reference's
coefficients, initial field, GetAccuracy, rates and dump format (checked
against the golden data made from the reference's own objects); the
standalone driver builds; the drop-in build against the reference's own
headers links (where the reference tree is present).

GPU: both drivers run RunBenchmark end to end and print the reference
driver's own known answers for its serial build (the plugin inherits
Baseline's InitializeInput): 2D 256^2/100 -> 4.972005e-07, 2D 256^2/1000
-> 4.756415e-06, 3D 64^3/100 -> 7.976800e-06, 3D 128^3/100 ->
7.232086e-07; --warmup and every kernel choice keep them; --dump writes
the reference's text format with the values the oracle computes.
"""
import ctypes
import hashlib
import os
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PLUGIN = os.path.join(ROOT, "benchmarks_b200", "plugin")
STANDALONE = os.path.join(PLUGIN, "_build", "diffusion_b200_standalone.exe")
DROPIN = os.path.join(ROOT, "oracle", "_ref", "diffusion_b200_dropin.exe")
PROBE_SO = os.path.join(ROOT, "tests", "_build",
                        "libmirror_probe_diffusion.so")
_f32p = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)


def _probe():
    src = [os.path.join(ROOT, "tests", "mirror_probe_diffusion.cc"),
           os.path.join(PLUGIN, "mirror", "surface_diffusion.cc")]
    deps = src + [os.path.join(PLUGIN, "mirror", "diffusion", h)
                  for h in ("diffusion.h", "baseline.h")]
    if (not os.path.exists(PROBE_SO) or os.path.getmtime(PROBE_SO)
            < max(os.path.getmtime(d) for d in deps)):
        os.makedirs(os.path.dirname(PROBE_SO), exist_ok=True)
        subprocess.run(["/usr/bin/g++", "--std=c++11", "-O3", "-fPIC",
                        "-shared", "-I" + os.path.join(PLUGIN, "mirror"),
                        "-o", PROBE_SO] + src, check=True)
    L = ctypes.CDLL(PROBE_SO)
    L.mirror_dif_params.argtypes = [ctypes.c_int, _ip, _f32p, _f32p]
    L.mirror_dif_initial_field.argtypes = [ctypes.c_int, _ip, _f32p]
    L.mirror_dif_accuracy.argtypes = [ctypes.c_int, _ip, _f32p, ctypes.c_int]
    L.mirror_dif_accuracy.restype = ctypes.c_float
    L.mirror_dif_dump.argtypes = [ctypes.c_int, _ip, _f32p]
    L.mirror_dif_rates.argtypes = [ctypes.c_int, _ip, ctypes.c_int,
                                   ctypes.c_float, _f32p]
    L.mirror_dif_rates.restype = ctypes.c_float
    return L


def _p(a):
    return a.ctypes.data_as(_f32p)


def _dims(case):
    d = (case["nx"], case["ny"]) + ((case["nz"],) if case["nd"] == 3 else ())
    return (ctypes.c_int * len(d))(*d)


def _shape(case):
    if case["nd"] == 2:
        return (case["ny"], case["nx"])
    return (case["nz"], case["ny"], case["nx"])


def test_mirror_surface_matches_reference_data(golden_diffusion, tmp_path):
    meta, fields = golden_diffusion
    L = _probe()
    for case in meta["cases"]:
        nd, d = case["nd"], _dims(case)
        c = np.zeros(7, np.float32)
        g = np.zeros(8, np.float32)
        L.mirror_dif_params(nd, d, _p(c), _p(g))
        oc, og = O.dif_params(nd, case["nx"], case["ny"], case["nz"])
        assert c.tobytes() == oc.tobytes() and g.tobytes() == og.tobytes()
        if case["nx"] * case["ny"] * case["nz"] > 300000:
            continue
        f = np.empty(_shape(case), np.float32)
        L.mirror_dif_initial_field(nd, d, _p(f))
        if case["noise_seed"] is None and case["backend"] == O.DIF_BASELINE:
            assert (hashlib.sha256(f.tobytes()).hexdigest()
                    == case["sha256_in"]), case["name"]
        assert f.tobytes() == O.dif_initialize(
            nd, case["nx"], case["ny"], case["nz"]).tobytes()
        key = case["name"] + "/out"
        if key in fields and "aniso" not in case["name"]:
            out = np.ascontiguousarray(fields[key])
            acc = L.mirror_dif_accuracy(nd, d, _p(out), case["count"])
            assert np.float32(acc) == np.float32(case["accuracy"])
    rates = meta["rates"]
    for nd, dims, key in ((2, (4096, 4096), "nd2_4096_n100_t1"),
                          (3, (256, 256, 256), "nd3_256_n100_t1")):
        gbs = np.zeros(1, np.float32)
        gf = L.mirror_dif_rates(nd, (ctypes.c_int * nd)(*dims), 100, 1.0,
                                _p(gbs))
        assert np.float32(gf) == np.float32(rates[key]["gflops"])
        assert np.float32(gbs[0]) == np.float32(rates[key]["gbs"])
    # Dump: one "%.7E" line per value, in index order.
    f = np.ascontiguousarray(fields["d2_37x23_n7/out"])
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        L.mirror_dif_dump(2, (ctypes.c_int * 2)(37, 23), _p(f))
        lines = open("diffusion_result.probe.out").read().splitlines()
    finally:
        os.chdir(cwd)
    assert lines == ["%.7E" % v for v in f.reshape(-1).astype(np.float64)]


def test_standalone_driver_builds():
    subprocess.run(["make", "-s", "-C", PLUGIN], check=True)
    assert os.path.exists(STANDALONE)


@pytest.mark.skipif(not os.path.isdir(O.REF_SRC),
                    reason="reference tree not present")
def test_dropin_builds_against_reference_headers():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"),
                    "REF_SRC=" + O.REF_SRC, "dropin"], check=True)
    assert os.path.exists(DROPIN)


def _run_driver(exe, *args, cwd=None):
    r = subprocess.run([exe] + list(args), capture_output=True, text=True,
                       cwd=cwd, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    acc = [ln for ln in r.stdout.splitlines() if ln.startswith("Accuracy")]
    assert acc, r.stdout
    return acc[0].split(":")[1].strip(), r.stdout


KATS = [("2", "256", "100", "4.972005e-07"), ("2", "256", "1000",
                                               "4.756415e-06"),
        ("3", "64", "100", "7.976800e-06"), ("3", "128", "100",
                                             "7.232086e-07")]


# Temporal blocking is a 3D kernel: the 2D cases run the other two.
DRIVER_CASES = [(k, kernel) for k in KATS
                for kernel in ("auto", "generic", "tb2", "tb4")
                if k[0] == "3" or not kernel.startswith("tb")]


@pytest.mark.gpu
@pytest.mark.parametrize("case,kernel", DRIVER_CASES)
def test_standalone_driver_prints_reference_known_answers(case, kernel):
    nd, size, count, kat = case
    acc, out = _run_driver(STANDALONE, "--nd", nd, "--size", size, "--count",
                           count, "--kernel", kernel)
    assert acc == kat, out
    assert "Kernel-only performance" in out


@pytest.mark.gpu
def test_standalone_driver_warmup_keeps_the_answer():
    acc, out = _run_driver(STANDALONE, "--nd", "2", "--size", "256",
                           "--count", "100", "--warmup")
    assert acc == "4.972005e-07"
    assert "Warming up the kernel" in out


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(DROPIN),
                    reason="the drop-in driver links the reference's own "
                           "objects, so it is built (oracle/Makefile dropin) "
                           "only where the reference tree is present, and "
                           "this machine has no build of it")
def test_dropin_driver_prints_reference_known_answers():
    for nd, size, count, kat in KATS:
        acc, _ = _run_driver(DROPIN, "--nd", nd, "--size", size, "--count",
                             count)
        assert acc == kat, (nd, size, count)


@pytest.mark.gpu
def test_driver_dump_matches_oracle(tmp_path):
    _run_driver(STANDALONE, "--nd", "2", "--size", "40", "--count", "13",
                "--dump", cwd=str(tmp_path))
    lines = open(tmp_path / "diffusion_result.b200.out").read().splitlines()
    c, _ = O.dif_params(2, 40, 40)
    ref = O.dif_run(O.dif_initialize(2, 40, 40), c, 13)
    assert lines == ["%.7E" % v for v in ref.reshape(-1).astype(np.float64)]


@pytest.mark.gpu
def test_driver_binary_dump_matches_oracle(tmp_path):
    import benchmarks_b200 as B
    _run_driver(STANDALONE, "--nd", "2", "--size", "40", "--count", "13",
                "--dump-binary", cwd=str(tmp_path))
    h, field = B.read_checkpoint(str(tmp_path / "diffusion_result.b200.d3d"))
    c, _ = O.dif_params(2, 40, 40)
    ref = O.dif_run(O.dif_initialize(2, 40, 40), c, 13)
    assert field.tobytes() == ref.tobytes()
    assert h["step"] == 13 and h["flags"] == 1 and h["ndim"] == 2
