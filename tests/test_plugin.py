"""The Diffusion3DB200 plugin and its driver (benchmarks_b200/plugin).

CPU: the restated plugin surface (plugin/mirror) computes the reference's
coefficients, initial field, GetAccuracy, rates and dump format (checked
against the golden data made from the reference's own objects); the
standalone driver builds; the drop-in build against the reference's own
headers and objects links (where the reference tree is present).

GPU: both drivers run RunBenchmark end to end and print the reference's
own known answers (64^3/100 -> 7.976817e-06, 128^3/100 -> 7.227031e-07),
for every kernel choice; --dump writes the reference's text format with
the values the oracle computes.
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
STANDALONE = os.path.join(PLUGIN, "_build", "d3d_b200_standalone.exe")
DROPIN = os.path.join(ROOT, "oracle", "_ref", "d3d_b200_dropin.exe")
PROBE_SO = os.path.join(ROOT, "tests", "_build", "libmirror_probe.so")
_f32p = ctypes.POINTER(ctypes.c_float)


def _probe():
    src = [os.path.join(ROOT, "tests", "mirror_probe.cc"),
           os.path.join(PLUGIN, "mirror", "surface.cc")]
    deps = src + [os.path.join(PLUGIN, "mirror", "diffusion3d", h)
                  for h in ("diffusion3d.h", "baseline.h")]
    if (not os.path.exists(PROBE_SO) or os.path.getmtime(PROBE_SO)
            < max(os.path.getmtime(d) for d in deps)):
        os.makedirs(os.path.dirname(PROBE_SO), exist_ok=True)
        subprocess.run(["/usr/bin/g++", "--std=c++11", "-O3", "-fPIC",
                        "-shared", "-I" + os.path.join(PLUGIN, "mirror"),
                        "-o", PROBE_SO] + src, check=True)
    L = ctypes.CDLL(PROBE_SO)
    L.mirror_params.argtypes = [ctypes.c_int] * 3 + [_f32p, _f32p]
    L.mirror_initial_field.argtypes = [ctypes.c_int] * 3 + [_f32p]
    L.mirror_accuracy.argtypes = [ctypes.c_int] * 3 + [_f32p, ctypes.c_int]
    L.mirror_accuracy.restype = ctypes.c_float
    L.mirror_dump.argtypes = [ctypes.c_int] * 3 + [_f32p]
    L.mirror_rates.argtypes = ([ctypes.c_int] * 4
                               + [ctypes.c_float, _f32p])
    L.mirror_rates.restype = ctypes.c_float
    return L


def _p(a):
    return a.ctypes.data_as(_f32p)


def test_mirror_surface_matches_reference_data(golden, tmp_path):
    meta, fields = golden
    L = _probe()
    for case in meta["cases"]:
        nx, ny, nz = case["nx"], case["ny"], case["nz"]
        c = np.zeros(7, np.float32)
        g = np.zeros(8, np.float32)
        L.mirror_params(nx, ny, nz, _p(c), _p(g))
        oc, og = O.params(nx, ny, nz)
        assert c.tobytes() == oc.tobytes() and g.tobytes() == og.tobytes()
        if nx * ny * nz > 300000:
            continue
        f = np.empty((nz, ny, nx), np.float32)
        L.mirror_initial_field(nx, ny, nz, _p(f))
        if case["noise_seed"] is None:
            assert (hashlib.sha256(f.tobytes()).hexdigest()
                    == case["sha256_in"]), case["name"]
        key = case["name"] + "/out"
        if key in fields:
            out = np.ascontiguousarray(fields[key])
            acc = L.mirror_accuracy(nx, ny, nz, _p(out), case["count"])
            assert np.float32(acc) == np.float32(case["accuracy"])
    gbs = np.zeros(1, np.float32)
    gf = L.mirror_rates(256, 256, 256, 100, 1.0, _p(gbs))
    rates = meta["rates_256_n100_t1"]
    assert np.float32(gf) == np.float32(rates["gflops"])
    assert np.float32(gbs[0]) == np.float32(rates["gbs"])
    # Dump: one "%.7E" line per value, in index order.
    f = np.ascontiguousarray(fields["r17x23x5_n7/out"])
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        L.mirror_dump(17, 23, 5, _p(f))
        lines = open("diffusion3d_result.probe.out").read().splitlines()
    finally:
        os.chdir(cwd)
    assert lines == ["%.7E" % v for v in f.reshape(-1).astype(np.float64)]


def test_standalone_driver_builds():
    subprocess.run(["make", "-s", "-C", PLUGIN], check=True)
    assert os.path.exists(STANDALONE)


@pytest.mark.skipif(not os.path.isdir(O.REF_SRC),
                    reason="reference tree not present")
def test_dropin_builds_against_reference_headers_and_objects():
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


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["auto", "generic", "tb2", "tb3", "tb4"])
def test_standalone_driver_prints_reference_known_answers(kernel):
    acc, out = _run_driver(STANDALONE, "--size", "64", "--count", "100",
                           "--kernel", kernel)
    assert acc == "7.976817e-06", out
    assert "Kernel-only performance" in out
    acc, _ = _run_driver(STANDALONE, "--size", "128", "--count", "100",
                         "--kernel", kernel)
    assert acc == "7.227031e-07"


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(DROPIN),
                    reason="the drop-in driver links the reference's own "
                           "objects, so it is built (oracle/Makefile dropin) "
                           "only where the reference tree is present, and "
                           "this machine has no build of it")
def test_dropin_driver_prints_reference_known_answers():
    acc, _ = _run_driver(DROPIN, "--size", "64", "--count", "100")
    assert acc == "7.976817e-06"
    acc, _ = _run_driver(DROPIN, "--size", "256", "--count", "100")
    assert acc == "4.336409e-07"


@pytest.mark.gpu
def test_driver_dump_matches_oracle(tmp_path):
    _run_driver(STANDALONE, "--size", "24", "--count", "13", "--dump",
                cwd=str(tmp_path))
    lines = open(tmp_path / "diffusion3d_result.b200.out").read().splitlines()
    c, _ = O.params(24, 24, 24)
    ref = O.run(O.initialize(24, 24, 24), c, 13)
    assert lines == ["%.7E" % v for v in ref.reshape(-1).astype(np.float64)]


@pytest.mark.gpu
def test_driver_binary_dump_matches_oracle(tmp_path):
    import benchmarks_b200 as B
    _run_driver(STANDALONE, "--size", "24", "--count", "13", "--dump-binary",
                cwd=str(tmp_path))
    h, field = B.read_checkpoint(str(tmp_path / "diffusion3d_result.b200.d3d"))
    c, _ = O.params(24, 24, 24)
    ref = O.run(O.initialize(24, 24, 24), c, 13)
    assert field.tobytes() == ref.tobytes()
    assert h["step"] == 13 and h["flags"] == 0
