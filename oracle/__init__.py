"""Test infrastructure only: the oracle, never the product.

ctypes bindings for
  * ``liboracle.so``        -- this repository's C restatement of the
                               reference's diffusion3d CPU path
                               (d3d_oracle.c / d3d_oracle_impl.h), and
  * ``_ref/libd3d_ref.so``  -- the reference's own Diffusion3DOpenMP /
                               Baseline / Diffusion3DOpenMPTemporalBlocking
                               objects compiled from its sources by
                               ``make -C oracle ref`` (present only where the
                               reference tree was available at build time),
  * ``_ref/libdif_ref.so``  -- the same for the reference's second plugin
                               surface, diffusion::DiffusionOpenMP /
                               diffusion::Baseline (2D and 3D grids); the
                               ``dif_*`` functions below.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, and only as the checker or as the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libd3d_ref.so")
DIF_REF_LIB_PATH = os.path.join(HERE, "_ref", "libdif_ref.so")
# Where the reference's sources lie (its src/ directory).  Only the build
# recipe (oracle/Makefile, `make ref`) and the tests that rebuild it read
# them; machines without the tree use what was built beforehand.
REF_SRC = os.environ.get("D3D_REFERENCE_SRC", "/root/reference/src")

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_lib = None
_ref = None
_dif_ref = None

# Backend ids understood by d3dref_run (oracle/ref_shim.cc).
REF_OPENMP, REF_BASELINE, REF_OPENMP_TB = 0, 1, 2
# Backend ids understood by difref_run (oracle/ref_shim_diffusion.cc).
DIF_OPENMP, DIF_BASELINE = 0, 1


def build(with_ref: bool | None = None) -> None:
    """Compile liboracle.so (and _ref/ when the reference tree exists)."""
    if with_ref is None:
        with_ref = os.path.isdir(REF_SRC)
    targets = ["all"] + (["ref"] if with_ref else [])
    subprocess.run(["make", "-s", "-C", HERE, "REF_SRC=" + REF_SRC]
                   + targets, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(with_ref=False)
        L = ctypes.CDLL(LIB_PATH)
        for sfx, T, P in (("f32", ctypes.c_float, _f32p),
                          ("f64", ctypes.c_double, _f64p)):
            getattr(L, "d3do_params_" + sfx).argtypes = [
                ctypes.c_int] * 3 + [P, P]
            getattr(L, "d3do_initialize_" + sfx).argtypes = (
                [P] + [ctypes.c_int] * 3 + [T] * 8)
            getattr(L, "d3do_step_" + sfx).argtypes = (
                [P, P] + [ctypes.c_int] * 3 + [P])
            getattr(L, "d3do_run_" + sfx).argtypes = (
                [P, P] + [ctypes.c_int] * 3 + [P, ctypes.c_int])
            fn = getattr(L, "d3do_accuracy_" + sfx)
            fn.argtypes = [P] + [ctypes.c_int] * 4
            fn.restype = T
            getattr(L, "difo_params_" + sfx).argtypes = [
                ctypes.c_int] * 4 + [P, P]
            getattr(L, "difo_initialize_" + sfx).argtypes = (
                [P] + [ctypes.c_int] * 3 + [T] * 8 + [ctypes.c_int] * 2)
            getattr(L, "difo_step_" + sfx).argtypes = (
                [P, P] + [ctypes.c_int] * 4 + [P])
            getattr(L, "difo_run_" + sfx).argtypes = (
                [P, P] + [ctypes.c_int] * 4 + [P, ctypes.c_int])
            fn = getattr(L, "difo_accuracy_" + sfx)
            fn.argtypes = [P] + [ctypes.c_int] * 5
            fn.restype = T
        for name, pa, pb in (("d3do_norms_f32_f32", _f32p, _f32p),
                             ("d3do_norms_f32_f64", _f32p, _f64p),
                             ("d3do_norms_f64_f64", _f64p, _f64p)):
            getattr(L, name).argtypes = [pa, pb, ctypes.c_long, _f64p]
        L.d3do_set_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_LIB_PATH)


def ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(REF_LIB_PATH)
        R = ctypes.CDLL(REF_LIB_PATH)
        R.d3dref_run.argtypes = ([ctypes.c_int] * 4 + [_f32p, _f32p, _f32p,
                                 ctypes.c_int, _f32p, ctypes.c_int])
        R.d3dref_run_timed.argtypes = (
            [ctypes.c_int] * 4 + [_f32p, _f32p, _f32p, ctypes.c_int, _f32p,
                                  ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_double)])
        R.d3dref_params.argtypes = [ctypes.c_int] * 3 + [_f32p, _f32p]
        R.d3dref_initialize.argtypes = ([_f32p] + [ctypes.c_int] * 3
                                        + [ctypes.c_float] * 8)
        R.d3dref_rates.argtypes = ([ctypes.c_int] * 4 + [ctypes.c_float,
                                   _f32p, _f32p])
        _ref = R
    return _ref


def _dt(dtype):
    dtype = np.dtype(dtype)
    if dtype == np.float32:
        return "f32", _f32p
    if dtype == np.float64:
        return "f64", _f64p
    raise TypeError(dtype)


def _ptr(a, P):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(P)


def set_threads(n: int) -> int:
    return lib().d3do_set_threads(n)


def params(nx, ny, nz, dtype=np.float32):
    """(coeff[7] = ce,cw,cn,cs,ct,cb,cc ; geom[8] = kappa,dx,dy,dz,kx,ky,kz,dt)."""
    sfx, P = _dt(dtype)
    c = np.zeros(7, dtype)
    g = np.zeros(8, dtype)
    getattr(lib(), "d3do_params_" + sfx)(nx, ny, nz, _ptr(c, P), _ptr(g, P))
    return c, g


def initialize(nx, ny, nz, time=0.0, dtype=np.float32):
    """Analytic field at `time` on the reference's cell-centred grid."""
    sfx, P = _dt(dtype)
    _, g = params(nx, ny, nz, dtype)
    buf = np.empty((nz, ny, nx), dtype)
    getattr(lib(), "d3do_initialize_" + sfx)(
        _ptr(buf, P), nx, ny, nz, g[4], g[5], g[6], g[1], g[2], g[3], g[0],
        time)
    return buf


def run(field, coeff, count):
    """`count` steps starting from `field` (nz, ny, nx); returns a new array."""
    f = np.ascontiguousarray(field)
    sfx, P = _dt(f.dtype)
    nz, ny, nx = f.shape
    f1 = f.copy()
    f2 = np.empty_like(f1)
    c = np.ascontiguousarray(coeff, dtype=f.dtype)
    getattr(lib(), "d3do_run_" + sfx)(_ptr(f1, P), _ptr(f2, P), nx, ny, nz,
                                      _ptr(c, P), count)
    return f1


def accuracy(field, count):
    """Baseline::GetAccuracy restated (RMS vs analytic, REAL accumulation)."""
    f = np.ascontiguousarray(field)
    sfx, P = _dt(f.dtype)
    nz, ny, nx = f.shape
    return float(getattr(lib(), "d3do_accuracy_" + sfx)(_ptr(f, P), nx, ny,
                                                        nz, count))


def norms(a, b):
    """FP64-accumulated (rms, max_abs, max_rel, sum(a)) of a against b."""
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert a.size == b.size
    out = np.zeros(4, np.float64)
    name = "d3do_norms_%s_%s" % (_dt(a.dtype)[0], _dt(b.dtype)[0])
    getattr(lib(), name)(_ptr(a, _dt(a.dtype)[1]), _ptr(b, _dt(b.dtype)[1]),
                         a.size, _ptr(out, _f64p))
    return out


def seeded_noise(shape, seed, amplitude=1e-3, dtype=np.float32):
    """Seeded U[0, amplitude) noise added to the analytic initial field."""
    rng = np.random.default_rng(seed)
    return (rng.random(shape) * amplitude).astype(dtype)


# --- the reference itself (oracle/_ref) ---------------------------------

def ref_params(nx, ny, nz):
    c = np.zeros(7, np.float32)
    g = np.zeros(8, np.float32)
    ref().d3dref_params(nx, ny, nz, _ptr(c, _f32p), _ptr(g, _f32p))
    return c, g


def ref_initialize(nx, ny, nz, time=0.0):
    _, g = ref_params(nx, ny, nz)
    buf = np.empty((nz, ny, nx), np.float32)
    ref().d3dref_initialize(_ptr(buf, _f32p), nx, ny, nz, g[4], g[5], g[6],
                            g[1], g[2], g[3], g[0], time)
    return buf


def ref_run(nx, ny, nz, count, field=None, coeff=None, backend=REF_OPENMP,
            want_accuracy=False, want_time=False, want_field=True):
    """Runs the reference backend; returns (field after count steps, acc),
    plus the seconds RunKernel(count) alone took when want_time."""
    out = np.empty((nz, ny, nx), np.float32) if want_field else None
    acc = np.zeros(1, np.float32)
    secs = ctypes.c_double(0.0)
    fin = None if field is None else np.ascontiguousarray(field, np.float32)
    cin = None if coeff is None else np.ascontiguousarray(coeff, np.float32)
    rc = ref().d3dref_run_timed(
        backend, nx, ny, nz,
        None if cin is None else _ptr(cin, _f32p),
        None if fin is None else _ptr(fin, _f32p),
        None if out is None else _ptr(out, _f32p), count,
        _ptr(acc, _f32p) if want_accuracy else None, 0, ctypes.byref(secs))
    if rc != 0:
        raise RuntimeError("d3dref_run failed: %d" % rc)
    res = (out, (float(acc[0]) if want_accuracy else None))
    return res + (secs.value,) if want_time else res


def ref_rates(nx, ny, nz, count, time):
    gf = np.zeros(1, np.float32)
    gb = np.zeros(1, np.float32)
    ref().d3dref_rates(nx, ny, nz, count, time, _ptr(gf, _f32p),
                       _ptr(gb, _f32p))
    return float(gf[0]), float(gb[0])


# --- the diffusion::Diffusion surface (2D and 3D) ------------------------
# Fields are (ny, nx) arrays in 2D and (nz, ny, nx) in 3D; nd follows the
# array's rank.

def _nd_shape(field):
    if field.ndim == 2:
        ny, nx = field.shape
        return 2, nx, ny, 1
    if field.ndim == 3:
        nz, ny, nx = field.shape
        return 3, nx, ny, nz
    raise ValueError("2D or 3D field expected, got shape %r" % (field.shape,))


def _dims(nd, nx, ny, nz):
    return (nx, ny) if nd == 2 else (nx, ny, nz)


def _shape(nd, nx, ny, nz):
    return (ny, nx) if nd == 2 else (nz, ny, nx)


def dif_params(nd, nx, ny, nz=1, dtype=np.float32):
    """diffusion::Diffusion's (coeff[7], geom[8]) for an nd-D grid."""
    sfx, P = _dt(dtype)
    c = np.zeros(7, dtype)
    g = np.zeros(8, dtype)
    getattr(lib(), "difo_params_" + sfx)(nd, nx, ny, nz if nd == 3 else 1,
                                         _ptr(c, P), _ptr(g, P))
    return c, g


def dif_initialize(nd, nx, ny, nz=1, time=0.0, dtype=np.float32, omp=False):
    """The header's Initialize (omp=False: Baseline's input and the analytic
    answer) or DiffusionOpenMP's InitializeInput (omp=True)."""
    nz = nz if nd == 3 else 1
    sfx, P = _dt(dtype)
    _, g = dif_params(nd, nx, ny, nz, dtype)
    buf = np.empty(_shape(nd, nx, ny, nz), dtype)
    getattr(lib(), "difo_initialize_" + sfx)(
        _ptr(buf, P), nx, ny, nz, g[4], g[5], g[6], g[1], g[2], g[3], g[0],
        time, nd, 1 if omp else 0)
    return buf


def dif_run(field, coeff, count):
    """`count` diffusion::DiffusionOpenMP steps from `field`; a new array."""
    f = np.ascontiguousarray(field)
    sfx, P = _dt(f.dtype)
    nd, nx, ny, nz = _nd_shape(f)
    f1 = f.copy()
    f2 = np.empty_like(f1)
    c = np.ascontiguousarray(coeff, dtype=f.dtype)
    getattr(lib(), "difo_run_" + sfx)(_ptr(f1, P), _ptr(f2, P), nd, nx, ny,
                                      nz, _ptr(c, P), count)
    return f1


def dif_accuracy(field, count):
    """diffusion::Baseline::GetAccuracy restated."""
    f = np.ascontiguousarray(field)
    sfx, P = _dt(f.dtype)
    nd, nx, ny, nz = _nd_shape(f)
    return float(getattr(lib(), "difo_accuracy_" + sfx)(_ptr(f, P), nd, nx,
                                                        ny, nz, count))


def dif_ref_available() -> bool:
    return os.path.exists(DIF_REF_LIB_PATH)


def dif_ref():
    global _dif_ref
    if _dif_ref is None:
        if not dif_ref_available():
            raise FileNotFoundError(DIF_REF_LIB_PATH)
        R = ctypes.CDLL(DIF_REF_LIB_PATH)
        _ip = ctypes.POINTER(ctypes.c_int)
        R.difref_run.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _f32p,
                                 _f32p, _f32p, _f32p, ctypes.c_int, _f32p]
        R.difref_params.argtypes = [ctypes.c_int, _ip, _f32p, _f32p]
        R.difref_initialize.argtypes = ([_f32p] + [ctypes.c_int] * 3
                                        + [ctypes.c_float] * 8
                                        + [ctypes.c_int])
        R.difref_rates.argtypes = [ctypes.c_int, _ip, ctypes.c_int,
                                   ctypes.c_float, _f32p, _f32p]
        _dif_ref = R
    return _dif_ref


def _int_array(vals):
    return (ctypes.c_int * len(vals))(*vals)


def difref_params(nd, nx, ny, nz=1):
    c = np.zeros(7, np.float32)
    g = np.zeros(8, np.float32)
    rc = dif_ref().difref_params(nd, _int_array(_dims(nd, nx, ny, nz)),
                                 _ptr(c, _f32p), _ptr(g, _f32p))
    if rc != 0:
        raise RuntimeError("difref_params failed: %d" % rc)
    return c, g


def difref_initialize(nd, nx, ny, nz=1, time=0.0):
    nz = nz if nd == 3 else 1
    _, g = difref_params(nd, nx, ny, nz)
    buf = np.empty(_shape(nd, nx, ny, nz), np.float32)
    dif_ref().difref_initialize(_ptr(buf, _f32p), nx, ny, nz, g[4], g[5],
                                g[6], g[1], g[2], g[3], g[0], time, nd)
    return buf


def difref_run(nd, nx, ny, nz=1, count=0, field=None, coeff=None,
               backend=DIF_OPENMP, want_accuracy=False):
    """Runs the reference backend; returns (its InitializeInput field, the
    field after `count` steps, GetAccuracy or None)."""
    nz = nz if nd == 3 else 1
    shape = _shape(nd, nx, ny, nz)
    init = np.empty(shape, np.float32)
    out = np.empty(shape, np.float32)
    acc = np.zeros(1, np.float32)
    fin = None if field is None else np.ascontiguousarray(field, np.float32)
    cin = None if coeff is None else np.ascontiguousarray(coeff, np.float32)
    rc = dif_ref().difref_run(
        backend, nd, _int_array(_dims(nd, nx, ny, nz)),
        None if cin is None else _ptr(cin, _f32p),
        None if fin is None else _ptr(fin, _f32p),
        _ptr(init, _f32p), _ptr(out, _f32p), count,
        _ptr(acc, _f32p) if want_accuracy else None)
    if rc != 0:
        raise RuntimeError("difref_run failed: %d" % rc)
    return init, out, (float(acc[0]) if want_accuracy else None)


def difref_rates(nd, nx, ny, nz, count, time):
    gf = np.zeros(1, np.float32)
    gb = np.zeros(1, np.float32)
    dif_ref().difref_rates(nd, _int_array(_dims(nd, nx, ny, nz)), count,
                           time, _ptr(gf, _f32p), _ptr(gb, _f32p))
    return float(gf[0]), float(gb[0])
