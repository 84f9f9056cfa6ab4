"""diffusion3d on B200: Python bindings over the C ABI of libd3d_b200.so.

The product is the CUDA library behind ``include/d3d_b200.h``; this module
binds it with ctypes so that tests, the benchmark and Python callers drive
exactly the entry points a C/C++ caller (the ``Diffusion3DB200`` plugin)
uses.  PyTorch is used only for device memory and streams.

There is no CPU fallback: if the library is missing or no CUDA device is
present, the compute entry points raise.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "libd3d_b200.so")
HEADER = os.path.join(ROOT, "include", "d3d_b200.h")

D3D_OK = 0
D3D_E_INVALID, D3D_E_CUDA, D3D_E_OOM = -1, -2, -3
D3D_E_TIMEOUT, D3D_E_UNSUPPORTED, D3D_E_BUSY, D3D_E_IO = -4, -5, -6, -7
D3D_E_TRANSPORT = -8
F32, F64 = 0, 1
KERNEL_AUTO, KERNEL_GENERIC, KERNEL_TMA, KERNEL_TB = 0, 1, 2, 3
NUM_TILE_VARIANTS = 6

_vp = ctypes.c_void_p
_vpp = ctypes.POINTER(ctypes.c_void_p)
_i = ctypes.c_int
_sz = ctypes.c_size_t
_dp = ctypes.POINTER(ctypes.c_double)

_SIGNATURES = {
    "d3d_version": ([], ctypes.c_char_p),
    "d3d_last_error": ([], ctypes.c_char_p),
    "d3d_launch_count": ([], ctypes.c_ulonglong),
    "d3d_coefficients": ([_i, _i, _i, _i, _vp, _vp], _i),
    "d3d_plan_create": ([_i, _i, _i, _i, _i, _i, _vpp], _i),
    "d3d_diffusion_coefficients": ([_i, ctypes.POINTER(ctypes.c_int), _i,
                                    _vp, _vp], _i),
    "d3d_diffusion_plan_create": ([_i, ctypes.POINTER(ctypes.c_int), _i, _i,
                                   _i, _vpp], _i),
    "d3d_plan_set_tile": ([_vp, _i, _i], _i),
    "d3d_plan_set_graphs": ([_vp, _i], _i),
    "d3d_plan_autotune": ([_vp, _vp, _vp, _vp, _i, _vp, _dp], _i),
    "d3d_plan_destroy": ([_vp], _i),
    "d3d_plan_info": ([_vp, ctypes.c_char_p, _sz], _i),
    "d3d_device_alloc": ([_sz, _vpp], _i),
    "d3d_device_free": ([_vp], _i),
    "d3d_host_alloc": ([_sz, _vpp], _i),
    "d3d_host_free": ([_vp], _i),
    "d3d_memcpy": ([_vp, _vp, _sz, _vp], _i),
    "d3d_stream_sync": ([_vp], _i),
    "d3d_step": ([_vp, _vp, _vp, _vp, _vp], _i),
    "d3d_step_planes": ([_vp, _vp, _vp, _i, _i, _vp, _vp], _i),
    "d3d_run": ([_vp, _vpp, _vpp, _vp, _i, _vp], _i),
    "d3d_slab_create": ([_i, _i, _i, _i, _i, _i, _i, _vpp,
                         ctypes.POINTER(ctypes.c_int)], _i),
    "d3d_slab_run": ([_vp, _vpp, _vpp, _vp, _i, _vp, _vp], _i),
    "d3d_slab_destroy": ([_vp], _i),
    "d3d_run_host": ([_vp, _vp, _vp, _vp, _vp, _i, _vp,
                      ctypes.POINTER(ctypes.c_float)], _i),
    "d3d_analytic": ([_vp, _vp, ctypes.c_double, _vp], _i),
    "d3d_compare": ([_vp, _vp, _i, _vp, _i, _sz, _dp, _vp], _i),
    "d3d_compare_noalloc": ([_vp, _i, _vp, _i, _sz, _dp, _vp], _i),
    "d3d_checkpoint_save": ([_vp, _vp, ctypes.c_longlong, ctypes.c_char_p,
                             _vp], _i),
    "d3d_checkpoint_load": ([_vp, ctypes.c_char_p, _vp,
                             ctypes.POINTER(ctypes.c_longlong), _vp], _i),
    "d3d_checkpoint_save_host": ([_vp, _vp, ctypes.c_longlong,
                                  ctypes.c_char_p], _i),
    "d3d_batch_coefficients": ([_i, _i, _i, ctypes.c_float,
                                ctypes.POINTER(ctypes.c_float)], _i),
    "d3d_batch_layout": ([_vp, _i, ctypes.POINTER(ctypes.c_size_t)], _i),
    "d3d_batch_create": ([_vp, _i, _vp, _sz, _vpp], _i),
    "d3d_batch_autotune": ([_vp, _vp], _i),
    "d3d_copy_calibrate": ([_vp, _vp, _sz, ctypes.c_float, _i, _vp,
                            ctypes.POINTER(ctypes.c_float)], _i),
    "d3d_batch_set_kind": ([_vp, _i], _i),
    "d3d_batch_set_resident_max_cluster": ([_vp, _i], _i),
    "d3d_batch_run": ([_vp, _vp, ctypes.POINTER(ctypes.c_float)], _i),
    "d3d_batch_info": ([_vp, ctypes.c_char_p, _sz], _i),
    "d3d_batch_progress": ([_vp, ctypes.POINTER(ctypes.c_int), _i], _i),
    "d3d_batch_destroy": ([_vp], _i),
    "d3d_server_set_resident": ([_vp, _i], _i),
    "d3d_server_set_large_kernel": ([_vp, _i, _i], _i),
    "d3d_server_create": ([_sz, _i, _vpp], _i),
    "d3d_server_submit": ([_vp, _i, _i, _i, _i,
                           ctypes.POINTER(ctypes.c_float), _vp, _vp,
                           ctypes.POINTER(ctypes.c_longlong)], _i),
    "d3d_server_tick": ([_vp, ctypes.POINTER(ctypes.c_longlong), _i,
                         ctypes.POINTER(ctypes.c_int)], _i),
    "d3d_server_pending": ([_vp, ctypes.POINTER(ctypes.c_int),
                            ctypes.POINTER(ctypes.c_int),
                            ctypes.POINTER(ctypes.c_int)], _i),
    "d3d_server_stats": ([_vp, ctypes.c_char_p, _sz], _i),
    "d3d_server_set_kernel": ([_vp, _i], _i),
    "d3d_server_set_lanes": ([_vp, _i], _i),
    "d3d_server_destroy": ([_vp], _i),
    "d3d_check_device_errors": ([ctypes.POINTER(ctypes.c_uint)], _i),
    "d3d_accuracy": ([_vp, _vp, _i, _dp, _vp], _i),
    "d3d_selftest_wait_timeout": ([ctypes.c_uint,
                                   ctypes.POINTER(ctypes.c_uint)], _i),
}

_lib = None


class D3DError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("d3d error %d: %s" % (code, msg))
        self.code = code


def declared_symbols(header: str = HEADER) -> list:
    """Function names declared in include/d3d_b200.h."""
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(d3d_[a-z0-9_]+)\s*\(", text)))


def build(force: bool = False) -> str:
    from . import _build
    return _build.build(force=force)


def lib():
    """The loaded library (built first if absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != D3D_OK:
        raise D3DError(rc, lib().d3d_last_error().decode())


def version() -> str:
    return lib().d3d_version().decode()


def launch_count() -> int:
    return int(lib().d3d_launch_count())


def np_dtype(dtype: int):
    return np.float64 if dtype == F64 else np.float32


def coefficients(nx, ny, nz, dtype=F32):
    """Reference-constructor coefficients (ce,cw,cn,cs,ct,cb,cc) and geometry
    (kappa,dx,dy,dz,kx,ky,kz,dt) in `dtype` -- a host-only entry point."""
    c = np.zeros(7, np_dtype(dtype))
    g = np.zeros(8, np_dtype(dtype))
    check(lib().d3d_coefficients(nx, ny, nz, dtype, c.ctypes.data,
                                 g.ctypes.data))
    return c, g


def _stream_handle(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _torch_dtype(dtype):
    import torch
    return torch.float64 if dtype == F64 else torch.float32


class Plan:
    """A d3d_plan: one grid shape, precision and kernel choice."""

    ndim = 3

    def __init__(self, nx, ny, nz, dtype=F32, kernel=KERNEL_AUTO, tb_depth=1,
                 variant=None, zchunk=0):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.dtype = dtype
        self.kernel = kernel
        self.tb_depth = tb_depth
        h = ctypes.c_void_p()
        check(self._create(ctypes.byref(h)))
        self._h = h
        if variant is not None or zchunk:
            self.set_tile(variant or 0, zchunk)

    def _create(self, out):
        return lib().d3d_plan_create(self.nx, self.ny, self.nz, self.dtype,
                                     self.kernel, self.tb_depth, out)

    @property
    def handle(self):
        return self._h

    @property
    def n(self):
        return self.nx * self.ny * self.nz

    @property
    def nbytes(self):
        return self.n * (8 if self.dtype == F64 else 4)

    def set_tile(self, variant, zchunk=0):
        check(lib().d3d_plan_set_tile(self._h, variant, zchunk))

    def autotune(self, f1, f2, steps=10, coeff=None, stream=None):
        """Times tile variants / z-chunks on f1, f2 (overwritten); keeps the
        fastest.  Returns (best ms per step, plan info)."""
        self._check_buf(f1)
        self._check_buf(f2)
        c = self._coeff(coeff)
        best = ctypes.c_double()
        check(lib().d3d_plan_autotune(self._h, f1.data_ptr(), f2.data_ptr(),
                                      c.ctypes.data, steps,
                                      _stream_handle(stream),
                                      ctypes.byref(best)))
        return best.value, self.info()

    def set_graphs(self, enable: bool):
        check(lib().d3d_plan_set_graphs(self._h, 1 if enable else 0))

    def info(self) -> dict:
        import json
        buf = ctypes.create_string_buffer(1024)
        check(lib().d3d_plan_info(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    def close(self):
        if getattr(self, "_h", None):
            lib().d3d_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- coefficient helpers -------------------------------------------
    def reference_coefficients(self):
        return coefficients(self.nx, self.ny, self.nz, self.dtype)[0]

    def _coeff(self, coeff):
        if coeff is None:
            coeff = self.reference_coefficients()
        c = np.ascontiguousarray(coeff, dtype=np_dtype(self.dtype))
        assert c.shape == (7,)
        return c

    # --- compute entry points (device buffers: torch tensors) -----------
    @property
    def shape(self):
        """Array shape of one field: (nz, ny, nx), or (ny, nx) in 2D."""
        if self.ndim == 2:
            return (self.ny, self.nx)
        return (self.nz, self.ny, self.nx)

    def empty(self):
        import torch
        return torch.empty(self.shape, dtype=_torch_dtype(self.dtype),
                           device="cuda")

    def _check_buf(self, t):
        assert t.is_cuda and t.is_contiguous() and t.numel() == self.n
        assert t.dtype == _torch_dtype(self.dtype)

    def step(self, f1, f2, coeff=None, stream=None):
        self._check_buf(f1)
        self._check_buf(f2)
        c = self._coeff(coeff)
        check(lib().d3d_step(self._h, f1.data_ptr(), f2.data_ptr(),
                             c.ctypes.data, _stream_handle(stream)))

    def step_planes(self, f1, f2, z_begin, z_end, coeff=None, stream=None):
        """One step of output planes [z_begin, z_end) (d3d_step_planes)."""
        self._check_buf(f1)
        self._check_buf(f2)
        c = self._coeff(coeff)
        check(lib().d3d_step_planes(self._h, f1.data_ptr(), f2.data_ptr(),
                                    int(z_begin), int(z_end), c.ctypes.data,
                                    _stream_handle(stream)))

    def run(self, f1, f2, count, coeff=None, stream=None):
        """`count` steps ping-ponging f1/f2; returns (result, other)."""
        self._check_buf(f1)
        self._check_buf(f2)
        c = self._coeff(coeff)
        a = ctypes.c_void_p(f1.data_ptr())
        b = ctypes.c_void_p(f2.data_ptr())
        check(lib().d3d_run(self._h, ctypes.byref(a), ctypes.byref(b),
                            c.ctypes.data, count, _stream_handle(stream)))
        if a.value == f1.data_ptr():
            return f1, f2
        return f2, f1

    def run_host(self, host, f1, f2, count, coeff=None, stream=None):
        """Diffusion3DCUDA::RunKernel semantics: host -> device, count steps,
        result back into `host` (a C-contiguous numpy array, ideally
        pinned).  Returns the kernel-only milliseconds."""
        assert host.flags["C_CONTIGUOUS"] and host.size == self.n
        assert host.dtype == np_dtype(self.dtype)
        self._check_buf(f1)
        self._check_buf(f2)
        c = self._coeff(coeff)
        ms = ctypes.c_float()
        check(lib().d3d_run_host(self._h, host.ctypes.data, f1.data_ptr(),
                                 f2.data_ptr(), c.ctypes.data, count,
                                 _stream_handle(stream), ctypes.byref(ms)))
        return ms.value

    def analytic(self, out, time, stream=None):
        self._check_buf(out)
        check(lib().d3d_analytic(self._h, out.data_ptr(), float(time),
                                 _stream_handle(stream)))

    def accuracy(self, field, count, stream=None):
        """FP64 (rms, max_abs, max_rel, sum) of `field` against the analytic
        solution after `count` steps, on the device."""
        self._check_buf(field)
        out = np.zeros(4, np.float64)
        check(lib().d3d_accuracy(self._h, field.data_ptr(), count,
                                 out.ctypes.data_as(_dp),
                                 _stream_handle(stream)))
        return out

    def save_checkpoint(self, field, path, step=0, stream=None):
        """Binary checkpoint of a device field (d3d_checkpoint_save)."""
        self._check_buf(field)
        check(lib().d3d_checkpoint_save(self._h, field.data_ptr(), int(step),
                                        os.fsencode(path),
                                        _stream_handle(stream)))

    def load_checkpoint(self, path, field, stream=None):
        """Reads a checkpoint into a device field; returns its step."""
        self._check_buf(field)
        step = ctypes.c_longlong()
        check(lib().d3d_checkpoint_load(self._h, os.fsencode(path),
                                        field.data_ptr(), ctypes.byref(step),
                                        _stream_handle(stream)))
        return step.value

    def compare(self, a, b, stream=None):
        """FP64 (rms, max_abs, max_rel, sum(a)) of device field a vs b."""
        import torch
        assert a.numel() == b.numel()
        dt = {torch.float32: F32, torch.float64: F64}
        out = np.zeros(4, np.float64)
        check(lib().d3d_compare(self._h, a.data_ptr(), dt[a.dtype],
                                b.data_ptr(), dt[b.dtype], a.numel(),
                                out.ctypes.data_as(_dp),
                                _stream_handle(stream)))
        return out


def diffusion_coefficients(nd, dims, dtype=F32):
    """(coeff[7], geom[8]) as diffusion::Diffusion(nd, dims) derives them
    (dims = (nx, ny) or (nx, ny, nz))."""
    c = np.zeros(7, np_dtype(dtype))
    g = np.zeros(8, np_dtype(dtype))
    d = (ctypes.c_int * len(dims))(*dims)
    check(lib().d3d_diffusion_coefficients(nd, d, dtype, c.ctypes.data,
                                           g.ctypes.data))
    return c, g


class DiffusionPlan(Plan):
    """A plan for the reference's diffusion::Diffusion surface: a 2D
    5-point grid (dims = (nx, ny)) or a 3D grid (dims = (nx, ny, nz)) summed
    in that surface's order.  Fields are (ny, nx) or (nz, ny, nx) arrays."""

    def __init__(self, dims, dtype=F32, kernel=KERNEL_AUTO, tb_depth=1,
                 variant=None, zchunk=0):
        dims = tuple(int(d) for d in dims)
        if len(dims) not in (2, 3):
            raise ValueError("dims must be (nx, ny) or (nx, ny, nz)")
        self.ndim = len(dims)
        self.dims = dims
        nz = dims[2] if self.ndim == 3 else 1
        super().__init__(dims[0], dims[1], nz, dtype, kernel, tb_depth,
                         variant, zchunk)

    def _create(self, out):
        d = (ctypes.c_int * self.ndim)(*self.dims)
        return lib().d3d_diffusion_plan_create(self.ndim, d, self.dtype,
                                               self.kernel, self.tb_depth,
                                               out)

    def reference_coefficients(self):
        return diffusion_coefficients(self.ndim, self.dims, self.dtype)[0]


# Kernel kinds of the batch API (d3d_batch_set_kind); kind 8 is the
# cluster-resident kernel for every grid it fits.
BATCH_NUM_KINDS = 9
BATCH_KIND_RESIDENT = 8


class BatchGrid(ctypes.Structure):
    """d3d_batch_grid: one grid of a batch."""
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("nz", ctypes.c_int), ("steps", ctypes.c_int),
                ("coeff", ctypes.c_float * 7),
                ("offset_a", ctypes.c_ulonglong),
                ("offset_b", ctypes.c_ulonglong)]


def copy_calibrate(f1, f2, passes=10, cc=0.4, stream=None):
    """HBM calibration (d3d_copy_calibrate): `passes` ping-pong passes of
    f2 = cc * f1 over two float32 CUDA tensors of equal size; returns
    (device ms, GB/s at 8 bytes per point per pass)."""
    assert str(f1.dtype) == "torch.float32" == str(f2.dtype)
    assert f1.numel() == f2.numel()
    ms = ctypes.c_float()
    check(lib().d3d_copy_calibrate(f1.data_ptr(), f2.data_ptr(), f1.numel(),
                                   cc, passes, _stream_handle(stream),
                                   ctypes.byref(ms)))
    return ms.value, 8.0 * f1.numel() * passes / (ms.value * 1e-3) / 1e9


def batch_coefficients(nx, ny, nz, kappa):
    """Stable coefficients for any grid shape (dt from the smallest spacing)."""
    c = (ctypes.c_float * 7)()
    check(lib().d3d_batch_coefficients(nx, ny, nz, kappa, c))
    return np.array(list(c), np.float32)


class Batch:
    """Many independent FP32 grids advanced by the batched multi-grid
    kernel.  `specs` is a list of (nx, ny, nz, steps, coeff7)."""

    def __init__(self, specs):
        import torch
        n = len(specs)
        arr = (BatchGrid * n)()
        for i, (nx, ny, nz, steps, coeff) in enumerate(specs):
            arr[i].nx, arr[i].ny, arr[i].nz, arr[i].steps = nx, ny, nz, steps
            for j in range(7):
                arr[i].coeff[j] = float(coeff[j])
        nbytes = ctypes.c_size_t()
        check(lib().d3d_batch_layout(arr, n, ctypes.byref(nbytes)))
        self.grids = arr
        self.arena = torch.zeros(max(nbytes.value // 4, 1),
                                 dtype=torch.float32, device="cuda")
        h = ctypes.c_void_p()
        check(lib().d3d_batch_create(arr, n, self.arena.data_ptr(),
                                     nbytes.value, ctypes.byref(h)))
        self._h = h

    def __len__(self):
        return len(self.grids)

    def _view(self, i, which):
        g = self.grids[i]
        off = g.offset_a if which == 0 else g.offset_b
        n = g.nx * g.ny * g.nz
        return self.arena[off:off + n].view(g.nz, g.ny, g.nx)

    def input(self, i):
        """Device view of grid i's input buffer (write the field here)."""
        return self._view(i, 0)

    def result(self, i):
        """Device view of grid i's field after its steps."""
        return self._view(i, self.grids[i].steps & 1)

    def autotune(self, stream=None):
        check(lib().d3d_batch_autotune(self._h, _stream_handle(stream)))

    def set_kind(self, kind):
        """Every size class to one kernel kind: 0..3 the march kernel's
        tile shapes, 4 and 5 the strip kernel (4 is the default), 6 and 7
        its two-step form (grids at most 248 floats wide), 8 the
        cluster-resident kernel for every grid it fits."""
        check(lib().d3d_batch_set_kind(self._h, int(kind)))

    def set_resident_max_cluster(self, n):
        """Cluster-resident kernel only for grids that fit clusters of at
        most n CTAs (1..16); 0 turns it off."""
        check(lib().d3d_batch_set_resident_max_cluster(self._h, int(n)))

    def run(self, stream=None, timed=True):
        ms = ctypes.c_float()
        check(lib().d3d_batch_run(self._h, _stream_handle(stream),
                                  ctypes.byref(ms) if timed else None))
        return ms.value

    def info(self):
        import json
        buf = ctypes.create_string_buffer(16384)
        check(lib().d3d_batch_info(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    def progress(self):
        """Per-grid step counters of the last run (d3d_batch_progress)."""
        out = np.zeros(len(self.grids), np.int32)
        check(lib().d3d_batch_progress(
            self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
            len(out)))
        return out

    def close(self):
        if getattr(self, "_h", None):
            lib().d3d_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching solve server (d3d_server_*).  submit() queues a
    solve with host input/output arrays (C-contiguous float32; pinned for
    asynchronous copies); tick() runs one scheduling round and returns the
    ids that finished."""

    def __init__(self, arena_bytes, chunk=8, kernel=None, lanes=None,
                 resident=None):
        h = ctypes.c_void_p()
        check(lib().d3d_server_create(int(arena_bytes), chunk,
                                      ctypes.byref(h)))
        self._h = h
        if kernel is not None:
            self.set_kernel(kernel)
        if lanes is not None:
            self.set_lanes(lanes)
        if resident is not None:
            self.set_resident(resident)
        self._keep = {}
        self._ids = (ctypes.c_longlong * 4096)()

    def submit(self, host_in, host_out, steps, coeff):
        assert host_in.dtype == np.float32 and host_out.dtype == np.float32
        assert host_in.flags["C_CONTIGUOUS"] and host_out.flags["C_CONTIGUOUS"]
        assert host_in.shape == host_out.shape and host_in.ndim == 3
        nz, ny, nx = host_in.shape
        c = (ctypes.c_float * 7)(*[float(v) for v in coeff])
        rid = ctypes.c_longlong()
        check(lib().d3d_server_submit(self._h, nx, ny, nz, steps, c,
                                      host_in.ctypes.data,
                                      host_out.ctypes.data,
                                      ctypes.byref(rid)))
        self._keep[rid.value] = (host_in, host_out)
        return rid.value

    def tick(self):
        n = ctypes.c_int()
        check(lib().d3d_server_tick(self._h, self._ids, len(self._ids),
                                    ctypes.byref(n)))
        done = [self._ids[i] for i in range(n.value)]
        for i in done:
            self._keep.pop(i, None)
        return done

    def set_kernel(self, kernel):
        """Step kernel of the idle server: 0..4 the pitched TMA kernel's
        tile shapes, 5 and 6 its strip form with 1 or 2 segments a thread
        (6 is the default), -1 the batch API's march kernel."""
        check(lib().d3d_server_set_kernel(self._h, int(kernel)))

    def set_lanes(self, lanes):
        """Compute streams of the idle server (1..8, default 4)."""
        check(lib().d3d_server_set_lanes(self._h, int(lanes)))

    def set_large_kernel(self, kernel, min_px=128):
        """Step kernel of the idle server's large solves (pitched rows of at
        least min_px floats), on the upper half of the lanes; kernel < 0
        turns it off."""
        check(lib().d3d_server_set_large_kernel(self._h, int(kernel),
                                                int(min_px)))

    def set_resident(self, on):
        """Whether the idle server runs the solves that fit it on the
        cluster-resident kernel (default off)."""
        check(lib().d3d_server_set_resident(self._h, int(bool(on))))

    def pending(self):
        q, a, r = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().d3d_server_pending(self._h, ctypes.byref(q),
                                       ctypes.byref(a), ctypes.byref(r)))
        return q.value, a.value, r.value

    def drain(self):
        """Ticks until every submitted request is done; returns their ids."""
        done = []
        while sum(self.pending()):
            done += self.tick()
        return done

    def stats(self):
        import json
        buf = ctypes.create_string_buffer(1024)
        check(lib().d3d_server_stats(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    def close(self):
        if getattr(self, "_h", None):
            lib().d3d_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


NOALLOC_MAX_ELEMENTS = 1 << 28


# --- binary checkpoints on the host (the d3d_checkpoint_* file format) ----
_CKPT_HEADER = np.dtype([("magic", "S8"), ("header_bytes", "<u4"),
                         ("dtype", "<u4"), ("ndim", "<u4"), ("nx", "<i4"),
                         ("ny", "<i4"), ("nz", "<i4"), ("step", "<i8"),
                         ("checksum", "<u8"), ("payload", "<u8"),
                         ("flags", "<u4"), ("reserved", "<u4")])
assert _CKPT_HEADER.itemsize == 64


def _word_sum(a):
    """The checksum: the sum of the 32-bit words modulo 2^64."""
    return int(np.ascontiguousarray(a).view(np.uint32).sum(dtype=np.uint64))


def read_checkpoint(path):
    """(header dict, field array) of a checkpoint file, on the host; the
    field is (ny, nx) in 2D, (nz, ny, nx) in 3D.  Raises ValueError on a bad
    magic, size or checksum."""
    with open(path, "rb") as f:
        raw = f.read(64)
        if len(raw) != 64:
            raise ValueError("%s: truncated header" % path)
        h = np.frombuffer(raw, _CKPT_HEADER)[0]
        if h["magic"] != b"D3DCKPT1" or h["header_bytes"] != 64:
            raise ValueError("%s is not a d3d checkpoint" % path)
        dt = np.float64 if h["dtype"] == F64 else np.float32
        shape = ((int(h["ny"]), int(h["nx"])) if h["ndim"] == 2 else
                 (int(h["nz"]), int(h["ny"]), int(h["nx"])))
        n = int(np.prod(shape))
        data = np.fromfile(f, dtype=dt, count=n)
    if data.size != n or data.nbytes != int(h["payload"]):
        raise ValueError("%s is truncated" % path)
    if _word_sum(data) != int(h["checksum"]):
        raise ValueError("%s failed its checksum" % path)
    head = {k: (h[k].item() if k != "magic" else h[k].decode())
            for k in _CKPT_HEADER.names}
    return head, data.reshape(shape)


def write_checkpoint(path, field, step=0, diffusion_surface=False):
    """Writes a host array as a checkpoint that d3d_checkpoint_load accepts
    ((ny, nx) arrays are 2D, (nz, ny, nx) arrays 3D)."""
    a = np.ascontiguousarray(field)
    if a.dtype not in (np.float32, np.float64) or a.ndim not in (2, 3):
        raise ValueError("FP32/FP64 2D or 3D array expected")
    h = np.zeros((), _CKPT_HEADER)
    h["magic"] = b"D3DCKPT1"
    h["header_bytes"] = 64
    h["dtype"] = F64 if a.dtype == np.float64 else F32
    h["ndim"] = a.ndim
    h["nx"], h["ny"] = a.shape[-1], a.shape[-2]
    h["nz"] = a.shape[0] if a.ndim == 3 else 1
    h["step"] = step
    h["checksum"] = _word_sum(a)
    h["payload"] = a.nbytes
    h["flags"] = 1 if diffusion_surface else 0
    with open(path, "wb") as f:
        f.write(h.tobytes())
        a.tofile(f)


def compare_noalloc(a, b, stream=None):
    """d3d_compare_noalloc: FP64 (rms, max_abs, max_rel, sum(a)) of device
    field a against b without any device allocation (n <= 2^28)."""
    import torch
    assert a.numel() == b.numel()
    dt = {torch.float32: F32, torch.float64: F64}
    out = np.zeros(4, np.float64)
    check(lib().d3d_compare_noalloc(a.data_ptr(), dt[a.dtype], b.data_ptr(),
                                    dt[b.dtype], a.numel(),
                                    out.ctypes.data_as(_dp),
                                    _stream_handle(stream)))
    return out


def check_device_errors() -> int:
    flags = ctypes.c_uint()
    rc = lib().d3d_check_device_errors(ctypes.byref(flags))
    if rc not in (D3D_OK, D3D_E_TIMEOUT):
        check(rc)
    return flags.value


def pinned_empty(shape, dtype=np.float32):
    """A numpy view of a pinned host buffer (torch pinned memory)."""
    import torch
    tdt = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
    t = torch.empty(tuple(shape), dtype=tdt, pin_memory=True)
    return t.numpy()
