"""C-ABI checks that need no GPU: the library loads, exports every symbol
include/d3d_b200.h declares, and its host-only entry points behave."""
import ctypes
import subprocess

import numpy as np
import pytest

import benchmarks_b200 as B
import oracle as O


def test_library_loads_and_exports_declared_symbols():
    L = B.lib()
    declared = B.declared_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
    # and nothing exported under d3d_ that the header does not declare
    out = subprocess.run(["nm", "-D", "--defined-only", B.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = sorted({ln.split()[-1] for ln in out.splitlines()
                       if ln.split() and ln.split()[-1].startswith("d3d_")})
    assert exported == declared


def test_version_and_last_error():
    assert "sm_100a" in B.version()
    rc = B.lib().d3d_coefficients(0, 4, 4, B.F32, None, None)
    assert rc == B.D3D_E_INVALID
    assert "bad dims" in B.lib().d3d_last_error().decode()


@pytest.mark.parametrize("dims", [(64, 64, 64), (17, 23, 5), (512, 512, 512),
                                  (24, 40, 16), (1, 1, 1), (96, 16, 33)])
def test_coefficients_match_oracle(dims):
    for dt, npdt in ((B.F32, np.float32), (B.F64, np.float64)):
        c, g = B.coefficients(*dims, dtype=dt)
        oc, og = O.params(*dims, dtype=npdt)
        assert c.tobytes() == oc.tobytes()
        assert g.tobytes() == og.tobytes()


def test_plan_create_rejects_bad_arguments():
    h = ctypes.c_void_p()
    L = B.lib()
    assert L.d3d_plan_create(0, 1, 1, B.F32, 0, 1, ctypes.byref(h)) \
        == B.D3D_E_INVALID
    assert L.d3d_plan_create(4, 4, 4, 7, 0, 1, ctypes.byref(h)) \
        == B.D3D_E_INVALID
    assert L.d3d_plan_create(4, 4, 4, B.F32, 9, 1, ctypes.byref(h)) \
        == B.D3D_E_INVALID
    assert L.d3d_plan_create(4, 4, 4, B.F32, B.KERNEL_TB, 7,
                             ctypes.byref(h)) == B.D3D_E_UNSUPPORTED
    assert L.d3d_plan_create(1 << 16, 1 << 16, 1, B.F32, 0, 1,
                             ctypes.byref(h)) == B.D3D_E_INVALID
    assert L.d3d_step(None, None, None, None, None) == B.D3D_E_INVALID
    assert L.d3d_run(None, None, None, None, 1, None) == B.D3D_E_INVALID


def test_slab_create_rejects_bad_geometry():
    """d3d_slab_create checks its geometry before any device work."""
    h = ctypes.c_void_p()
    L = B.lib()
    bad = [
        (0, 4, 16, 0, 8, 1),     # nx < 1
        (4, 4, 16, 8, 8, 1),     # empty slab
        (4, 4, 16, 0, 17, 1),    # past the grid
        (4, 4, 16, 0, 8, 0),     # halo < 1
        (4, 4, 16, 1, 9, 2),     # the rank below holds 1 plane < halo
        (4, 4, 16, 8, 15, 2),    # the rank above holds 1 plane < halo
        (4, 4, 16, 4, 7, 2),     # 3 owned planes < 2 x halo with neighbours
    ]
    for nx, ny, nz, z0, z1, halo in bad:
        assert L.d3d_slab_create(nx, ny, nz, z0, z1, halo, B.F32,
                                 ctypes.byref(h), None) == B.D3D_E_INVALID
    assert L.d3d_slab_create(4, 4, 16, 0, 16, 1, 5, ctypes.byref(h),
                             None) == B.D3D_E_INVALID       # dtype
    assert L.d3d_slab_create(4, 4, 16, 0, 16, 1, B.F32, None,
                             None) == B.D3D_E_INVALID       # no output
    assert L.d3d_slab_run(None, None, None, None, 1, None, None) \
        == B.D3D_E_INVALID
    assert L.d3d_slab_destroy(None) == B.D3D_OK


@pytest.mark.parametrize("nd,dims", [(2, (256, 256)), (2, (37, 23)),
                                     (2, (1, 1)), (3, (64, 64, 64)),
                                     (3, (17, 23, 5)), (3, (24, 40, 16))])
def test_diffusion_coefficients_match_oracle(nd, dims):
    """diffusion::Diffusion's constructor (its cc sums the z pair as a unit)
    through d3d_diffusion_coefficients, against the pinned restatement."""
    nz = dims[2] if nd == 3 else 1
    for dt, npdt in ((B.F32, np.float32), (B.F64, np.float64)):
        c, g = B.diffusion_coefficients(nd, dims, dt)
        oc, og = O.dif_params(nd, dims[0], dims[1], nz, npdt)
        assert c.tobytes() == oc.tobytes()
        assert g.tobytes() == og.tobytes()


def test_diffusion_plan_rejects_bad_arguments():
    h = ctypes.c_void_p()
    L = B.lib()
    d2 = (ctypes.c_int * 2)(16, 16)
    d3 = (ctypes.c_int * 3)(16, 16, 0)
    assert L.d3d_diffusion_plan_create(4, d2, B.F32, 0, 1,
                                       ctypes.byref(h)) == B.D3D_E_INVALID
    assert L.d3d_diffusion_plan_create(2, None, B.F32, 0, 1,
                                       ctypes.byref(h)) == B.D3D_E_INVALID
    assert L.d3d_diffusion_plan_create(3, d3, B.F32, 0, 1,
                                       ctypes.byref(h)) == B.D3D_E_INVALID
    for kernel in (B.KERNEL_TMA, B.KERNEL_TB):
        assert L.d3d_diffusion_plan_create(2, d2, B.F32, kernel, 2,
                                           ctypes.byref(h)) \
            == B.D3D_E_UNSUPPORTED
    assert L.d3d_diffusion_coefficients(1, d2, B.F32, None, None) \
        == B.D3D_E_INVALID


def test_copy_calibrate_rejects_bad_arguments():
    """Argument checks run before any device work."""
    L = B.lib()
    ms = ctypes.c_float()
    assert L.d3d_copy_calibrate(None, None, 8, 0.4, 1, None,
                                ctypes.byref(ms)) == B.D3D_E_INVALID
    # overlapping buffers
    assert L.d3d_copy_calibrate(4096, 4096 + 16, 64, 0.4, 1, None,
                                ctypes.byref(ms)) == B.D3D_E_INVALID
    assert L.d3d_copy_calibrate(4096, 1 << 20, 64, 0.4, 0, None,
                                ctypes.byref(ms)) == B.D3D_E_INVALID


@pytest.mark.gpu
@pytest.mark.parametrize("n,offset", [(1 << 20, 0), (1000003, 0), (4099, 1),
                                      (3, 0), (1, 2)])
def test_copy_calibrate_scales_exactly(n, offset):
    """One pass writes cc * f1 into f2 bit-exactly (16-byte vector body and
    scalar tail, or scalar throughout for misaligned buffers); a second
    pass writes cc * f2 back into f1."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(7)
    buf1 = torch.rand(n + offset, device="cuda", generator=g)
    buf2 = torch.zeros(n + offset, device="cuda")
    f1, f2 = buf1[offset:], buf2[offset:]
    x = f1.cpu().numpy().copy()
    cc = np.float32(0.4)
    ms, gbs = B.copy_calibrate(f1, f2, passes=1, cc=float(cc))
    assert ms > 0 and gbs > 0
    assert f2.cpu().numpy().tobytes() == (cc * x).astype(np.float32).tobytes()
    B.copy_calibrate(f1, f2, passes=2, cc=float(cc))
    y = (cc * (cc * x).astype(np.float32)).astype(np.float32)
    assert f1.cpu().numpy().tobytes() == y.tobytes()
