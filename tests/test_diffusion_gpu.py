"""GPU parity for the reference's second plugin surface, diffusion::Diffusion
(src/diffusion): the 2D 5-point kernel and the 3D kernels in that surface's
order, through the C ABI (d3d_diffusion_plan_create), against the committed
fixtures (tests/golden/make_golden_diffusion.py, made from the reference's
own objects) and the pinned oracle.  FP32 results must be bit-identical to
diffusion::DiffusionOpenMP; FP64 to the FP64 restatement.
"""
import hashlib

import numpy as np
import pytest

import benchmarks_b200 as B
import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

KERNELS_2D = [B.KERNEL_AUTO, B.KERNEL_GENERIC]
KERNELS_3D = [(B.KERNEL_GENERIC, 1), (B.KERNEL_AUTO, 1), (B.KERNEL_TB, 2),
              (B.KERNEL_TB, 4)]


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _dims(field):
    return tuple(reversed(field.shape))


def gpu_run(field, coeff, count, kernel=B.KERNEL_AUTO, tb=1, zchunk=0,
            offset=0):
    """`count` steps of a DiffusionPlan; `offset` elements of slack in front
    of each device buffer make it misaligned (forcing narrower accesses)."""
    field = np.ascontiguousarray(field)
    dtype = B.F64 if field.dtype == np.float64 else B.F32
    plan = B.DiffusionPlan(_dims(field), dtype, kernel, tb, zchunk=zchunk)
    tdt = torch.float64 if dtype == B.F64 else torch.float32
    n = field.size
    raw1 = torch.empty(n + offset, dtype=tdt, device="cuda")
    raw2 = torch.empty(n + offset, dtype=tdt, device="cuda")
    f1 = raw1[offset:]
    f2 = raw2[offset:]
    f1.copy_(torch.from_numpy(field.reshape(-1)))
    res, _ = plan.run(f1, f2, count, coeff)
    torch.cuda.synchronize()
    assert B.check_device_errors() == 0
    out = res.cpu().numpy().reshape(field.shape)
    info = plan.info()
    plan.close()
    return out, info


def bits_equal(a, b):
    return a.dtype == b.dtype and a.tobytes() == b.tobytes()


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


def _kernels(nd):
    return ([(k, 1) for k in KERNELS_2D] if nd == 2 else KERNELS_3D)


def test_golden_cases_bit_exact(golden_diffusion):
    meta, fields = golden_diffusion
    for case in meta["cases"]:
        fin = _case_input(case, fields)
        for kernel, tb in _kernels(case["nd"]):
            out, info = gpu_run(fin, _coeff(case), case["count"], kernel, tb)
            assert _sha(out) == case["sha256_out"], (case["name"], kernel, tb)
            if case["nd"] == 2 and case["count"] > 0:
                assert info["last_kernel"] == "step2d"
            assert info["surface"] == "diffusion"


def test_driver_known_answers_from_gpu_fields(golden_diffusion):
    """The reference driver's `Accuracy : %e` lines, reproduced from fields
    the GPU computed (Baseline::GetAccuracy restated on the host)."""
    meta, _ = golden_diffusion
    for k in meta["driver_kats"]:
        nd, size, count = k["nd"], k["size"], k["count"]
        nz = size if nd == 3 else 1
        c, _ = O.dif_params(nd, size, size, nz)
        f = O.dif_initialize(nd, size, size, nz,
                             omp=k["backend"] == "openmp")
        out, _ = gpu_run(f, c, count)
        assert "%e" % O.dif_accuracy(out, count) == k["accuracy"], k


@pytest.mark.parametrize("shape", [(1, 1), (1, 7), (7, 1), (3, 2), (9, 130),
                                   (33, 131), (5, 4096), (300, 257),
                                   (64, 128), (2, 1000), (129, 4)])
@pytest.mark.parametrize("offset", [0, 1, 2])
def test_ragged_2d_shapes_and_alignments_vs_oracle(shape, offset):
    """Every (ny, nx) above with 16-, 8- and 4-byte accesses (misaligned
    buffers force the narrower lanes) against the oracle."""
    ny, nx = shape
    c, _ = O.dif_params(2, nx, ny)
    f = O.dif_initialize(2, nx, ny) + O.seeded_noise((ny, nx), nx * ny)
    ref = O.dif_run(f, c, 5)
    out, _ = gpu_run(f, c, 5, offset=offset)
    assert bits_equal(out, ref), (shape, offset)


@pytest.mark.parametrize("ychunk", [1, 2, 3, 4, 5, 6, 7, 13, 64, 1000])
def test_2d_row_chunks(ychunk):
    """Every row-chunk length, including ones shorter than the register
    ring and ones that leave a ragged last chunk."""
    ny, nx = 97, 520
    c, _ = O.dif_params(2, nx, ny)
    f = O.dif_initialize(2, nx, ny) + O.seeded_noise((ny, nx), 5)
    ref = O.dif_run(f, c, 4)
    out, info = gpu_run(f, c, 4, zchunk=ychunk)
    assert info["launch_zchunk"] == min(ychunk, ny)
    assert bits_equal(out, ref)


@pytest.mark.parametrize("variant", range(B.NUM_TILE_VARIANTS))
@pytest.mark.parametrize("ychunk", [0, 3, 16])
@pytest.mark.parametrize("offset", [0, 1])
def test_2d_variants(variant, ychunk, offset):
    """Every register-ring variant of the 2D kernel, with 16-byte and scalar
    lanes, against the oracle."""
    ny, nx = 150, 1028
    c, _ = O.dif_params(2, nx, ny)
    f = O.dif_initialize(2, nx, ny) + O.seeded_noise((ny, nx), 6)
    ref = O.dif_run(f, c, 3)
    field = np.ascontiguousarray(f)
    plan = B.DiffusionPlan((nx, ny), variant=variant, zchunk=ychunk)
    raw1 = torch.empty(field.size + offset, device="cuda")
    raw2 = torch.empty(field.size + offset, device="cuda")
    f1, f2 = raw1[offset:], raw2[offset:]
    f1.copy_(torch.from_numpy(field.reshape(-1)))
    res, _ = plan.run(f1, f2, 3, c)
    out = res.cpu().numpy().reshape(field.shape)
    assert plan.info()["variant"] == variant
    plan.close()
    assert bits_equal(out, ref)


def test_2d_anisotropic_coefficients():
    aniso = np.array([0.11, 0.07, 0.09, 0.13, 0.0, 0.0, 0.6], np.float32)
    ny, nx = 45, 200
    f = O.dif_initialize(2, nx, ny) + O.seeded_noise((ny, nx), 8)
    assert bits_equal(gpu_run(f, aniso, 9)[0], O.dif_run(f, aniso, 9))


@pytest.mark.parametrize("shape", [(23, 37), (64, 64), (40, 6), (17, 131)])
@pytest.mark.parametrize("offset", [0, 1])
def test_2d_fp64_bit_exact_vs_fp64_oracle(shape, offset):
    ny, nx = shape
    c, _ = O.dif_params(2, nx, ny, dtype=np.float64)
    f = (O.dif_initialize(2, nx, ny, dtype=np.float64)
         + O.seeded_noise((ny, nx), 9, dtype=np.float64))
    out, _ = gpu_run(f, c, 7, offset=offset)
    assert bits_equal(out, O.dif_run(f, c, 7))


@pytest.mark.parametrize("kernel,tb", KERNELS_3D + [(B.KERNEL_TB, 3)])
@pytest.mark.parametrize("dims", [(17, 23, 5), (64, 20, 9), (33, 8, 40),
                                  (128, 64, 16)])
def test_3d_surface_order_vs_oracle(kernel, tb, dims):
    """3D through diffusion::Diffusion: the y-1 term summed before y+1 and
    its own cc, on every 3D kernel; and the diffusion3d order differs."""
    nx, ny, nz = dims
    c, _ = O.dif_params(3, nx, ny, nz)
    f = O.dif_initialize(3, nx, ny, nz) + O.seeded_noise((nz, ny, nx), 10)
    ref = O.dif_run(f, c, 6)
    out, info = gpu_run(f, c, 6, kernel, tb)
    assert bits_equal(out, ref), (kernel, tb, dims, info)
    assert not bits_equal(ref, O.run(f, c, 6))


def test_3d_surface_fp64():
    nx, ny, nz = 40, 24, 12
    c, _ = O.dif_params(3, nx, ny, nz, np.float64)
    f = (O.dif_initialize(3, nx, ny, nz, dtype=np.float64)
         + O.seeded_noise((nz, ny, nx), 12, dtype=np.float64))
    for kernel, tb in KERNELS_3D:
        out, _ = gpu_run(f, c, 5, kernel, tb)
        assert bits_equal(out, O.dif_run(f, c, 5)), (kernel, tb)


def test_2d_run_host_and_autotune():
    ny, nx = 512, 768
    plan = B.DiffusionPlan((nx, ny))
    c = plan.reference_coefficients()
    f = O.dif_initialize(2, nx, ny) + O.seeded_noise((ny, nx), 13)
    ref = O.dif_run(f, c, 20)
    f1, f2 = plan.empty(), plan.empty()
    best, info = plan.autotune(f1, f2, steps=4)
    assert best > 0 and info["zchunk"] >= 0
    host = B.pinned_empty((ny, nx))
    host[...] = f
    ms = plan.run_host(host, f1, f2, 20)
    assert ms > 0
    assert bits_equal(np.asarray(host), ref)
    plan.close()


def test_2d_device_accuracy_and_analytic():
    """The FP64 device accuracy report and analytic field of a 2D plan (no
    z factor) against the same closed form evaluated by numpy in double."""
    nx, ny = 256, 192
    plan = B.DiffusionPlan((nx, ny))
    c = plan.reference_coefficients()
    out = O.dif_run(O.dif_initialize(2, nx, ny), c, 100)
    dev = torch.from_numpy(out).cuda()
    _, g32 = B.diffusion_coefficients(2, (nx, ny), B.F32)
    _, g = B.diffusion_coefficients(2, (nx, ny), B.F64)
    kappa, dx, dy, k = g[0], g[1], g[2], g[4]
    t = float(np.float32(100) * g32[7])
    xs = dx * (np.arange(nx) + 0.5)
    ys = dy * (np.arange(ny) + 0.5)
    ana = (0.125 * (1.0 - np.exp(-kappa * t * k * k) * np.cos(k * xs))[None, :]
           * (1.0 - np.exp(-kappa * t * k * k) * np.cos(k * ys))[:, None])
    d = out.astype(np.float64) - ana
    rms, mx, _, total = plan.accuracy(dev, 100)
    assert rms == pytest.approx(np.sqrt(np.mean(d * d)), rel=1e-9)
    assert mx == pytest.approx(np.abs(d).max(), rel=1e-9)
    assert total == pytest.approx(out.astype(np.float64).sum(), rel=1e-12)
    # The reference's own report rounds each analytic value to float (up to
    # half an ulp, 1.5e-8 near 0.25), which is the size of the error itself
    # here: the two reports agree to that rounding.
    assert abs(rms - O.dif_accuracy(out, 100)) < 3e-8
    buf = plan.empty()
    plan.analytic(buf, t)
    assert np.abs(buf.cpu().numpy() - ana).max() < 1e-7
    plan.close()


@pytest.mark.parametrize("shape", [(3, 1 << 24), (1 << 20, 4),
                                   (16384, 16384), (32767, 65536)])
def test_2d_large_and_maximum_sizes(shape):
    """Wide, tall, 1 GiB and 8 GiB (just under the 2^31-point plane limit)
    2D grids: a constant field stays exactly uniform, and sampled points of
    a random field match the reference formula."""
    ny, nx = shape
    c, _ = O.dif_params(2, nx, ny)
    plan = B.DiffusionPlan((nx, ny))
    f1 = torch.full((ny, nx), 0.375, device="cuda")
    f2 = torch.empty_like(f1)
    plan.step(f1, f2, c)
    expect = O.dif_run(np.full((3, 3), 0.375, np.float32), c, 1)[1, 1]
    assert bool((f2 == float(expect)).all())
    gen = torch.Generator(device="cuda").manual_seed(17)
    f1 = torch.rand((ny, nx), device="cuda", generator=gen)
    plan.step(f1, f2, c)
    torch.cuda.synchronize()
    rng = np.random.default_rng(4)
    pts = [(y, x) for y in {0, ny - 1, ny // 2} for x in {0, nx - 1, nx // 3}]
    pts += [(int(rng.integers(ny)), int(rng.integers(nx))) for _ in range(32)]
    ce, cw, cn, cs, _, _, cc = (np.float32(v) for v in c)

    def g(y, x):
        y = min(max(y, 0), ny - 1)
        x = min(max(x, 0), nx - 1)
        return np.float32(f1[y, x].item())

    for y, x in pts:
        v = np.float32(cc * g(y, x))
        v = np.float32(v + np.float32(cw * g(y, x - 1)))
        v = np.float32(v + np.float32(ce * g(y, x + 1)))
        v = np.float32(v + np.float32(cs * g(y - 1, x)))
        v = np.float32(v + np.float32(cn * g(y + 1, x)))
        assert np.float32(f2[y, x].item()) == v, (y, x)
    assert B.check_device_errors() == 0
    plan.close()
