"""GPU parity: every kernel, through the C ABI, against the oracle.

FP32 results must be bit-identical to the reference's Diffusion3DOpenMP
(tests/golden, generated from the reference's own objects, and the pinned
oracle for other shapes); FP64 results bit-identical to the FP64
restatement.  At full sizes, where the CPU oracle is too slow, kernels are
checked against each other (a size-independent property: every kernel
computes the same bits).
"""
import hashlib

import numpy as np
import pytest

import benchmarks_b200 as B
import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

ALL_KERNELS = [(B.KERNEL_GENERIC, 1), (B.KERNEL_AUTO, 1), (B.KERNEL_TB, 2),
               (B.KERNEL_TB, 3), (B.KERNEL_TB, 4)]


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def gpu_run(field, coeff, count, kernel=B.KERNEL_AUTO, tb=1, variant=None,
            zchunk=0):
    field = np.ascontiguousarray(field)
    dtype = B.F64 if field.dtype == np.float64 else B.F32
    nz, ny, nx = field.shape
    plan = B.Plan(nx, ny, nz, dtype, kernel, tb, variant=variant,
                  zchunk=zchunk)
    f1 = torch.from_numpy(field).cuda()
    f2 = torch.empty_like(f1)
    res, _ = plan.run(f1, f2, count, coeff)
    torch.cuda.synchronize()
    assert B.check_device_errors() == 0
    out = res.cpu().numpy()
    plan.close()
    return out


def bits_equal(a, b):
    return a.dtype == b.dtype and a.tobytes() == b.tobytes()


def _coeff(case):
    return np.array(case["coeff_hex"], np.uint32).view(np.float32)


def _case_input(case, fields):
    key = case["name"] + "/in"
    if key in fields:
        return fields[key]
    f = O.initialize(case["nx"], case["ny"], case["nz"])
    if case["noise_seed"] is not None:
        f = f + O.seeded_noise(f.shape, case["noise_seed"])
    return f


@pytest.mark.parametrize("kernel,tb", ALL_KERNELS)
def test_golden_small_cases_bit_exact(golden, kernel, tb):
    meta, fields = golden
    for case in meta["cases"]:
        if case["name"] + "/out" not in fields:
            continue
        out = gpu_run(fields[case["name"] + "/in"], _coeff(case),
                      case["count"], kernel, tb)
        assert bits_equal(out, fields[case["name"] + "/out"]), case["name"]


@pytest.mark.parametrize("kernel,tb", ALL_KERNELS)
@pytest.mark.parametrize("name", ["c64_n100", "c128_n100", "c256_n100",
                                  "c128_n1000_noise"])
def test_golden_reference_configs_bit_exact(golden, kernel, tb, name):
    """The reference's own runs (64^3/100, 128^3/100, 256^3/100 and a
    1000-step noisy 128^3 run): same sha256 of the output bytes, same
    GetAccuracy."""
    meta, fields = golden
    case = {c["name"]: c for c in meta["cases"]}[name]
    out = gpu_run(_case_input(case, fields), _coeff(case), case["count"],
                  kernel, tb)
    assert _sha(out) == case["sha256_out"]
    acc = O.accuracy(out, case["count"])
    assert np.float32(acc) == np.float32(case["accuracy"])


SHAPES = [(1, 1, 1), (4, 1, 1), (1, 5, 3), (8, 8, 1), (8, 8, 2), (16, 3, 7),
          (33, 17, 9), (36, 20, 11), (128, 9, 5), (132, 18, 12),
          (260, 33, 6), (64, 130, 3), (7, 300, 4)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("kernel,tb", ALL_KERNELS)
def test_ragged_shapes_vs_oracle(shape, kernel, tb):
    nx, ny, nz = shape
    c, _ = O.params(nx, ny, nz)
    fin = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 21)
    for count in (0, 1, 5):
        ref = O.run(fin, c, count)
        out = gpu_run(fin, c, count, kernel, tb)
        assert bits_equal(out, ref), (shape, count)


@pytest.mark.parametrize("kernel,tb", ALL_KERNELS)
def test_anisotropic_coefficients(kernel, tb):
    nx, ny, nz = 44, 27, 19
    c = np.array([0.11, 0.07, 0.09, 0.13, 0.05, 0.08, 0.47], np.float32)
    fin = O.seeded_noise((nz, ny, nx), 5, amplitude=1.0)
    out = gpu_run(fin, c, 9, kernel, tb)
    assert bits_equal(out, O.run(fin, c, 9))


@pytest.mark.parametrize("kernel,tb", ALL_KERNELS)
@pytest.mark.parametrize("shape", [(20, 12, 9), (64, 64, 64), (36, 5, 40)])
def test_fp64_bit_exact_vs_fp64_oracle(kernel, tb, shape):
    nx, ny, nz = shape
    c, _ = O.params(nx, ny, nz, np.float64)
    fin = O.initialize(nx, ny, nz, dtype=np.float64)
    fin = fin + O.seeded_noise(fin.shape, 3).astype(np.float64)
    out = gpu_run(fin, c, 7, kernel, tb)
    assert bits_equal(out, O.run(fin, c, 7))


@pytest.mark.parametrize("variant", range(B.NUM_TILE_VARIANTS))
@pytest.mark.parametrize("zchunk", [0, 1, 5, 64])
def test_tile_variants_and_zchunks(variant, zchunk):
    nx, ny, nz = 136, 40, 23
    c, _ = O.params(nx, ny, nz)
    fin = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 8)
    ref = O.run(fin, c, 3)
    out = gpu_run(fin, c, 3, B.KERNEL_TMA, 1, variant=variant, zchunk=zchunk)
    assert bits_equal(out, ref)


@pytest.mark.parametrize("k", [2, 3, 4])
@pytest.mark.parametrize("zchunk", [1, 3, 7])
def test_temporal_blocking_short_chunks(k, zchunk):
    nx, ny, nz = 64, 24, 21
    c, _ = O.params(nx, ny, nz)
    fin = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 9)
    for count in (k, 2 * k + 1):
        out = gpu_run(fin, c, count, B.KERNEL_TB, k, zchunk=zchunk)
        assert bits_equal(out, O.run(fin, c, count)), count


@pytest.mark.parametrize("dims", [(128, 14, 7), (132, 30, 9), (260, 29, 33),
                                  (256, 64, 40), (64, 1, 1), (128, 15, 2),
                                  (136, 17, 3), (4, 3, 5)])
@pytest.mark.parametrize("zchunk", [0, 1, 2, 5])
def test_tb2_warp_row_kernel_vs_generic_and_oracle(dims, zchunk):
    """The K = 2 FP32 warp-row kernel (TB variant 0) against the generic-K
    kernel (variant 1) and the oracle: tiles of 128 x 14 cut by every edge
    case (nx not a multiple of 128, ny not a multiple of 14, nz of 1..3,
    one-plane z-chunks), even and odd step counts."""
    nx, ny, nz = dims
    c, _ = O.params(nx, ny, nz)
    fin = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 21)
    for count in (2, 5):
        ref = O.run(fin, c, count)
        outs = []
        for variant in (0, 1):
            out = gpu_run(fin, c, count, B.KERNEL_TB, 2, variant=variant,
                          zchunk=zchunk)
            outs.append(out)
        assert bits_equal(outs[0], ref), (dims, zchunk, count)
        assert bits_equal(outs[1], ref), (dims, zchunk, count)


def test_tb2_warp_row_kernel_is_the_default():
    plan = B.Plan(128, 28, 8, B.F32, B.KERNEL_TB, 2)
    f1, f2 = plan.empty(), plan.empty()
    f1.uniform_()
    plan.run(f1, f2, 2)
    torch.cuda.synchronize()
    assert plan.info()["last_kernel"] == "steps_tb2w"
    plan.set_tile(1, 0)
    plan.run(f1, f2, 2)
    torch.cuda.synchronize()
    assert plan.info()["last_kernel"] == "steps_tb"
    plan.close()


def test_tma_rejects_ineligible_and_auto_falls_to_generic():
    nx, ny, nz = 17, 8, 4  # row pitch 68 B: not a multiple of 16
    plan = B.Plan(nx, ny, nz, B.F32, B.KERNEL_TMA)
    f1 = torch.rand((nz, ny, nx), device="cuda")
    f2 = torch.empty_like(f1)
    with pytest.raises(B.D3DError) as ei:
        plan.step(f1, f2)
    assert ei.value.code == B.D3D_E_UNSUPPORTED
    # misaligned base pointer: AUTO still runs (generic kernel), same bits
    nx = 64
    c, _ = O.params(nx, ny, nz)
    fin = O.seeded_noise((nz, ny, nx), 4, amplitude=1.0)
    big = torch.zeros(fin.size + 1, device="cuda")
    big[1:] = torch.from_numpy(fin.reshape(-1)).cuda()
    f1 = big[1:].view(nz, ny, nx)
    f2 = torch.empty_like(f1)
    plan = B.Plan(nx, ny, nz, B.F32, B.KERNEL_AUTO)
    plan.step(f1, f2, c)
    assert plan.info()["last_kernel"] == "step_generic"
    assert bits_equal(f2.cpu().numpy(), O.run(fin, c, 1))


def test_run_host_matches_device_run():
    nx, ny, nz = 96, 64, 48
    c, _ = O.params(nx, ny, nz)
    fin = O.initialize(nx, ny, nz)
    plan = B.Plan(nx, ny, nz)
    host = B.pinned_empty((nz, ny, nx))
    host[...] = fin
    f1 = plan.empty()
    f2 = plan.empty()
    ms = plan.run_host(host, f1, f2, 11, c)
    assert ms > 0
    assert bits_equal(host, O.run(fin, c, 11))


def test_full_size_512_kernels_agree():
    """512^3: every kernel produces the same bits (TMA z-march, generic,
    temporal blocking k=2,3,4) over 12 steps, and the FP64 device norm
    between them is exactly zero."""
    n = 512
    c, _ = O.params(n, n, n)
    gen = torch.Generator(device="cuda").manual_seed(1234)
    base = torch.rand((n, n, n), device="cuda", generator=gen)
    outs = {}
    for kernel, tb in ALL_KERNELS:
        plan = B.Plan(n, n, n, B.F32, kernel, tb)
        f1 = base.clone()
        f2 = torch.empty_like(f1)
        res, _ = plan.run(f1, f2, 12, c)
        torch.cuda.synchronize()
        outs[(kernel, tb)] = res
        del f2
    ref = outs[(B.KERNEL_AUTO, 1)]
    plan = B.Plan(n, n, n)
    for key, v in outs.items():
        assert torch.equal(v, ref), key
        nrm = plan.compare(v, ref)
        assert nrm[0] == 0.0 and nrm[1] == 0.0
    assert B.check_device_errors() == 0


@pytest.mark.parametrize("dims,dtype,fine", [
    ((1024, 1024, 65), np.float32, 16), ((1024, 512, 61), np.float64, 12)])
def test_fine_zchunks_on_wide_grids_vs_oracle(dims, dtype, fine):
    """Grids wide enough that the TMA z-march cuts short chunks (16 planes
    FP32, 12 FP64; four or more waves of CTAs): nz leaves a last chunk of
    one plane.  The automatic launch shape is checked, then the bits
    against the oracle."""
    nx, ny, nz = dims
    c, _ = O.params(nx, ny, nz, dtype)
    fin = O.seeded_noise((nz, ny, nx), 61, amplitude=1.0).astype(dtype)
    plan = B.Plan(nx, ny, nz, B.F64 if dtype == np.float64 else B.F32,
                  B.KERNEL_TMA)
    f1 = torch.from_numpy(fin).cuda()
    f2 = torch.empty_like(f1)
    res, _ = plan.run(f1, f2, 3, c)
    torch.cuda.synchronize()
    info = plan.info()
    assert info["launch_zchunk"] == fine, info
    assert B.check_device_errors() == 0
    assert bits_equal(res.cpu().numpy(), O.run(fin, c, 3))
    plan.close()


def test_device_compare_matches_oracle_norms():
    a = O.seeded_noise((40, 30, 20), 1, amplitude=1.0) + np.float32(0.5)
    b = a + O.seeded_noise(a.shape, 2, amplitude=1e-3)
    plan = B.Plan(20, 30, 40)
    got = plan.compare(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
    exp = O.norms(a, b)
    np.testing.assert_allclose(got, exp, rtol=1e-12, atol=0)


def test_device_analytic_close_to_reference_initialize():
    nx, ny, nz = 64, 48, 40
    plan = B.Plan(nx, ny, nz, B.F64)
    out = plan.empty()
    _, g = O.params(nx, ny, nz, np.float64)
    t = 37 * g[7]
    plan.analytic(out, t)
    ref = O.initialize(nx, ny, nz, time=t, dtype=np.float64)
    # 1 - a*cos(theta) cancels near the origin; libm and CUDA cos may differ
    # by an ulp, which the cancellation magnifies to ~1e-13 relative.
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-11, atol=1e-15)
    # The FP32 analytic field agrees with the reference's own float
    # Initialize to float rounding.
    plan32 = B.Plan(nx, ny, nz, B.F32)
    o32 = plan32.empty()
    _, g32 = O.params(nx, ny, nz)
    plan32.analytic(o32, float(np.float32(37) * g32[7]))
    ref32 = O.initialize(nx, ny, nz, time=np.float32(37) * g32[7])
    np.testing.assert_allclose(o32.cpu().numpy(), ref32, rtol=1e-5, atol=1e-7)


@pytest.mark.parametrize("kernel,tb", [(B.KERNEL_AUTO, 1), (B.KERNEL_TB, 2)])
def test_autotune_then_bit_exact(kernel, tb):
    nx, ny, nz = 128, 96, 72
    c, _ = O.params(nx, ny, nz)
    plan = B.Plan(nx, ny, nz, B.F32, kernel, tb)
    s1 = torch.rand((nz, ny, nx), device="cuda")
    s2 = torch.empty_like(s1)
    ms, info = plan.autotune(s1, s2, steps=4, coeff=c)
    assert ms > 0
    assert 0 <= info["variant"] < B.NUM_TILE_VARIANTS
    fin = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 12)
    f1 = torch.from_numpy(fin).cuda()
    f2 = torch.empty_like(f1)
    res, _ = plan.run(f1, f2, 9, c)
    assert bits_equal(res.cpu().numpy(), O.run(fin, c, 9))


def test_graph_replay_matches_direct_launches():
    nx, ny, nz = 64, 40, 33
    c, _ = O.params(nx, ny, nz)
    fin = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 13)
    ref = O.run(fin, c, 6)
    for graphs in (True, False):
        plan = B.Plan(nx, ny, nz)
        plan.set_graphs(graphs)
        f1 = torch.from_numpy(fin).cuda()
        f2 = torch.empty_like(f1)
        for _ in range(3):  # replays of the cached graph
            g1, g2 = f1.clone(), torch.empty_like(f1)
            res, _ = plan.run(g1, g2, 6, c)
            assert bits_equal(res.cpu().numpy(), ref)
        assert plan.info()["graphs"] == int(graphs)


def _reference_points(field, c, idx):
    """The reference's one-step formula at sampled (z, y, x) points, in
    float32 with its summation order and clamped neighbours."""
    nz, ny, nx = field.shape
    f = np.float32
    out = []
    for z, y, x in idx:
        g = lambda zz, yy, xx: field[min(max(zz, 0), nz - 1),
                                     min(max(yy, 0), ny - 1),
                                     min(max(xx, 0), nx - 1)]
        cc, cw, ce, cs, cn, cb, ct = (c[6], c[1], c[0], c[3], c[2], c[5],
                                      c[4])
        v = f(cc * g(z, y, x))
        v = f(v + f(cw * g(z, y, x - 1)))
        v = f(v + f(ce * g(z, y, x + 1)))
        v = f(v + f(cs * g(z, y + 1, x)))
        v = f(v + f(cn * g(z, y - 1, x)))
        v = f(v + f(cb * g(z - 1, y, x)))
        v = f(v + f(ct * g(z + 1, y, x)))
        out.append(v)
    return np.array(out, np.float32)


@pytest.mark.parametrize("dims", [(1024, 1024, 1024), (32768, 65535, 2)])
def test_maximum_sizes(dims):
    """A 4 GiB-per-buffer field and a plane just under the 2^31-point limit
    of the C ABI: the TMA and generic kernels agree bit for bit, and
    sampled points (edges, corners, interior) match the reference formula."""
    nx, ny, nz = dims
    c, _ = O.params(nx, ny, nz)
    gen = torch.Generator(device="cuda").manual_seed(31)
    f1 = torch.rand((nz, ny, nx), device="cuda", generator=gen)
    outs = []
    for kernel in (B.KERNEL_TMA, B.KERNEL_GENERIC):
        plan = B.Plan(nx, ny, nz, B.F32, kernel)
        f2 = torch.empty_like(f1)
        plan.step(f1, f2, c)
        torch.cuda.synchronize()
        outs.append(f2)
        plan.close()
    assert torch.equal(outs[0], outs[1])
    rng = np.random.default_rng(3)
    idx = [(z, y, x) for z in {0, nz - 1, nz // 2} for y in {0, ny - 1}
           for x in {0, nx - 1, nx // 3}]
    idx += [(int(rng.integers(nz)), int(rng.integers(ny)),
             int(rng.integers(nx))) for _ in range(24)]
    class Planes:  # device values fetched one by one (fields are huge)
        shape = (nz, ny, nx)

        def __getitem__(self, key):
            z, y, x = key
            return np.float32(f1[z, y, x].item())

    ref = _reference_points(Planes(), c, idx)
    got = np.array([outs[0][z, y, x].item() for z, y, x in idx], np.float32)
    assert got.tobytes() == ref.tobytes()
    assert B.check_device_errors() == 0


def test_device_accuracy_matches_oracle_fp64_report():
    """d3d_accuracy (analytic form evaluated per point in double, errors
    summed in double) against the oracle's FP64 analytic field and norms;
    the reference's float GetAccuracy agrees to float rounding."""
    nx, ny, nz, count = 48, 40, 36, 23
    c, g = O.params(nx, ny, nz)
    fin = O.initialize(nx, ny, nz)
    ref = O.run(fin, c, count)
    plan = B.Plan(nx, ny, nz)
    got = plan.accuracy(torch.from_numpy(ref).cuda(), count)
    t = float(np.float32(count) * g[7])
    ana = O.initialize(nx, ny, nz, time=t, dtype=np.float64)
    exp = O.norms(ref, ana)
    np.testing.assert_allclose(got[[0, 3]], exp[[0, 3]], rtol=1e-9)
    np.testing.assert_allclose(got[1], exp[1], rtol=1e-9)
    # the reference's figure: float analytic field, float running sum
    assert got[0] == pytest.approx(O.accuracy(ref, count), rel=1e-3)


def test_bounded_wait_timeout_leaves_context_usable():
    """The failure path of every bounded mbarrier wait: a wait that can
    never complete runs out, sets the device error word, and the next
    kernels run normally."""
    flags = B.ctypes.c_uint()
    rc = B.lib().d3d_selftest_wait_timeout(2000, B.ctypes.byref(flags))
    assert rc == B.D3D_E_TIMEOUT and flags.value & 1
    assert B.check_device_errors() == 0  # read-and-clear
    nx, ny, nz = 64, 16, 9
    c, _ = O.params(nx, ny, nz)
    fin = O.seeded_noise((nz, ny, nx), 1, amplitude=1.0)
    assert bits_equal(gpu_run(fin, c, 3), O.run(fin, c, 3))
