"""Batched solves (d3d_batch_*): many grids of different shapes, coefficients
and step counts in one run.  Every grid's result must be bit-identical to
the oracle's RunKernel on that grid, and to the same grid run alone."""
import ctypes

import numpy as np
import pytest

import benchmarks_b200 as B
import oracle as O


def policy_coefficients(nx, ny, nz, kappa):
    """The stability policy in plain float32 arithmetic: the reference's
    constructor expressions with dt from the smallest spacing."""
    f = np.float32
    dx, dy, dz = f(1.0) / f(nx), f(1.0) / f(ny), f(1.0) / f(nz)
    h = min(dx, dy, dz)
    dt = f(0.1 * float(h) * float(h) / float(f(kappa)))
    k = f(kappa)
    ce = k * dt / (dx * dx)
    cn = k * dt / (dy * dy)
    ct = k * dt / (dz * dz)
    cc = f(1.0 - float(ce + ce + cn + cn + ct + ct))
    return np.array([ce, ce, cn, cn, ct, ct, cc], np.float32)


@pytest.mark.parametrize("dims,kappa", [((16, 96, 40), 0.1),
                                        ((96, 16, 17), 0.05),
                                        ((33, 33, 33), 0.2),
                                        ((64, 64, 64), 0.1)])
def test_policy_coefficients(dims, kappa):
    c = B.batch_coefficients(*dims, kappa)
    assert c.tobytes() == policy_coefficients(*dims, kappa).tobytes()
    assert c[6] >= 0.39  # stable: cc >= 0.4 up to rounding
    if dims[0] == dims[1] == dims[2] and kappa == np.float32(0.1):
        # cubic grids: the reference constructor's coefficients
        assert c.tobytes() == O.params(*dims)[0].tobytes()


def test_layout_packs_aligned_disjoint_buffers():
    specs = [(17, 5, 3, 1), (96, 80, 33, 4), (16, 16, 16, 0)]
    arr = (B.BatchGrid * len(specs))()
    for i, (nx, ny, nz, st) in enumerate(specs):
        arr[i].nx, arr[i].ny, arr[i].nz, arr[i].steps = nx, ny, nz, st
    nbytes = ctypes.c_size_t()
    B.check(B.lib().d3d_batch_layout(arr, len(specs), ctypes.byref(nbytes)))
    spans = []
    for g in arr:
        n = g.nx * g.ny * g.nz
        for off in (g.offset_a, g.offset_b):
            assert (off * 4) % 256 == 0
            spans.append((off, off + n))
    spans.sort()
    for (a0, a1), (b0, b1) in zip(spans, spans[1:]):
        assert a1 <= b0
    assert spans[-1][1] * 4 <= nbytes.value


def test_create_rejects_bad_batches():
    L = B.lib()
    arr = (B.BatchGrid * 1)()
    arr[0].nx, arr[0].ny, arr[0].nz, arr[0].steps = 8, 8, 8, 1
    arr[0].offset_a, arr[0].offset_b = 0, 256
    h = ctypes.c_void_p()
    # second buffer past the end of the arena
    assert L.d3d_batch_create(arr, 1, 4096, 1024 * 4,
                              ctypes.byref(h)) == B.D3D_E_INVALID
    # overlapping buffers
    arr[0].offset_b = 100
    assert L.d3d_batch_create(arr, 1, 4096, 4096 * 4,
                              ctypes.byref(h)) == B.D3D_E_INVALID
    arr[0].nx = 0
    assert L.d3d_batch_create(arr, 1, 4096, 4096 * 4,
                              ctypes.byref(h)) == B.D3D_E_INVALID
    # a plane under 2^31 points whose padded rows (ceil4(nx)) are not
    arr[0].nx, arr[0].ny, arr[0].nz = 46341, 46340, 1
    assert 46341 * 46340 < 2 ** 31 <= 46344 * 46340
    assert L.d3d_batch_create(arr, 1, 4096, 1 << 62,
                              ctypes.byref(h)) == B.D3D_E_INVALID


def _mixed_specs(seed, n, max_side=40, max_steps=24):
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n):
        nx, ny, nz = (int(v) for v in rng.integers(1, max_side + 1, 3))
        steps = int(rng.integers(0, max_steps + 1))
        kappa = float(rng.uniform(0.05, 0.2))
        specs.append((nx, ny, nz, steps, B.batch_coefficients(nx, ny, nz,
                                                              kappa)))
    return specs


def _fields(specs, seed):
    out = []
    for i, (nx, ny, nz, _, _) in enumerate(specs):
        f = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), seed + i)
        out.append(f)
    return out


def _run_batch(specs, fields, autotune=False, kind=None):
    torch = pytest.importorskip("torch")
    batch = B.Batch(specs)
    if autotune:
        batch.autotune()
    if kind is not None:
        batch.set_kind(kind)
    for i, f in enumerate(fields):
        batch.input(i).copy_(torch.from_numpy(f))
    batch.run()
    torch.cuda.synchronize()
    return [batch.result(i).cpu().numpy() for i in range(len(specs))], batch


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [1, 2])
def test_batch_bit_exact_vs_oracle(seed):
    specs = _mixed_specs(seed, 40)
    # include the edge shapes explicitly
    specs += [(1, 1, 1, 5, B.batch_coefficients(1, 1, 1, 0.1)),
              (96, 3, 2, 7, B.batch_coefficients(96, 3, 2, 0.1)),
              (70, 70, 9, 11, B.batch_coefficients(70, 70, 9, 0.15)),
              (20, 20, 20, 0, B.batch_coefficients(20, 20, 20, 0.1))]
    fields = _fields(specs, 100 * seed)
    outs, batch = _run_batch(specs, fields)
    for (nx, ny, nz, steps, c), f, o in zip(specs, fields, outs):
        ref = O.run(f, c, steps)
        assert o.tobytes() == ref.tobytes(), (nx, ny, nz, steps)
    info = batch.info()
    assert info["grids"] == len(specs)


@pytest.mark.gpu
def test_each_grid_same_alone_and_in_the_mix():
    specs = _mixed_specs(7, 24, max_side=64, max_steps=16)
    fields = _fields(specs, 700)
    mixed, _ = _run_batch(specs, fields)
    for i in (0, 5, 11, 23):
        alone, _ = _run_batch([specs[i]], [fields[i]])
        assert alone[0].tobytes() == mixed[i].tobytes()


@pytest.mark.gpu
def test_autotuned_batch_still_bit_exact():
    specs = _mixed_specs(3, 30, max_side=96, max_steps=10)
    fields = _fields(specs, 300)
    outs, batch = _run_batch(specs, fields, autotune=True)
    for (nx, ny, nz, steps, c), f, o in zip(specs, fields, outs):
        assert o.tobytes() == O.run(f, c, steps).tobytes()
    for c in batch.info()["classes"]:
        if c["kernel"] == "march":
            assert tuple(c["tile"]) in {(64, 8), (32, 16), (32, 8), (16, 16)}
        else:
            assert c["kernel"] in ("strip", "strip2")
            assert c["segments_per_thread"] in (1, 2)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", range(B.BATCH_NUM_KINDS))
def test_every_kernel_kind_bit_exact(kind):
    """Each march tile shape, both strip forms, both two-step strip forms
    and the cluster-resident kernel on grids of every size class, nx
    leaving 0..3 pad columns in the pitched copies (nx = 1 included),
    zero-step grids, odd and even step counts (a two-step class ends odd
    counts with one strip step)."""
    dims = [(1, 1, 1), (1, 5, 7), (3, 2, 9), (17, 23, 5), (24, 9, 13),
            (25, 30, 2), (40, 41, 11), (41, 3, 6), (72, 17, 8), (73, 70, 9),
            (96, 96, 4), (13, 1, 30)]
    specs = [(nx, ny, nz, (i * 5) % 9,
              B.batch_coefficients(nx, ny, nz, 0.05 + 0.01 * i))
             for i, (nx, ny, nz) in enumerate(dims)]
    fields = _fields(specs, 1100 + kind)
    outs, batch = _run_batch(specs, fields, kind=kind)
    for (nx, ny, nz, steps, c), f, o in zip(specs, fields, outs):
        assert o.tobytes() == O.run(f, c, steps).tobytes(), (kind, nx, ny,
                                                              nz, steps)
    assert B.check_device_errors() == 0


@pytest.mark.gpu
def test_two_step_kinds_need_narrow_grids():
    specs = [(249, 3, 4, 2, B.batch_coefficients(249, 3, 4, 0.1)),
             (20, 20, 20, 3, B.batch_coefficients(20, 20, 20, 0.1))]
    batch = B.Batch(specs)
    with pytest.raises(B.D3DError) as ei:
        batch.set_kind(6)
    assert ei.value.code == B.D3D_E_UNSUPPORTED
    batch.set_kind(5)
    batch.autotune()  # skips the two-step kinds for the wide grid's class
    batch.close()


@pytest.mark.gpu
def test_batch_replay_is_repeatable():
    torch = pytest.importorskip("torch")
    specs = _mixed_specs(9, 12, max_side=48, max_steps=9)
    fields = _fields(specs, 900)
    batch = B.Batch(specs)
    results = []
    for _ in range(3):  # the graph is captured once and replayed
        for i, f in enumerate(fields):
            batch.input(i).copy_(torch.from_numpy(f))
        batch.run()
        torch.cuda.synchronize()
        results.append([batch.result(i).cpu().numpy().tobytes()
                        for i in range(len(specs))])
    assert results[0] == results[1] == results[2]


@pytest.mark.gpu
def test_more_grids_than_one_launch_row():
    """70,000 grids: the repitch launches stride over grids in steps of
    65,535 (the grid-y limit) and the step launch has 70,000 CTAs."""
    torch = pytest.importorskip("torch")
    n = 70000
    shapes = [(1, 1, 1), (5, 2, 3), (3, 4, 2)]
    specs = []
    for i in range(n):
        nx, ny, nz = shapes[i % 3]
        specs.append((nx, ny, nz, 1 + (i % 2),
                      B.batch_coefficients(nx, ny, nz, 0.1)))
    batch = B.Batch(specs)
    batch.arena.zero_()
    fields = {}
    for j in range(6):  # shape x step parity
        nx, ny, nz = shapes[j % 3]
        fields[j] = O.seeded_noise((nz, ny, nx), 50 + j, amplitude=1.0)
    for i in (0, 1, 2, 3, 4, 5, n - 6, n - 5, n - 4, n - 3, n - 2, n - 1,
              65534, 65535, 65536):
        batch.input(i).copy_(torch.from_numpy(fields[i % 6]))
    batch.run()
    torch.cuda.synchronize()
    for i in (0, 1, 2, 3, 4, 5, n - 6, n - 5, n - 4, n - 3, n - 2, n - 1,
              65534, 65535, 65536):
        nx, ny, nz, steps, c = specs[i]
        want = O.run(fields[i % 6], c, steps)
        assert batch.result(i).cpu().numpy().tobytes() == want.tobytes(), i
    assert B.check_device_errors() == 0
    batch.close()


# Grids for the cluster-resident kernel.  A CTA holds at most 57,856 floats:
# pc planes (or their row parts, with a halo row on each side) and one halo
# plane, in at most 16 CTAs.  These cover clusters of 1 to 16 CTAs, a last
# CTA with fewer planes, one-plane slabs, planes cut into 2 and 4 row parts
# (a last part with fewer rows), every thread shape (the 512 x 4 and
# 384 x 6 ones for wide planes of few rows), rows of one segment, nx
# leaving 0..3 pad columns, and a grid it does not fit (96^3: 20 CTAs),
# which runs on the strip kind.
RESIDENT_DIMS = [(1, 1, 1), (5, 1, 9), (17, 23, 5), (13, 1, 30),
                 (64, 64, 64), (88, 80, 37), (96, 96, 80), (95, 7, 300),
                 (33, 60, 45), (96, 90, 12), (40, 40, 200), (96, 96, 96),
                 (100, 96, 10), (57, 31, 128), (16, 96, 96), (96, 16, 3),
                 (500, 9, 20), (700, 12, 11), (93, 67, 40)]


def _resident_specs(steps_of):
    return [(nx, ny, nz, steps_of(i),
             B.batch_coefficients(nx, ny, nz, 0.05 + 0.01 * i))
            for i, (nx, ny, nz) in enumerate(RESIDENT_DIMS)]


@pytest.mark.gpu
def test_cluster_resident_kind_bit_exact_with_step_counters():
    specs = _resident_specs(lambda i: 1 + (i * 7) % 12)
    fields = _fields(specs, 1300)
    outs, batch = _run_batch(specs, fields, kind=B.BATCH_KIND_RESIDENT)
    for (nx, ny, nz, steps, c), f, o in zip(specs, fields, outs):
        assert o.tobytes() == O.run(f, c, steps).tobytes(), (nx, ny, nz,
                                                              steps)
    assert B.check_device_errors() == 0
    info = batch.info()
    res = info["resident"]
    assert res["on"]
    # (96, 96, 96) needs 20 CTAs: it runs on the strip kind, every other
    # grid on the resident one
    assert res["grids"] == len(specs) - 1
    clusters = {c["cluster"] for c in res["classes"]}
    assert 1 in clusters and 16 in clusters
    assert {c["threads"] for c in res["classes"]} == {128, 256, 512, 384}
    # every grid's counter reached its step count
    assert list(batch.progress()) == [s for _, _, _, s, _ in specs]
    batch.close()


@pytest.mark.gpu
@pytest.mark.parametrize("bound", [0, 1, 4, 8, 12])
def test_cluster_resident_split_by_cluster_size(bound):
    """Only grids that fit clusters of at most `bound` CTAs run resident
    (0: none); the others take the strip kind in the same run.  Every grid
    keeps the oracle's bits and reaches its step count either way."""
    torch = pytest.importorskip("torch")
    specs = _resident_specs(lambda i: 2 + (i * 5) % 9)
    fields = _fields(specs, 1350)
    batch = B.Batch(specs)
    batch.set_kind(B.BATCH_KIND_RESIDENT)
    every = batch.info()["resident"]["classes"]
    batch.set_resident_max_cluster(bound)
    for i, f in enumerate(fields):
        batch.input(i).copy_(torch.from_numpy(f))
    batch.run()
    torch.cuda.synchronize()
    for i, ((nx, ny, nz, steps, c), f) in enumerate(zip(specs, fields)):
        assert batch.result(i).cpu().numpy().tobytes() == \
            O.run(f, c, steps).tobytes(), (bound, nx, ny, nz)
    assert list(batch.progress()) == [s for _, _, _, s, _ in specs]
    res = batch.info()["resident"]
    assert res["on"] == (bound > 0)
    want = sum(c["grids"] for c in every if c["cluster"] <= bound)
    assert res["grids"] == want
    assert all(c["cluster"] <= bound for c in res["classes"])
    for bad in (-1, 17):
        with pytest.raises(B.D3DError) as ei:
            batch.set_resident_max_cluster(bad)
        assert ei.value.code == B.D3D_E_INVALID
    assert B.check_device_errors() == 0
    batch.close()


@pytest.mark.gpu
def test_cluster_resident_same_alone_and_in_the_mix():
    specs = _resident_specs(lambda i: 3 + i % 5)
    fields = _fields(specs, 1400)
    mixed, _ = _run_batch(specs, fields, kind=B.BATCH_KIND_RESIDENT)
    for i in (0, 4, 6, 7, 11):
        alone, _ = _run_batch([specs[i]], [fields[i]],
                              kind=B.BATCH_KIND_RESIDENT)
        assert alone[0].tobytes() == mixed[i].tobytes(), i


@pytest.mark.gpu
def test_cluster_resident_replays_and_long_runs():
    """The captured graph replays (work counters reset each run), and a
    few hundred steps keep the bits of the oracle's run."""
    torch = pytest.importorskip("torch")
    specs = [(48, 40, 36, 301, B.batch_coefficients(48, 40, 36, 0.1)),
             (96, 64, 70, 257, B.batch_coefficients(96, 64, 70, 0.1)),
             (23, 19, 11, 500, B.batch_coefficients(23, 19, 11, 0.1))]
    fields = _fields(specs, 1500)
    batch = B.Batch(specs)
    batch.set_kind(B.BATCH_KIND_RESIDENT)
    for _ in range(2):
        for i, f in enumerate(fields):
            batch.input(i).copy_(torch.from_numpy(f))
        batch.run()
        torch.cuda.synchronize()
        for i, ((nx, ny, nz, steps, c), f) in enumerate(zip(specs, fields)):
            assert batch.result(i).cpu().numpy().tobytes() == \
                O.run(f, c, steps).tobytes(), i
        assert list(batch.progress()) == [s for _, _, _, s, _ in specs]
    assert batch.info()["launches_per_run"] < 10
    batch.close()
