"""The continuous-batching server (d3d_server_*): every served result must be
bit-identical to the oracle's RunKernel, whether the request runs alone or
in a mix, arrives while others are on the GPU, or waits for arena space."""
import numpy as np
import pytest

import benchmarks_b200 as B
import oracle as O

pytestmark = pytest.mark.gpu


def _requests(seed, n, max_side=48, max_steps=40, cubic=False):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        if cubic:
            nx = ny = nz = int(rng.integers(4, max_side + 1))
        else:
            nx, ny, nz = (int(v) for v in rng.integers(1, max_side + 1, 3))
        steps = int(rng.integers(0, max_steps + 1))
        c = B.batch_coefficients(nx, ny, nz, float(rng.uniform(0.05, 0.2)))
        f = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), seed + i)
        reqs.append((f, steps, c))
    return reqs


def _serve(reqs, arena_bytes=1 << 28, chunk=8, interleave=False,
           kernel=None, lanes=None, resident=None):
    server = B.Server(arena_bytes, chunk, kernel, lanes, resident)
    outs = [np.full_like(f, np.nan) for f, _, _ in reqs]
    ids = {}
    done = set()
    for k, ((f, steps, c), o) in enumerate(zip(reqs, outs)):
        ids[server.submit(f, o, steps, c)] = k
        if interleave and k % 3 == 2:
            done.update(server.tick())  # others are running meanwhile
    done.update(server.drain())
    assert done == set(ids)
    stats = server.stats()
    server.close()
    return outs, stats


def test_served_results_bit_exact_vs_oracle():
    reqs = _requests(1, 30)
    outs, stats = _serve(reqs)
    for (f, steps, c), o in zip(reqs, outs):
        assert o.tobytes() == O.run(f, c, steps).tobytes()
    assert stats["completed"] == len(reqs)


def test_same_alone_and_in_the_mix():
    reqs = _requests(2, 18, max_side=40, max_steps=30)
    mixed, _ = _serve(reqs, interleave=True)
    for k in (0, 4, 9, 17):
        alone, _ = _serve([reqs[k]])
        assert alone[0].tobytes() == mixed[k].tobytes()


@pytest.mark.parametrize("kernel,lanes", [(-1, 1), (-1, 2), (0, 3), (1, 1),
                                          (1, 2), (2, 4), (3, 2), (4, 1),
                                          (5, 1), (5, 4), (6, 2)])
def test_every_step_kernel_bit_exact(kernel, lanes):
    """Each tile shape of the pitched TMA kernel, its strip forms (5, 6)
    and the march kernel, on 1 to 4 compute streams, on grids whose nx
    leaves 0..3 pad columns (nx = 1 included), rows split into several
    strip pieces (nx > 248), single rows and planes, and grids deeper than
    one z slab."""
    dims = [(1, 1, 1), (1, 7, 5), (2, 3, 40), (3, 1, 9), (5, 33, 17),
            (8, 8, 8), (13, 17, 19), (64, 16, 3), (130, 9, 35),
            (131, 70, 6), (257, 5, 4), (36, 35, 70), (249, 11, 3),
            (500, 7, 2)]
    reqs = []
    for i, (nx, ny, nz) in enumerate(dims):
        c = B.batch_coefficients(nx, ny, nz, 0.05 + 0.01 * i)
        f = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 70 + i)
        reqs.append((f, (i * 7) % 13, c))
    outs, stats = _serve(reqs, chunk=5, interleave=True, kernel=kernel,
                         lanes=lanes, resident=False)
    assert stats["kernel"] == kernel and stats["lanes"] == lanes
    assert stats["resident_solves"] == 0
    for (f, steps, c), o in zip(reqs, outs):
        assert o.tobytes() == O.run(f, c, steps).tobytes()
    assert B.check_device_errors() == 0


@pytest.mark.parametrize("base,large,min_px,lanes", [(6, 2, 64, 4),
                                                     (5, 1, 128, 2),
                                                     (6, 2, 64, 1),
                                                     (2, 6, 32, 3)])
def test_large_solve_kernel_bit_exact(base, large, min_px, lanes):
    """A second step kernel for the wide solves on their own lanes: every
    result stays bit-exact, whichever side of the threshold a solve is."""
    dims = [(1, 1, 1), (5, 33, 17), (61, 9, 35), (64, 16, 3), (130, 9, 35),
            (131, 70, 6), (257, 5, 4), (36, 35, 70), (249, 11, 3),
            (500, 7, 2), (127, 40, 20), (128, 3, 9)]
    reqs = []
    for i, (nx, ny, nz) in enumerate(dims):
        c = B.batch_coefficients(nx, ny, nz, 0.05 + 0.01 * i)
        f = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 170 + i)
        reqs.append((f, 1 + (i * 7) % 13, c))
    server = B.Server(1 << 28, 4, base, lanes, False)
    server.set_large_kernel(large, min_px)
    outs = [np.full_like(f, np.nan) for f, _, _ in reqs]
    for k, ((f, steps, c), o) in enumerate(zip(reqs, outs)):
        server.submit(f, o, steps, c)
        if k % 3 == 2:
            server.tick()
    server.drain()
    server.close()
    for (f, steps, c), o in zip(reqs, outs):
        assert o.tobytes() == O.run(f, c, steps).tobytes()
    assert B.check_device_errors() == 0


def test_kernel_and_lanes_change_only_when_idle():
    server = B.Server(1 << 24, 4)
    f = np.zeros((4, 4, 5), np.float32)
    o = np.empty_like(f)
    server.submit(f, o, 3, B.batch_coefficients(5, 4, 4, 0.1))
    with pytest.raises(B.D3DError) as ei:
        server.set_kernel(-1)
    assert ei.value.code == B.D3D_E_BUSY
    with pytest.raises(B.D3DError) as ei:
        server.set_lanes(1)
    assert ei.value.code == B.D3D_E_BUSY
    server.drain()
    server.set_kernel(-1)
    server.set_lanes(3)
    for bad in (0, 9):
        with pytest.raises(B.D3DError):
            server.set_lanes(bad)
    with pytest.raises(B.D3DError):
        server.set_kernel(7)
    server.set_resident(False)
    server.set_resident(True)
    server.close()


def test_large_grids_cut_into_z_slabs():
    """Grids deep enough to be cut into z slabs (one alone, then beside
    small ones); odd depths leave a short last slab."""
    dims = [(150, 70, 101), (33, 9, 200), (64, 64, 47), (7, 5, 31)]
    reqs = []
    for i, (nx, ny, nz) in enumerate(dims):
        c = B.batch_coefficients(nx, ny, nz, 0.1 + 0.02 * i)
        f = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 40 + i)
        reqs.append((f, 5 + 2 * i, c))
    alone, _ = _serve(reqs[:1], chunk=3)
    f0, st0, c0 = reqs[0]
    assert alone[0].tobytes() == O.run(f0, c0, st0).tobytes()
    outs, _ = _serve(reqs, chunk=4, interleave=True)
    for (f, steps, c), o in zip(reqs, outs):
        assert o.tobytes() == O.run(f, c, steps).tobytes()


@pytest.mark.parametrize("chunk", [1, 3, 16])
def test_chunk_sizes_and_late_arrivals(chunk):
    reqs = _requests(3, 15, max_side=32, max_steps=25)
    outs, stats = _serve(reqs, chunk=chunk, interleave=True)
    for (f, steps, c), o in zip(reqs, outs):
        assert o.tobytes() == O.run(f, c, steps).tobytes()
    assert stats["chunk"] == chunk


def test_small_arena_queues_until_space_frees():
    # Room for about one 40^3 solve at a time: admission must wait.
    reqs = _requests(4, 8, max_side=40, max_steps=12, cubic=True)
    arena = 2 * 4 * 40 ** 3 + 4096
    outs, stats = _serve(reqs, arena_bytes=arena)
    for (f, steps, c), o in zip(reqs, outs):
        assert o.tobytes() == O.run(f, c, steps).tobytes()
    assert stats["peak_arena_bytes"] <= arena


def test_rejects_solves_that_can_never_fit():
    server = B.Server(1 << 20, resident=False)
    f = np.zeros((64, 64, 64), np.float32)  # 2 x 1 MiB > 1 MiB arena
    o = np.zeros_like(f)
    with pytest.raises(B.D3DError) as ei:
        server.submit(f, o, 3, O.params(64, 64, 64)[0])
    assert ei.value.code == B.D3D_E_BUSY
    server.close()
    # On the cluster-resident path the same solve needs one buffer only.
    server = B.Server(1 << 20, resident=True)
    f = O.seeded_noise((64, 64, 64), 3, amplitude=1.0)
    server.submit(f, o, 3, O.params(64, 64, 64)[0])
    server.drain()
    assert o.tobytes() == O.run(f, O.params(64, 64, 64)[0], 3).tobytes()
    assert server.stats()["resident_solves"] == 1
    f = np.zeros((64, 64, 65), np.float32)  # 1 MiB + 16 KiB: never fits
    o = np.zeros_like(f)
    with pytest.raises(B.D3DError) as ei:
        server.submit(f, o, 3, O.params(65, 64, 64)[0])
    assert ei.value.code == B.D3D_E_BUSY
    server.close()


@pytest.mark.parametrize("lanes", [1, 4])
def test_resident_path_matches_the_tick_path(lanes):
    """Solves the cluster-resident kernel fits (all its cluster sizes,
    every pad count, single planes and rows) and larger ones beside them:
    every result equals the oracle's with the resident path on and off,
    alone and interleaved with later arrivals."""
    dims = [(1, 1, 1), (5, 3, 2), (17, 23, 5), (64, 64, 64), (88, 80, 37),
            (96, 96, 80), (95, 7, 300), (33, 60, 45), (130, 80, 30),
            (96, 96, 96), (250, 40, 9), (40, 40, 200)]
    reqs = []
    for i, (nx, ny, nz) in enumerate(dims):
        c = B.batch_coefficients(nx, ny, nz, 0.05 + 0.01 * i)
        f = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 90 + i)
        reqs.append((f, 1 + (i * 5) % 17, c))
    on, st_on = _serve(reqs, arena_bytes=1 << 30, chunk=4, interleave=True,
                       lanes=lanes, resident=True)
    off, st_off = _serve(reqs, arena_bytes=1 << 30, chunk=4,
                         interleave=True, lanes=lanes, resident=False)
    for (f, steps, c), a, b in zip(reqs, on, off):
        ref = O.run(f, c, steps)
        assert a.tobytes() == ref.tobytes()
        assert b.tobytes() == ref.tobytes()
    # (96, 96, 96) needs 20 CTAs: it runs on the ticks
    assert st_on["resident_solves"] == len(reqs) - 1
    assert st_off["resident_solves"] == 0
    alone, _ = _serve([reqs[5]], arena_bytes=1 << 30, resident=True)
    assert alone[0].tobytes() == on[5].tobytes()
    assert B.check_device_errors() == 0


def test_zero_step_requests_return_their_input():
    reqs = [(O.seeded_noise((5, 6, 7), 1, amplitude=1.0), 0,
             O.params(7, 6, 5)[0])]
    outs, _ = _serve(reqs)
    assert outs[0].tobytes() == reqs[0][0].tobytes()


def test_arena_allocation_failure_is_reported():
    """Host-visible failure: an arena larger than the device fails cleanly
    with D3D_E_OOM and leaves the process usable."""
    with pytest.raises(B.D3DError) as ei:
        B.Server(1 << 50)
    assert ei.value.code == B.D3D_E_OOM
    server = B.Server(1 << 24)
    f = O.seeded_noise((8, 8, 8), 1, amplitude=1.0)
    o = np.zeros_like(f)
    server.submit(f, o, 2, O.params(8, 8, 8)[0])
    server.drain()
    assert o.tobytes() == O.run(f, O.params(8, 8, 8)[0], 2).tobytes()
    server.close()
