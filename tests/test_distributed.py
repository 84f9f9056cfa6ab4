"""Multi-rank paths on CPU (gloo, 127.0.0.1), no GPU needed.

* z-slab decomposition with halo exchange: ranks run the oracle's step on
  their local slab; the gathered field must be bit-identical to a
  single-process run, for several world sizes, halo depths and uneven
  slabs.
* (GPU) the same with the CUDA kernels: 2 or 3 gloo ranks share one GPU,
  each stepping its slab through the C ABI (the halo-1 overlapped schedule
  with d3d_step_planes, the overlapped schedule of k-step passes, and the
  halo-h schedule with whole-buffer runs), the planes staged through host
  memory; no kernel waits on another rank's.
* bench-style max-over-ranks timing reduction.
"""
import os
import socket

import numpy as np
import pytest

from benchmarks_b200.distributed import SlabDecomposition, slab_bounds


def test_slab_bounds_cover_the_grid():
    for nz in (5, 16, 17, 100):
        for world in range(1, 6):
            if world > nz:
                continue
            spans = [slab_bounds(nz, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == nz
            for (a0, a1), (b0, b1) in zip(spans, spans[1:]):
                assert a1 == b0
            sizes = [z1 - z0 for z0, z1 in spans]
            assert max(sizes) - min(sizes) <= 1


def test_decomposition_slices():
    d = SlabDecomposition(20, 1, 3, halo=2)  # owns [7, 14)
    assert (d.z0, d.z1, d.lo, d.hi) == (7, 14, 5, 16)
    assert d.owned() == slice(2, 9)
    assert d.send_down() == slice(2, 4) and d.recv_down() == slice(0, 2)
    assert d.send_up() == slice(7, 9) and d.recv_up() == slice(9, 11)
    edge = SlabDecomposition(20, 0, 3, halo=2)
    assert edge.lo == 0 and edge.down is None and edge.recv_down() == slice(0, 0)
    with pytest.raises(ValueError):
        SlabDecomposition(4, 0, 3, halo=3)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _slab_worker(rank, world, port, nx, ny, nz, count, halo, seed, out,
                 overlap=False):
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    import oracle as O
    from benchmarks_b200.distributed import SlabSolver

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        c, _ = O.params(nx, ny, nz)
        field = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), seed)
        lib = O.lib()

        def step(src, dst):  # the oracle's step on the local slab
            s = src.numpy()
            d = dst.numpy()
            lib.d3do_step_f32(s.ctypes.data_as(O._f32p),
                              d.ctypes.data_as(O._f32p), nx, ny, s.shape[0],
                              c.ctypes.data_as(O._f32p))

        solver = SlabSolver(dist, nx, ny, nz, c, halo=halo, step_fn=step,
                            device=torch.device("cpu"), overlap=overlap)
        solver.load(torch.from_numpy(field))
        solver.run(count)
        full = solver.gather().numpy()
        # max-over-ranks reduction as bench.py does it
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            np.save(out, full)
            assert t.item() == world
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,halo,overlap,dims,count", [
    (2, 1, False, (12, 9, 16), 7),
    (2, 3, False, (10, 7, 15), 8),
    (3, 2, False, (8, 8, 17), 11),
    (3, 1, False, (5, 6, 7), 5),
    # the overlapped schedule of k-step passes (pieces around each rank
    # boundary first), with a shorter last pass when count % halo != 0
    (2, 2, True, (12, 9, 16), 7),
    (3, 3, True, (10, 7, 20), 8),
    (4, 2, True, (6, 5, 19), 9),
])
def test_slab_solver_matches_single_process(tmp_path, world, halo, overlap,
                                            dims, count):
    import torch.multiprocessing as mp

    import oracle as O
    nx, ny, nz = dims
    out = str(tmp_path / "full.npy")
    mp.start_processes(_slab_worker,
                       args=(world, _free_port(), nx, ny, nz, count, halo, 5,
                             out, overlap),
                       nprocs=world, join=True, start_method="spawn")
    full = np.load(out)
    c, _ = O.params(nx, ny, nz)
    field = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 5)
    assert full.tobytes() == O.run(field, c, count).tobytes()


def _slab_cuda_worker(rank, world, port, nx, ny, nz, count, halo, overlap,
                      seed, out):
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    import oracle as O
    from benchmarks_b200.distributed import SlabSolver

    torch.cuda.set_device(0)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        c, _ = O.params(nx, ny, nz)
        field = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), seed)
        solver = SlabSolver(dist, nx, ny, nz, c, halo=halo, overlap=overlap)
        solver.load(torch.from_numpy(field).cuda())
        solver.run(count)
        torch.cuda.synchronize()
        full = solver.gather().cpu().numpy()
        solver.close()
        if rank == 0:
            np.save(out, full)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("world,halo,overlap,dims,count", [
    (2, 1, True, (64, 40, 36), 9),
    (3, 1, True, (136, 17, 23), 6),
    (2, 2, False, (64, 40, 36), 9),
    (2, 3, False, (130, 24, 31), 7),
    (2, 2, True, (128, 40, 36), 9),
    (3, 2, True, (136, 17, 23), 6),
    (2, 3, True, (130, 24, 31), 7),
])
def test_slab_solver_cuda_kernels_across_ranks(tmp_path, world, halo, overlap,
                                               dims, count):
    """Ranks on one GPU, exchange through host memory (gloo): the gathered
    field equals the oracle's run and the one-GPU run, bit for bit."""
    import torch
    import torch.multiprocessing as mp

    import benchmarks_b200 as B
    import oracle as O
    nx, ny, nz = dims
    out = str(tmp_path / "full.npy")
    mp.start_processes(_slab_cuda_worker,
                       args=(world, _free_port(), nx, ny, nz, count, halo,
                             overlap, 6, out),
                       nprocs=world, join=True, start_method="spawn")
    full = np.load(out)
    c, _ = O.params(nx, ny, nz)
    field = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 6)
    assert full.tobytes() == O.run(field, c, count).tobytes()
    plan = B.Plan(nx, ny, nz)
    f1 = torch.from_numpy(field).cuda()
    res, _ = plan.run(f1, torch.empty_like(f1), count, c)
    assert res.cpu().numpy().tobytes() == full.tobytes()
    plan.close()


@pytest.mark.gpu
def test_step_planes_writes_only_its_planes():
    """d3d_step_planes: the planes asked for equal a whole step's, the
    others keep their contents; bad ranges are refused."""
    import torch

    import benchmarks_b200 as B
    import oracle as O
    for dims in ((128, 24, 20), (37, 11, 9)):  # TMA and generic paths
        nx, ny, nz = dims
        c, _ = O.params(nx, ny, nz)
        fin = O.seeded_noise((nz, ny, nx), 8, amplitude=1.0)
        ref = O.run(fin, c, 1)
        plan = B.Plan(nx, ny, nz)
        f1 = torch.from_numpy(fin).cuda()
        for zb, ze in ((0, 1), (nz - 1, nz), (3, 7), (0, nz), (1, nz - 1)):
            f2 = torch.full_like(f1, -5.0)
            plan.step_planes(f1, f2, zb, ze, c)
            got = f2.cpu().numpy()
            assert got[zb:ze].tobytes() == ref[zb:ze].tobytes(), (dims, zb)
            assert (got[:zb] == -5.0).all() and (got[ze:] == -5.0).all()
        for zb, ze in ((-1, 2), (3, 3), (0, nz + 1)):
            with pytest.raises(B.D3DError) as ei:
                plan.step_planes(f1, f2, zb, ze, c)
            assert ei.value.code == B.D3D_E_INVALID
        plan.close()


@pytest.mark.gpu
def test_slab_solver_cuda_kernels_world_one():
    """The default step (our CUDA kernels through the C ABI) inside the slab
    solver, on one GPU with an NCCL group of one."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    import oracle as O
    from benchmarks_b200.distributed import SlabSolver

    nx, ny, nz, count = 64, 40, 36, 9
    c, _ = O.params(nx, ny, nz)
    field = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 2)
    store = dist.TCPStore("127.0.0.1", _free_port(), 1, True)
    dist.init_process_group("nccl", store=store, rank=0, world_size=1,
                            timeout=timedelta(seconds=60))
    try:
        fulls = []
        for halo, overlap in ((2, False), (1, True), (2, True)):
            solver = SlabSolver(dist, nx, ny, nz, c, halo=halo,
                                overlap=overlap)
            solver.load(torch.from_numpy(field).cuda())
            solver.run(count)
            torch.cuda.synchronize()
            fulls.append(solver.gather().cpu().numpy())
            solver.close()
    finally:
        dist.destroy_process_group()
    for full in fulls:
        assert full.tobytes() == O.run(field, c, count).tobytes()


@pytest.mark.gpu
def test_slab_transport_failure_is_reported():
    """A transport callback that fails ends d3d_slab_run with
    D3D_E_TRANSPORT after the work it queued; the Python exception comes
    back to the caller, and the slab stays usable."""
    import ctypes

    import torch

    import benchmarks_b200 as B
    import oracle as O
    from benchmarks_b200.distributed import SlabDecomposition, _SlabTransport

    nx, ny, nz = 32, 16, 24
    c, _ = O.params(nx, ny, nz)
    dec = SlabDecomposition(nz, 1, 2, halo=2)   # owns [12, 24), one below

    class Boom(RuntimeError):
        pass

    class Group:      # post() raises before any transfer
        @staticmethod
        def get_backend():
            return "nccl"

        @staticmethod
        def batch_isend_irecv(ops):
            raise Boom("no peer")

        P2POp = staticmethod(lambda *a: a)
        isend = irecv = None

    slab = ctypes.c_void_p()
    lnz = ctypes.c_int()
    B.check(B.lib().d3d_slab_create(nx, ny, nz, dec.z0, dec.z1, 2, B.F32,
                                    ctypes.byref(slab), ctypes.byref(lnz)))
    try:
        assert lnz.value == dec.local_nz == 14
        f1 = torch.zeros((lnz.value, ny, nx), device="cuda")
        f2 = torch.zeros_like(f1)
        t = _SlabTransport(Group, dec, f1.device, torch.float32)
        a = ctypes.c_void_p(f1.data_ptr())
        b = ctypes.c_void_p(f2.data_ptr())
        rc = B.lib().d3d_slab_run(slab, ctypes.byref(a), ctypes.byref(b),
                                  c.ctypes.data, 2, ctypes.byref(t.struct),
                                  torch.cuda.current_stream().cuda_stream)
        assert rc == B.D3D_E_TRANSPORT
        assert isinstance(t.error, Boom)
        assert "transport" in B.lib().d3d_last_error().decode()
        # a neighbour and no transport: refused before any launch
        rc = B.lib().d3d_slab_run(slab, ctypes.byref(a), ctypes.byref(b),
                                  c.ctypes.data, 2, None, None)
        assert rc == B.D3D_E_INVALID
        torch.cuda.synchronize()
    finally:
        B.lib().d3d_slab_destroy(slab)


@pytest.mark.gpu
@pytest.mark.parametrize("world,halo,dims,count", [
    (2, 2, (128, 40, 36), 9),
    (3, 3, (96, 24, 40), 7),
    (4, 2, (64, 17, 33), 10),
])
def test_slab_runner_threads_exchange_device_planes(world, halo, dims,
                                                    count):
    """d3d_slab_run with a transport of the caller's own: each rank is a
    host thread with its own stream and slab, and the planes move device to
    device (no torch.distributed, no host staging).  Waits are host-side and
    bounded (a barrier with a timeout); no kernel waits on another rank's.
    The owned planes gathered from all ranks equal the oracle's run."""
    import ctypes
    import threading

    import benchmarks_b200 as B
    import oracle as O
    import torch
    from benchmarks_b200.distributed import SlabDecomposition, _SlabTransport

    nx, ny, nz = dims
    c, _ = O.params(nx, ny, nz)
    field = O.initialize(nx, ny, nz) + O.seeded_noise((nz, ny, nx), 9)
    g = torch.from_numpy(field).cuda()
    decs = [SlabDecomposition(nz, r, world, halo) for r in range(world)]
    posted = [None] * world           # this pass's (send, recv) per rank
    barrier = threading.Barrier(world, timeout=60)
    errors = [None] * world
    results = [None] * world

    def rank_main(r):
        d = decs[r]
        stream = torch.cuda.Stream()
        slab = ctypes.c_void_p()
        lnz = ctypes.c_int()
        try:
            B.check(B.lib().d3d_slab_create(nx, ny, nz, d.z0, d.z1, halo,
                                            B.F32, ctypes.byref(slab),
                                            ctypes.byref(lnz)))
            assert lnz.value == d.local_nz
            f1 = g[d.lo:d.hi].clone()
            f2 = torch.empty_like(f1)
            torch.cuda.synchronize()

            def post(user, send, recv, nbytes, s):
                try:  # the planes to send are ready once this stream is
                    B.check(B.lib().d3d_stream_sync(s))
                except Exception as e:
                    errors[r] = e
                    barrier.abort()
                    return 1
                posted[r] = ([send[0], send[1]], [recv[0], recv[1]], nbytes)
                return 0

            def wait(user, s):
                try:
                    barrier.wait()           # every rank has posted
                    _, recv, nbytes = posted[r]
                    for side, peer, their in ((0, r - 1, 1), (1, r + 1, 0)):
                        if recv[side]:
                            B.check(B.lib().d3d_memcpy(
                                recv[side], posted[peer][0][their], nbytes,
                                s))
                    B.check(B.lib().d3d_stream_sync(s))
                    barrier.wait()           # every rank has copied
                    return 0
                except Exception as e:  # reported as a transport failure
                    errors[r] = e
                    barrier.abort()
                    return 1

            keep = (_SlabTransport.POST(post), _SlabTransport.WAIT(wait))
            t = _SlabTransport.Struct(
                ctypes.cast(keep[0], ctypes.c_void_p),
                ctypes.cast(keep[1], ctypes.c_void_p), None)
            a = ctypes.c_void_p(f1.data_ptr())
            b = ctypes.c_void_p(f2.data_ptr())
            B.check(B.lib().d3d_slab_run(slab, ctypes.byref(a),
                                         ctypes.byref(b), c.ctypes.data,
                                         count, ctypes.byref(t),
                                         stream.cuda_stream))
            torch.cuda.synchronize()
            res = f1 if a.value == f1.data_ptr() else f2
            results[r] = res[d.owned()].cpu().numpy()
        except Exception as e:
            if errors[r] is None:
                errors[r] = e
            barrier.abort()
        finally:
            B.lib().d3d_slab_destroy(slab)

    threads = [threading.Thread(target=rank_main, args=(r,))
               for r in range(world)]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=300)
    assert not any(th.is_alive() for th in threads)
    assert errors == [None] * world, errors
    full = np.concatenate(results)
    assert full.tobytes() == O.run(field, c, count).tobytes()
    assert B.check_device_errors() == 0
