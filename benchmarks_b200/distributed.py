"""Multi-GPU diffusion3d: one grid split into z-slabs across ranks.

The reference has no in-tree multi-node path (its only one is the external
Physis MPI runtime, src/diffusion3d/Makefile:253-268).  Here each rank of a
torch.distributed process group (NCCL over NVLink between GPUs) owns planes
[z0, z1) of the global nx*ny*nz field plus up to `halo` ghost planes on each
side that has a neighbour.  Planes move by send/recv into the
neighbours' ghost planes, landing in the receiver's own memory (NCCL
between GPUs; through host memory on gloo).  SlabSolver has two schedules
(its docstring): an overlapped one that steps the two boundary planes
first, exchanges them while the interior steps, and never computes a plane
twice; and a halo-h one that exchanges h planes every h steps and runs the
h steps on the whole local buffer in one call.  The local stencil clamps at
the local buffer's edges; that is the reference's rule exactly at the
global boundary, and at a ghost edge it corrupts one more ghost plane per
step -- never an owned plane within h steps.  So the owned planes are
bit-identical to a single-GPU run.

Communication per exchange: 2 * halo planes of nx*ny values per interior
rank boundary.
"""
from __future__ import annotations

import ctypes

import numpy as np


def slab_bounds(nz, rank, world):
    """Owned planes [z0, z1) of `rank`: contiguous, sizes differ by <= 1."""
    base, extra = divmod(nz, world)
    z0 = rank * base + min(rank, extra)
    z1 = z0 + base + (1 if rank < extra else 0)
    return z0, z1


class SlabDecomposition:
    """Index bookkeeping for one rank (no device work)."""

    def __init__(self, nz, rank, world, halo=1):
        if world < 1 or not 0 <= rank < world:
            raise ValueError("bad rank/world")
        if nz < world:
            raise ValueError("fewer planes than ranks")
        self.nz, self.rank, self.world, self.halo = nz, rank, world, halo
        self.z0, self.z1 = slab_bounds(nz, rank, world)
        if self.z1 - self.z0 < halo:
            raise ValueError("slab thinner than the halo depth")
        self.lo = max(self.z0 - halo, 0)      # first local plane (global z)
        self.hi = min(self.z1 + halo, nz)     # one past the last
        self.down = rank - 1 if rank > 0 else None
        self.up = rank + 1 if rank < world - 1 else None

    @property
    def local_nz(self):
        return self.hi - self.lo

    def owned(self):
        """Owned planes as a local slice."""
        return slice(self.z0 - self.lo, self.z1 - self.lo)

    def send_down(self):  # my lowest owned planes -> rank-1's upper ghosts
        return slice(self.z0 - self.lo, self.z0 - self.lo + self.halo)

    def recv_down(self):  # my lower ghosts <- rank-1's highest owned planes
        return slice(0, self.z0 - self.lo)

    def send_up(self):    # my highest owned planes -> rank+1's lower ghosts
        return slice(self.z1 - self.lo - self.halo, self.z1 - self.lo)

    def recv_up(self):    # my upper ghosts <- rank+1's lowest owned planes
        return slice(self.z1 - self.lo, self.hi - self.lo)


class SingleProcess:
    """The process-group calls SlabSolver makes, for one rank alone (no
    torch.distributed group): no neighbours, so nothing is exchanged."""

    @staticmethod
    def get_rank():
        return 0

    @staticmethod
    def get_world_size():
        return 1

    @staticmethod
    def get_backend():
        return "nccl"

    @staticmethod
    def all_gather(parts, t):
        parts[0].copy_(t)


def _host_staged(dist, tensor):
    """Whether send/recv of `tensor` must go through host memory: a CUDA
    tensor on a backend without device transport (gloo)."""
    return tensor.is_cuda and dist.get_backend() != "nccl"


class _Exchange:
    """Posted sends and receives of whole planes (contiguous slices of a
    (planes, ny, nx) buffer).  On NCCL the planes move between GPUs, into
    the receiver's own memory, on the library's stream, ordered after the
    work already queued on the caller's stream; wait() orders the caller's
    stream after them.  On gloo with CUDA tensors the planes are staged
    through host memory (the send copies are taken when the exchange is
    posted, the receive copies land in wait())."""

    def __init__(self, dist, sends, recvs, group=None):
        # sends / recvs: [(peer, tensor)]
        self.dist = dist
        self.recvs = recvs
        self.staged = []
        ops = []
        for peer, t in sends:
            if _host_staged(dist, t):
                t = t.cpu()
            ops.append(dist.P2POp(dist.isend, t, peer, group))
        for peer, t in recvs:
            if _host_staged(dist, t):
                h = torch_empty_like_cpu(t)
                self.staged.append((t, h))
                t = h
            ops.append(dist.P2POp(dist.irecv, t, peer, group))
        self.reqs = dist.batch_isend_irecv(ops) if ops else []

    def wait(self):
        for r in self.reqs:
            r.wait()
        for dev, host in self.staged:
            dev.copy_(host)


def torch_empty_like_cpu(t):
    import torch
    return torch.empty(t.shape, dtype=t.dtype, device="cpu")


def exchange(dist, field, dec, group=None):
    """Fills the ghost planes of `field` (local_nz, ny, nx) from the
    neighbours.  Every rank calls this the same number of times."""
    sends, recvs = [], []
    if dec.down is not None:
        sends.append((dec.down, field[dec.send_down()]))
        recvs.append((dec.down, field[dec.recv_down()]))
    if dec.up is not None:
        sends.append((dec.up, field[dec.send_up()]))
        recvs.append((dec.up, field[dec.recv_up()]))
    _Exchange(dist, sends, recvs, group).wait()


class _CudaArray:
    """Device memory the library owns, seen through the CUDA array
    interface so torch can wrap it without a copy."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {
            "shape": (count,), "typestr": typestr, "data": (ptr, False),
            "version": 2}


class _SlabTransport:
    """d3d_slab_transport over a torch.distributed group: post() starts
    the send/recv of the planes the library names (_Exchange: NCCL into
    the receiver's memory, or host staging on gloo), wait() finishes it.
    A Python exception in a callback is kept and re-raised by the caller
    once the library has returned D3D_E_TRANSPORT."""

    POST = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p,
                            ctypes.POINTER(ctypes.c_void_p),
                            ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t,
                            ctypes.c_void_p)
    WAIT = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p)

    class Struct(ctypes.Structure):
        _fields_ = [("post", ctypes.c_void_p), ("wait", ctypes.c_void_p),
                    ("user", ctypes.c_void_p)]

    def __init__(self, dist, dec, device, dtype):
        import torch
        self.dist, self.dec, self.device = dist, dec, device
        self.dtype = dtype
        self.esize = 8 if dtype == torch.float64 else 4
        self.typestr = "<f8" if dtype == torch.float64 else "<f4"
        self.error = None
        self._xchg = None
        self._post = self.POST(self._on_post)  # kept alive with the struct
        self._wait = self.WAIT(self._on_wait)
        self.struct = self.Struct(
            ctypes.cast(self._post, ctypes.c_void_p),
            ctypes.cast(self._wait, ctypes.c_void_p), None)

    def _view(self, ptr, nbytes):
        import torch
        return torch.as_tensor(
            _CudaArray(ptr, nbytes // self.esize, self.typestr),
            device=self.device)

    def _on_post(self, user, send, recv, nbytes, stream):
        try:
            peers = (self.dec.down, self.dec.up)
            sends, recvs = [], []
            for i in range(2):
                if send[i]:
                    sends.append((peers[i], self._view(send[i], nbytes)))
                    recvs.append((peers[i], self._view(recv[i], nbytes)))
            if any(_host_staged(self.dist, t) for _, t in sends):
                import torch
                torch.cuda.synchronize(self.device)
            self._xchg = _Exchange(self.dist, sends, recvs)
            return 0
        except BaseException as e:  # reported through the return code
            self.error = e
            return 1

    def _on_wait(self, user, stream):
        try:
            xchg, self._xchg = self._xchg, None
            xchg.wait()
            return 0
        except BaseException as e:
            self.error = e
            return 1


class SlabSolver:
    """Runs `count` steps of one global field split across the group.

    Three schedules, all bit-identical to a one-GPU run:
    * overlap=True, halo 1: every step first computes the two owned planes
      the neighbours need (d3d_step_planes), posts their exchange into the
      neighbours' ghost planes of the output buffer, computes the interior
      planes while the planes travel, then waits.  No plane is computed
      twice.
    * overlap=True, halo k >= 2 (passes of k steps; d3d_slab_run, the
      pass loop in the library, with this group's send/recv as its
      transport): each pass first runs k steps on a 3k-plane piece around
      every rank boundary ([lo-k, lo+2k) below, [hi-2k, hi+k) above, on
      copies), whose middle k planes are then exact; they go to the
      neighbour while the owned planes [lo, hi) run k steps in one call
      (the plan's kernels: fused two-step passes where it uses them), exact
      except the k planes at each rank boundary, which the pieces' planes
      overwrite.  The received planes land in side buffers and become the
      next pass's ghosts.  The pieces cost 2k extra planes of stepping per
      boundary; a pass exchanges once.
    * overlap=False (halo h >= 1): every h steps the ranks exchange their h
      outermost owned planes, then each rank runs h steps on its whole
      local buffer with one RunKernel-style call; the ghost planes are
      computed redundantly and go stale one plane per step, never reaching
      an owned plane within h steps.

    step_fn(src, dst), when given, replaces the CUDA plan (one whole-buffer
    step; overlap is then unavailable): the CPU tests pass the oracle's
    step there.
    """

    def __init__(self, dist, nx, ny, nz, coeff, halo=1, step_fn=None,
                 device=None, dtype=None, overlap=False):
        import torch
        self.dist = dist
        if overlap and halo == 1 and step_fn is not None:
            raise ValueError("the halo-1 overlapped schedule runs on the "
                             "CUDA plan")
        self.overlap = overlap
        self.dec = SlabDecomposition(nz, dist.get_rank(),
                                     dist.get_world_size(), halo)
        d = self.dec
        if (overlap and halo > 1 and (d.down is not None or d.up is not None)
                and d.z1 - d.z0 < 2 * halo):
            raise ValueError("the overlapped schedule needs at least "
                             "2 x halo owned planes a rank")
        self.nx, self.ny, self.nz = nx, ny, nz
        self.coeff = np.ascontiguousarray(coeff)
        self.device = device if device is not None else torch.device("cuda")
        self.dtype = dtype if dtype is not None else torch.float32
        shape = (self.dec.local_nz, ny, nx)
        self.f1 = torch.zeros(shape, dtype=self.dtype, device=self.device)
        self.f2 = torch.zeros_like(self.f1)
        self._plan = None
        self._slab = None          # the C-ABI slab (CUDA, overlapped passes)
        self._transport = None
        self._pieces = {}          # the same schedule for a step_fn
        self.step_fn = step_fn
        neighbours = d.down is not None or d.up is not None
        if step_fn is None:
            from . import F32, F64, Plan, check, lib
            dt = F64 if self.dtype == torch.float64 else F32
            if overlap and halo > 1:
                self._slab = ctypes.c_void_p()
                lnz = ctypes.c_int()
                check(lib().d3d_slab_create(nx, ny, nz, d.z0, d.z1, halo, dt,
                                            ctypes.byref(self._slab),
                                            ctypes.byref(lnz)))
                assert lnz.value == d.local_nz
                if neighbours:
                    self._transport = _SlabTransport(dist, d, self.device,
                                                     self.dtype)
            else:
                self._plan = Plan(nx, ny, d.local_nz, dt)
        elif overlap and halo > 1:
            # per neighbour: the piece's two buffers and the ghost landing
            for side in ("down", "up"):
                if getattr(d, side) is not None:
                    self._pieces[side] = (
                        torch.empty((3 * halo, ny, nx), dtype=self.dtype,
                                    device=self.device),
                        torch.empty((3 * halo, ny, nx), dtype=self.dtype,
                                    device=self.device),
                        torch.empty((halo, ny, nx), dtype=self.dtype,
                                    device=self.device))

    def load(self, global_field):
        """Copies this rank's planes (with ghosts) of a global field."""
        import torch
        g = torch.as_tensor(global_field)
        self.f1.copy_(g[self.dec.lo:self.dec.hi])

    def _step_overlapped(self):
        d, plan, c = self.dec, self._plan, self.coeff
        f1, f2 = self.f1, self.f2
        lo, hi = d.z0 - d.lo, d.z1 - d.lo  # owned planes, local indices
        edge = []
        if d.down is not None:
            edge.append(lo)
        if d.up is not None and hi - 1 not in edge:
            edge.append(hi - 1)
        for z in edge:
            plan.step_planes(f1, f2, z, z + 1, c)
        sends, recvs = [], []
        if d.down is not None:
            sends.append((d.down, f2[lo:lo + 1]))
            recvs.append((d.down, f2[lo - 1:lo]))
        if d.up is not None:
            sends.append((d.up, f2[hi - 1:hi]))
            recvs.append((d.up, f2[hi:hi + 1]))
        if any(_host_staged(self.dist, t) for _, t in sends):
            import torch
            torch.cuda.synchronize(self.device)
        xchg = _Exchange(self.dist, sends, recvs)
        ilo = lo + (1 if d.down is not None else 0)
        ihi = hi - (1 if d.up is not None else 0)
        if ilo < ihi:
            plan.step_planes(f1, f2, ilo, ihi, c)
        xchg.wait()
        self.f1, self.f2 = f2, f1

    def _steps(self, a, b, k):
        """k steps of step_fn ping-ponging (a, b); returns the buffer
        holding the result."""
        for _ in range(k):
            self.step_fn(a, b)
            a, b = b, a
        return a

    def _pass_fused(self, k):
        """One k-step pass (k <= halo) of the overlapped-pass schedule on
        step_fn: the pass loop of d3d_slab_run, written out for the host
        tests (the CUDA path runs it in the library)."""
        d, h = self.dec, self.dec.halo
        f1, f2 = self.f1, self.f2
        lo, hi = d.z0 - d.lo, d.z1 - d.lo  # owned planes, local indices
        first = {"down": lo - h, "up": hi - 2 * h}
        peer = {"down": d.down, "up": d.up}
        exact = {}
        sends, recvs = [], []
        for side, (pa, pb, ghost) in self._pieces.items():
            pa.copy_(f1[first[side]:first[side] + 3 * h])
            r = self._steps(pa, pb, k)
            exact[side] = r[h:2 * h]   # exact after k <= h steps
            sends.append((peer[side], exact[side]))
            recvs.append((peer[side], ghost))
        xchg = _Exchange(self.dist, sends, recvs)
        own = self._steps(f1[lo:hi], f2[lo:hi], k)
        res, other = (f1, f2) if own.data_ptr() == f1[lo:hi].data_ptr() \
            else (f2, f1)
        if "down" in exact:
            res[lo:lo + h].copy_(exact["down"])
        if "up" in exact:
            res[hi - h:hi].copy_(exact["up"])
        xchg.wait()
        if "down" in self._pieces:
            res[lo - h:lo].copy_(self._pieces["down"][2])
        if "up" in self._pieces:
            res[hi:hi + h].copy_(self._pieces["up"][2])
        self.f1, self.f2 = res, other

    def _run_slab(self, count):
        """`count` steps through d3d_slab_run (the pass loop in the
        library; this group's send/recv as its transport)."""
        import torch
        from . import D3D_E_TRANSPORT, check, lib
        a = ctypes.c_void_p(self.f1.data_ptr())
        b = ctypes.c_void_p(self.f2.data_ptr())
        t = self._transport
        rc = lib().d3d_slab_run(
            self._slab, ctypes.byref(a), ctypes.byref(b),
            self.coeff.ctypes.data, count,
            ctypes.byref(t.struct) if t is not None else None,
            torch.cuda.current_stream(self.device).cuda_stream)
        if rc == D3D_E_TRANSPORT and t is not None and t.error is not None:
            err, t.error = t.error, None
            raise err
        check(rc)
        if a.value != self.f1.data_ptr():
            self.f1, self.f2 = self.f2, self.f1

    def run(self, count):
        if self.overlap and self.dec.halo > 1:
            d = self.dec
            if d.down is not None or d.up is not None:
                exchange(self.dist, self.f1, d)  # current ghosts to start
            if self._slab is not None:
                self._run_slab(count)
            else:
                h, done = d.halo, 0
                while done < count:
                    k = min(h, count - done)
                    self._pass_fused(k)
                    done += k
            return self.f1[d.owned()]
        if self.overlap:
            for _ in range(count):
                self._step_overlapped()
            return self.f1[self.dec.owned()]
        h = self.dec.halo
        done = 0
        while done < count:
            exchange(self.dist, self.f1, self.dec)
            k = min(h, count - done)
            if self.step_fn is not None:
                for _ in range(k):
                    self.step_fn(self.f1, self.f2)
                    self.f1, self.f2 = self.f2, self.f1
            else:
                a, b = self._plan.run(self.f1, self.f2, k, self.coeff)
                self.f1, self.f2 = a, b
            done += k
        return self.f1[self.dec.owned()]

    def gather(self):
        """The full field on every rank (all_gather of owned slabs)."""
        import torch
        owned = self.f1[self.dec.owned()].contiguous()
        sizes = [slab_bounds(self.nz, r, self.dec.world)
                 for r in range(self.dec.world)]
        maxn = max(z1 - z0 for z0, z1 in sizes)
        staged = _host_staged(self.dist, owned)
        dev = torch.device("cpu") if staged else self.device
        pad = torch.zeros((maxn, self.ny, self.nx), dtype=self.dtype,
                          device=dev)
        pad[:owned.shape[0]] = owned.to(dev)
        parts = [torch.empty_like(pad) for _ in sizes]
        self.dist.all_gather(parts, pad)
        return torch.cat([p[:z1 - z0] for p, (z0, z1) in zip(parts, sizes)])

    def close(self):
        if self._plan is not None:
            self._plan.close()
            self._plan = None
        if self._slab is not None:
            from . import lib
            lib().d3d_slab_destroy(self._slab)
            self._slab = None
