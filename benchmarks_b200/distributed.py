"""Multi-GPU diffusion3d: one grid split into z-slabs across ranks.

The reference has no in-tree multi-node path (its only one is the external
Physis MPI runtime, src/diffusion3d/Makefile:253-268).  Here each rank of a
torch.distributed process group (NCCL over NVLink between GPUs) owns planes
[z0, z1) of the global nx*ny*nz field plus up to `halo` ghost planes on each
side that has a neighbour.  Every `halo` steps the ranks exchange their
`halo` outermost owned planes with both neighbours (send/recv into the
neighbours' ghost planes, landing in the receiver's own memory), then each
rank runs `halo` ordinary steps on its local buffer with the single-grid
kernels.  The local stencil clamps at the local buffer's edges; that is the
reference's rule exactly at the global boundary, and at a ghost edge it
corrupts one more ghost plane per step -- never an owned plane within
`halo` steps.  So the owned planes are bit-identical to a single-GPU run.

Communication per exchange: 2 * halo planes of nx*ny values per interior
rank boundary; compute overhead: 2 * halo extra planes per step.
"""
from __future__ import annotations

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


def exchange(dist, field, dec, group=None):
    """Fills the ghost planes of `field` (local_nz, ny, nx) from the
    neighbours.  Every rank calls this the same number of times."""
    ops = []
    if dec.down is not None:
        ops.append(dist.P2POp(dist.isend, field[dec.send_down()].contiguous(),
                              dec.down, group))
        rd = field[dec.recv_down()]
        ops.append(dist.P2POp(dist.irecv, rd, dec.down, group))
    if dec.up is not None:
        ops.append(dist.P2POp(dist.isend, field[dec.send_up()].contiguous(),
                              dec.up, group))
        ru = field[dec.recv_up()]
        ops.append(dist.P2POp(dist.irecv, ru, dec.up, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


class SlabSolver:
    """Runs `count` steps of one global field split across the group.

    step_fn(src, dst) advances a local (local_nz, ny, nx) buffer by one
    step; the default uses this rank's GPU through the C ABI
    (Plan.step on the local buffer).
    """

    def __init__(self, dist, nx, ny, nz, coeff, halo=1, step_fn=None,
                 device=None, dtype=None):
        import torch
        self.dist = dist
        self.dec = SlabDecomposition(nz, dist.get_rank(),
                                     dist.get_world_size(), halo)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.coeff = np.ascontiguousarray(coeff)
        self.device = device if device is not None else torch.device("cuda")
        self.dtype = dtype if dtype is not None else torch.float32
        shape = (self.dec.local_nz, ny, nx)
        self.f1 = torch.zeros(shape, dtype=self.dtype, device=self.device)
        self.f2 = torch.zeros_like(self.f1)
        if step_fn is None:
            from . import F32, F64, Plan
            plan = Plan(nx, ny, self.dec.local_nz,
                        F64 if self.dtype == torch.float64 else F32)
            self._plan = plan

            def step_fn(src, dst):
                plan.step(src, dst, self.coeff)
        self.step_fn = step_fn

    def load(self, global_field):
        """Copies this rank's planes (with ghosts) of a global field."""
        import torch
        g = torch.as_tensor(global_field)
        self.f1.copy_(g[self.dec.lo:self.dec.hi])

    def run(self, count):
        h = self.dec.halo
        done = 0
        while done < count:
            exchange(self.dist, self.f1, self.dec)
            for _ in range(min(h, count - done)):
                self.step_fn(self.f1, self.f2)
                self.f1, self.f2 = self.f2, self.f1
                done += 1
        return self.f1[self.dec.owned()]

    def gather(self):
        """The full field on every rank (all_gather of owned slabs)."""
        import torch
        owned = self.f1[self.dec.owned()].contiguous()
        sizes = [slab_bounds(self.nz, r, self.dec.world)
                 for r in range(self.dec.world)]
        maxn = max(z1 - z0 for z0, z1 in sizes)
        pad = torch.zeros((maxn, self.ny, self.nx), dtype=self.dtype,
                          device=self.device)
        pad[:owned.shape[0]] = owned
        parts = [torch.empty_like(pad) for _ in sizes]
        self.dist.all_gather(parts, pad)
        return torch.cat([p[:z1 - z0] for p, (z0, z1) in zip(parts, sizes)])
