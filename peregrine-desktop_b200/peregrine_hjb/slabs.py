"""One table split into x slabs over ranks.

The backup reaches only a bounded distance in x: nothing in the dynamics
reads x or y (solver/src/Tiles.jl:94-103), so the successor and every swept
probe of a cell lie within the largest successor offset of it -- the same
property the reference's out-of-core tiling rests on (Tiles.jl:311-340,
halo = reach + 2; only x and y can be cut).  A table therefore splits into
contiguous x slabs, one per rank, each loaded with `halo` extra rows either
side.  One Jacobi sweep is then:

  1. every rank sweeps the interior rows of its slab;
  2. neighbours exchange the `halo` rows at each end of their interiors
     (paired sends and receives, so no rank waits on a cycle);
  3. the ranks take the sum and the max of their residuals.

The sweep itself and the row copies are the sweeper's (an object with
`sweep(phase) -> (l1, maxnorm)`, `rows(r0, r1) -> tensor` and
`set_rows(r0, r1, tensor)`, rows local to the slab, row 0 = global row a);
this module owns the partition, the exchange and the stop rule, over
torch.distributed (NCCL between GPUs, gloo on CPUs).  With a halo at least
the reach, every interior cell reads only rows its slab holds, and the split
solve equals the single-table solve bit for bit.
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class Slab:
    x0: int  # interior rows [x0, x1), global
    x1: int
    a: int   # loaded rows [a, b), global (interior plus halo, clipped to the table)
    b: int

    @property
    def rows(self) -> int:
        return self.b - self.a


def plan_slabs(n1: int, world: int, halo: int) -> list:
    """Contiguous, balanced x slabs of a table of n1 rows over `world`
    ranks.  Refuses an interior thinner than the halo: a neighbour's halo
    would then reach past this slab into the next one's rows."""
    if world < 1 or halo < 0:
        raise ValueError("world must be >= 1 and halo >= 0")
    if n1 < world:
        raise ValueError(f"{n1} rows cannot be split over {world} ranks")
    out = []
    for r in range(world):
        x0 = (r * n1) // world
        x1 = ((r + 1) * n1) // world
        if world > 1 and x1 - x0 < halo:
            raise ValueError(f"slab {r} has {x1 - x0} interior rows, fewer than the {halo}-row "
                             "halo; use fewer ranks or a coarser x axis")
        out.append(Slab(x0, x1, max(0, x0 - halo), min(n1, x1 + halo)))
    return out


def exchange_halos(slabs, rank: int, world: int, sweeper) -> None:
    """Send the ends of this rank's interior to its neighbours' halos and
    receive theirs into this slab's halo rows."""
    import torch.distributed as dist
    s = slabs[rank]
    ops, recvs = [], []
    if rank > 0:
        lo = slabs[rank - 1]
        n = s.x0 - s.a  # the rows below the interior = the lower neighbour's top interior rows
        if n > 0:
            ops.append(dist.P2POp(dist.isend, sweeper.rows(s.x0 - s.a, s.x0 - s.a + (lo.b - lo.x1)).contiguous(),
                                  rank - 1))
            buf = sweeper.rows(0, n).clone()
            ops.append(dist.P2POp(dist.irecv, buf, rank - 1))
            recvs.append((0, n, buf))
    if rank < world - 1:
        hi = slabs[rank + 1]
        n = s.b - s.x1
        if n > 0:
            ops.append(dist.P2POp(dist.isend, sweeper.rows(s.x1 - s.a - (hi.x0 - hi.a), s.x1 - s.a).contiguous(),
                                  rank + 1))
            buf = sweeper.rows(s.x1 - s.a, s.b - s.a).clone()
            ops.append(dist.P2POp(dist.irecv, buf, rank + 1))
            recvs.append((s.x1 - s.a, s.b - s.a, buf))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for r0, r1, buf in recvs:
        sweeper.set_rows(r0, r1, buf)


def solve_slabs(sweeper, slabs, rank: int, world: int, iters: int, tol: float,
                device=None) -> tuple:
    """Jacobi sweeps of a table split into x slabs until the largest
    single-cell change over every rank is <= tol or `iters` sweeps ran
    (the max-norm stop rule).  Returns (sweeps, last L1 total, last max)."""
    import torch
    import torch.distributed as dist
    multi = world > 1 and dist.is_available() and dist.is_initialized()
    d = dm = float("inf")
    done = 0
    for it in range(1, iters + 1):
        l1, mx = sweeper.sweep(it - 1)
        if multi:
            exchange_halos(slabs, rank, world, sweeper)
            t = torch.tensor([float(mx)], dtype=torch.float64, device=device or "cpu")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            u = torch.tensor([float(l1)], dtype=torch.float64, device=device or "cpu")
            dist.all_reduce(u, op=dist.ReduceOp.SUM)
            mx, l1 = float(t.item()), float(u.item())
        d, dm, done = l1, mx, it
        if dm <= tol:
            break
    return done, d, dm


def exchange_in_process(slabs, sweepers) -> None:
    """The halo exchange of exchange_halos for slabs held by one process
    (several contexts on one GPU, swept one after another): each slab's halo
    rows are copied from its neighbours' interiors after every slab's sweep."""
    got = []
    for r, s in enumerate(slabs):
        if r > 0:
            lo, n = slabs[r - 1], s.x0 - s.a
            if n > 0:
                got.append((r, 0, n, sweepers[r - 1].rows(s.a - lo.a, s.x0 - lo.a)))
        if r < len(slabs) - 1:
            hi, n = slabs[r + 1], s.b - s.x1
            if n > 0:
                got.append((r, s.x1 - s.a, s.b - s.a, sweepers[r + 1].rows(s.x1 - hi.a, s.b - hi.a)))
    for r, r0, r1, t in got:
        sweepers[r].set_rows(r0, r1, t)


class DeviceSlab:
    """One slab on this process's GPU (pg_load_slab), swept by the row stencil
    (the fast masked sweeps keep whole tables); rows move as torch tensors on
    the device, so the exchange runs over NCCL without touching the host."""

    def __init__(self, grid, model, params, occ, ctl, seeds, slab: Slab, device: int = 0,
                 kernel=None, exact: bool = False):
        import numpy as np

        from . import _lib
        self._lib = _lib
        self.slab = slab
        self.device = device
        self.kernel = _lib.KERNEL_STENCIL_EXACT if exact else _lib.KERNEL_STENCIL_ROWS
        self.ctx = _lib.Context(device)
        row0, rows = self.ctx.load_slab(grid, model, params, occ, ctl, slab.x0, slab.x1,
                                        max(slab.x0 - slab.a, slab.b - slab.x1))
        if (row0, rows) != (slab.a, slab.b - slab.a):
            raise ValueError("the library's slab differs from the plan")
        per = self.ctx.row_cells
        seeds = np.asarray(seeds, np.int64)
        loc = seeds[(seeds >= slab.a * per) & (seeds < slab.b * per)] - slab.a * per
        # seed the slab (cap everywhere, zero at the seeds) without sweeping
        self.ctx.solve(loc, 0, 0.0, _lib.default_opts(kernel=self.kernel))

    def sweep(self, phase: int):
        d, dm, _ = self.ctx.sweep(phase=phase, kernel=self.kernel)
        return d, dm

    def rows(self, r0: int, r1: int):
        import torch
        t = torch.empty((r1 - r0) * self.ctx.row_cells, dtype=torch.float32,
                        device=f"cuda:{self.device}")
        torch.cuda.synchronize(self.device)
        self.ctx.get_rows(r0, r1, t.data_ptr(), on_device=True)
        return t

    def set_rows(self, r0: int, r1: int, t) -> None:
        import torch
        torch.cuda.synchronize(self.device)
        self.ctx.set_rows(r0, r1, t.contiguous().data_ptr(), on_device=True)

    def interior(self):
        """The slab's interior rows, FP32 row-major (host)."""
        s = self.slab
        return self.ctx.get_rows(s.x0 - s.a, s.x1 - s.a)

    def close(self) -> None:
        self.ctx.close()
