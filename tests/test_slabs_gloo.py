"""One table split into x slabs over two gloo ranks (peregrine_hjb/slabs.py):
each rank sweeps its interior with the CPU oracle from a table that holds
only its slab (NaN everywhere else, so a read outside the slab would show),
the ranks exchange halos after every sweep, and the gathered table equals the
single-table Jacobi solve bit for bit."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import PKG, ROOT

N = (12, 12, 8, 5, 5, 5)
SWEEPS = 8
HALO = 3  # the tiny grid's reach is one row (7.5 cm per step on 33 cm rows), plus two


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _structs(og, pr):
    return (og.copy_struct(pr.grid.to_c(), og.OGrid), og.copy_struct(pr.model.to_c(), og.OModel),
            og.copy_struct(pr.params, og.OParams))


class OracleSlab:
    """The oracle's sweep of one slab's interior, on a whole-size table that
    holds only the slab's rows."""

    def __init__(self, og, pr, slab):
        import torch
        self.og, self.pr, self.slab, self.torch = og, pr, slab, torch
        self.g, self.m, self.p = _structs(og, pr)
        self.per = pr.ncells // pr.grid.n[0]
        self.V = np.full(pr.ncells, np.nan, np.float32)
        self.V[slab.a * self.per:slab.b * self.per] = np.float32(pr.params.cap)
        lo, hi = slab.x0 * self.per, slab.x1 * self.per
        self.seeds = pr.seeds[(pr.seeds >= slab.a * self.per) & (pr.seeds < slab.b * self.per)]
        self.V[self.seeds] = 0.0
        self.inner = pr.seeds[(pr.seeds >= lo) & (pr.seeds < hi)]

    def sweep(self, phase):
        lo, hi = self.slab.x0 * self.per, self.slab.x1 * self.per
        out, tot, mx = self.og.sweep_jacobi_slab(self.V, self.pr.occ, self.g, self.m, self.pr.ctl,
                                                 self.p, lo, hi, phase)
        self.V[lo:hi] = out
        self.V[self.inner] = 0.0
        return tot, mx

    def rows(self, r0, r1):
        a = self.slab.a
        return self.torch.from_numpy(self.V[(a + r0) * self.per:(a + r1) * self.per].copy())

    def set_rows(self, r0, r1, t):
        a = self.slab.a
        self.V[(a + r0) * self.per:(a + r1) * self.per] = t.numpy()


def _worker(rank, world, port, q):
    for p in (ROOT, PKG):
        sys.path.insert(0, p)
    import torch.distributed as dist
    from oracle import oracle as og
    from peregrine_hjb import slabs as S
    from peregrine_hjb.synth import Problem
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pr = Problem("tiny", seed=5, n=N)
        plan = S.plan_slabs(pr.grid.n[0], world, HALO)
        sw = OracleSlab(og, pr, plan[rank])
        done, d, dm = S.solve_slabs(sw, plan, rank, world, SWEEPS, 0.0)
        s = plan[rank]
        mine = sw.V[s.x0 * sw.per:s.x1 * sw.per].copy()
        parts = [None] * world
        dist.all_gather_object(parts, (s.x0, mine))
        q.put((rank, done, d, dm, sorted(parts, key=lambda t: t[0])))
    finally:
        dist.destroy_process_group()


def test_plan_slabs():
    sys.path.insert(0, PKG)
    from peregrine_hjb.slabs import plan_slabs
    p = plan_slabs(12, 2, 3)
    assert [(s.x0, s.x1, s.a, s.b) for s in p] == [(0, 6, 0, 9), (6, 12, 3, 12)]
    p = plan_slabs(96, 8, 3)
    assert p[0].x0 == 0 and p[-1].x1 == 96
    assert all(p[i].x1 == p[i + 1].x0 for i in range(7))
    with pytest.raises(ValueError, match="fewer than"):
        plan_slabs(12, 6, 3)


def test_two_ranks_reproduce_the_single_table_solve(og):
    from peregrine_hjb.synth import Problem
    pr = Problem("tiny", seed=5, n=N)
    g, m, p = _structs(og, pr)
    V = np.full(pr.ncells, np.float32(pr.params.cap), np.float32)
    V[pr.seeds] = 0.0
    for it in range(SWEEPS):
        V, tot, mx, _ = og.sweep_jacobi(V, pr.occ, g, m, pr.ctl, p, phase=it)
        V[pr.seeds] = 0.0
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pp in procs:
        pp.start()
    out = sorted(q.get(timeout=300) for _ in procs)
    for pp in procs:
        pp.join(timeout=60)
        assert pp.exitcode == 0
    for rank, done, d, dm, parts in out:
        assert done == SWEEPS
        assert dm == mx                      # the max over ranks is the whole table's
        got = np.concatenate([v for _, v in parts])
        assert np.array_equal(got, V), f"max |dV| {np.nanmax(np.abs(got - V))}"
