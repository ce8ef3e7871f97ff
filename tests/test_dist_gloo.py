"""The N>1 path on CPU: two gloo ranks split a set of independent tables,
take the max of their timings and gather every table's record -- the same
steps `bench.py --gpus N` and a sharded run take over NCCL, with the solve
replaced by a host stand-in (no GPU here)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import PKG


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, jobs, q):
    sys.path.insert(0, PKG)
    import torch.distributed as dist
    from peregrine_hjb import dist as pdist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        recs = pdist.solve_sharded(
            jobs, lambda i, j: {"cells": pdist.table_cost(j["n"], 1), "checksum": sum(j["n"]) * 7},
            rank, world)
        t = pdist.max_over_ranks(1.5 + rank)
        q.put((rank, recs, t))
    finally:
        dist.destroy_process_group()


def test_assignment_is_a_partition_and_balanced():
    sys.path.insert(0, PKG)
    from peregrine_hjb.dist import assign_tables
    costs = [5, 9, 3, 9, 1, 7, 2, 8]
    for world in (1, 2, 3, 4):
        parts = assign_tables(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
        assert parts == assign_tables(costs, world)  # deterministic


def test_two_gloo_ranks_split_tables_and_agree():
    rng_jobs = [{"n": [24 + 8 * (i % 4), 24 + 8 * ((i + 1) % 4), 16, 9, 9, 9], "nctl": 125}
                for i in range(10)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, rng_jobs, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    (r0, recs0, t0), (r1, recs1, t1) = out
    assert recs0 == recs1                       # everyone holds the full list
    assert [r["index"] for r in recs0] == list(range(10))
    assert {r["rank"] for r in recs0} == {0, 1}  # both ranks did work
    assert t0 == t1 == 2.5                       # the max over ranks
