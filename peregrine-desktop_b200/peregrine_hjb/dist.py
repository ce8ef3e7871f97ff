"""Multi-GPU plumbing: independent target tables sharded across ranks.

The reference solves one table at a time on one GPU (solver/cloud/README.md:197).
Tables are independent units -- no value ever crosses between two targets'
tables -- so several GPUs split a run's tables with no data-path collective:
each rank solves a disjoint subset, and the only collectives are the ones
that report (the max of the timings, the gathered per-table records).

Process model: one process per GPU, launched by torchrun; `torch.distributed`
with NCCL on GPUs or gloo on CPUs (the tests).
"""
from __future__ import annotations

import heapq


def table_cost(n, nctl: int) -> int:
    """Work of one sweep of a table: cells x controls."""
    c = 1
    for v in n:
        c *= int(v)
    return c * int(nctl)


def assign_tables(costs, world: int):
    """Deterministic longest-processing-time-first assignment of tables to
    ranks: returns, per rank, the sorted list of table indices.  Ties go to
    the lower table index and the lower rank, so every rank computes the same
    assignment without communicating."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-int(costs[i]), i))
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(costs[i]), r))
    return [sorted(v) for v in out]


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over all ranks (the bench's timing rule); the
    identity without an initialised process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_records(records):
    """All ranks' per-table records (lists of dicts), merged and sorted by
    table index; each rank gets the full list."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return sorted(records, key=lambda r: r["index"])
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, list(records))
    merged = [r for p in parts for r in p]
    return sorted(merged, key=lambda r: r["index"])


def solve_sharded(jobs, solve_one, rank: int, world: int):
    """Solve this rank's share of `jobs` with `solve_one(index, job) -> dict`
    and return every rank's records (gathered)."""
    costs = [table_cost(j["n"], j["nctl"]) for j in jobs]
    mine = assign_tables(costs, world)[rank]
    recs = []
    for i in mine:
        rec = dict(solve_one(i, jobs[i]))
        rec["index"] = i
        rec["rank"] = rank
        recs.append(rec)
    return gather_records(recs)
