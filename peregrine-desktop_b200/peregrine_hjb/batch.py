"""Batched solves of many independent tables, and the tile autotuner.

The reference solves its targets one after another (`run_solve`, Run.jl:
1851-1958), each a full `solve_value!`.  Independent tables have no data in
common, so the library sweeps a whole batch of them in one persistent
launch per sweep, replayed as a CUDA graph (`pg_batch_*`).  The tile shape
of the blend-then-shift sweep (rows of a plane per block) depends on the
table's (Nx, Ny); `autotune` times the candidate shapes on the device and
keeps the fastest per shape.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .synth import Problem


def tile_candidates(n1: int, n2: int) -> list[int]:
    """Rows per block worth trying in a batch (256-thread blocks, 4 cells per
    thread): whole rows, tiles of equal height, at most 1024 cells per block
    and at least 3/4 of the balanced tiling with the fewest tiles."""
    rmax = min(n1, 1024 // n2)
    r0 = -(-n1 // -(-n1 // rmax))  # the balanced tiling with the fewest tiles
    out = []
    for nt in range(-(-n1 // rmax), n1 + 1):
        r = -(-n1 // nt)
        if r * n2 < 0.75 * r0 * n2 or len(out) >= 4:
            break
        if r not in out:
            out.append(r)
    return out


def autotune(problems, device: int = 0, sweeps: int = 4) -> dict:
    """{(n1, n2): rows} for the problems' position shapes: each candidate
    tiling timed as a one-table batch (the launch the batch runs) on one
    table of that shape, the fastest kept."""
    best = {}
    for pr in problems:
        n1, n2 = int(pr.grid.n[0]), int(pr.grid.n[1])
        if (n1, n2) in best:
            continue
        cands = tile_candidates(n1, n2)
        if len(cands) == 1:
            best[(n1, n2)] = cands[0]
            continue
        times = {}
        for r in cands:
            with _lib.Batch(device, "fp16") as b:
                b.add(pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.seeds, pr.ctl, r)
                times[r] = b.solve(sweeps, 0.0, 0, True).kernel_ms
        best[(n1, n2)] = min(times, key=times.get)
    return best


def batch_problems(count: int = 64, seed: int = 0, control_set: str = "cube5", dt: float = 0.04,
                   xy=(24, 32, 40, 48), heading=(16, 24, 32), vel=(9, 11, 15)):
    """Independent tables of uneven size: position axes from `xy`, headings
    from `heading`, each velocity axis from `vel`; each table its own seeded
    drivetrain, target disk and 2-6 rectangles."""
    rng = np.random.default_rng(seed)
    out = []
    for t in range(count):
        n = [int(rng.choice(xy)), int(rng.choice(xy)), int(rng.choice(heading)),
             int(rng.choice(vel)), int(rng.choice(vel)), int(rng.choice(vel))]
        out.append(Problem("tiny", seed=int(seed * 1000 + t), n=n, control_set=control_set, dt=dt,
                           rects=int(rng.integers(2, 7))))
    return out


def solve_batch(problems, storage: str = "fp16", iters: int = 4000, tol: float = 1e-4,
                polish_sweeps: int = 4000, graph: bool = True, tiles: dict | None = None,
                device: int = 0):
    """Solve `problems` as one batch; returns (result, [V per table],
    [(sweeps, last max-norm change) per table])."""
    with _lib.Batch(device, storage) as b:
        for pr in problems:
            rows = (tiles or {}).get((int(pr.grid.n[0]), int(pr.grid.n[1])), 0)
            b.add(pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.seeds, pr.ctl, rows)
        res = b.solve(iters, tol, polish_sweeps, graph)
        Vs = [b.get_value(t) for t in range(len(problems))]
        info = [b.table(t) for t in range(len(problems))]
    return res, Vs, info
