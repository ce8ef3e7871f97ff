"""Generate the committed golden fixtures from the CPU oracle.

    python tests/golden/make_golden.py [tiny|small] [--checkpoint DIR]

tiny_fixed_point.npz: the oracle's Jacobi solve of the 12x12x8x5x5x5
synthetic workload (seed 5, 27 controls, max-norm stop 1e-4 s) -- V at the
fixed point, the sweep count, and the argmin control of one more sweep.
The oracle takes minutes on the CPU for this, so the GPU parity test reads
the fixture instead of re-solving.

small_fixed_point.npz: the same for the 24x24x16x9x9x9 workload (seed 0,
6,718,464 cells, 27 controls, dt 0.05 s, max-norm stop 1e-4 s).  The oracle
needs ~22 s per sweep on 8 cores and several hundred sweeps, so this runs for
hours; with --checkpoint it saves V every 25 sweeps and resumes from the
last save.  The full table is 27 MB, so the fixture keeps:
  * the SHA-256 of the whole table's bytes (float32, row-major) and of each
    x slab -- the exact kernels must reproduce them bit for bit;
  * V, the argmin of one more sweep and, for cells whose best two
    lookaheads lie within 1e-3 s, that gap, on three whole x slabs (the
    target's, the farthest from it, and one between);
  * the sweep count and the last max-norm change.
"""
import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "peregrine-desktop_b200"))

from oracle import oracle as og  # noqa: E402
from peregrine_hjb.synth import Problem  # noqa: E402

GAP_KEEP = 1e-3  # s: gaps between the best two lookaheads stored per cell


def structs(pr):
    g = og.copy_struct(pr.grid.to_c(), og.OGrid)
    m = og.copy_struct(pr.model.to_c(), og.OModel)
    p = og.copy_struct(pr.params, og.OParams)
    return g, m, p


def tiny():
    pr = Problem("tiny", seed=5)
    g, m, p = structs(pr)
    t0 = time.time()
    V, it, ld, lm = og.solve_value(pr.occ, g, m, pr.seeds, pr.ctl, p, 3000, 1e-4, stop_rule=1,
                                   jacobi=True)
    _, _, mx, am = og.sweep_jacobi(V, pr.occ, g, m, pr.ctl, p, phase=it, argmin=True)
    np.savez_compressed(os.path.join(HERE, "tiny_fixed_point.npz"), V=V, iterations=it,
                        last_delta=ld, last_maxnorm=lm, argmin=am, workload="tiny", seed=5)
    print(f"tiny: {it} sweeps, {time.time() - t0:.0f} s, last max-norm {lm:.3g}")


def solve_checkpointed(pr, tol, iters, ckpt):
    """og_solve_value's Jacobi loop (max-norm stop), one oracle sweep at a
    time so that it can be saved and resumed."""
    g, m, p = structs(pr)
    V = np.full(pr.ncells, np.float32(pr.params.cap), np.float32)
    V[pr.seeds] = 0.0
    it0 = 0
    path = os.path.join(ckpt, "small_V.npy") if ckpt else None
    if path and os.path.exists(path):
        V = np.load(path)
        with open(os.path.join(ckpt, "small_it.txt")) as fh:
            it0, done = (int(x) for x in fh.read().split())
        if done:
            lm = float(np.load(os.path.join(ckpt, "small_lm.npy")))
            return V, it0, lm
    lm = np.inf
    t0 = time.time()
    for it in range(it0 + 1, iters + 1):
        V, tot, lm, _ = og.sweep_jacobi(V, pr.occ, g, m, pr.ctl, p, phase=it - 1)
        V[pr.seeds] = 0.0
        done = lm <= tol
        if path and (it % 25 == 0 or done):
            np.save(path + ".tmp.npy", V)
            os.replace(path + ".tmp.npy", path)
            np.save(os.path.join(ckpt, "small_lm.npy"), np.float64(lm))
            with open(os.path.join(ckpt, "small_it.txt"), "w") as fh:
                fh.write(f"{it} {int(done)}")
        print(f"sweep {it} delta {tot:.6g} maxnorm {lm:.6g} ({time.time() - t0:.0f} s)",
              flush=True)
        if done:
            return V, it, lm
    raise RuntimeError(f"no convergence in {iters} sweeps")


def small(ckpt):
    pr = Problem("small", seed=0)
    g, m, p = structs(pr)
    V, it, lm = solve_checkpointed(pr, 1e-4, 3000, ckpt)
    n = pr.grid.n
    slab = pr.ncells // n[0]
    sha = hashlib.sha256(V.tobytes()).hexdigest()
    slab_sha = np.array([hashlib.sha256(V[i * slab:(i + 1) * slab].tobytes()).hexdigest()
                         for i in range(n[0])])
    # the target's x slab, the farthest one, and one between
    tx = int(np.clip(round((pr.target[0] - pr.grid.lo[0]) / pr.grid.step[0]), 0, n[0] - 1))
    far = 0 if tx >= n[0] // 2 else n[0] - 1
    slabs = np.array(sorted({tx, (tx + far) // 2, far}), np.int32)
    cells = np.concatenate([np.arange(i * slab, (i + 1) * slab, dtype=np.int64) for i in slabs])
    _, _, _, am = og.sweep_jacobi(V, pr.occ, g, m, pr.ctl, p, phase=it, argmin=True)
    la = og.cell_lookaheads(V, pr.occ, g, m, pr.ctl, p, cells)
    two = np.sort(la, axis=1)[:, :2]
    gap = (two[:, 1].astype(np.float64) - two[:, 0]).astype(np.float32)
    near = np.nonzero(gap < GAP_KEEP)[0].astype(np.int32)
    np.savez_compressed(os.path.join(HERE, "small_fixed_point.npz"), workload="small", seed=0,
                        tol=1e-4, iterations=it, last_maxnorm=lm, sha256=sha, slab_sha256=slab_sha,
                        slabs=slabs, V=V[cells], argmin=am[cells], near=near, near_gap=gap[near],
                        gap_keep=GAP_KEEP)
    print(f"small: {it} sweeps, last max-norm {lm:.3g}, sha256 {sha}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("which", nargs="?", default="tiny", choices=["tiny", "small", "all"])
    ap.add_argument("--checkpoint", default=None,
                    help="directory for the small workload's resumable state")
    a = ap.parse_args()
    if a.checkpoint:
        os.makedirs(a.checkpoint, exist_ok=True)
    if a.which in ("tiny", "all"):
        tiny()
    if a.which in ("small", "all"):
        small(a.checkpoint)


if __name__ == "__main__":
    main()
