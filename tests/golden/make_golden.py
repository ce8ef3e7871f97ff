"""Generate the committed golden fixtures from the CPU oracle.

    python tests/golden/make_golden.py

tiny_fixed_point.npz: the oracle's Jacobi solve of the 12x12x8x5x5x5
synthetic workload (seed 5, 27 controls, max-norm stop 1e-4 s) -- V at the
fixed point, the sweep count, and the argmin control of one more sweep.
The oracle takes minutes on the CPU for this, so the GPU parity test reads
the fixture instead of re-solving.
"""
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


def main():
    pr = Problem("tiny", seed=5)
    g = og.copy_struct(pr.grid.to_c(), og.OGrid)
    m = og.copy_struct(pr.model.to_c(), og.OModel)
    p = og.copy_struct(pr.params, og.OParams)
    t0 = time.time()
    V, it, ld, lm = og.solve_value(pr.occ, g, m, pr.seeds, pr.ctl, p, 3000, 1e-4, stop_rule=1,
                                   jacobi=True)
    _, _, mx, am = og.sweep_jacobi(V, pr.occ, g, m, pr.ctl, p, phase=it, argmin=True)
    np.savez_compressed(os.path.join(HERE, "tiny_fixed_point.npz"), V=V, iterations=it,
                        last_delta=ld, last_maxnorm=lm, argmin=am, workload="tiny", seed=5)
    print(f"tiny: {it} sweeps, {time.time() - t0:.0f} s, last max-norm {lm:.3g}")


if __name__ == "__main__":
    main()
