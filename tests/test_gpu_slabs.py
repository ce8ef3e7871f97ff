"""One table split into x slabs (pg_load_slab, peregrine_hjb/slabs.py) on the
device: the slabs of several contexts on one GPU are swept one after another
and exchange halos in process (their kernels never wait on each other), and
the gathered table equals the whole-table solve bit for bit -- the path a
table split over several GPUs takes, with NCCL doing the exchange."""
import numpy as np
import pytest

from conftest import gpu_available
from peregrine_hjb import _lib
from peregrine_hjb import slabs as S
from peregrine_hjb.synth import Problem

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

N = (40, 24, 8, 5, 5, 5)
SWEEPS = 12


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("exact", [False, True])
def test_slabs_reproduce_the_whole_table(world, exact):
    pr = Problem("tiny", seed=3, n=N)
    g, m = pr.grid.to_c(), pr.model.to_c()
    kernel = _lib.KERNEL_STENCIL_EXACT if exact else _lib.KERNEL_STENCIL_ROWS
    opts = _lib.default_opts(stop_rule=_lib.STOP_MAXNORM, kernel=kernel)
    want, res = _lib.solve_value(g, m, pr.params, pr.occ, pr.seeds, pr.ctl, SWEEPS, 0.0, opts)
    halo = _lib.reach_rows(g, m, pr.params, pr.ctl) + 2
    plan = S.plan_slabs(N[0], world, halo)
    sw = [S.DeviceSlab(g, m, pr.params, pr.occ, pr.ctl, pr.seeds, s, exact=exact) for s in plan]
    try:
        for it in range(SWEEPS):
            mx = max(w.sweep(it)[1] for w in sw)
            S.exchange_in_process(plan, sw)
        got = np.concatenate([w.interior() for w in sw])
    finally:
        for w in sw:
            w.close()
    assert np.array_equal(got, want), f"max |dV| {np.max(np.abs(got - want))}"
    assert mx == res.last_maxnorm


def test_slab_refuses_the_cell_form_sweep():
    pr = Problem("tiny", seed=3, n=N)
    with _lib.Context(0) as ctx:
        ctx.load_slab(pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.ctl, 0, 20, 3)
        with pytest.raises(_lib.PeregrineError):
            ctx.sweep(kernel=_lib.KERNEL_CELLFORM)
