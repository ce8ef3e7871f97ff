"""Batched solves: many independent tables swept together in one persistent
launch per sweep (optionally a CUDA graph) give each table exactly what its
own solve gives with the same number of sweeps; 16-bit storage with the FP32
polish lands within the storage tolerance of the FP32 batch."""
import numpy as np
import pytest

from conftest import gpu_available
from peregrine_hjb import _lib
from peregrine_hjb import batch as pb

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


@pytest.fixture(scope="module")
def problems():
    return pb.batch_problems(4, seed=3, control_set="cube3", dt=0.05, xy=(12, 16, 24),
                             heading=(8,), vel=(5, 7))


@pytest.mark.parametrize("graph", [True, False])
def test_batch_matches_individual_solves(problems, graph):
    res, Vs, info = pb.solve_batch(problems, storage="fp32", iters=3000, tol=1e-4, graph=graph)
    assert res.tables == len(problems) and res.converged == len(problems)
    for pr, V, (sweeps, mx) in zip(problems, Vs, info):
        assert mx <= 1e-4
        with _lib.Context(0) as ctx:
            ctx.load_problem(pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.ctl, "fp32")
            ctx.solve(pr.seeds, sweeps, 0.0,
                      _lib.default_opts(stop_rule=_lib.STOP_MAXNORM, kernel=_lib.KERNEL_STENCIL))
            want = ctx.get_value()
        assert np.array_equal(V, want), f"max |dV| {np.max(np.abs(V - want))}"


@pytest.mark.parametrize("storage", ["fp16", "bf16", "q16"])
def test_batch_16bit_with_polish_matches_fp32(problems, storage):
    _, V32, _ = pb.solve_batch(problems, storage="fp32", iters=3000, tol=1e-5)
    res, V16, info = pb.solve_batch(problems, storage=storage, iters=3000, tol=1e-5,
                                    polish_sweeps=3000)
    assert res.polish_sweeps > 0 and res.converged == len(problems)
    for a, b in zip(V32, V16):
        assert np.max(np.abs(a.astype(np.float64) - b)) <= 5e-3


def test_autotune_picks_a_candidate(problems):
    tiles = pb.autotune(problems[:2], sweeps=2)
    for (n1, n2), r in tiles.items():
        assert r in pb.tile_candidates(n1, n2)
    res, _, _ = pb.solve_batch(problems, storage="fp16", iters=3000, tol=1e-4, tiles=tiles)
    assert res.converged == len(problems)
