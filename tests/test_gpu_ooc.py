"""The out-of-core driver (pg_solve_ooc) against the in-core solve, on grids
that fit: the reference's SelfTest [10] (tiled vs in-core, and a starved halo
as the control that must come out worse, solver/src/SelfTest.jl:684-851) and
its halo refusal (solver/src/Run.jl:1688-1691)."""
import numpy as np
import pytest

from conftest import gpu_available
from peregrine_hjb import _lib
from peregrine_hjb.synth import Problem

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

N = (40, 24, 8, 5, 5, 5)  # 40 x rows: five 8-row tiles


@pytest.fixture(scope="module")
def pr():
    return Problem("tiny", seed=3, n=N)


def in_core(pr, sweeps, kernel, tol=0.0):
    opts = _lib.default_opts(stop_rule=_lib.STOP_MAXNORM, kernel=kernel)
    return _lib.solve_value(pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.seeds,
                            pr.ctl, sweeps, tol, opts)


def ooc(pr, rounds, tol=0.0, **kw):
    o = _lib.ooc_opts(**kw)
    return _lib.solve_ooc(pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.seeds, pr.ctl,
                          rounds, tol, o)


@pytest.mark.parametrize("kernel", [_lib.KERNEL_STENCIL_ROWS, _lib.KERNEL_STENCIL_EXACT])
def test_tiled_jacobi_round_is_the_whole_table_sweep(pr, kernel):
    """Jacobi tiles, one sweep per residency, a full halo: every round is
    one whole-table sweep, bit for bit, and the last round's max-norm is the
    whole-table sweep's."""
    Vi, ri = in_core(pr, 12, kernel)
    Vo, ro = ooc(pr, 12, tile_rows=8, tile_sweeps=1, jacobi=1, kernel=kernel)
    assert ro.tiles_per_round == 5 and ro.rounds == 12
    assert ro.halo_rows >= ro.reach_rows + 2
    assert np.array_equal(Vo, Vi), f"max |dV| {np.max(np.abs(Vo - Vi))}"
    assert ro.last_maxnorm == ri.last_maxnorm


def test_halo_below_the_reach_is_refused(pr):
    with pytest.raises(_lib.PeregrineError) as ei:
        ooc(pr, 2, tile_rows=8, halo_rows=1, jacobi=1)
    assert ei.value.code == _lib.PG_EINVAL and "halo" in str(ei.value)


def test_starved_halo_is_worse():
    """The control of SelfTest [10]: on 4.6 cm rows one backup reaches two
    rows, so with a one-row halo the tiles read rows that were never loaded
    and the table comes out different from the in-core one, where a full
    halo matches it exactly."""
    pr = Problem("tiny", seed=3, n=(80, 24, 8, 5, 5, 5))
    Vi, _ = in_core(pr, 80, _lib.KERNEL_STENCIL_ROWS)
    Vs, rs = ooc(pr, 80, tile_rows=16, halo_rows=1, allow_starved_halo=1, tile_sweeps=1, jacobi=1)
    Vf, _ = ooc(pr, 80, tile_rows=16, tile_sweeps=1, jacobi=1)
    assert rs.reach_rows >= 2
    assert np.array_equal(Vf, Vi)
    assert np.max(np.abs(Vs.astype(np.float64) - Vi)) > 1e-3


def test_in_place_tiles_reach_the_same_fixed_point(pr):
    """The reference's store: tiles written back in place, four sweeps per
    residency.  A different iteration order of the same monotone update, so
    it settles on the in-core fixed point (both stop when no cell moves by
    more than 1e-7 s)."""
    Vi, ri = in_core(pr, 5000, _lib.KERNEL_STENCIL_ROWS, tol=1e-7)
    Vo, ro = ooc(pr, 5000, tol=1e-7, tile_rows=8, tile_sweeps=4, jacobi=0)
    assert ro.rounds < ri.iterations
    assert np.max(np.abs(Vo.astype(np.float64) - Vi)) <= 1e-5


def test_fp16_store(pr):
    """FP16 in the host store: the tiles sweep in FP32 arithmetic from FP16
    values and round back, as the in-core FP16 storage does."""
    Vi, _ = in_core(pr, 6, _lib.KERNEL_STENCIL_ROWS)
    Vh, ro = ooc(pr, 6, tile_rows=8, tile_sweeps=1, jacobi=1, storage="fp16")
    assert Vh.dtype == np.float16 and ro.h2d_bytes > 0
    assert np.max(np.abs(Vh.astype(np.float64) - Vi)) <= 0.05
