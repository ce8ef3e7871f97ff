"""The drop-in boundary on the device: the reference's hot-path self-tests
(`solve.py --self-test`, solver/solve.jl:30) and the bounded sweep wait
(PG_ETIMEOUT)."""
import numpy as np
import pytest

from conftest import gpu_available
from peregrine_hjb import _lib
from peregrine_hjb.synth import Problem

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def test_self_test_passes():
    from peregrine_hjb.selftest import self_test, _FAIL, _PASS
    assert self_test() == 0
    assert _FAIL[0] == 0 and _PASS[0] >= 40


def test_bounded_wait_returns_timeout_and_leaves_the_context_usable():
    """A sweep that outlasts the wait limit makes the solve return
    PG_ETIMEOUT; the sweep still completes, and the context then runs the
    same solve to the same table as a context with no limit."""
    pr = Problem("small", seed=0)
    opts = _lib.default_opts(stop_rule=_lib.STOP_MAXNORM, kernel=_lib.KERNEL_STENCIL)
    with _lib.Context(0) as ref:
        ref.load_problem(pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.ctl)
        ref.solve(pr.seeds, 20, 0.0, opts)
        want = ref.get_value()
    with _lib.Context(0) as ctx:
        ctx.load_problem(pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.ctl)
        # a sweep of 6.7M cells x 27 controls takes about a millisecond
        ctx.set_wait_timeout(1e-7)
        with pytest.raises(_lib.PeregrineError) as ei:
            ctx.solve(pr.seeds, 20, 0.0, opts)
        assert ei.value.code == _lib.PG_ETIMEOUT
        ctx.set_wait_timeout(60.0)
        ctx.solve(pr.seeds, 20, 0.0, opts)
        assert np.array_equal(ctx.get_value(), want)
    with pytest.raises(_lib.PeregrineError):
        with _lib.Context(0) as c2:
            c2.set_wait_timeout(-1.0)
