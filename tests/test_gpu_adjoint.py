"""The adjoint (dL/dtheta of a loss on the converged table, 18 model entries)
against an independent CPU FP64 reference and against central finite
differences of FP64 solves.  The loss is the mean table value over start
states at rest, as in the differentiation benchmark.

Tolerances: the GPU adjoint accumulates lambda in FP64 with atomic adds (in
an order that changes from sweep to sweep, so FP32 would leave a residual
floor near 1e-5 of |c|_1) and the 18 sums per block in FP32, so its gradient
carries ~1e-5 relative noise; the CPU reference (FP64, finite-
difference successor derivatives) agrees within 1e-4 of the largest entry.
Finite differences of full solves (relative step 1e-3) also see the
policy's switches between neighbouring controls; 1e-3 of the largest entry
plus 2 % of the entry bounds them (observed: < 5e-5 and < 2 %).
"""
import numpy as np
import pytest
import torch

from conftest import gpu_available
from peregrine_hjb import _lib
from peregrine_hjb import autograd as ag
from peregrine_hjb.synth import Problem

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

REF_TOL = 1e-4       # of max |g|, GPU adjoint vs CPU FP64 reference
FD_TOL_ABS = 1e-3    # of max |g|, GPU adjoint vs central differences
FD_TOL_REL = 2e-2    # of |g_fd|
FD_PARAMS = ("B22", "A11", "q2", "S22", "D11", "c0")


@pytest.fixture(scope="module")
def setup():
    pr = Problem("tiny", seed=5)
    spec = ag.SolveSpec.from_problem(pr, iters=6000, tol=1e-7)
    th0 = ag.theta_of(spec.model)
    states = ag.start_states(spec.grid, pr.occ, 512, seed=1)
    idx, w = ag.interp_weights(spec.grid, states)
    c = np.zeros(pr.ncells, np.float64)
    np.add.at(c, idx.ravel(), (w / len(states)).ravel())
    V, res, ctx = ag.solve(spec, th0, keep=True)
    try:
        g_gpu, ares = ctx.adjoint(c.astype(np.float32))
        _, _, pol = ctx.sweep(phase=0, kernel=_lib.KERNEL_STENCIL, argmin=True)
    finally:
        ctx.close()
    return dict(pr=pr, spec=spec, th0=th0, idx=idx, w=w, c=c, V=V, pol=pol, g=g_gpu, ares=ares)


def test_adjoint_converges(setup):
    ares = setup["ares"]
    assert ares.active_cells > 0
    assert ares.last_residual <= 1e-5 * ares.c_norm
    assert np.all(np.isfinite(setup["g"])) and np.max(np.abs(setup["g"])) > 0


def test_adjoint_matches_cpu_fp64_reference(og, setup):
    s = setup
    g_ = og.copy_struct(s["spec"].grid, og.OGrid)
    m_ = og.copy_struct(s["spec"].model, og.OModel)
    p_ = og.copy_struct(s["spec"].params, og.OParams)
    g_ref, _, nact = og.adjoint_grad_f64(s["V"].astype(np.float64), s["pol"], s["pr"].occ, g_, m_,
                                         s["pr"].ctl, p_, s["c"], iters=20000, tol=1e-9)
    assert abs(nact - s["ares"].active_cells) <= 0.001 * nact
    err = np.abs(s["g"] - g_ref) / np.max(np.abs(g_ref))
    assert err.max() <= REF_TOL, dict(zip(ag.THETA_NAMES, err))


def test_adjoint_matches_central_differences(setup):
    s = setup
    for name in FD_PARAMS:
        k = ag.THETA_NAMES.index(name)
        d = 1e-3 * max(abs(s["th0"][k]), 1e-2)
        vals = []
        for sign in (+1, -1):
            th = s["th0"].copy()
            th[k] += sign * d
            Vk, _, _ = ag.solve(s["spec"], th, storage="fp64")
            vals.append(float((Vk.astype(np.float64)[s["idx"]] * s["w"]).sum(1).mean()))
        fd = (vals[0] - vals[1]) / (2 * d)
        bound = FD_TOL_ABS * np.max(np.abs(s["g"])) + FD_TOL_REL * abs(fd)
        assert abs(s["g"][k] - fd) <= bound, (name, s["g"][k], fd)


def test_adjoint_on_more_cells_than_one_launch_wave(og):
    """24x24x8x9x9x9 = 3.4M cells: more than one pass of a capped grid, so
    every cell-parallel kernel of the adjoint must cover the whole table."""
    pr = Problem("tiny", seed=7, n=(24, 24, 8, 9, 9, 9))
    spec = ag.SolveSpec.from_problem(pr, iters=6000, tol=1e-6)
    th0 = ag.theta_of(spec.model)
    states = ag.start_states(spec.grid, pr.occ, 1024, seed=2)
    idx, w = ag.interp_weights(spec.grid, states)
    c = np.zeros(pr.ncells, np.float64)
    np.add.at(c, idx.ravel(), (w / len(states)).ravel())
    V, _, ctx = ag.solve(spec, th0, keep=True)
    try:
        g, ares = ctx.adjoint(c.astype(np.float32))
        _, _, pol = ctx.sweep(phase=0, kernel=_lib.KERNEL_STENCIL, argmin=True)
    finally:
        ctx.close()
    g_ = og.copy_struct(spec.grid, og.OGrid)
    m_ = og.copy_struct(spec.model, og.OModel)
    p_ = og.copy_struct(spec.params, og.OParams)
    g_ref, _, nact = og.adjoint_grad_f64(V.astype(np.float64), pol, pr.occ, g_, m_, pr.ctl, p_, c,
                                         iters=20000, tol=1e-9)
    assert abs(nact - ares.active_cells) <= 0.001 * nact
    err = np.abs(g - g_ref) / np.max(np.abs(g_ref))
    assert err.max() <= REF_TOL, dict(zip(ag.THETA_NAMES, err))


def test_adjoint_on_the_24x24x16x9x9x9_grid_with_125_controls(og):
    """The config-0 grid (6.7M cells) with the 125 controls of the benchmark
    ({-1, -0.5, 0, 0.5, 1}^3): the GPU adjoint against the CPU FP64 reference
    run on the same converged table and policy, within 1e-4 of max |g|."""
    pr = Problem("small", seed=0, control_set="cube5")
    spec = ag.SolveSpec.from_problem(pr, iters=6000, tol=1e-6)
    th0 = ag.theta_of(spec.model)
    states = ag.start_states(spec.grid, pr.occ, 4096, seed=3)
    idx, w = ag.interp_weights(spec.grid, states)
    c = np.zeros(pr.ncells, np.float64)
    np.add.at(c, idx.ravel(), (w / len(states)).ravel())
    V, _, ctx = ag.solve(spec, th0, keep=True)
    try:
        g, ares = ctx.adjoint(c.astype(np.float32))
        _, _, pol = ctx.sweep(phase=0, kernel=_lib.KERNEL_STENCIL, argmin=True)
    finally:
        ctx.close()
    g_ = og.copy_struct(spec.grid, og.OGrid)
    m_ = og.copy_struct(spec.model, og.OModel)
    p_ = og.copy_struct(spec.params, og.OParams)
    g_ref, _, nact = og.adjoint_grad_f64(V.astype(np.float64), pol, pr.occ, g_, m_, pr.ctl, p_, c,
                                         iters=20000, tol=1e-9)
    assert abs(nact - ares.active_cells) <= 0.001 * nact
    err = np.abs(g - g_ref) / np.max(np.abs(g_ref))
    assert err.max() <= REF_TOL, dict(zip(ag.THETA_NAMES, err))


def test_autograd_function_matches_the_direct_call(setup):
    s = setup
    theta = torch.tensor(s["th0"], requires_grad=True)
    V = ag.ValueTable.apply(theta, s["spec"])
    loss = ag.start_state_loss(V, s["idx"], s["w"])
    loss.backward()
    g = theta.grad.numpy()
    assert np.allclose(g, s["g"], rtol=1e-4, atol=1e-6 * np.max(np.abs(s["g"])))
    assert abs(float(loss) - float((s["V"][s["idx"]] * s["w"]).sum(1).mean())) < 1e-5
