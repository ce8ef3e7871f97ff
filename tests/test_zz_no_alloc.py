"""pg_sweep_noalloc, the sweep that allocates nothing, against pg_sweep.

pg_sweep_noalloc runs the cell-form sweep on buffers the caller owns, with
its block partials in a fixed array inside the library.  Two calls in a row
must give what pg_sweep gives with the cell-form kernel on the same state,
bit for bit (the same kernel and the same fixed-order reduction), including
the residuals; a call that changes nothing must report zero even though the
array still holds the previous call's partials.  This file sorts last so the
array has been through the other tests' processes' sweeps when it runs after
them; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import gpu_available
from peregrine_hjb import _lib
from peregrine_hjb.synth import Problem


def plane_major(V, n):
    """Row-major (x, y, h, vx, vy, w) to the plane-major device order."""
    return np.ascontiguousarray(V.reshape(n).transpose(2, 3, 4, 5, 0, 1)).ravel()


def row_major(V, n):
    """Plane-major (h, vx, vy, w, x, y) back to row-major."""
    nx, ny, nh, n4, n5, n6 = n
    return np.ascontiguousarray(V.reshape(nh, n4, n5, n6, nx, ny).transpose(4, 5, 0, 1, 2, 3)).ravel()


def test_refuses_grids_beyond_the_working_array():
    """Sizes beyond the fixed array are refused before any device work."""
    lib = _lib.load_library()
    pr_grid = _lib.Grid6()
    for k, (n, lo, st) in enumerate(zip((48, 48, 32, 15, 15, 15), (0, 0, -3, -2, -2, -3),
                                        (0.1, 0.1, 0.2, 0.3, 0.3, 0.4))):
        pr_grid.n[k], pr_grid.lo[k], pr_grid.step[k] = n, lo, st
    m, p = _lib.Model(), _lib.Params()
    p.dt, p.nsub, p.checks, p.cap = 0.04, 1, 1, 100.0
    d = C.c_double()
    fake = C.c_void_p(256)  # never dereferenced: the size check comes first
    rc = lib.pg_sweep_noalloc(C.byref(pr_grid), C.byref(m), C.byref(p), fake, fake, 27,
                              fake, C.c_void_p(512), 0, None, C.byref(d), None)
    assert rc == _lib.PG_EINVAL
    assert "8388608" in lib.pg_last_error().decode()


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")
def test_two_calls_match_pg_sweep():
    import torch

    pr = Problem("tiny", seed=5)
    n = tuple(pr.grid.n)
    g, m, p = pr.grid.to_c(), pr.model.to_c(), pr.params
    V0 = np.full(pr.ncells, np.float32(p.cap), np.float32)
    V0[pr.seeds] = 0.0

    # The existing entry point: three sweeps to give the table structure,
    # then the two sweeps to compare against.
    with _lib.Context(0) as ctx:
        ctx.load_problem(g, m, p, pr.occ, pr.ctl, "fp32")
        ctx.set_value(V0)
        for ph in range(3):
            ctx.sweep(phase=ph, kernel=_lib.KERNEL_CELLFORM)
        Vs = ctx.get_value()
        d1, dm1, _ = ctx.sweep(phase=3, kernel=_lib.KERNEL_CELLFORM)
        W1 = ctx.get_value()
        d2, dm2, _ = ctx.sweep(phase=4, kernel=_lib.KERNEL_CELLFORM)
        W2 = ctx.get_value()
    assert d1 > 0 and d2 > 0

    # The caller's own buffers, in the documented layouts.
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    occ_hxy = np.ascontiguousarray(pr.occ.reshape(n[0], n[1], n[2]).transpose(2, 0, 1)).ravel()
    occ_t = torch.from_numpy((occ_hxy != 0).astype(np.uint8)).to(dev)
    ctl_t = torch.from_numpy(np.ascontiguousarray(pr.ctl, np.float32)).to(dev)
    a = torch.from_numpy(plane_major(Vs, n)).to(dev)
    b = torch.empty_like(a)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream

    e1, em1 = _lib.sweep_noalloc(g, m, p, occ_t.data_ptr(), ctl_t.data_ptr(), pr.nctl,
                                 a.data_ptr(), b.data_ptr(), phase=3, stream=stream)
    got1 = row_major(b.cpu().numpy(), n)
    e2, em2 = _lib.sweep_noalloc(g, m, p, occ_t.data_ptr(), ctl_t.data_ptr(), pr.nctl,
                                 b.data_ptr(), a.data_ptr(), phase=4, stream=stream)
    got2 = row_major(a.cpu().numpy(), n)

    assert np.array_equal(got1, W1), f"first call: max |dV| {np.max(np.abs(got1 - W1))}"
    assert np.array_equal(got2, W2), f"second call: max |dV| {np.max(np.abs(got2 - W2))}"
    assert (e1, em1) == (d1, dm1)
    assert (e2, em2) == (d2, dm2)

    # A sweep that lowers nothing reports zero: the previous call's partials
    # and totals left in the array do not leak into it.
    z = torch.zeros_like(a)
    e3, em3 = _lib.sweep_noalloc(g, m, p, occ_t.data_ptr(), ctl_t.data_ptr(), pr.nctl,
                                 z.data_ptr(), b.data_ptr(), phase=0, stream=stream)
    assert (e3, em3) == (0.0, 0.0)
    assert torch.count_nonzero(b).item() == 0
