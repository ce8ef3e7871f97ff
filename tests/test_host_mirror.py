"""Host-side mirrors of the reference (grid, control tables, seeds,
occupancy, params) against the oracle, and the C ABI's exports.  No GPU."""
import math
import os
import re
import subprocess

import numpy as np
import pytest

from peregrine_hjb import grid as pgrid
from peregrine_hjb import params as pparams
from peregrine_hjb import seeds as pseeds
from peregrine_hjb.geometry import build_occupancy

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
f32 = np.float32


def to_og(og, g):
    return og.grid(g.n, [float(v) for v in g.lo], [float(v) for v in g.step])


def test_grid_make_matches_oracle(og):
    for n, lo, hi in [((24, 24, 16, 9, 9, 9), (0, 0, -math.pi, -150, -150, -6), (365.8, 365.8, math.pi, 150, 150, 6)),
                      ((46, 46, 24, 13, 13, 13), (23, 23, -math.pi, -170, -170, -8), (343, 343, math.pi, 170, 170, 8))]:
        g = pgrid.Grid6.make(n, lo, hi)
        o = og.grid_make(n, lo, hi)
        for k in range(6):
            assert np.float32(o.lo[k]) == g.lo[k]
            assert np.float32(o.step[k]) == g.step[k]


@pytest.mark.parametrize("level", [1, 2, 3, 4, 6])
def test_control_set_matches_oracle(og, level):
    a = pparams.control_set(level)
    b = og.control_set(level)
    assert a.dtype == np.float32 and np.array_equal(a, b)


def test_cube_sets():
    c3 = pparams.cube_set([-1, 0, 1]).reshape(3, -1).T
    c5 = pparams.cube_set([-1, -0.5, 0, 0.5, 1]).reshape(3, -1).T
    assert len(c3) == 27 and len(c5) == 125
    assert np.all(c3[0] == 0) and np.all(c5[0] == 0)
    l1 = np.abs(c5).sum(axis=1)
    assert np.all(np.diff(l1) >= -1e-6)


def test_substeps_default_is_five():
    """dt/4 is an exact power-of-two division, so tau/hmax is exactly 4 and
    substeps_for gives 5 (PeregrineSolver.jl:985-989, Run.jl:260)."""
    for dt in (0.05, 0.04, 0.03):
        g = pgrid.Grid6.make((4, 4, 4, 3, 3, 3), (0, 0, 0, -1, -1, -1), (1, 1, 1, 1, 1, 1))
        sp = pparams.solver_params({"dt": dt}, g)
        tau = f32(dt)
        hmax = f32(sp.p.hmax)
        k = int(min(f32(tau / hmax), f32(1e4))) + 1
        assert k == 5


def test_target_cells_match_oracle(og):
    rng = np.random.default_rng(3)
    g = pgrid.Grid6.make((20, 18, 12, 7, 7, 7), (0, 0, -math.pi, -150, -150, -6), (300, 280, math.pi, 150, 150, 6))
    o = to_og(og, g)
    for _ in range(40):
        s = (rng.uniform(-10, 310), rng.uniform(-10, 290), rng.uniform(-7, 7),
             rng.uniform(-160, 160), rng.uniform(-160, 160), rng.uniform(-7, 7))
        tol = tuple(f32(g.step[k] * f32(rng.uniform(0.2, 1.6))) for k in range(6))
        a = pseeds.target_cells(g, [f32(v) for v in s], tol)
        b = og.target_cells(o, [f32(v) for v in s], tol)
        assert list(a) == list(b)


def _rects(rng, k, field=365.8):
    out = []
    for _ in range(k):
        w, h = rng.uniform(20, 60, 2)
        x0, y0 = rng.uniform(0, field - w), rng.uniform(0, field - h)
        out.append([[x0, y0], [x0 + w, y0], [x0 + w, y0 + h], [x0, y0 + h]])
    return out


@pytest.mark.parametrize("robot", [None, [[-18, -18], [18, -18], [18, 18], [-18, 18]],
                                   [[-20, -10], [22, -12], [25, 15], [-5, 20], [-21, 5]]])
@pytest.mark.parametrize("clearance", [0.0, 5.0])
def test_occupancy_matches_oracle(og, robot, clearance):
    rng = np.random.default_rng(11)
    g = pgrid.Grid6.make((30, 28, 8, 3, 3, 3), (20, 25, -math.pi, -1, -1, -1), (345, 340, math.pi, 1, 1, 1))
    polys = _rects(rng, 4)
    polys.append([[150, 150], [200, 160], [170, 210], [180, 175]])  # concave
    bounds = (0.0, 0.0, 365.8, 365.8)
    a = build_occupancy(g, polys, 2.0, robot, 3, clearance, bounds=bounds, wall_clearance_cm=clearance)
    b = og.build_occupancy(to_og(og, g), polys, 2.0, robot, 3, clearance, bounds, clearance)
    if robot is not None and len(robot) >= 3:
        # the reference rotates the footprint with a BLAS matrix product whose
        # rounding is not pinned; allow a vanishing share of boundary cells
        assert np.mean(a != b) < 1e-3
    else:
        assert np.array_equal(a, b)


def test_solver_params_defaults():
    g = pgrid.Grid6.make((4, 4, 4, 3, 3, 3), (0, 0, 0, -1, -1, -1), (1, 1, 1, 1, 1, 1))
    sp = pparams.solver_params({}, g)
    p = sp.p
    assert abs(p.dt - 0.05) < 1e-8 and p.nsub == 4 and p.checks == 3 and p.adaptive_checks == 1
    assert p.cap == 60.0 and p.ntau == 5 and p.cfl == 2.0 and p.ncoarse == 8 and p.rounds == 2
    assert p.simplex == 1 and p.rk2 == 1 and p.vclamp == 0 and abs(p.tau_max - 0.5) < 1e-9
    assert sp.nctl == 67 and sp.warm and sp.iters == 400 and sp.tol == 1e-3


def test_storage_key_accepts_the_library_storages():
    g = pgrid.Grid6.make((4, 4, 4, 3, 3, 3), (0, 0, 0, -1, -1, -1), (1, 1, 1, 1, 1, 1))
    for name in ("fp32", "fp16", "bf16", "q16", "fp64"):
        assert pparams.solver_params({"storage": name}, g).storage == name
    import pytest
    with pytest.raises(ValueError):
        pparams.solver_params({"storage": "fp8"}, g)


def test_region_seeds_are_disk_and_slow():
    from peregrine_hjb.synth import Problem
    pr = Problem("small", seed=1)
    g = pr.grid
    i1, i2, i3, i4, i5, i6 = g.unflatten(pr.seeds)
    x = g.axisvalue(0, i1).astype(np.float64)
    y = g.axisvalue(1, i2).astype(np.float64)
    vx = g.axisvalue(3, i4).astype(np.float64)
    vy = g.axisvalue(4, i5).astype(np.float64)
    assert np.all((x - pr.target[0]) ** 2 + (y - pr.target[1]) ** 2 <= 100.0 + 1e-9)
    assert np.all(vx * vx + vy * vy < 400.0)
    assert len(set(i3.tolist())) == g.n[2] and len(set(i6.tolist())) == g.n[5]


def test_library_exports_every_declared_symbol():
    """libperegrine_hjb.so loads without a GPU and exports every entry point
    include/peregrine_hjb.h declares."""
    from peregrine_hjb import _lib
    hdr = open(os.path.join(ROOT, "include", "peregrine_hjb.h")).read()
    declared = set(re.findall(r"^\s*(?:int|int32_t|void|const char\*)\s+(pg_\w+)\s*\(", hdr, re.M))
    assert declared == set(_lib.EXPORTS)
    lib = _lib.load_library()
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (pg_\w+)$", out, re.M))
    assert declared <= exported
    assert lib.pg_abi_version() == 1


def test_library_refuses_bad_arguments_without_a_gpu():
    from peregrine_hjb import _lib
    lib = _lib.load_library()
    import ctypes as C
    assert lib.pg_destroy(None) == 0
    assert lib.pg_create(None, 0) == _lib.PG_EINVAL
    assert b"null" in lib.pg_last_error()
    # the adjoint binding converts its arguments and refuses a null context
    grad = np.zeros(18)
    res = _lib.AdjointResult()
    dl = np.zeros(4, dtype=np.float32)
    assert lib.pg_adjoint(None, dl.ctypes.data, 0, 10, 1e-6, grad.ctypes.data,
                          C.byref(res)) == _lib.PG_EINVAL


def test_binding_constants_match_the_header():
    """The ctypes binding's kernel and storage selectors are the header's."""
    from peregrine_hjb import _lib
    hdr = open(os.path.join(ROOT, "include", "peregrine_hjb.h")).read()
    defs = {k: int(v) for k, v in re.findall(r"^#define\s+(PG_(?:KERNEL|STORE)_\w+)\s+(-?\d+)", hdr, re.M)}
    for name, value in defs.items():
        if name.startswith("PG_KERNEL_"):
            assert getattr(_lib, "KERNEL_" + name[len("PG_KERNEL_"):]) == value, name
    assert _lib.STORE_Q16 == defs["PG_STORE_Q16"]
