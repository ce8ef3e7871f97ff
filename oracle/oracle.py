"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of liboracle.so, the CPU
restatement of the reference solver's hot path (pg_oracle.c).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use
this module; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"


class OGrid(C.Structure):
    _fields_ = [("n", C.c_int32 * 6), ("lo", C.c_float * 6), ("step", C.c_float * 6)]


class OModel(C.Structure):
    _fields_ = [("B", C.c_float * 9), ("A", C.c_float * 9), ("q", C.c_float * 3),
                ("S", C.c_float * 9), ("D", C.c_float * 9), ("c", C.c_float * 3),
                ("eps", C.c_float * 3), ("knee", C.c_float)]


class OParams(C.Structure):
    _fields_ = [("dt", C.c_float), ("nsub", C.c_int32), ("checks", C.c_int32),
                ("adaptive_checks", C.c_int32), ("nearest", C.c_int32), ("cap", C.c_float),
                ("ntau", C.c_int32), ("tau_ratio", C.c_float), ("cfl", C.c_float),
                ("tau_min", C.c_float), ("tau_max", C.c_float), ("hmax", C.c_float),
                ("ncoarse", C.c_int32), ("rounds", C.c_int32), ("delta0", C.c_float),
                ("rk2", C.c_int32), ("vclamp", C.c_int32), ("simplex", C.c_int32)]


class OState(C.Structure):
    _fields_ = [(k, C.c_float) for k in ("x", "y", "h", "vx", "vy", "w")]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    L = C.CDLL(str(LIB))
    vp, i32, i64, f32, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_float, C.c_double
    P = C.POINTER
    L.og_grid_make.argtypes = [P(OGrid), vp, vp, vp]
    L.og_traction_gain.restype = f32
    L.og_traction_gain.argtypes = [f32, f32, f32, f32]
    L.og_body_accel.argtypes = [P(OModel), f32, f32, f32, f32, f32, f32, vp]
    L.og_step_state.restype = OState
    L.og_step_state.argtypes = [P(OModel), OState, f32, f32, f32, f32, i32]
    L.og_step_state_rk2.restype = OState
    L.og_step_state_rk2.argtypes = [P(OModel), OState, f32, f32, f32, f32, i32]
    L.og_control_set.restype = C.c_int
    L.og_control_set.argtypes = [C.c_int, vp, C.c_int]
    L.og_interp.restype = f32
    L.og_interp.argtypes = [vp, P(OGrid), OState, C.c_int, f32, C.c_int]
    L.og_interp_kuhn.restype = f32
    L.og_interp_kuhn.argtypes = [vp, P(OGrid), OState, f32, C.c_int, vp]
    L.og_cell_update.restype = f32
    L.og_cell_update.argtypes = [i64, vp, vp, vp, P(OGrid), P(OModel), vp, i32, P(OParams), i32,
                                 C.c_int, vp]
    L.og_sweep_jacobi.argtypes = [vp, vp, vp, vp, P(OGrid), P(OModel), vp, i32, P(OParams), i32,
                                  i64, i64, C.c_int, P(f64), P(f64), vp]
    L.og_sweep_inplace.restype = f64
    L.og_sweep_inplace.argtypes = [vp, vp, vp, P(OGrid), P(OModel), vp, i32, P(OParams), i32,
                                   C.c_int]
    L.og_sweep_jacobi_slab.argtypes = [vp, vp, vp, P(OGrid), P(OModel), vp, i32, P(OParams), i32,
                                       i64, i64, C.c_int, P(f64), P(f64)]
    L.og_cell_lookaheads.argtypes = [vp, vp, P(OGrid), P(OModel), vp, i32, P(OParams), vp, i64,
                                     C.c_int, vp]
    L.og_sweep_escape_jacobi.argtypes = [vp, vp, vp, P(OGrid), P(OModel), vp, i32, P(OParams),
                                         i32, C.c_int, P(f64)]
    L.og_solve_value.restype = C.c_int
    L.og_solve_value.argtypes = [vp, vp, vp, P(OGrid), P(OModel), vp, i64, vp, i32, P(OParams),
                                 i32, f64, C.c_int, C.c_int, C.c_int, P(f64), P(f64)]
    L.og_target_cells.restype = i64
    L.og_target_cells.argtypes = [P(OGrid), vp, vp, vp, i64]
    L.og_encode.restype = C.c_int
    L.og_encode.argtypes = [vp, i64, C.c_int, f64, f32, f64, vp, P(i64), P(i64)]
    L.og_build_occupancy.argtypes = [P(OGrid), C.c_int, vp, vp, f64, C.c_int, vp, C.c_int, f64,
                                     vp, f64, vp]
    L.og_adjoint_grad_f64.restype = C.c_int
    L.og_adjoint_grad_f64.argtypes = [vp, vp, vp, P(OGrid), P(OModel), vp, i32, P(OParams), vp, i32,
                                      f64, C.c_int, vp, P(i32), P(i64)]
    _lib = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def grid(n, lo, step) -> OGrid:
    g = OGrid()
    for k in range(6):
        g.n[k] = int(n[k])
        g.lo[k] = float(lo[k])
        g.step[k] = float(step[k])
    return g


def grid_make(n, lo, hi) -> OGrid:
    g = OGrid()
    lib().og_grid_make(C.byref(g), _p(np.asarray(n, np.int32)), _p(np.asarray(lo, np.float64)),
                       _p(np.asarray(hi, np.float64)))
    return g


def model(B, A, q, S, D, c, eps, knee) -> OModel:
    m = OModel()
    for name, v in (("B", B), ("A", A), ("S", S), ("D", D)):
        arr = np.asarray(v, np.float32).reshape(-1)
        for i in range(9):
            getattr(m, name)[i] = float(arr[i])
    for name, v in (("q", q), ("c", c), ("eps", eps)):
        arr = np.asarray(v, np.float32).reshape(-1)
        for i in range(3):
            getattr(m, name)[i] = float(arr[i])
    m.knee = float(np.float32(knee))
    return m


def params(**kw) -> OParams:
    """Defaults of Params() (PeregrineSolver.jl:918-927)."""
    d = dict(dt=0.05, nsub=4, checks=3, adaptive_checks=1, nearest=0, cap=60.0, ntau=1,
             tau_ratio=2.0, cfl=0.0, tau_min=0.004, tau_max=0.5, hmax=0.0125, ncoarse=0,
             rounds=0, delta0=0.35, rk2=1, vclamp=0, simplex=1)
    d.update(kw)
    p = OParams()
    for k, v in d.items():
        setattr(p, k, float(v) if isinstance(getattr(p, k), float) else int(v))
    return p


def copy_struct(src, dst_type):
    dst = dst_type()
    C.memmove(C.byref(dst), C.byref(src), C.sizeof(dst_type))
    return dst


def state(x, y, h, vx, vy, w) -> OState:
    return OState(x, y, h, vx, vy, w)


def control_set(level: int) -> np.ndarray:
    out = np.zeros(3 * (1 + 8 * (level + 1) * (level + 2) // 2), np.float32)
    n = lib().og_control_set(level, _p(out), out.size // 3)
    return out[: 3 * n].copy().reshape(3, n).reshape(-1)


def sweep_jacobi(V, occ, g, m, ctl, p, phase=0, lo=0, hi=None, threads=0, argmin=False,
                 pol=None):
    V = np.ascontiguousarray(V, np.float32)
    occ = np.ascontiguousarray(occ, np.uint8)
    ctl = np.ascontiguousarray(ctl, np.float32)
    n = V.size
    hi = n if hi is None else hi
    out = V.copy()
    tot = C.c_double()
    mx = C.c_double()
    am = np.full(n, -2, np.int16) if argmin else None
    lib().og_sweep_jacobi(_p(V), _p(out), _p(occ), _p(pol), C.byref(g), C.byref(m), _p(ctl),
                          ctl.size // 3, C.byref(p), phase, lo, hi, threads, C.byref(tot),
                          C.byref(mx), _p(am))
    return out, tot.value, mx.value, am


def sweep_jacobi_slab(V, occ, g, m, ctl, p, lo, hi, phase=0, threads=0):
    """One Jacobi sweep of the cells [lo, hi) only: returns (V' on the slab,
    L1 total, max-norm); V is the whole table it reads from."""
    V = np.ascontiguousarray(V, np.float32)
    ctl = np.ascontiguousarray(ctl, np.float32)
    out = np.empty(hi - lo, np.float32)
    tot = C.c_double()
    mx = C.c_double()
    lib().og_sweep_jacobi_slab(_p(V), _p(out), _p(np.ascontiguousarray(occ, np.uint8)), C.byref(g),
                               C.byref(m), _p(ctl), ctl.size // 3, C.byref(p), phase, lo, hi,
                               threads, C.byref(tot), C.byref(mx))
    return out, tot.value, mx.value


def cell_lookaheads(V, occ, g, m, ctl, p, cells, threads=0):
    """Every control's lookahead value for the listed cells, [len(cells), nctl]."""
    V = np.ascontiguousarray(V, np.float32)
    ctl = np.ascontiguousarray(ctl, np.float32)
    cells = np.ascontiguousarray(cells, np.int64)
    nctl = ctl.size // 3
    out = np.empty((cells.size, nctl), np.float32)
    lib().og_cell_lookaheads(_p(V), _p(np.ascontiguousarray(occ, np.uint8)), C.byref(g),
                             C.byref(m), _p(ctl), nctl, C.byref(p), _p(cells), cells.size,
                             threads, _p(out))
    return out


def sweep_escape_jacobi(V, occ, g, m, ctl, p, phase=0, threads=0):
    V = np.ascontiguousarray(V, np.float32)
    out = V.copy()
    tot = C.c_double()
    lib().og_sweep_escape_jacobi(_p(V), _p(out), _p(np.ascontiguousarray(occ, np.uint8)),
                                 C.byref(g), C.byref(m), _p(np.ascontiguousarray(ctl, np.float32)),
                                 ctl.size // 3, C.byref(p), phase, threads, C.byref(tot))
    return out, tot.value


def sweep_inplace(V, occ, g, m, ctl, p, phase=0, rev=False, pol=None):
    V = np.ascontiguousarray(V, np.float32).copy()
    d = lib().og_sweep_inplace(_p(V), _p(np.ascontiguousarray(occ, np.uint8)), _p(pol), C.byref(g),
                               C.byref(m), _p(np.ascontiguousarray(ctl, np.float32)),
                               ctl.size // 3, C.byref(p), phase, int(rev))
    return V, d


def solve_value(occ, g, m, tidx, ctl, p, iters, tol, stop_rule=0, jacobi=True, threads=0,
                warm=False):
    n = 1
    for k in range(6):
        n *= g.n[k]
    V = np.empty(n, np.float32)
    pol = np.zeros(3 * n, np.int8) if warm else None
    tidx = np.ascontiguousarray(tidx, np.int64)
    ld = C.c_double()
    lm = C.c_double()
    it = lib().og_solve_value(_p(V), _p(np.ascontiguousarray(occ, np.uint8)), _p(pol), C.byref(g),
                              C.byref(m), _p(tidx), tidx.size,
                              _p(np.ascontiguousarray(ctl, np.float32)), ctl.size // 3,
                              C.byref(p), iters, tol, stop_rule, int(jacobi), threads,
                              C.byref(ld), C.byref(lm))
    return V, it, ld.value, lm.value


def target_cells(g, s, tol) -> np.ndarray:
    out = np.zeros(1 << 16, np.int64)
    n = lib().og_target_cells(C.byref(g), _p(np.asarray(s, np.float32)),
                              _p(np.asarray(tol, np.float32)), _p(out), out.size)
    if n < 0:
        raise ValueError("too many target cells for the oracle buffer")
    return out[:n].copy()


def encode(V, dtype, scale, cap, escape_scale=0.0):
    V = np.ascontiguousarray(V, np.float32)
    code = {"u8": 0, "u16": 1, "f16": 2, "f32": 3}[dtype]
    eb = {"u8": 1, "u16": 2, "f16": 2, "f32": 4}[dtype]
    out = np.zeros(V.size * eb, np.uint8)
    r = C.c_int64()
    e = C.c_int64()
    lib().og_encode(_p(V), V.size, code, scale, cap, escape_scale, _p(out), C.byref(r), C.byref(e))
    return out, r.value, e.value


def build_occupancy(g, polys, margin, robot=None, substeps=3, clearance=0.0, bounds=None,
                    wall_clearance=None):
    if wall_clearance is None:
        wall_clearance = clearance
    nverts = np.array([len(P) for P in polys] or [0], np.int32)
    pts = np.array([v for P in polys for v in P] or [[0.0, 0.0]], np.float64).reshape(-1)
    rb = None if robot is None else np.asarray(robot, np.float64).reshape(-1)
    bd = None if bounds is None else np.asarray(bounds, np.float64)
    out = np.zeros(g.n[0] * g.n[1] * g.n[2], np.uint8)
    lib().og_build_occupancy(C.byref(g), len(polys), _p(nverts), _p(pts), float(margin),
                             0 if robot is None else len(robot), _p(rb), int(substeps),
                             float(clearance), _p(bd), float(wall_clearance), _p(out))
    return out


def adjoint_grad_f64(V, pol, occ, g, m, ctl, p, c, iters=20000, tol=1e-10, threads=0):
    """FP64 reference gradient dL/dtheta (18) of a loss with dL/dV = c on the
    converged table V (row-major) with policy pol; returns (grad, sweeps,
    active cells)."""
    V = np.ascontiguousarray(V, dtype=np.float64)
    pol = np.ascontiguousarray(pol, dtype=np.int16)
    occ = np.ascontiguousarray(occ, dtype=np.uint8)
    ctl = np.ascontiguousarray(ctl, dtype=np.float32)
    c = np.ascontiguousarray(c, dtype=np.float64)
    grad = np.zeros(18, dtype=np.float64)
    it, na = C.c_int32(), C.c_int64()
    rc = lib().og_adjoint_grad_f64(_p(V), _p(pol), _p(occ), C.byref(g), C.byref(m), _p(ctl),
                                   int(ctl.size // 3), C.byref(p), _p(c), int(iters), float(tol),
                                   int(threads), _p(grad), C.byref(it), C.byref(na))
    if rc != 0:
        raise MemoryError("og_adjoint_grad_f64 ran out of memory")
    return grad, it.value, na.value


def available_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
