"""Solver knobs, control tables and input files.

Mirrors solver/src/Run.jl:203-294 (solver_params), PeregrineSolver.jl:318-346
(control_set), PeregrineSolver.jl:897-927 (Params defaults) and
Pipeline.jl:406-490 (load_model / load_field / load_targets).

Additive job-JSON keys (absent = the reference's behaviour):
  control_set   "octahedron" (default: the reference lattice at control_level),
                "cube3" = {-1,0,1}^3, "cube5" = {-1,-0.5,0,0.5,1}^3
  target_region {"kind": "disk", "radius_cm": r, "speed_max_cm_s": s}
  stop_rule     "l1_quiet" (default) | "maxnorm"
  storage       "fp32" (default) | "fp16" | "bf16" | "q16" (16-bit fixed point,
                2^-11 s steps, value_cap below 32 s) | "fp64"
  polish_sweeps FP32 sweeps allowed after a 16-bit solve converges (64)
  sweep         "jacobi" (the only sweep order on the GPU)
"""
from __future__ import annotations

import json
import math
import tomllib
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .grid import getc

f32 = np.float32
TAU_REF = 0.5  # Advise.jl:19


def control_set(level: int) -> np.ndarray:
    """control_set(level) (PeregrineSolver.jl:318-346); planar [u1|u2|u3]."""
    if level < 1:
        raise ValueError("control level must be >= 1")
    out = [(f32(0), f32(0), f32(0))]
    seen = {out[0]}
    L = f32(level)
    for sd in (-1, 1):
        for ss in (-1, 1):
            for st in (-1, 1):
                for i in range(level + 1):
                    for j in range(level - i + 1):
                        k = level - i - j
                        a, b, c = f32(i) / L, f32(j) / L, f32(k) / L
                        p = (f32(0) if a == 0 else f32(sd) * a,
                             f32(0) if b == 0 else f32(ss) * b,
                             f32(0) if c == 0 else f32(st) * c)
                        if p not in seen:
                            seen.add(p)
                            out.append(p)
    return _planar(_effort_sorted(out))


def _effort_sorted(pts):
    def key(p):
        l1 = f32(f32(abs(p[0]) + abs(p[1])) + abs(p[2]))
        l2 = f32(f32(p[0] * p[0] + p[1] * p[1]) + p[2] * p[2])
        return (float(l1), float(l2))
    return sorted(pts, key=key)  # stable, like Julia's default sort!


def _planar(pts) -> np.ndarray:
    a = np.array(pts, dtype=np.float32).reshape(-1, 3)
    return np.ascontiguousarray(a.T.reshape(-1))


def cube_set(values) -> np.ndarray:
    """{values}^3, coast first then increasing (L1, L2) effort with the
    reference's tie order (its generation order, stable)."""
    vals = [f32(v) for v in values]
    pts = [(a, b, c) for a in vals for b in vals for c in vals]
    return _planar(_effort_sorted(pts))


def control_table(cfg) -> tuple[np.ndarray, int, str]:
    kind = str(getc(cfg, "control_set", "octahedron")).lower()
    level = int(getc(cfg, "control_level", 4))
    if kind in ("octahedron", "lattice"):
        ctl = control_set(level)
    elif kind == "cube3":
        ctl = cube_set([-1, 0, 1])
    elif kind == "cube5":
        ctl = cube_set([-1, -0.5, 0, 0.5, 1])
    else:
        raise ValueError(f"unknown control_set '{kind}' (octahedron, cube3 or cube5)")
    return ctl, level, kind


@dataclass
class SolverParams:
    """What solver_params returns (Run.jl:287-293), plus the additive keys."""
    p: _lib.Params
    level: int
    control_kind: str
    ctl: np.ndarray
    nctl: int
    warm: bool
    iters: int
    tol: float
    cap: float
    ttol: tuple
    margin: float
    clearance: float
    stop_rule: int
    storage: str
    polish_sweeps: int
    raw: dict = field(default_factory=dict)


def solver_params(cfg, g) -> SolverParams:
    """solver_params (Run.jl:203-294)."""
    dt = f32(getc(cfg, "dt", 0.05))
    nsub = int(getc(cfg, "substeps", 4))
    checks = int(getc(cfg, "sweep_checks", 3))
    nearest = bool(getc(cfg, "nearest", False))
    iters = int(getc(cfg, "iterations", 400))
    tol = float(getc(cfg, "tolerance", 1e-3))
    margin = float(getc(cfg, "margin_cm", 0.0))
    clearance = float(getc(cfg, "clearance_cm", 5.0))
    tt = getc(cfg, "target_tol", None)
    ttol = tuple(f32(v) for v in tt) if tt is not None else tuple(
        f32(g.step[k] * f32(0.5)) for k in range(6))
    cap = f32(getc(cfg, "value_cap", 60.0))
    scan = int(getc(cfg, "control_scan", 8))
    rounds = int(getc(cfg, "refine_rounds", 2))
    delta0 = float(getc(cfg, "refine_delta", 0.35))
    warm = bool(getc(cfg, "warm_start", True))
    ntau = int(getc(cfg, "tau_levels", 5))
    tau_ratio = float(getc(cfg, "tau_ratio", 2.0))
    cfl = float(getc(cfg, "cfl", 2.0))
    tau_min = float(getc(cfg, "tau_min", 0.004))
    tm = getc(cfg, "tau_max", TAU_REF)
    tau_max = float(tm) if isinstance(tm, (int, float)) and not isinstance(tm, bool) else TAU_REF
    # dt/max(nsub,1) is a Float32 division in the reference (dt is Float32)
    hmax = float(getc(cfg, "substep_max", float(dt / f32(max(nsub, 1)))))
    achecks = bool(getc(cfg, "adaptive_checks", True))
    rk2 = bool(getc(cfg, "rk2", True))
    vclamp = bool(getc(cfg, "velocity_clamp", False))
    simplex = bool(getc(cfg, "simplex", True))

    p = _lib.Params()
    p.dt = float(dt); p.nsub = nsub; p.checks = checks; p.adaptive_checks = int(achecks)
    p.nearest = int(nearest); p.cap = float(cap); p.ntau = ntau; p.tau_ratio = tau_ratio
    p.cfl = cfl; p.tau_min = tau_min; p.tau_max = tau_max; p.hmax = hmax
    p.ncoarse = scan; p.rounds = rounds; p.delta0 = delta0; p.rk2 = int(rk2)
    p.vclamp = int(vclamp); p.simplex = int(simplex)

    ctl, level, kind = control_table(cfg)
    stop = str(getc(cfg, "stop_rule", "l1_quiet")).lower()
    if stop not in ("l1_quiet", "maxnorm"):
        raise ValueError(f"unknown stop_rule '{stop}'")
    storage = str(getc(cfg, "storage", "fp32")).lower()
    if storage not in _lib.STORAGES:
        raise ValueError(f"unknown storage '{storage}'")
    sweep = str(getc(cfg, "sweep", "jacobi")).lower()
    if sweep != "jacobi":
        raise ValueError("only the Jacobi sweep order is implemented on the GPU")
    raw = dict(dt=float(dt), nsub=nsub, checks=checks, nearest=nearest, scan=scan, rounds=rounds,
               delta0=delta0, ntau=ntau, tau_ratio=tau_ratio, cfl=cfl, tau_min=tau_min,
               tau_max=tau_max, hmax=hmax, achecks=achecks, rk2=rk2, vclamp=vclamp,
               simplex=simplex)
    return SolverParams(p=p, level=level, control_kind=kind, ctl=ctl, nctl=ctl.size // 3,
                        warm=warm, iters=iters, tol=tol, cap=float(cap), ttol=ttol,
                        margin=margin, clearance=clearance,
                        stop_rule=_lib.STOP_MAXNORM if stop == "maxnorm" else _lib.STOP_L1_QUIET,
                        storage=storage, polish_sweeps=int(getc(cfg, "polish_sweeps", 64)),
                        raw=raw)


# ---------------------------------------------------------------------------
# Input files (Pipeline.jl:406-490)
# ---------------------------------------------------------------------------

def readjson(path):
    """readjson (Pipeline.jl:17-27): tolerates a UTF-8 BOM."""
    with open(path, "r", encoding="utf-8-sig") as fh:
        return json.load(fh)


@dataclass
class Drivetrain:
    B: np.ndarray
    A: np.ndarray
    q: np.ndarray
    S: np.ndarray
    D: np.ndarray
    c: np.ndarray
    eps: np.ndarray
    knee: float

    def to_c(self) -> _lib.Model:
        m = _lib.Model()
        for name in ("B", "A", "S", "D"):
            arr = getattr(self, name).astype(np.float32).reshape(-1)
            for i in range(9):
                getattr(m, name)[i] = float(arr[i])
        for name in ("q", "c", "eps"):
            arr = getattr(self, name).astype(np.float32).reshape(-1)
            for i in range(3):
                getattr(m, name)[i] = float(arr[i])
        m.knee = float(np.float32(self.knee))
        return m

    def zeroed_c(self) -> "Drivetrain":
        return Drivetrain(self.B, self.A, self.q, self.S, self.D, np.zeros(3, np.float32),
                          self.eps, self.knee)


def load_model(path):
    """load_model (Pipeline.jl:406-440)."""
    with open(path, "rb") as fh:
        cfg = tomllib.load(fh)
    if "mecanum_basis" not in cfg:
        raise ValueError(f"{path} has no [mecanum_basis]; is it a drivetrain_fit.toml?")
    mb = cfg["mecanum_basis"]

    def mat(key):
        return np.array([[float(mb[key][r][c]) for c in range(3)] for r in range(3)],
                        dtype=np.float32)

    B, A = mat("B"), mat("A")
    q = np.array([float(v) for v in mb["q"]], dtype=np.float32)
    c = np.array([float(v) for v in mb["c"]], dtype=np.float32)
    S = mat("S") if "S" in mb else np.zeros((3, 3), np.float32)
    D = mat("D") if "D" in mb else np.zeros((3, 3), np.float32)
    if "traction_knee" not in mb or mb["traction_knee"] is None:
        raise ValueError("regression has no traction_knee; refit with "
                         "fit_drivetrain.py --traction-knee auto")
    knee = np.float32(float(mb["traction_knee"]))
    if math.isnan(knee) or knee <= 0:
        raise ValueError(f"regression traction_knee is {mb['traction_knee']}; "
                         "a positive knee is required")
    eps = (np.array([float(v) for v in mb["coulomb_eps"]], dtype=np.float32)
           if "coulomb_eps" in mb else np.array([5.0, 5.0, 0.15], dtype=np.float32))
    return Drivetrain(B, A, q, S, D, c, eps, float(knee)), cfg


def _poly(pts, what):
    if len(pts) < 3:
        raise ValueError(f"{what} has fewer than 3 vertices")
    out = []
    for p in pts:
        if len(p) != 2:
            raise ValueError(f"{what} has a vertex that is not [x, y]")
        out.append((float(p[0]), float(p[1])))
    return out


def load_field(path):
    """load_field (Pipeline.jl:462-475)."""
    cfg = readjson(path)
    f = cfg["field"]
    bounds = (float(f["x_min"]), float(f["y_min"]), float(f["x_max"]), float(f["y_max"]))
    polys = [_poly(ob["polygon"], f"obstacle '{ob.get('name', '?')}'")
             for ob in cfg.get("obstacles", []) or []]
    robot = None
    if "robot" in cfg and cfg["robot"] and "polygon" in cfg["robot"]:
        robot = _poly(cfg["robot"]["polygon"], "robot footprint")
    return bounds, polys, robot, cfg


def load_targets(path):
    """load_targets (Pipeline.jl:478-490)."""
    cfg = readjson(path)
    names, states = [], []
    for t in cfg["targets"]:
        s = t["state"]
        if len(s) != 6:
            raise ValueError(f"target '{t.get('name', '?')}' state must be 6 numbers")
        names.append(str(t.get("name", f"target{len(names)}")))
        states.append(tuple(f32(v) for v in s))
    if not states:
        raise ValueError(f"{path} lists no targets")
    return names, states, cfg
