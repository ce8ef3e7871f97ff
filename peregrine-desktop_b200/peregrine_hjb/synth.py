"""Seeded synthetic jobs for the benchmark configurations.

The reference ships no benchmark suite for this path, so every workload is
drawn from numpy's PCG64 (`default_rng(seed)`) and written in the reference's
own input schemas (drivetrain_fit.toml `[mecanum_basis]`, field.json,
targets.json, config.json), so the GPU solver, the CPU oracle and any other
reader see identical files.

Workloads (grid n, controls, dt, obstacles):
  small   24 x 24 x 16 x 9 x 9 x 9   (6.7M cells), {-1,0,1}^3, dt 0.05, 3 rects
  medium  48 x 48 x 32 x 15 x 15 x 15 (249M cells), {-1,-.5,0,.5,1}^3, dt 0.04, 6 rects
  large   96 x 96 x 64 x 21 x 21 x 21 (5.46e9 cells), same controls, dt 0.03, 8 rects
Field 365.8 cm square, point robot, velocity axes +-150 cm/s, omega +-6 rad/s,
unreached cells at 30 s, a 10 cm target disk (any heading, |v| < 20 cm/s),
max-norm stop at 1e-4 s.  The plain scheme: full control scan, one horizon,
fixed probes, 64-corner multilinear, RK2, no warm start, no escape pass.
"""
from __future__ import annotations

import json
import os

import numpy as np

from .grid import Grid6, getc
from .geometry import build_occupancy
from .params import Drivetrain, solver_params
from .seeds import region_cells

FIELD = 365.8
WORKLOADS = {
    "tiny": dict(n=[12, 12, 8, 5, 5, 5], control_set="cube3", dt=0.05, rects=2),
    "small": dict(n=[24, 24, 16, 9, 9, 9], control_set="cube3", dt=0.05, rects=3),
    "medium": dict(n=[48, 48, 32, 15, 15, 15], control_set="cube5", dt=0.04, rects=6),
    # the medium workload's planes and controls with a quarter of the headings:
    # the same per-block work, small enough for a profiler capture
    "medium_h8": dict(n=[48, 48, 8, 15, 15, 15], control_set="cube5", dt=0.04, rects=6),
    "large": dict(n=[96, 96, 64, 21, 21, 21], control_set="cube5", dt=0.03, rects=8),
    # the large workload's planes and controls with 2 headings: the same
    # per-block work, a few GB on the device, for profiler captures
    "large_h2": dict(n=[96, 96, 2, 21, 21, 21], control_set="cube5", dt=0.03, rects=8),
    # the out-of-core variant: 5.5e10 cells, 110 GB per table in FP16, swept a
    # tile of x rows at a time from host memory
    "xlarge_ooc": dict(n=[192, 192, 96, 25, 25, 25], control_set="cube5", dt=0.03, rects=8),
}


def draw_model(rng) -> Drivetrain:
    B = np.diag([rng.uniform(150, 250), rng.uniform(150, 250), rng.uniform(8, 14)])
    A = np.diag(-rng.uniform(1.5, 3.0, size=3))
    q = rng.normal(0.0, 0.5, size=3)
    S = np.diag(-rng.uniform(5.0, 15.0, size=3))
    D = np.diag(-rng.uniform(0.002, 0.006, size=3))
    c = rng.normal(0.0, 2.0, size=3)
    f = np.float32
    return Drivetrain(B.astype(f), A.astype(f), q.astype(f), S.astype(f), D.astype(f),
                      c.astype(f), np.array([5.0, 5.0, 0.15], f), 0.55)


def draw_field(rng, nrect: int):
    rects = []
    for _ in range(nrect):
        w, h = rng.uniform(20, 60), rng.uniform(20, 60)
        x0 = rng.uniform(0, FIELD - w)
        y0 = rng.uniform(0, FIELD - h)
        rects.append([[x0, y0], [x0 + w, y0], [x0 + w, y0 + h], [x0, y0 + h]])
    return rects


def draw_target(rng, rects, radius=10.0):
    for _ in range(10000):
        x, y = rng.uniform(radius, FIELD - radius, size=2)
        ok = True
        for r in rects:
            (x0, y0), (x1, y1) = r[0], r[2]
            if x0 - radius <= x <= x1 + radius and y0 - radius <= y <= y1 + radius:
                ok = False
                break
        if ok:
            return float(x), float(y)
    raise RuntimeError("no free target position")


def job(workload: str = "small", seed: int = 0, n=None, control_set=None, dt=None, rects=None):
    """Draw one job as plain dicts (config, model, field, targets)."""
    w = dict(WORKLOADS[workload])
    if n is not None:
        w["n"] = list(n)
    if control_set is not None:
        w["control_set"] = control_set
    if dt is not None:
        w["dt"] = dt
    if rects is not None:
        w["rects"] = rects
    rng = np.random.default_rng(seed)
    model = draw_model(rng)
    rr = draw_field(rng, int(w["rects"]))
    tx, ty = draw_target(rng, rr)
    cfg = {
        "grid": {"n": w["n"], "bounds": [0.0, 0.0, FIELD, FIELD], "vmax": 150.0, "wmax": 6.0},
        "dt": w["dt"], "substeps": 4, "sweep_checks": 3, "adaptive_checks": False,
        "iterations": 3000, "tolerance": 1e-4, "stop_rule": "maxnorm",
        "control_set": w["control_set"], "control_scan": 0, "refine_rounds": 0,
        "warm_start": False, "tau_levels": 1, "cfl": 0.0, "rk2": True, "simplex": False,
        "velocity_clamp": False, "nearest": False, "value_cap": 30.0, "zero_c": False,
        "clearance_cm": 0.0, "wall_clearance_cm": 0.0, "margin_cm": 0.0,
        "heading_substeps": 3, "escape": False, "dtype": "u16",
        "target_region": {"kind": "disk", "radius_cm": 10.0, "speed_max_cm_s": 20.0},
    }
    field = {"schema_version": 2,
             "field": {"x_min": 0.0, "y_min": 0.0, "x_max": FIELD, "y_max": FIELD},
             "obstacles": [{"name": f"rect{i}", "polygon": r} for i, r in enumerate(rr)]}
    targets = {"schema_version": 1,
               "targets": [{"name": "disk", "state": [tx, ty, 0.0, 0.0, 0.0, 0.0]}]}
    return cfg, model, field, targets


def write_toml(path, m: Drivetrain):
    def mat(M):
        return "[" + ", ".join("[" + ", ".join(repr(float(v)) for v in row) + "]" for row in M) + "]"

    def vec(v):
        return "[" + ", ".join(repr(float(x)) for x in v) + "]"

    with open(path, "w") as fh:
        fh.write("[units]\ndistance = \"cm\"\n\n[mecanum_basis]\n")
        fh.write(f"B = {mat(m.B)}\nA = {mat(m.A)}\nq = {vec(m.q)}\nS = {mat(m.S)}\n")
        fh.write(f"D = {mat(m.D)}\nc = {vec(m.c)}\ncoulomb_eps = {vec(m.eps)}\n")
        fh.write(f"traction_knee = {float(m.knee)!r}\n")


def write_job(dirpath, workload="small", seed=0, **kw) -> str:
    """Write a complete job directory; returns the config.json path."""
    os.makedirs(dirpath, exist_ok=True)
    cfg, model, field, targets = job(workload, seed, **kw)
    write_toml(os.path.join(dirpath, "drivetrain_fit.toml"), model)
    with open(os.path.join(dirpath, "field.json"), "w") as fh:
        json.dump(field, fh, indent=1)
    with open(os.path.join(dirpath, "targets.json"), "w") as fh:
        json.dump(targets, fh, indent=1)
    cfg = dict(cfg)
    cfg["regression"] = os.path.join(dirpath, "drivetrain_fit.toml")
    cfg["field"] = os.path.join(dirpath, "field.json")
    cfg["targets"] = os.path.join(dirpath, "targets.json")
    cfg["out_dir"] = os.path.join(dirpath, "out")
    p = os.path.join(dirpath, "config.json")
    with open(p, "w") as fh:
        json.dump(cfg, fh, indent=1)
    return p


class Problem:
    """A job built in memory through the same host functions run_solve uses."""

    def __init__(self, workload="small", seed=0, **kw):
        cfg, model, field, targets = job(workload, seed, **kw)
        self.cfg = cfg
        self.model = model
        gc = cfg["grid"]
        b = gc["bounds"]
        self.grid = Grid6.make(gc["n"], (b[0], b[1], -np.pi, -gc["vmax"], -gc["vmax"], -gc["wmax"]),
                               (b[2], b[3], np.pi, gc["vmax"], gc["vmax"], gc["wmax"]))
        self.sp = solver_params(cfg, self.grid)
        polys = [o["polygon"] for o in field["obstacles"]]
        self.polys = polys
        self.occ = build_occupancy(self.grid, polys, 0.0, None, int(getc(cfg, "heading_substeps", 3)),
                                   0.0, bounds=(0.0, 0.0, FIELD, FIELD), wall_clearance_cm=0.0)
        s = targets["targets"][0]["state"]
        self.target = s
        self.seeds = region_cells(self.grid, s, cfg["target_region"])
        self.ctl = self.sp.ctl
        self.nctl = self.sp.nctl
        self.params = self.sp.p

    @property
    def ncells(self) -> int:
        return self.grid.ncells
