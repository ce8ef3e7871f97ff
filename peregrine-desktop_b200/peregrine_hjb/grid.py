"""Grid construction, mirroring solver/src/PeregrineSolver.jl:47-81 and
solver/src/Run.jl:20-162.

Float32 is kept wherever the reference keeps it: `lo` and `step` are Float32
(Grid6), axis values are `lo + Float32(i) * step` rounded in Float32.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import _lib

AXES = ("x", "y", "h", "vx", "vy", "w")
DEFAULT_VMAX = 170.0
DEFAULT_WMAX = 8.0
DEFAULT_XY_CM = 8.0
DEFAULT_HEADING_DEG = 22.5
DEFAULT_V_CM_S = 34.0
DEFAULT_W_RAD_S = 1.6

f32 = np.float32


def getc(cfg, key, default):
    """`getc` (Run.jl:18): the key's value unless absent or null."""
    if cfg is None:
        return default
    v = cfg.get(key) if hasattr(cfg, "get") else None
    return default if v is None else v


@dataclass(frozen=True)
class Grid6:
    """Grid6 (PeregrineSolver.jl:47-51)."""
    n: tuple
    lo: tuple  # np.float32 each
    step: tuple

    @staticmethod
    def make(n, lo, hi) -> "Grid6":
        """Grid6(n, lo, hi) (PeregrineSolver.jl:53-60)."""
        n = tuple(int(v) for v in n)
        if any(v < 2 for v in n):
            raise ValueError(f"every axis needs at least 2 samples, got {n}")
        st = tuple(f32(2 * math.pi / n[k]) if k == 2 else f32((float(hi[k]) - float(lo[k])) / (n[k] - 1))
                   for k in range(6))
        lo3 = tuple(f32(-math.pi) if k == 2 else f32(float(lo[k])) for k in range(6))
        return Grid6(n, lo3, st)

    @property
    def ncells(self) -> int:
        c = 1
        for v in self.n:
            c *= v
        return c

    def axisvalue(self, k: int, i):
        """lo + Float32(i)*step, each operation rounded in Float32."""
        i = np.asarray(i)
        return (self.lo[k] + (i.astype(np.float32) * self.step[k]).astype(np.float32)).astype(np.float32)

    def axis(self, k: int) -> np.ndarray:
        return self.axisvalue(k, np.arange(self.n[k]))

    def flatten(self, i1, i2, i3, i4, i5, i6):
        n = self.n
        return (((((np.int64(i1) * n[1] + i2) * n[2] + i3) * n[3] + i4) * n[4] + i5) * n[5] + i6)

    def unflatten(self, idx):
        idx = np.asarray(idx, dtype=np.int64)
        out = []
        r = idx
        for k in range(5, 0, -1):
            out.append(r % self.n[k])
            r = r // self.n[k]
        out.append(r)
        return tuple(reversed(out))

    def to_c(self) -> _lib.Grid6:
        g = _lib.Grid6()
        for k in range(6):
            g.n[k] = self.n[k]
            g.lo[k] = float(self.lo[k])
            g.step[k] = float(self.step[k])
        return g

    def span_max(self, k: int) -> float:
        """Manifest `grid.max` (Run.jl:2008): lo + step * (n or n - 1), each
        operation in Float32 as the reference's Grid6 fields are, then
        widened."""
        m = self.n[k] if k == 2 else self.n[k] - 1
        return float(f32(self.lo[k] + f32(self.step[k] * f32(m))))


def axis_samples(span: float, cell: float):
    """Run.jl:55-59"""
    if not cell > 0:
        raise ValueError(f"resolution must be positive, got {cell}")
    n = max(2, math.ceil(span / cell - 1.0e-9) + 1)
    return n, (n - 1) * cell


def symmetric_samples(limit: float, cell: float):
    """Run.jl:61-65"""
    if not cell > 0:
        raise ValueError(f"resolution must be positive, got {cell}")
    half = max(1, math.ceil(limit / cell - 1.0e-9))
    return 2 * half + 1, half * cell


def grid_resolution(cfg):
    """Run.jl:68-74"""
    r = getc(cfg, "resolution", {})
    return (float(getc(r, "xy_cm", DEFAULT_XY_CM)), float(getc(r, "heading_deg", DEFAULT_HEADING_DEG)),
            float(getc(r, "v_cm_s", DEFAULT_V_CM_S)), float(getc(r, "w_rad_s", DEFAULT_W_RAD_S)))


def julia_round_int(x: float) -> int:
    """round(Int, x): nearest, ties to even (Python's round does the same)."""
    return int(round(x))


def build_grid(gcfg, bounds, robot=None, wall_clearance: float = 0.0, hsub: int = 3) -> Grid6:
    """build_grid (Run.jl:99-138).  `gcfg` is the config's `grid` block."""
    from .geometry import feasible_bounds

    vmax = float(getc(gcfg, "vmax", DEFAULT_VMAX))
    wmax = float(getc(gcfg, "wmax", DEFAULT_WMAX))
    xy_cm, heading_deg, v_cm_s, w_rad_s = grid_resolution(gcfg)
    nfix = getc(gcfg, "n", None)
    nh = int(nfix[2]) if nfix is not None else max(4, julia_round_int(360.0 / heading_deg))
    ov = getc(gcfg, "bounds", None)
    if ov is not None:
        fb = dict(xlo=float(ov[0]), ylo=float(ov[1]), xhi=float(ov[2]), yhi=float(ov[3]))
    else:
        fb = feasible_bounds(bounds, robot, wall_clearance, nh, hsub)
    if nfix is not None:
        n = tuple(int(v) for v in nfix)
        lo = (fb["xlo"], fb["ylo"], -math.pi, -vmax, -vmax, -wmax)
        hi = (fb["xhi"], fb["yhi"], math.pi, vmax, vmax, wmax)
        return Grid6.make(n, lo, hi)
    ax_n, ax_span = axis_samples(fb["xhi"] - fb["xlo"], xy_cm)
    ay_n, ay_span = axis_samples(fb["yhi"] - fb["ylo"], xy_cm)
    av_n, av_lim = symmetric_samples(vmax, v_cm_s)
    aw_n, aw_lim = symmetric_samples(wmax, w_rad_s)
    padx = (ax_span - (fb["xhi"] - fb["xlo"])) / 2
    pady = (ay_span - (fb["yhi"] - fb["ylo"])) / 2
    n = (ax_n, ay_n, nh, av_n, av_n, aw_n)
    lo = (fb["xlo"] - padx, fb["ylo"] - pady, -math.pi, -av_lim, -av_lim, -aw_lim)
    hi = (fb["xhi"] + padx, fb["yhi"] + pady, math.pi, av_lim, av_lim, aw_lim)
    return Grid6.make(n, lo, hi)


def grid_inputs(cfg, bounds, robot):
    """grid_inputs (Run.jl:148-159)."""
    clearance = float(getc(cfg, "clearance_cm", 5.0))
    return dict(bounds=bounds, robot=robot, clearance=clearance,
                wall_clearance=float(getc(cfg, "wall_clearance_cm", clearance)),
                hsub=int(getc(cfg, "heading_substeps", 3)))
