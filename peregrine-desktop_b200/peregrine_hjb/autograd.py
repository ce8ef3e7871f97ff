"""Differentiating the value table with respect to the drivetrain model.

`ValueTable.apply(theta, spec)` solves the table on the GPU for the model
with its 18 differentiable entries set to `theta` and returns V (row-major,
FP32); its backward runs the library's adjoint (`pg_adjoint`) at the
converged policy and returns dL/dtheta.  `theta` is the diagonals of B, A,
S, D and the vectors q and c (THETA_NAMES); every other model entry stays as
`spec.model` has it.  The reference never differentiates its tables; the
model and the solve it differentiates through are its `Model` and
`solve_value!` (PeregrineSolver.jl:100-171, Run.jl:1434-1474).

torch is only the autograd plumbing here: the solve and the adjoint are the
library's CUDA kernels, and there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib

THETA_NAMES = ("B00", "B11", "B22", "A00", "A11", "A22", "q0", "q1", "q2",
               "S00", "S11", "S22", "D00", "D11", "D22", "c0", "c1", "c2")
_SLOTS = [("B", 0), ("B", 4), ("B", 8), ("A", 0), ("A", 4), ("A", 8), ("q", 0), ("q", 1),
          ("q", 2), ("S", 0), ("S", 4), ("S", 8), ("D", 0), ("D", 4), ("D", 8), ("c", 0),
          ("c", 1), ("c", 2)]


def theta_of(model: _lib.Model) -> np.ndarray:
    """The 18 differentiable entries of a model, in THETA_NAMES order."""
    return np.array([getattr(model, f)[k] for f, k in _SLOTS], dtype=np.float64)


def model_with(model: _lib.Model, theta) -> _lib.Model:
    """A copy of `model` with its 18 differentiable entries set to theta."""
    m = _lib.Model()
    C.memmove(C.byref(m), C.byref(model), C.sizeof(_lib.Model))
    for (f, k), v in zip(_SLOTS, np.asarray(theta, dtype=np.float64)):
        getattr(m, f)[k] = float(v)
    return m


@dataclass
class SolveSpec:
    """Everything a solve needs besides theta."""
    grid: _lib.Grid6
    model: _lib.Model
    params: _lib.Params
    occ: np.ndarray
    seeds: np.ndarray
    ctl: np.ndarray
    iters: int = 5000
    tol: float = 1e-6
    storage: str = "fp32"
    kernel: int = _lib.KERNEL_STENCIL
    adjoint_iters: int = 20000
    adjoint_tol: float = 1e-5
    device: int = 0

    @classmethod
    def from_problem(cls, pr, **kw):
        return cls(grid=pr.grid.to_c(), model=pr.model.to_c(), params=pr.params, occ=pr.occ,
                   seeds=pr.seeds, ctl=pr.ctl, **kw)


def solve(spec: SolveSpec, theta, storage: str | None = None, keep: bool = False):
    """Solve the table for theta; returns (V row-major float32, result, context
    or None).  The context (kept when `keep`) still holds the converged table
    on the device for the adjoint."""
    ctx = _lib.Context(spec.device)
    try:
        ctx.load_problem(spec.grid, model_with(spec.model, theta), spec.params, spec.occ, spec.ctl,
                         storage or spec.storage)
        opts = _lib.default_opts(stop_rule=_lib.STOP_MAXNORM, kernel=spec.kernel,
                                 storage=storage or spec.storage, polish_sweeps=0)
        res = ctx.solve(spec.seeds, spec.iters, spec.tol, opts)
        V = ctx.get_value()
    except BaseException:
        ctx.close()
        raise
    if keep:
        return V, res, ctx
    ctx.close()
    return V, res, None


class ValueTable(torch.autograd.Function):
    """V(theta): the converged minimum-time table as a function of the model."""

    @staticmethod
    def forward(fctx, theta: torch.Tensor, spec: SolveSpec):
        V, res, ctx = solve(spec, theta.detach().cpu().numpy(), keep=True)
        fctx.pg = ctx
        fctx.spec = spec
        fctx.sweeps = res.iterations
        return torch.from_numpy(V)

    @staticmethod
    def backward(fctx, grad_v: torch.Tensor):
        ctx = fctx.pg
        try:
            g = np.ascontiguousarray(grad_v.detach().to("cpu", torch.float32).numpy())
            grad, res = ctx.adjoint(g, fctx.spec.adjoint_iters, fctx.spec.adjoint_tol)
        finally:
            ctx.close()
            fctx.pg = None
        fctx.adjoint = res
        return torch.from_numpy(grad), None


def start_states(grid: _lib.Grid6, occ: np.ndarray, count: int = 4096, seed: int = 0) -> np.ndarray:
    """`count` start states uniform over the free (x, y, h) space at rest:
    (x, y, h, 0, 0, 0), free meaning the nearest occupancy cell is free."""
    rng = np.random.default_rng(seed)
    n = [int(v) for v in grid.n]
    lo = np.array([grid.lo[k] for k in range(6)], dtype=np.float64)
    st = np.array([grid.step[k] for k in range(6)], dtype=np.float64)
    occ3 = np.asarray(occ, dtype=np.uint8).reshape(n[0], n[1], n[2])
    out = []
    while len(out) < count:
        x = rng.uniform(lo[0], lo[0] + st[0] * (n[0] - 1))
        y = rng.uniform(lo[1], lo[1] + st[1] * (n[1] - 1))
        h = rng.uniform(-math.pi, math.pi)
        i = int(round((x - lo[0]) / st[0]))
        j = int(round((y - lo[1]) / st[1]))
        k = int(round((h - lo[2]) / st[2])) % n[2]
        if occ3[i, j, k] == 0:
            out.append((x, y, h, 0.0, 0.0, 0.0))
    return np.array(out, dtype=np.float64)


def interp_weights(grid: _lib.Grid6, states: np.ndarray):
    """Row-major corner indices and weights (k, 64) of the 64-corner
    multilinear interpolation (PeregrineSolver.jl:399-466) at each state."""
    n = np.array([int(v) for v in grid.n])
    lo = np.array([grid.lo[k] for k in range(6)], dtype=np.float64)
    st = np.array([grid.step[k] for k in range(6)], dtype=np.float64)
    f = (np.asarray(states, dtype=np.float64) - lo) / st
    f[:, 2] = f[:, 2] - np.floor(f[:, 2] / n[2]) * n[2]
    for k in (0, 1, 3, 4, 5):
        f[:, k] = np.clip(f[:, k], 0, n[k] - 1)
    b = np.floor(f).astype(np.int64)
    t = f - b
    idx = np.zeros((len(f), 64), dtype=np.int64)
    w = np.ones((len(f), 64), dtype=np.float64)
    for d in range(64):
        flat = np.zeros(len(f), dtype=np.int64)
        for ax in range(6):
            bit = (d >> ax) & 1
            w[:, d] *= t[:, ax] if bit else 1.0 - t[:, ax]
            j = (b[:, ax] + bit) % n[2] if ax == 2 else np.minimum(b[:, ax] + bit, n[ax] - 1)
            flat = flat * n[ax] + j
        idx[:, d] = flat
    return idx, w


def start_state_loss(V: torch.Tensor, idx: np.ndarray, w: np.ndarray) -> torch.Tensor:
    """Mean interpolated V over the start states (differentiable in V)."""
    ti = torch.from_numpy(idx).to(V.device)
    tw = torch.from_numpy(w).to(V.device, V.dtype)
    return (V[ti] * tw).sum(dim=1).mean()
