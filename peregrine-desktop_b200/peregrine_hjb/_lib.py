"""ctypes binding of libperegrine_hjb.so (include/peregrine_hjb.h).

The library is the only compute path: there is no CPU fallback.  Loading
fails loudly when the shared object is missing, and every call that returns a
negative status raises :class:`PeregrineError` with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_NAME = "libperegrine_hjb.so"
LIB_PATH = Path(__file__).resolve().parent / LIB_NAME

PG_OK = 0
PG_EINVAL, PG_ECUDA, PG_ENOMEM, PG_ETIMEOUT, PG_ESTATE, PG_EUNSUPPORTED, PG_ECANCELLED = (
    -1, -2, -3, -4, -5, -6, -7)

STOP_L1_QUIET, STOP_MAXNORM = 0, 1
STORE_F32, STORE_F16, STORE_BF16, STORE_F64 = 0, 1, 2, 3
STORE_Q16 = 4
STORAGES = {"fp32": STORE_F32, "fp16": STORE_F16, "bf16": STORE_BF16, "fp64": STORE_F64,
            "q16": STORE_Q16}
(KERNEL_AUTO, KERNEL_STENCIL, KERNEL_CELLFORM, KERNEL_STENCIL_EXACT, KERNEL_STENCIL_ROWS,
 KERNEL_STENCIL_GATHER, KERNEL_STENCIL_BLEND) = (0, 1, 2, 3, 4, 5, 6)
DTYPE_CODES = {"u8": 0, "u16": 1, "f16": 2, "f32": 3}

# Every symbol include/peregrine_hjb.h declares.
EXPORTS = (
    "pg_abi_version", "pg_last_error", "pg_default_opts", "pg_create", "pg_destroy",
    "pg_solve_value", "pg_load_problem", "pg_solve", "pg_get_value", "pg_set_value",
    "pg_sweep", "pg_escape_sweep", "pg_solve_escape", "pg_encode", "pg_time_sweeps",
    "pg_launch_count", "pg_set_tile_rows", "pg_batch_create", "pg_batch_destroy",
    "pg_batch_add", "pg_batch_solve", "pg_batch_table", "pg_adjoint", "pg_measure_peaks",
    "pg_sweep_noalloc", "pg_set_wait_timeout", "pg_default_ooc_opts", "pg_solve_ooc",
    "pg_reach_rows", "pg_load_slab", "pg_get_rows", "pg_set_rows",
    "pg_probe_step", "pg_probe_traction_gain", "pg_probe_interp",
)


class PeregrineError(RuntimeError):
    """A negative status from the library, with its message."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (status {code})")
        self.code = code


class Grid6(C.Structure):
    _fields_ = [("n", C.c_int32 * 6), ("lo", C.c_float * 6), ("step", C.c_float * 6)]


class Model(C.Structure):
    _fields_ = [("B", C.c_float * 9), ("A", C.c_float * 9), ("q", C.c_float * 3),
                ("S", C.c_float * 9), ("D", C.c_float * 9), ("c", C.c_float * 3),
                ("eps", C.c_float * 3), ("knee", C.c_float)]


class Params(C.Structure):
    _fields_ = [("dt", C.c_float), ("nsub", C.c_int32), ("checks", C.c_int32),
                ("adaptive_checks", C.c_int32), ("nearest", C.c_int32), ("cap", C.c_float),
                ("ntau", C.c_int32), ("tau_ratio", C.c_float), ("cfl", C.c_float),
                ("tau_min", C.c_float), ("tau_max", C.c_float), ("hmax", C.c_float),
                ("ncoarse", C.c_int32), ("rounds", C.c_int32), ("delta0", C.c_float),
                ("rk2", C.c_int32), ("vclamp", C.c_int32), ("simplex", C.c_int32)]


class SolveOpts(C.Structure):
    _fields_ = [("stop_rule", C.c_int32), ("storage", C.c_int32), ("kernel", C.c_int32),
                ("warm_start", C.c_int32), ("polish_sweeps", C.c_int32),
                ("progress_every", C.c_int32), ("reserved", C.c_int32 * 6)]


class SolveResult(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("polish_iterations", C.c_int32),
                ("last_delta", C.c_double), ("last_maxnorm", C.c_double),
                ("kernel_ms", C.c_double), ("elapsed_ms", C.c_double),
                ("cell_controls", C.c_int64)]


class BatchResult(C.Structure):
    _fields_ = [("tables", C.c_int32), ("converged", C.c_int32), ("sweeps", C.c_int32),
                ("polish_sweeps", C.c_int32), ("graph", C.c_int32), ("kernel_ms", C.c_double),
                ("elapsed_ms", C.c_double), ("cell_controls", C.c_int64)]


class AdjointResult(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("active_cells", C.c_int32),
                ("last_residual", C.c_double), ("c_norm", C.c_double),
                ("kernel_ms", C.c_double)]


class OocOpts(C.Structure):
    _fields_ = [("tile_rows", C.c_int32), ("halo_rows", C.c_int32), ("tile_sweeps", C.c_int32),
                ("jacobi", C.c_int32), ("kernel", C.c_int32), ("storage", C.c_int32),
                ("stop_rule", C.c_int32), ("allow_starved_halo", C.c_int32),
                ("device_budget_bytes", C.c_int64), ("reserved", C.c_int32 * 4)]


class OocResult(C.Structure):
    _fields_ = [("rounds", C.c_int32), ("tiles_per_round", C.c_int32), ("tile_rows", C.c_int32),
                ("halo_rows", C.c_int32), ("reach_rows", C.c_int32), ("reserved", C.c_int32),
                ("last_delta", C.c_double), ("last_maxnorm", C.c_double),
                ("kernel_ms", C.c_double), ("elapsed_ms", C.c_double),
                ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64), ("launches", C.c_int64)]


PROGRESS_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.c_double, C.c_double)

_lib = None


def load_library(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load libperegrine_hjb.so once; raise if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path or os.environ.get("PEREGRINE_HJB_LIB") or LIB_PATH)
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build the CUDA library first "
            "(make -C peregrine-desktop_b200/csrc, or __graft_entry__.build()). "
            "There is no CPU fallback.")
    lib = C.CDLL(str(p))
    vp, i32, i64, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    P = C.POINTER
    sig = {
        "pg_abi_version": (i32, []),
        "pg_last_error": (C.c_char_p, []),
        "pg_default_opts": (None, [P(SolveOpts)]),
        "pg_create": (C.c_int, [P(vp), C.c_int]),
        "pg_destroy": (C.c_int, [vp]),
        "pg_solve_value": (C.c_int, [vp, P(Grid6), P(Model), P(Params), vp, vp, i64, vp, i32,
                                     i32, f64, P(SolveOpts), vp, P(SolveResult), PROGRESS_CB, vp]),
        "pg_load_problem": (C.c_int, [vp, P(Grid6), P(Model), P(Params), vp, vp, i32, i32]),
        "pg_solve": (C.c_int, [vp, vp, i64, i32, f64, P(SolveOpts), P(SolveResult),
                               PROGRESS_CB, vp]),
        "pg_get_value": (C.c_int, [vp, vp]),
        "pg_set_value": (C.c_int, [vp, vp]),
        "pg_sweep": (C.c_int, [vp, i32, i32, P(f64), P(f64), vp]),
        "pg_escape_sweep": (C.c_int, [vp, i32, P(f64)]),
        "pg_solve_escape": (C.c_int, [vp, i32, f64, P(SolveResult), PROGRESS_CB, vp]),
        "pg_encode": (C.c_int, [vp, i32, f64, f64, i64, i64, vp, P(i64), P(i64)]),
        "pg_time_sweeps": (C.c_int, [vp, i32, i32, i32, P(f64)]),
        "pg_launch_count": (C.c_int, [vp, P(i64)]),
        "pg_set_tile_rows": (C.c_int, [vp, i32]),
        "pg_batch_create": (C.c_int, [P(vp), C.c_int, i32]),
        "pg_batch_destroy": (C.c_int, [vp]),
        "pg_batch_add": (C.c_int, [vp, P(Grid6), P(Model), P(Params), vp, vp, i64, vp, i32, i32,
                                   P(i32)]),
        "pg_batch_solve": (C.c_int, [vp, i32, f64, i32, i32, P(BatchResult)]),
        "pg_batch_table": (C.c_int, [vp, i32, P(i32), P(f64), P(vp)]),
        "pg_adjoint": (C.c_int, [vp, vp, i32, i32, f64, vp, P(AdjointResult)]),
        "pg_measure_peaks": (C.c_int, [C.c_int, P(f64), P(f64), P(f64)]),
        "pg_sweep_noalloc": (C.c_int, [P(Grid6), P(Model), P(Params), vp, vp, i32, vp, vp, i32,
                                       vp, P(f64), P(f64)]),
        "pg_set_wait_timeout": (C.c_int, [vp, f64]),
        "pg_default_ooc_opts": (None, [P(OocOpts)]),
        "pg_reach_rows": (C.c_int, [C.c_int, P(Grid6), P(Model), P(Params), vp, i32, P(i32)]),
        "pg_load_slab": (C.c_int, [vp, P(Grid6), P(Model), P(Params), vp, vp, i32, i32, i32, i32,
                                   P(i32), P(i32)]),
        "pg_get_rows": (C.c_int, [vp, i32, i32, vp, i32]),
        "pg_set_rows": (C.c_int, [vp, i32, i32, vp, i32]),
        "pg_solve_ooc": (C.c_int, [C.c_int, P(Grid6), P(Model), P(Params), vp, vp, i64, vp, i32,
                                   i32, f64, P(OocOpts), vp, P(OocResult), PROGRESS_CB, vp]),
        "pg_probe_step": (C.c_int, [C.c_int, P(Model), i32, vp, vp, vp, vp, i64, vp]),
        "pg_probe_traction_gain": (C.c_int, [C.c_int, vp, C.c_float, i64, vp]),
        "pg_probe_interp": (C.c_int, [vp, vp, i64, i32, i32, i32, C.c_float, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.pg_abi_version() != 1:
        raise RuntimeError(f"{p}: unexpected ABI version {lib.pg_abi_version()}")
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != PG_OK:
        msg = _lib.pg_last_error().decode("utf-8", "replace") if _lib else "library not loaded"
        raise PeregrineError(rc, msg)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def default_opts(**kw) -> SolveOpts:
    lib = load_library()
    o = SolveOpts()
    lib.pg_default_opts(C.byref(o))
    for k, v in kw.items():
        if k == "storage" and isinstance(v, str):
            v = STORAGES[v]
        setattr(o, k, int(v))
    return o


class Context:
    """One device context: a stream plus the buffers of one loaded problem."""

    def __init__(self, device: int = 0):
        self._lib = load_library()
        h = C.c_void_p()
        _check(self._lib.pg_create(C.byref(h), int(device)))
        self._h = h
        self.ncells = 0
        self.nctl = 0

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.pg_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_problem(self, grid: Grid6, model: Model, params: Params, occ: np.ndarray,
                     ctl: np.ndarray, storage: int | str = STORE_F32) -> None:
        if isinstance(storage, str):
            storage = STORAGES[storage]
        occ = np.ascontiguousarray(occ, dtype=np.uint8)
        ctl = np.ascontiguousarray(ctl, dtype=np.float32)
        nctl = ctl.size // 3
        n = [int(v) for v in grid.n]
        if occ.size != n[0] * n[1] * n[2]:
            raise ValueError(f"occupancy has {occ.size} entries, expected {n[0] * n[1] * n[2]}")
        _check(self._lib.pg_load_problem(self._h, C.byref(grid), C.byref(model),
                                         C.byref(params), _ptr(occ), _ptr(ctl), nctl,
                                         int(storage)))
        self.ncells = int(np.prod(np.array(n, dtype=np.int64)))
        self.nctl = nctl
        self._cap = float(params.cap)
        self._keep = (occ, ctl)

    def solve(self, tidx: np.ndarray, iters: int, tol: float, opts: SolveOpts | None = None,
              progress=None) -> SolveResult:
        tidx = np.ascontiguousarray(tidx, dtype=np.int64)
        res = SolveResult()
        cb = _wrap_cb(progress)
        _check(self._lib.pg_solve(self._h, _ptr(tidx), tidx.size, int(iters), float(tol),
                                  C.byref(opts) if opts is not None else None, C.byref(res),
                                  cb, None))
        return res

    def solve_escape(self, iters: int, tol: float, progress=None) -> SolveResult:
        res = SolveResult()
        _check(self._lib.pg_solve_escape(self._h, int(iters), float(tol), C.byref(res),
                                         _wrap_cb(progress), None))
        return res

    def get_value(self) -> np.ndarray:
        out = np.empty(self.ncells, dtype=np.float32)
        _check(self._lib.pg_get_value(self._h, _ptr(out)))
        return out

    def set_value(self, V: np.ndarray) -> None:
        V = np.ascontiguousarray(V, dtype=np.float32)
        if V.size != self.ncells:
            raise ValueError("value array has the wrong size")
        _check(self._lib.pg_set_value(self._h, _ptr(V)))

    def sweep(self, phase: int = 0, kernel: int = KERNEL_AUTO, argmin: bool = False):
        d = C.c_double()
        dm = C.c_double()
        am = np.empty(self.ncells, dtype=np.int16) if argmin else None
        _check(self._lib.pg_sweep(self._h, int(phase), int(kernel), C.byref(d), C.byref(dm),
                                  _ptr(am)))
        return d.value, dm.value, am

    def escape_sweep(self, phase: int = 0) -> float:
        d = C.c_double()
        _check(self._lib.pg_escape_sweep(self._h, int(phase), C.byref(d)))
        return d.value

    def encode(self, dtype: str, scale: float, escape_scale: float, lo: int, n: int,
               out: np.ndarray | None = None):
        eb = {"u8": 1, "u16": 2, "f16": 2, "f32": 4}[dtype]
        if out is None:
            out = np.empty(n * eb, dtype=np.uint8)
        r = C.c_int64()
        e = C.c_int64()
        _check(self._lib.pg_encode(self._h, DTYPE_CODES[dtype], float(scale), float(escape_scale),
                                   int(lo), int(n), _ptr(out), C.byref(r), C.byref(e)))
        return out[: n * eb], r.value, e.value

    def time_sweeps(self, warmup: int, steps: int, kernel: int = KERNEL_AUTO) -> float:
        ms = C.c_double()
        _check(self._lib.pg_time_sweeps(self._h, int(warmup), int(steps), int(kernel),
                                        C.byref(ms)))
        return ms.value

    def adjoint(self, dl_dv, iters: int = 20000, tol: float = 1e-5):
        """dL/dtheta (18 model entries) at the current converged FP32 table for
        dl_dv = dL/dV (row-major: a host array, or a device address as int)."""
        grad = np.zeros(18, dtype=np.float64)
        res = AdjointResult()
        if isinstance(dl_dv, int):
            ptr, on_dev = C.c_void_p(dl_dv), 1
        else:
            dl_dv = np.ascontiguousarray(dl_dv, dtype=np.float32)
            if dl_dv.size != self.ncells:
                raise ValueError("dL/dV has the wrong size")
            ptr, on_dev = _ptr(dl_dv), 0
        _check(self._lib.pg_adjoint(self._h, ptr, on_dev, int(iters), float(tol), _ptr(grad),
                                    C.byref(res)))
        return grad, res

    def set_tile_rows(self, rows: int) -> None:
        _check(self._lib.pg_set_tile_rows(self._h, int(rows)))

    def launch_count(self) -> int:
        n = C.c_int64()
        _check(self._lib.pg_launch_count(self._h, C.byref(n)))
        return n.value

    def load_slab(self, grid: Grid6, model: Model, params: Params, occ: np.ndarray,
                  ctl: np.ndarray, x0: int, x1: int, halo: int):
        """pg_load_slab: rows [x0, x1) of the table with `halo` rows either
        side; returns (first global row, rows held)."""
        occ = np.ascontiguousarray(occ, dtype=np.uint8)
        ctl = np.ascontiguousarray(ctl, dtype=np.float32)
        r0, nr = C.c_int32(), C.c_int32()
        _check(self._lib.pg_load_slab(self._h, C.byref(grid), C.byref(model), C.byref(params),
                                      _ptr(occ), _ptr(ctl), ctl.size // 3, int(x0), int(x1),
                                      int(halo), C.byref(r0), C.byref(nr)))
        per = 1
        for k in range(1, 6):
            per *= int(grid.n[k])
        self.ncells = per * nr.value
        self.nctl = ctl.size // 3
        self._cap = float(params.cap)
        self._keep = (occ, ctl)
        self.row_cells = per
        return r0.value, nr.value

    def get_rows(self, r0: int, r1: int, out=None, on_device: bool = False):
        """Rows [r0, r1) (FP32 row-major): into `out` (a numpy array, or with
        on_device a device pointer / tensor data_ptr)."""
        if out is None:
            out = np.empty((r1 - r0) * self.row_cells, np.float32)
        p = out if on_device else _ptr(out)
        _check(self._lib.pg_get_rows(self._h, int(r0), int(r1), p, int(on_device)))
        return out

    def set_rows(self, r0: int, r1: int, src, on_device: bool = False) -> None:
        p = src if on_device else _ptr(np.ascontiguousarray(src, np.float32))
        _check(self._lib.pg_set_rows(self._h, int(r0), int(r1), p, int(on_device)))

    def set_wait_timeout(self, seconds: float) -> None:
        """Limit each wait for a sweep (0 = no limit); a sweep that outlasts it
        makes the solve raise PeregrineError with code PG_ETIMEOUT."""
        _check(self._lib.pg_set_wait_timeout(self._h, float(seconds)))

    def probe_interp(self, states, kuhn=False, nearest=False, vclamp=False, cap=None,
                     grads=False):
        """interp / interp_kuhn of the current V at states [n, 6] (field-frame
        velocity) on the device; returns values (and [n, 6] Kuhn gradients)."""
        st = np.ascontiguousarray(np.asarray(states, np.float32).reshape(-1, 6))
        n = st.shape[0]
        out = np.empty(n, np.float32)
        gr = np.empty((n, 6), np.float32) if grads else None
        cap = float(self._cap if cap is None else cap)
        _check(self._lib.pg_probe_interp(self._h, _ptr(st), n, int(kuhn), int(nearest),
                                         int(vclamp), cap, _ptr(out), _ptr(gr)))
        return (out, gr) if grads else out


def ooc_opts(**kw) -> OocOpts:
    lib = load_library()
    o = OocOpts()
    lib.pg_default_ooc_opts(C.byref(o))
    for k, v in kw.items():
        if k == "storage" and isinstance(v, str):
            v = STORAGES[v]
        setattr(o, k, int(v))
    return o


def solve_ooc(grid: Grid6, model: Model, params: Params, occ: np.ndarray, tidx: np.ndarray,
              ctl: np.ndarray, rounds: int, tol: float, opts: OocOpts | None = None,
              progress=None, device: int = 0, out: np.ndarray | None = None):
    """pg_solve_ooc: the table solved a tile of x rows at a time with the
    table on the host; returns (V row-major in the store's type, result)."""
    lib = load_library()
    o = opts if opts is not None else ooc_opts()
    n = 1
    for k in range(6):
        n *= int(grid.n[k])
    dt = {STORE_F32: np.float32, STORE_F16: np.float16, STORE_BF16: np.uint16}[o.storage]
    V = out if out is not None else np.empty(n, dtype=dt)
    occ = np.ascontiguousarray(occ, np.uint8)
    tidx = np.ascontiguousarray(tidx, np.int64)
    ctl = np.ascontiguousarray(ctl, np.float32)
    res = OocResult()
    _check(lib.pg_solve_ooc(int(device), C.byref(grid), C.byref(model), C.byref(params),
                            _ptr(occ), _ptr(tidx), tidx.size, _ptr(ctl), ctl.size // 3,
                            int(rounds), float(tol), C.byref(o), _ptr(V), C.byref(res),
                            _wrap_cb(progress), None))
    return V, res


def reach_rows(grid: Grid6, model: Model, params: Params, ctl: np.ndarray, device: int = 0) -> int:
    """pg_reach_rows: one backup's largest x offset, in rows."""
    lib = load_library()
    ctl = np.ascontiguousarray(ctl, np.float32)
    r = C.c_int32()
    _check(lib.pg_reach_rows(int(device), C.byref(grid), C.byref(model), C.byref(params), _ptr(ctl),
                             ctl.size // 3, C.byref(r)))
    return r.value


def probe_step(model: Model, states, controls, dt, nsub, rk2=True, device: int = 0):
    """step_state / step_state_rk2 on the device for states [n, 6] under
    controls [n, 3]; dt and nsub are scalars or [n]; NaN rows = diverged."""
    lib = load_library()
    st = np.ascontiguousarray(np.asarray(states, np.float32).reshape(-1, 6))
    n = st.shape[0]
    u = np.ascontiguousarray(np.broadcast_to(np.asarray(controls, np.float32).reshape(-1, 3), (n, 3)))
    dts = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, np.float32), (n,)))
    ns = np.ascontiguousarray(np.broadcast_to(np.asarray(nsub, np.int32), (n,)))
    out = np.empty((n, 6), np.float32)
    _check(lib.pg_probe_step(int(device), C.byref(model), int(rk2), _ptr(st), _ptr(u), _ptr(dts),
                             _ptr(ns), n, _ptr(out)))
    return out


def probe_traction_gain(controls, knee, device: int = 0):
    """traction_gain on the device for controls [n, 3]."""
    lib = load_library()
    u = np.ascontiguousarray(np.asarray(controls, np.float32).reshape(-1, 3))
    out = np.empty(u.shape[0], np.float32)
    _check(lib.pg_probe_traction_gain(int(device), _ptr(u), C.c_float(knee), u.shape[0], _ptr(out)))
    return out


def measure_peaks(device: int = 0) -> dict:
    """Shared-memory and L2 read bandwidth (GB/s) and FP32 FMA TFLOP/s of the
    device, measured by the library's own probe kernels."""
    lib = load_library()
    s, l2, f = C.c_double(), C.c_double(), C.c_double()
    _check(lib.pg_measure_peaks(int(device), C.byref(s), C.byref(l2), C.byref(f)))
    return {"smem_gbs": s.value, "l2_gbs": l2.value, "fma_tflops": f.value}


class Batch:
    """Many independent tables solved side by side (pg_batch_*)."""

    def __init__(self, device: int = 0, storage: str = "fp16"):
        self._lib = load_library()
        h = C.c_void_p()
        _check(self._lib.pg_batch_create(C.byref(h), int(device), STORAGES[storage]))
        self._h = h
        self.ncells = []

    def close(self) -> None:
        if self._h:
            self._lib.pg_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, grid: Grid6, model: Model, params: Params, occ: np.ndarray, seeds: np.ndarray,
            ctl: np.ndarray, tile_rows: int = 0) -> int:
        occ = np.ascontiguousarray(occ, dtype=np.uint8)
        seeds = np.ascontiguousarray(seeds, dtype=np.int64)
        ctl = np.ascontiguousarray(ctl, dtype=np.float32)
        idx = C.c_int32()
        _check(self._lib.pg_batch_add(self._h, C.byref(grid), C.byref(model), C.byref(params),
                                      _ptr(occ), _ptr(seeds), seeds.size, _ptr(ctl),
                                      ctl.size // 3, int(tile_rows), C.byref(idx)))
        self.ncells.append(int(np.prod(np.array([int(v) for v in grid.n], dtype=np.int64))))
        return idx.value

    def solve(self, iters: int, tol: float, polish_sweeps: int = 0, graph: bool = True):
        res = BatchResult()
        _check(self._lib.pg_batch_solve(self._h, int(iters), float(tol), int(polish_sweeps),
                                        1 if graph else 0, C.byref(res)))
        return res

    def table(self, t: int):
        """(sweeps, last max-norm change) of table t."""
        sw, mx = C.c_int32(), C.c_double()
        _check(self._lib.pg_batch_table(self._h, int(t), C.byref(sw), C.byref(mx), None))
        return sw.value, mx.value

    def get_value(self, t: int) -> np.ndarray:
        ctx = C.c_void_p()
        _check(self._lib.pg_batch_table(self._h, int(t), None, None, C.byref(ctx)))
        out = np.empty(self.ncells[t], dtype=np.float32)
        _check(self._lib.pg_get_value(ctx, _ptr(out)))
        return out


def sweep_noalloc(grid: Grid6, model: Model, params: Params, occ_dev: int, ctl_dev: int,
                  nctl: int, v_in_dev: int, v_out_dev: int, phase: int = 0,
                  stream: int = 0) -> tuple[float, float]:
    """One cell-form sweep on device buffers the caller owns, allocating nothing.

    For callers that cannot allocate device memory themselves (their own pool
    or a fixed budget owns the device).  The arguments are raw device
    addresses (e.g. ``tensor.data_ptr()``) in the layouts pg_sweep_noalloc
    documents: V plane-major, occupancy (h, x, y), controls as three columns.
    Returns (L1 decrease, max decrease).  Grids above 8,388,608 cells are
    refused.
    """
    lib = load_library()
    d, dm = C.c_double(), C.c_double()
    _check(lib.pg_sweep_noalloc(C.byref(grid), C.byref(model), C.byref(params),
                                C.c_void_p(occ_dev), C.c_void_p(ctl_dev), int(nctl),
                                C.c_void_p(v_in_dev), C.c_void_p(v_out_dev), int(phase),
                                C.c_void_p(stream), C.byref(d), C.byref(dm)))
    return d.value, dm.value


def _wrap_cb(progress):
    if progress is None:
        return PROGRESS_CB()

    def _cb(_user, it, d, dm):
        try:
            return 1 if progress(int(it), float(d), float(dm)) else 0
        except Exception:  # never let a Python exception unwind through C
            return 1

    return PROGRESS_CB(_cb)


def solve_value(grid: Grid6, model: Model, params: Params, occ: np.ndarray, tidx: np.ndarray,
                ctl: np.ndarray, iters: int, tol: float, opts: SolveOpts | None = None,
                device: int = 0, progress=None):
    """One-shot mirror of solve_value! (Run.jl:1434-1474): host buffers in,
    host V (row-major float32) and the result record out."""
    lib = load_library()
    with Context(device) as ctx:
        occ = np.ascontiguousarray(occ, dtype=np.uint8)
        ctl = np.ascontiguousarray(ctl, dtype=np.float32)
        tidx = np.ascontiguousarray(tidx, dtype=np.int64)
        n = int(np.prod(np.array([int(v) for v in grid.n], dtype=np.int64)))
        V = np.empty(n, dtype=np.float32)
        res = SolveResult()
        _check(lib.pg_solve_value(ctx._h, C.byref(grid), C.byref(model), C.byref(params),
                                  _ptr(occ), _ptr(tidx), tidx.size, _ptr(ctl), ctl.size // 3,
                                  int(iters), float(tol),
                                  C.byref(opts) if opts is not None else None, _ptr(V),
                                  C.byref(res), _wrap_cb(progress), None))
        return V, res
