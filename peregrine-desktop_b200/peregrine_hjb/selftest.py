"""`solve.py --self-test`: the reference's hot-path self-tests, run on this
library's device code (solver/src/SelfTest.jl).

The reference's rule is that a self-test tests what the tool is for
(SelfTest.jl:3-23); the solver is for minimum-time value tables, so these
are the tests that pin the arithmetic of the table: [6] the control lattice,
[8] the Kuhn simplex interpolant, [5] the traction knee, [4] the velocity
envelope, [2] the integrators' order and divergence, [1] the closed-form
minimum time of a double integrator, and [16]'s encoding checks (dtype round
trips and the u16 saturation guard).  Each runs the device implementation
through the library's probe entry points or a real solve; the output format
and the exit code (0 all passed, 1 otherwise) are the reference's
(SelfTest.jl:29-40, 2040-2064).  The reference's tiling, advice, cost-model
and honing tests cover parts of its tool this library does not replace.

Sample points come from numpy's PCG64 with the reference's seed (4242); the
checks are the reference's properties and bars, not its random stream.
"""
from __future__ import annotations

import math
import sys

import numpy as np

from . import _lib
from .grid import Grid6
from .params import Drivetrain, control_set
from .seeds import target_cells
from .tables import DTYPES, escape_codes, escape_scale_for

f32 = np.float32

_PASS = [0]
_FAIL = [0]


def _check(ok: bool, name: str, detail: str = "") -> bool:
    ok = bool(ok)
    if ok:
        _PASS[0] += 1
    else:
        _FAIL[0] += 1
    print(("  PASS  " if ok else "  FAIL  ") + name + (f"   ({detail})" if detail else ""),
          flush=True)
    return ok


def make_params(**kw) -> _lib.Params:
    """Params() with the reference defaults (PeregrineSolver.jl:918-927)."""
    d = dict(dt=0.05, nsub=4, checks=3, adaptive_checks=1, nearest=0, cap=60.0, ntau=1,
             tau_ratio=2.0, cfl=0.0, tau_min=0.004, tau_max=0.5, hmax=0.0125, ncoarse=0,
             rounds=0, delta0=0.35, rk2=1, vclamp=0, simplex=1)
    d.update(kw)
    p = _lib.Params()
    for k, v in d.items():
        setattr(p, k, float(v) if isinstance(getattr(p, k), float) else int(v))
    return p


def _model(B, A=None, q=None, S=None, D=None, c=None, eps=(5.0, 5.0, 0.15), knee=0.0):
    z9 = np.zeros((3, 3), f32)
    z3 = np.zeros(3, f32)

    def m3(v):
        return z9 if v is None else np.asarray(v, f32).reshape(3, 3)

    return Drivetrain(m3(B), m3(A), z3 if q is None else np.asarray(q, f32), m3(S), m3(D),
                      z3 if c is None else np.asarray(c, f32), np.asarray(eps, f32), float(knee))


def double_integrator(amax: float) -> Drivetrain:
    """A pure double integrator a = amax*u (SelfTest.jl:43-49)."""
    return _model(np.diag([amax, amax, amax]))


def realistic() -> Drivetrain:
    """A model with the shape of a real fit (SelfTest.jl:51-61)."""
    B = [-849.0, -25.8, -69.5, 5.0, -846.8, 0.6, -0.2, -9.6, -64.9]
    A = [-2.13, -0.007, -8.72, -0.064, -4.96, -0.013, 0.039, 0.078, -4.67]
    S = [-11.6, -3.37, 3.29, 2.07, 6.33, 1.00, -0.56, -1.17, -0.28]
    D = [0.021, 0.003, 0.729, 0.001, 0.049, 0.871, -0.0004, -0.0006, 0.312]
    return _model(B, A, (0.0, 0.0, 0.0), S, D, (0.0, 0.0, 0.0), (5.0, 5.0, 0.15), 0.45)


def _context(g: Grid6, V: np.ndarray, cap: float) -> _lib.Context:
    """A context holding table V (row-major) on grid g."""
    ctx = _lib.Context(0)
    occ = np.zeros(g.n[0] * g.n[1] * g.n[2], np.uint8)
    ctx.load_problem(g.to_c(), double_integrator(1.0).to_c(), make_params(cap=cap), occ,
                     control_set(1))
    ctx.set_value(np.ascontiguousarray(V, np.float32))
    return ctx


def _axis_values(g: Grid6) -> list:
    return [g.axis(k) for k in range(6)]


def _table(g: Grid6, fn) -> np.ndarray:
    """fn of the six axis values over every cell, row-major."""
    ax = _axis_values(g)
    mesh = np.meshgrid(*ax, indexing="ij")
    return np.asarray(fn(*mesh), np.float32).reshape(-1)


def test_control_set() -> bool:
    """[6] every lattice control is admissible (SelfTest.jl:574-593)."""
    print("\n[6] control set")
    ok = True
    for level in range(1, 7):
        cs = control_set(level).reshape(3, -1).T
        l1 = np.abs(cs).sum(axis=1)
        worst = float(l1.max())
        onbound = int(np.sum(np.abs(l1 - 1) < 1e-5))
        uniq = len({tuple(r) for r in cs.tolist()})
        ok &= _check(worst <= 1 + 1e-5 and onbound == len(cs) - 1 and uniq == len(cs),
                     f"level {level} admissible, on the boundary, no duplicates",
                     f"{len(cs)} controls, max 1-norm {worst:.6f}")
    u = control_set(4).reshape(3, -1).T
    mix = np.stack([u[:, 0] + u[:, 1] - u[:, 2], u[:, 0] - u[:, 1] - u[:, 2],
                    u[:, 0] - u[:, 1] + u[:, 2], u[:, 0] + u[:, 1] + u[:, 2]], axis=1)
    worst = float(np.abs(mix).max())
    ok &= _check(worst <= 1 + 1e-5, "no wheel power exceeds 1", f"max |wheel| = {worst:.6f}")
    return ok


def test_kuhn() -> bool:
    """[8] the Kuhn simplex interpolant on the device (SelfTest.jl:407-515)."""
    print("\n[8] Kuhn simplex interpolation")
    g = Grid6.make((7, 6, 8, 5, 5, 5), (0.0, 0.0, -math.pi, -100.0, -100.0, -4.0),
                   (120.0, 100.0, math.pi, 100.0, 100.0, 4.0))
    cap = 1.0e6
    co = np.array([0.017, -0.023, 0.31, 0.0041, -0.0072, 0.11], f32)
    c0 = f32(3.5)

    def fexact(s):
        s = np.asarray(s, f32)
        acc = np.full(s.shape[0], c0, f32)
        for k in range(6):
            acc = (acc + (co[k] * s[:, k]).astype(f32)).astype(f32)
        return acc

    V = _table(g, lambda *a: fexact(np.stack([x.reshape(-1) for x in a], axis=1)))
    rng = np.random.default_rng(4242)

    def samples(n, lo, span):
        return (np.asarray(lo) + rng.random((n, 6)) * np.asarray(span)).astype(f32)

    lo = [0.0, 0.0, -3.0, -90.0, -90.0, -3.5]
    span = [110.0, 90.0, 5.2, 180.0, 180.0, 7.0]
    with _context(g, V, cap) as ctx:
        s = samples(4000, lo, span)
        v, gr = ctx.probe_interp(s, kuhn=True, cap=cap, grads=True)
        worst_v = float(np.max(np.abs(v.astype(np.float64) - fexact(s))))
        worst_g = float(np.max(np.abs(gr.astype(np.float64) - co[None, :])))
        ok = _check(worst_v < 2.0e-3, "exact on affine data", f"worst value error {worst_v:.3g}")
        ok &= _check(worst_g < 2.0e-4, "gradient exact on affine data",
                     f"worst gradient error {worst_g:.3g}")
        s = samples(2000, lo, span)
        m = ctx.probe_interp(s, kuhn=False, cap=cap)
        vk = ctx.probe_interp(s, kuhn=True, cap=cap)
        worst_m = float(np.max(np.abs(vk.astype(np.float64) - m)))
        off = ctx.probe_interp(np.array([[5, 5, 0, 400, 0, 0]], f32), kuhn=True, cap=cap)[0]
        nan = ctx.probe_interp(np.array([[5, 5, 0, np.nan, 0, 0]], f32), kuhn=True, cap=cap)[0]
    with _context(g, np.full(g.ncells, 2.75, f32), cap) as ctx:
        vc = ctx.probe_interp(samples(2000, lo, span), kuhn=True, cap=cap)
        worst_c = float(np.max(np.abs(vc.astype(np.float64) - 2.75)))
    ok &= _check(worst_c < 1.0e-5, "weights are a partition of unity",
                 f"worst constant error {worst_c:.3g}")
    Vr = (rng.random(g.ncells) * 10).astype(f32)
    base = samples(3000, [0.0, 0.0, -3.0, -80.0, -80.0, -3.0], [100.0, 80.0, 5.2, 160.0, 160.0, 6.0])
    ks = rng.integers(0, 6, size=3000)
    lo_s, hi_s = base.copy(), base.copy()
    for i, k in enumerate(ks):
        pl = int(rng.integers(1, g.n[k] - 1))
        base[i, k] = g.axisvalue(k, pl)
        d = f32(f32(1e-3) * g.step[k])
        lo_s[i] = base[i]
        hi_s[i] = base[i]
        lo_s[i, k] = f32(base[i, k] - d)
        hi_s[i, k] = f32(base[i, k] + d)
    with _context(g, Vr, cap) as ctx:
        a = ctx.probe_interp(lo_s, kuhn=True, cap=cap)
        b = ctx.probe_interp(hi_s, kuhn=True, cap=cap)
        am = ctx.probe_interp(lo_s, kuhn=False, cap=cap)
        bm = ctx.probe_interp(hi_s, kuhn=False, cap=cap)
    worst_j = float(np.max(np.abs(a.astype(np.float64) - b)))
    worst_ml = float(np.max(np.abs(am.astype(np.float64) - bm)))
    ok &= _check(worst_j < 0.2, "continuous across cell faces",
                 f"largest jump {worst_j:.4f} over 0.002 of a cell on a 0..10 table "
                 f"(multilinear {worst_ml:.4f})")
    ok &= _check(worst_m < 3.0e-3, "agrees with multilinear on affine data",
                 f"worst disagreement {worst_m:.3g}")
    ok &= _check(off == cap and nan == cap, "rejects out-of-envelope and non-finite states",
                 f"{off}, {nan}")
    return ok


def test_nan_knee() -> bool:
    """[5] a NaN or zero knee means no saturation (SelfTest.jl:554-564)."""
    print("\n[5] NaN traction knee")
    g = _lib.probe_traction_gain([[0.5, 0.5, 0.0], [0.5, 0.5, 0.0]], float("nan"))
    ok = _check(g[0] == 1.0, "NaN knee gives unit gain")
    ok &= _check(_lib.probe_traction_gain([[0.5, 0.5, 0.0]], 0.0)[0] == 1.0,
                 "zero knee gives unit gain")
    gn = float(_lib.probe_traction_gain([[1.0, 0.0, 0.0]], 0.45)[0])
    ok &= _check(0.0 < gn < 1.0, "an active knee saturates", f"gain {gn:.4f}")
    return ok


def test_velocity_envelope() -> bool:
    """[4] outside the velocity envelope is rejected, not clamped
    (SelfTest.jl:524-540)."""
    print("\n[4] velocity envelope")
    g = Grid6.make((5, 5, 4, 5, 5, 5), (0.0, 0.0, -math.pi, -150.0, -150.0, -8.0),
                   (100.0, 100.0, math.pi, 150.0, 150.0, 8.0))
    cap = 30.0
    with _context(g, np.ones(g.ncells, f32), cap) as ctx:
        pts = np.array([[50, 50, 0, 100, 0, 0], [50, 50, 0, 400, 0, 0],
                        [50, 50, 0, np.nan, 0, 0]], f32)
        inside, outside, nan = ctx.probe_interp(pts, cap=cap)
        clamped = ctx.probe_interp(pts[1:2], cap=cap, vclamp=True)[0]
    ok = _check(abs(inside - 1.0) <= 1e-6, "inside the envelope interpolates", f"{inside}")
    ok &= _check(outside == cap, "outside the envelope is rejected", f"{outside}")
    ok &= _check(abs(clamped - 1.0) <= 1e-6, "vclamp = true restores clamping", f"{clamped}")
    ok &= _check(nan == cap, "a NaN coordinate is rejected, not rounded", f"{nan}")
    return ok


def test_integrator() -> bool:
    """[2] RK2 is second order, Euler first; divergence is reported
    (SelfTest.jl:208-258)."""
    print("\n[2] integrator order")
    m = realistic().to_c()
    s0 = np.array([[10.0, 20.0, 0.3, 40.0, -25.0, 1.5]], f32)
    u = np.array([[0.6, -0.3, 0.1]], f32)
    dt = 0.05
    ref = _lib.probe_step(m, s0, u, dt, 4096, rk2=True)[0].astype(np.float64)

    def err(rk2, nsub):
        return float(np.max(np.abs(_lib.probe_step(m, s0, u, dt, nsub, rk2=rk2)[0] - ref)))

    e_eul, e_rk2 = err(False, 4), err(True, 4)
    ok = _check(e_rk2 < e_eul / 5, "midpoint beats Euler at the same substeps",
                f"Euler {e_eul:.4g}, midpoint {e_rk2:.4g}, {e_eul / e_rk2:.1f}x better")
    order = math.log2(err(True, 4) / err(True, 8))
    ok &= _check(order > 1.5, "midpoint converges at order > 1.5", f"observed order {order:.2f}")
    oe = math.log2(err(False, 4) / err(False, 8))
    ok &= _check(oe < 1.4, "Euler converges at order ~1", f"observed order {oe:.2f}")
    spin = np.array([[0.0, 0.0, 0.0, 0.0, 0.0, 30.0]], f32)
    for rk2, name in ((False, "step_state"), (True, "step_state_rk2")):
        got = _lib.probe_step(m, spin, [[0.0, 0.0, 1.0]], 2.0, 160, rk2=rk2)[0]
        ok &= _check(not np.all(np.isfinite(got)), f"{name} reports divergence instead of throwing",
                     "non-finite state returned")
    return ok


def test_min_time() -> bool:
    """[1] the closed-form minimum time of a double integrator
    (SelfTest.jl:90-199), solved on the device."""
    print("\n[1] minimum time against the closed-form bang-bang solution")
    amax = 100.0
    m = double_integrator(amax).to_c()
    g = Grid6.make((81, 5, 4, 33, 5, 5), (0.0, 0.0, -math.pi, -100.0, -100.0, -2.0),
                   (200.0, 200.0, math.pi, 100.0, 100.0, 2.0))
    occ = np.zeros(g.n[0] * g.n[1] * g.n[2], np.uint8)
    cap = 30.0
    ttol = [float(f32(g.step[k] * f32(0.5))) for k in range(6)]
    tcells = target_cells(g, (100.0, 100.0, 0.0, 0.0, 0.0, 0.0), ttol)
    ctl = control_set(4)
    common = dict(dt=0.05, nsub=4, cap=cap)
    schemes = {
        "legacy": make_params(**common, checks=3, adaptive_checks=0, ntau=1, cfl=0.0, ncoarse=0,
                              rounds=0, rk2=0, vclamp=0),
        "ladder": make_params(**common, checks=2, adaptive_checks=1, ntau=4, cfl=1.0,
                              hmax=0.0125, ncoarse=0, rounds=0, rk2=1),
        "now": make_params(**common, checks=2, adaptive_checks=1, ntau=4, cfl=1.0, hmax=0.0125,
                           ncoarse=8, rounds=2, rk2=1),
    }
    ds = (20.0, 40.0, 60.0)
    want = [2.0 * math.sqrt(d / amax) for d in ds]
    pts = np.array([[100.0 - d, 100.0, 0.0, 0.0, 0.0, 0.0] for d in ds], f32)
    got = {}
    for name, p in schemes.items():
        opts = _lib.default_opts(warm_start=int(p.ncoarse > 0))
        with _lib.Context(0) as ctx:
            ctx.load_problem(g.to_c(), m, p, occ, ctl)
            ctx.solve(tcells, 600, 1e-4, opts)
            got[name] = [float(v) for v in ctx.probe_interp(pts, kuhn=True, cap=cap)]
    gl, gd, gn = got["legacy"], got["ladder"], got["now"]
    for i, d in enumerate(ds):
        print(f"        d = {d:2.0f} cm  exact {want[i]:.3f}  fixed-dt {gl[i]:.3f} "
              f"({100 * (gl[i] - want[i]) / want[i]:+.1f}%)  +ladder {gd[i]:.3f} "
              f"({100 * (gd[i] - want[i]) / want[i]:+.1f}%)  +fast-search {gn[i]:.3f} "
              f"({100 * (gn[i] - want[i]) / want[i]:+.1f}%)")
    ml, md, mn = sum(gl) / 3, sum(gd) / 3, sum(gn) / 3
    ok = _check(mn <= md * 1.08, "cheap search costs little where it can gain nothing",
                f"exhaustive {md:.3f} s, rotating scan {mn:.3f} s, {100 * (mn - md) / md:+.1f}%")
    ok &= _check(md <= ml * 1.02, "the horizon ladder does not lose ground either",
                 f"fixed dt {ml:.3f} s, ladder {md:.3f} s, {100 * (md - ml) / ml:+.1f}%")
    ex = [gn[i] - want[i] for i in range(3)]
    slope = (ex[2] - ex[0]) / (want[2] - want[0])
    intercept = ex[0] - slope * want[0]
    print(f"        excess = {intercept:.3f} s fixed + {100 * slope:.1f}% of the journey")
    ok &= _check(intercept < 0.45, "terminal excess is bounded", f"{intercept:.3f} s")
    ok &= _check(slope < 0.20, "no significant per-second loss in the cruise",
                 f"{100 * slope:.1f}% per second")
    return ok


def _decode(dt, buf, sc, es, base):
    """Section 6 / 6.1 decoding of one encoded buffer: (time or inf, escape
    time or None) per cell."""
    if dt == "f32":
        fl = np.frombuffer(buf, np.float32)
        out = []
        for v in fl:
            if np.isnan(v):
                out.append((math.inf, None))
            elif v < 0:
                out.append((math.inf, -float(v)))
            else:
                out.append((float(v), None))
        return out
    raws = np.frombuffer(buf, np.uint8 if dt == "u8" else np.uint16).astype(np.int64)
    sentinel = int(DTYPES[dt]["sentinel"])
    out = []
    for r in raws:
        if r == sentinel:
            out.append((math.inf, None))
        elif r >= base:
            out.append((math.inf, es * (r - base) ** 2))
        else:
            out.append((r * sc, None))
    return out


def test_encoding() -> bool:
    """[16] the escape band survives encoding and a real value never lands in
    it (SelfTest.jl:1623-1702), through the device encoder."""
    print("\n[16] table encoding and the escape band")
    cap = 30.0
    g = Grid6.make((4, 4, 4, 4, 4, 4), (0.0, 0.0, -math.pi, -1.0, -1.0, -1.0),
                   (3.0, 3.0, math.pi, 1.0, 1.0, 1.0))
    rng = np.random.default_rng(4242)
    n = g.ncells
    after = (rng.random(n) * cap).astype(f32)
    kind = rng.integers(0, 3, size=n)
    after[kind == 1] = f32(cap)                      # unreached
    esc = kind == 2
    after[esc] = -(rng.random(int(esc.sum())) * cap).astype(f32)  # escape times
    nesc = int(esc.sum())
    ok = True
    with _context(g, after, cap) as ctx:
        for dt in ("u16", "u8", "f32"):
            sc = DTYPES[dt]["scale"]
            es = escape_scale_for(dt, cap)
            base = int(DTYPES[dt]["escape_base"])
            buf, _, _ = ctx.encode(dt, sc, es, 0, n)
            dec = _decode(dt, bytes(buf[: n * DTYPES[dt]["bytes"]]), sc, es, base)
            nboth = nesc_rt = nreach = 0
            worst = 0.0
            for i, (v, e) in enumerate(dec):
                if math.isfinite(v):
                    nreach += 1
                if after[i] < 0:
                    nesc_rt += 1
                    if math.isfinite(v):
                        nboth += 1
                    if e is not None:
                        worst = max(worst, abs(e - float(-after[i])))
                elif 0 <= after[i] < cap:
                    if e is not None:
                        nboth += 1
            ok &= _check(nboth == 0, f"{dt}: no cell decodes as both reachable and escapable",
                         f"{nboth} of {n}")
            ok &= _check(nesc_rt == nesc, f"{dt}: every escape cell survived encoding",
                         f"{nesc_rt} of {nesc}")
            tol = 1.0e-3 if dt == "f32" else es * (2 * (escape_codes(dt) - 1) + 1) + 1.0e-6
            ok &= _check(worst <= tol, f"{dt}: escape times round-trip inside the band's step",
                         f"worst {worst:.4f} s, band step at the top {tol:.4f} s")
            nterm = int(np.sum((after >= 0) & (after < cap)))
            if base == 0 or cap / sc < base:
                ok &= _check(nreach == nterm,
                             f"{dt}: reachable count is unchanged by the escape band",
                             f"{nreach} vs {nterm}")
            else:
                ok &= _check(nreach <= nterm, f"{dt}: cannot represent a {cap} s cap, so it "
                             "saturates", f"{nreach} of {nterm} representable below "
                             f"{base * sc:.3f} s")
    probe = np.full(g.ncells, 1.0, f32)
    probe[0] = f32(0.9 * 0xFC00 * 0.001)
    probe[1] = f32(1.1 * 0xFC00 * 0.001)
    with _context(g, probe, 100.0) as ctx:
        buf, _, _ = ctx.encode("u16", 0.001, escape_scale_for("u16", 100.0), 0, 2)
    p16 = np.frombuffer(bytes(buf[:4]), np.uint16)
    ok &= _check(p16[0] < 0xFC00 and p16[1] == 0xFFFF,
                 "a real value above the band saturates to unreachable, not into it",
                 f"{int(p16[0])}, {int(p16[1])}")
    return ok


def self_test() -> int:
    """Run every self-test; returns the process exit code."""
    _PASS[0] = _FAIL[0] = 0
    print("PeregrineSolver self-test")
    try:
        _lib.load_library()
        c = _lib.Context(0)
        c.close()
        backend = "cuda"
    except Exception as e:  # no device: the product has no CPU path
        print("backend: none")
        print(f"ERROR the self-test needs the CUDA library and a device: {e}", file=sys.stderr)
        return 1
    print("backend:", backend)
    for t in (test_control_set, test_kuhn, test_nan_knee, test_velocity_envelope,
              test_integrator, test_min_time, test_encoding):
        try:
            t()
        except Exception as e:
            _check(False, f"{t.__name__} raised", f"{type(e).__name__}: {e}")
    print(f"\n{_PASS[0]} passed, {_FAIL[0]} failed")
    return 0 if _FAIL[0] == 0 else 1
