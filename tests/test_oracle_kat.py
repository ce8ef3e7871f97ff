"""The CPU oracle against the reference's own known answers.

Every test here pins the oracle (oracle/pg_oracle.c) to a fixed point the
reference states: its self-tests (solver/src/SelfTest.jl) and the worked
examples of docs/TABLE_FORMAT.md.  No GPU.
"""
import math

import numpy as np
import pytest

f32 = np.float32


def realistic(og):
    """_realistic() (SelfTest.jl:51-61)"""
    B = (-849.0, -25.8, -69.5, 5.0, -846.8, 0.6, -0.2, -9.6, -64.9)
    A = (-2.13, -0.007, -8.72, -0.064, -4.96, -0.013, 0.039, 0.078, -4.67)
    S = (-11.6, -3.37, 3.29, 2.07, 6.33, 1.00, -0.56, -1.17, -0.28)
    D = (0.021, 0.003, 0.729, 0.001, 0.049, 0.871, -0.0004, -0.0006, 0.312)
    return og.model(B, A, (0, 0, 0), S, D, (0, 0, 0), (5.0, 5.0, 0.15), 0.45)


def test_body_accel_worked_example(og):
    """TABLE_FORMAT.md §8.7: u_raw=(1,0,0), knee 0.55 -> gain 0.5218,
    a = (166.2, -2.78, 0.067) from rest."""
    Au = (318.44, 6.12, -4.87, -5.33, 241.07, 3.94, 0.128, -0.061, 13.706)
    z9 = (0,) * 9
    m = og.model(Au, z9, (0, 0, 0), z9, z9, (0, 0, 0), (5, 5, 0.15), 0.55)
    L = og.lib()
    gain = L.og_traction_gain(1.0, 0.0, 0.0, 0.55)
    assert abs(gain - 0.5218) < 5e-5
    out = np.zeros(3, np.float32)
    L.og_body_accel(m, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, out.ctypes.data)
    # the worked example multiplies by the printed (4-digit) gain, so allow
    # half a printed digit plus 318.44 * 5e-5 of gain rounding
    assert abs(out[0] - 166.2) < 0.05 + 318.44 * 5e-5
    assert abs(out[1] - (-2.78)) < 0.005 + 5.33 * 5e-5
    assert abs(out[2] - 0.067) < 0.0005 + 0.128 * 5e-5
    # and exactly A_u * gain in Float32
    assert out[0] == np.float32(np.float32(318.44) * np.float32(gain))


def test_nan_knee(og):
    """SelfTest [5] (SelfTest.jl:554-564)"""
    L = og.lib()
    assert L.og_traction_gain(0.5, 0.5, 0.0, float("nan")) == 1.0
    assert L.og_traction_gain(0.5, 0.5, 0.0, 0.0) == 1.0
    g = L.og_traction_gain(1.0, 0.0, 0.0, 0.45)
    assert 0.0 < g < 1.0


@pytest.mark.parametrize("level,count", [(1, 7), (2, 19), (3, 39), (4, 67), (5, 103), (6, 147)])
def test_control_set(og, level, count):
    """SelfTest [6] (SelfTest.jl:574-593): admissible, on the boundary, unique,
    coast first; the counts of PeregrineSolver.jl:315-316."""
    c = og.control_set(level).reshape(3, -1).T
    assert len(c) == count
    assert np.all(c[0] == 0)
    l1 = np.abs(c).sum(axis=1)
    assert l1.max() <= 1 + 1e-5
    assert np.sum(np.abs(l1 - 1) < 1e-5) == len(c) - 1
    assert len({tuple(r) for r in c}) == len(c)
    mix = np.stack([c[:, 0] + c[:, 1] - c[:, 2], c[:, 0] - c[:, 1] - c[:, 2],
                    c[:, 0] - c[:, 1] + c[:, 2], c[:, 0] + c[:, 1] + c[:, 2]], axis=1)
    assert np.abs(mix).max() <= 1 + 1e-5
    # effort order: L1 then L2 non-decreasing
    l2 = (c ** 2).sum(axis=1)
    keys = list(zip(l1.round(6), l2.round(6)))
    assert keys == sorted(keys)


def _state_err(a, b):
    return max(abs(float(getattr(a, k)) - float(getattr(b, k))) for k in ("x", "y", "h", "vx", "vy", "w"))


def test_integrator_order(og):
    """SelfTest [2] (SelfTest.jl:207-258)"""
    m = realistic(og)
    L = og.lib()
    s0 = og.state(10.0, 20.0, 0.3, 40.0, -25.0, 1.5)
    u = (0.6, -0.3, 0.1)
    dt = 0.05
    ref = L.og_step_state_rk2(m, s0, *u, dt, 4096)
    e_eul = _state_err(L.og_step_state(m, s0, *u, dt, 4), ref)
    e_rk2 = _state_err(L.og_step_state_rk2(m, s0, *u, dt, 4), ref)
    assert e_rk2 < e_eul / 5
    e8 = _state_err(L.og_step_state_rk2(m, s0, *u, dt, 8), ref)
    assert math.log2(e_rk2 / e8) > 1.5
    e8e = _state_err(L.og_step_state(m, s0, *u, dt, 8), ref)
    assert math.log2(e_eul / e8e) < 1.4


def test_divergence_is_reported(og):
    """SelfTest [2] second half: a diverging step returns a non-finite state."""
    m = realistic(og)
    L = og.lib()
    spin = og.state(0, 0, 0, 0, 0, 30.0)
    for f in (L.og_step_state, L.og_step_state_rk2):
        s = f(m, spin, 0.0, 0.0, 1.0, 2.0, 160)
        vals = [getattr(s, k) for k in ("x", "y", "h", "vx", "vy", "w")]
        assert not all(math.isfinite(v) for v in vals)


def test_velocity_envelope(og):
    """SelfTest [4] (SelfTest.jl:524-540)"""
    g = og.grid_make((5, 5, 4, 5, 5, 5), (0, 0, -math.pi, -150, -150, -8),
                     (100, 100, math.pi, 150, 150, 8))
    V = np.ones(5 * 5 * 4 * 5 * 5 * 5, np.float32)
    L = og.lib()
    cap = 30.0
    inside = L.og_interp(V.ctypes.data, g, og.state(50, 50, 0, 100, 0, 0), 0, cap, 0)
    outside = L.og_interp(V.ctypes.data, g, og.state(50, 50, 0, 400, 0, 0), 0, cap, 0)
    clamped = L.og_interp(V.ctypes.data, g, og.state(50, 50, 0, 400, 0, 0), 0, cap, 1)
    nan = L.og_interp(V.ctypes.data, g, og.state(50, 50, 0, float("nan"), 0, 0), 0, cap, 0)
    assert abs(inside - 1) < 1e-6 and outside == cap and abs(clamped - 1) < 1e-6 and nan == cap


def test_kuhn_and_multilinear_on_affine_data(og):
    """SelfTest [8] (SelfTest.jl:407-515), with a numpy stream in place of
    MersenneTwister(4242): the properties, not the sample sequence."""
    n = (7, 6, 8, 5, 5, 5)
    g = og.grid_make(n, (0, 0, -math.pi, -100, -100, -4), (120, 100, math.pi, 100, 100, 4))
    co = np.array([0.017, -0.023, 0.31, 0.0041, -0.0072, 0.11], np.float32)
    c0 = f32(3.5)
    axes = [np.array([f32(g.lo[k]) + f32(i) * f32(g.step[k]) for i in range(n[k])], np.float32)
            for k in range(6)]
    mesh = np.meshgrid(*axes, indexing="ij")
    V = (c0 + sum(co[k] * mesh[k] for k in range(6))).astype(np.float32).reshape(-1)
    L = og.lib()
    cap = 1.0e6
    rng = np.random.default_rng(4242)
    grad = np.zeros(6, np.float32)
    wv = wg = wm = 0.0
    for _ in range(1500):
        s = (rng.random() * 110, rng.random() * 90, -3.0 + rng.random() * 5.2,
             -90 + rng.random() * 180, -90 + rng.random() * 180, -3.5 + rng.random() * 7)
        sf = [float(f32(v)) for v in s]
        exact = float(c0 + sum(co[k] * f32(sf[k]) for k in range(6)))
        v = L.og_interp_kuhn(V.ctypes.data, g, og.state(*sf), cap, 0, grad.ctypes.data)
        b = L.og_interp(V.ctypes.data, g, og.state(*sf), 0, cap, 0)
        wv = max(wv, abs(v - exact))
        wg = max(wg, float(np.max(np.abs(grad - co))))
        wm = max(wm, abs(v - b))
    assert wv < 2e-3 and wg < 2e-4 and wm < 3e-3
    Vc = np.full(V.size, 2.75, np.float32)
    for _ in range(500):
        sf = (rng.random() * 110, rng.random() * 90, -3.0 + rng.random() * 5.2,
              -90 + rng.random() * 180, -90 + rng.random() * 180, -3.5 + rng.random() * 7)
        assert abs(L.og_interp_kuhn(Vc.ctypes.data, g, og.state(*sf), cap, 0, None) - 2.75) < 1e-5
    # continuity across a cell face
    Vr = (rng.random(V.size) * 10).astype(np.float32)
    worst = 0.0
    for _ in range(500):
        base = [rng.random() * 100, rng.random() * 80, -3.0 + rng.random() * 5.2,
                -80 + rng.random() * 160, -80 + rng.random() * 160, -3.0 + rng.random() * 6]
        k = int(rng.integers(0, 6))
        pl = int(rng.integers(1, n[k] - 1))
        base[k] = float(axes[k][pl])
        lo = list(base); hi = list(base)
        lo[k] -= 1e-3 * float(g.step[k]); hi[k] += 1e-3 * float(g.step[k])
        a = L.og_interp_kuhn(Vr.ctypes.data, g, og.state(*lo), cap, 0, None)
        b = L.og_interp_kuhn(Vr.ctypes.data, g, og.state(*hi), cap, 0, None)
        worst = max(worst, abs(a - b))
    assert worst < 0.2
    off = L.og_interp_kuhn(V.ctypes.data, g, og.state(5, 5, 0, 400, 0, 0), cap, 0, None)
    nan = L.og_interp_kuhn(V.ctypes.data, g, og.state(5, 5, 0, float("nan"), 0, 0), cap, 0, None)
    assert off == cap and nan == cap


def _escape_scale_for(dtype, cap):
    codes = {"u8": 0xFF - 0xE0, "u16": 0xFFFF - 0xFC00}.get(dtype, 0)
    return 0.0 if codes <= 1 else cap / (codes - 1) ** 2


def test_u16_band_saturation_kat(og):
    """SelfTest.jl:1697-1702: a real value above the band saturates to the
    sentinel instead of decoding as an escape."""
    probe = np.array([f32(0.9 * 0xFC00 * 0.001), f32(1.1 * 0xFC00 * 0.001)], np.float32)
    buf, _, _ = og.encode(probe, "u16", 0.001, 100.0, _escape_scale_for("u16", 100.0))
    codes = buf.view(np.uint16)
    assert codes[0] < 0xFC00 and codes[1] == 0xFFFF


@pytest.mark.parametrize("dtype", ["u16", "u8", "f32"])
def test_encode_round_trip(og, dtype):
    """The card round trip of SelfTest.jl:1618-1693, decoded by the rules of
    TABLE_FORMAT.md §6 / §6.1."""
    cap = 30.0
    rng = np.random.default_rng(7)
    reach = rng.uniform(0, cap, 400).astype(np.float32)
    esc = -rng.uniform(0.0, cap, 200).astype(np.float32)
    V = np.concatenate([reach, esc, np.array([cap, np.inf, np.nan, 0.0, -0.0], np.float32)])
    sc = {"u16": 0.001, "u8": 0.025, "f32": 1.0}[dtype]
    es = _escape_scale_for(dtype, cap)
    buf, nreach, nesc = og.encode(V, dtype, sc, cap, es)
    base = {"u16": 0xFC00, "u8": 0xE0, "f32": 0}[dtype]
    sentinel = {"u16": 0xFFFF, "u8": 0xFF, "f32": 0}[dtype]
    if dtype == "f32":
        fl = buf.view(np.float32)
    else:
        raws = buf.view(np.uint16) if dtype == "u16" else buf
    assert nesc == 200
    both = 0
    worst = 0.0
    for i, v in enumerate(V):
        if dtype == "f32":
            r = fl[i]
            if math.isnan(r):
                dv, de = math.inf, None
            elif r < 0:
                dv, de = math.inf, -float(r)
            else:
                dv, de = float(r), None
        else:
            r = int(raws[i])
            if r == sentinel:
                dv, de = math.inf, None
            elif r >= base:
                dv, de = math.inf, es * (r - base) ** 2
            else:
                dv, de = r * sc, None
        if v < 0 and math.isfinite(v):
            if math.isfinite(dv):
                both += 1
            if de is not None:
                worst = max(worst, abs(de - (-float(v))))
        elif 0 <= v < cap and de is not None:
            both += 1
    assert both == 0
    codes = 0 if dtype == "f32" else sentinel - base
    tol = 1e-3 if dtype == "f32" else es * (2 * (codes - 1) + 1) + 1e-6
    assert worst <= tol


def test_table_format_worked_example():
    """TABLE_FORMAT.md §7: state -> indices -> flat index 28035145 -> chunk 3,
    byte 5738642; and the §6 decode of three raw codes."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "peregrine-desktop_b200"))
    from peregrine_hjb.tables import escape_scale_for

    n = [46, 46, 24, 13, 13, 13]
    mn = [23.0, 23.0, -3.14159265, -170.0, -170.0, -8.0]
    mx = [343.0, 343.0, 3.14159265, 170.0, 170.0, 8.0]
    wrap = [False, False, True, False, False, False]
    step = [(2 * math.pi / n[k]) if wrap[k] else (mx[k] - mn[k]) / (n[k] - 1) for k in range(6)]
    state = [100.0, 200.0, 1.0, 50.0, -30.0, 2.5]
    idx6 = []
    for k in range(6):
        i = round((state[k] - mn[k]) / step[k])
        idx6.append(i % n[k] if wrap[k] else min(max(i, 0), n[k] - 1))
    assert idx6 == [11, 25, 16, 8, 5, 8]
    flat = 0
    for k in range(6):
        flat = flat * n[k] + idx6[k]
    assert flat == 28035145
    shift = 23
    assert flat >> shift == 3
    assert (flat & ((1 << shift) - 1)) * 2 == 5738642
    es = escape_scale_for("u16", 60.0)
    assert abs(es - 5.7448e-05) < 1e-8
    decode = lambda r: (r * 0.001, None) if r < 0xFC00 else (math.inf, None if r == 0xFFFF else es * (r - 0xFC00) ** 2)
    assert abs(decode(12345)[0] - 12.345) < 1e-12
    v, e = decode(64612)
    assert v == math.inf and abs(e - 0.57) < 0.005
    assert decode(65535) == (math.inf, None)


def test_target_cells_nearest_fallback(og):
    """target_cells (Pipeline.jl:504-536): a tolerance below half a cell still
    seeds the single nearest cell."""
    g = og.grid_make((10, 10, 8, 5, 5, 5), (0, 0, -math.pi, -100, -100, -4), (90, 90, math.pi, 100, 100, 4))
    cells = og.target_cells(g, (33.0, 47.0, 0.1, 0, 0, 0), (0.1,) * 6)
    assert len(cells) == 1
    half = [float(g.step[k]) * 0.5 for k in range(6)]
    many = og.target_cells(g, (30.0, 40.0, 0.0, 0, 0, 0), half)
    assert len(many) >= 1


def test_golden_fixed_point_is_a_fixed_point(og):
    """tests/golden/tiny_fixed_point.npz (made by make_golden.py from the
    oracle) really is the oracle's converged table: one more oracle sweep
    moves no cell by more than the 1e-4 s stop tolerance, and its argmin is
    the one stored."""
    import os
    from peregrine_hjb.synth import Problem
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "tiny_fixed_point.npz"))
    pr = Problem("tiny", seed=5)
    g = og.copy_struct(pr.grid.to_c(), og.OGrid)
    m = og.copy_struct(pr.model.to_c(), og.OModel)
    p = og.copy_struct(pr.params, og.OParams)
    V = gold["V"]
    assert V.shape == (pr.ncells,) and np.all(V[pr.seeds] == 0)
    _, _, mx, am = og.sweep_jacobi(V, pr.occ, g, m, pr.ctl, p, phase=int(gold["iterations"]),
                                   argmin=True)
    assert mx <= 1e-4
    assert np.array_equal(am, gold["argmin"])
