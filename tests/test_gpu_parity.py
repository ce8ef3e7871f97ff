"""The CUDA path against the CPU oracle, through the C ABI.

Bit-exact where the kernel keeps the reference's operation order (the
cell-form kernel and the exact stencil instantiation); within a stated
tolerance where it does not (the FMA stencils: 2e-5 s per sweep; at the
fixed point 1e-3 s max and 1.5e-4 s RMS; argmin agreement >= 99.9%).
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

from conftest import gpu_available
from peregrine_hjb import _lib
from peregrine_hjb.synth import Problem

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

FMA_SWEEP_TOL = 2e-5        # s, one sweep, FMA stencils vs oracle
FMA_FIXED_POINT_MAX = 1e-3  # s, converged tables, FMA stencils vs oracle, max
# s, converged tables, FMA stencils vs oracle, RMS.  Two FP32 evaluations of
# the same ~945 undiscounted sweeps in different rounding orders each
# random-walk a few ulp per sweep; the oracle's own walk is ~7e-5 s RMS, so
# 1e-4 is the noise floor of the comparison and 1.5e-4 leaves it room.
FMA_FIXED_POINT_RMS = 1.5e-4
ARGMIN_AGREE = 0.999


def oracle_structs(og, pr):
    g = og.copy_struct(pr.grid.to_c(), og.OGrid)
    m = og.copy_struct(pr.model.to_c(), og.OModel)
    p = og.copy_struct(pr.params, og.OParams)
    return g, m, p


def init_value(pr):
    V = np.full(pr.ncells, np.float32(pr.params.cap), np.float32)
    V[pr.seeds] = 0.0
    return V


@pytest.fixture(scope="module")
def tiny():
    return Problem("tiny", seed=5)


@pytest.fixture(scope="module")
def tiny_state(og, tiny):
    """A structured V: the initial table after four oracle sweeps."""
    g, m, p = oracle_structs(og, tiny)
    V = init_value(tiny)
    for it in range(4):
        V, _, _, _ = og.sweep_jacobi(V, tiny.occ, g, m, tiny.ctl, p, phase=it)
        V[tiny.seeds] = 0.0
    return V


def gpu_ctx(pr, storage="fp32", params=None):
    ctx = _lib.Context(0)
    ctx.load_problem(pr.grid.to_c(), pr.model.to_c(), params or pr.params, pr.occ, pr.ctl, storage)
    return ctx


@pytest.mark.parametrize("kernel", [_lib.KERNEL_CELLFORM, _lib.KERNEL_STENCIL_EXACT])
def test_one_sweep_bit_exact(og, tiny, tiny_state, kernel):
    g, m, p = oracle_structs(og, tiny)
    want, tot, mx, am = og.sweep_jacobi(tiny_state, tiny.occ, g, m, tiny.ctl, p, phase=4, argmin=True)
    with gpu_ctx(tiny) as ctx:
        ctx.set_value(tiny_state)
        d, dm, gam = ctx.sweep(phase=4, kernel=kernel, argmin=True)
        got = ctx.get_value()
    assert np.array_equal(got, want), f"max |dV| {np.max(np.abs(got - want))}"
    assert np.array_equal(gam, am)
    assert mx == dm
    assert abs(d - tot) <= 1e-9 * max(1.0, tot)


@pytest.mark.parametrize("kernel", [_lib.KERNEL_STENCIL, _lib.KERNEL_STENCIL_ROWS,
                                    _lib.KERNEL_STENCIL_GATHER])
def test_one_sweep_fma_stencil_within_tolerance(og, tiny, tiny_state, kernel):
    g, m, p = oracle_structs(og, tiny)
    want, tot, mx, am = og.sweep_jacobi(tiny_state, tiny.occ, g, m, tiny.ctl, p, phase=4, argmin=True)
    with gpu_ctx(tiny) as ctx:
        ctx.set_value(tiny_state)
        _, _, gam = ctx.sweep(phase=4, kernel=kernel, argmin=True)
        got = ctx.get_value()
    assert np.max(np.abs(got - want)) <= FMA_SWEEP_TOL
    free = am >= 0
    assert np.mean(gam[free] == am[free]) >= ARGMIN_AGREE


@pytest.mark.parametrize("storage", ["fp32", "fp16", "bf16", "q16"])
@pytest.mark.parametrize("n", [(40, 48, 8, 5, 5, 5), (36, 44, 8, 5, 5, 5)])
def test_one_sweep_blend_tiles(og, n, storage):
    """The blend-then-shift sweep on grids that need several row tiles per
    plane (and, for 44 columns, the scalar blend of the 16-bit types): one
    sweep against the oracle run on the same stored values, within the FMA
    tolerance plus half a storage ulp of the result."""
    pr = Problem("tiny", seed=3, n=n)
    g, m, p = oracle_structs(og, pr)
    V = init_value(pr)
    for it in range(3):
        V, _, _, _ = og.sweep_jacobi(V, pr.occ, g, m, pr.ctl, p, phase=it)
    with gpu_ctx(pr, storage) as ctx:
        ctx.set_value(V)
        Vs = ctx.get_value()  # V as stored
        want, _, _, am = og.sweep_jacobi(Vs, pr.occ, g, m, pr.ctl, p, phase=3, argmin=True)
        _, _, gam = ctx.sweep(phase=3, kernel=_lib.KERNEL_STENCIL, argmin=True)
        got = ctx.get_value()
    if storage == "fp32":
        half_ulp = 0.0
    elif storage == "q16":
        half_ulp = 2.0 ** -12
    else:
        mant = 10 if storage == "fp16" else 7
        half_ulp = np.ldexp(1.0, np.frexp(np.abs(want).astype(np.float64))[1] - 1 - mant - 1)
    err = np.abs(got.astype(np.float64) - want) - half_ulp
    assert err.max() <= FMA_SWEEP_TOL, f"max excess {err.max()}"
    free = am >= 0
    assert np.mean(gam[free] == am[free]) >= ARGMIN_AGREE


@pytest.mark.parametrize("storage", ["fp32", "fp16", "bf16", "q16"])
@pytest.mark.parametrize("n,rows,cs", [((40, 48, 8, 5, 5, 5), 0, "cube3"),
                                       ((36, 44, 8, 5, 5, 5), 0, "cube3"),
                                       ((24, 96, 4, 5, 5, 5), 0, "cube3"),
                                       ((40, 48, 8, 5, 5, 5), 5, "cube3"),
                                       ((17, 20, 8, 5, 5, 5), 0, "cube3"),
                                       ((24, 48, 8, 7, 7, 7), 0, "cube5"),
                                       ((10, 192, 2, 5, 5, 5), 0, "cube5")])
def test_register_blend_matches_blend_bit_for_bit(n, rows, cs, storage):
    """The register-resident blend (controls of a plane in corner-group
    order, corner values held in registers) against the re-reading blend:
    same FMA chain, same successor rounding, so four sweeps give the same
    stored values, residuals and argmin bit for bit -- on one- and multi-tile
    planes, row groups of 44, 48 and 96 columns, blocks with idle threads,
    an explicit tiling, and 192 columns, where a block stages its 125
    controls in two chunks."""
    pr = Problem("tiny", seed=7, n=n, control_set=cs)
    V = init_value(pr)
    out = {}
    for kern in (_lib.KERNEL_STENCIL, _lib.KERNEL_STENCIL_BLEND):
        with gpu_ctx(pr, storage) as ctx:
            if rows:
                ctx.set_tile_rows(rows)
            ctx.set_value(V)
            res = [ctx.sweep(phase=ph, kernel=kern)[:2] for ph in range(4)]
            _, _, am = ctx.sweep(phase=4, kernel=kern, argmin=True)
            out[kern] = (ctx.get_value(), res, am)
    a, b = out[_lib.KERNEL_STENCIL], out[_lib.KERNEL_STENCIL_BLEND]
    assert np.array_equal(a[0], b[0]), f"max |dV| {np.max(np.abs(a[0] - b[0]))}"
    assert a[1] == b[1]
    assert np.array_equal(a[2], b[2])


def test_one_sweep_small_slab_bit_exact(og):
    """The 24x24x16x9x9x9 workload (27 controls), one x-slab against the oracle."""
    pr = Problem("small", seed=0)
    g, m, p = oracle_structs(og, pr)
    V0 = init_value(pr)
    with gpu_ctx(pr) as ctx:
        ctx.set_value(V0)
        for it in range(6):
            ctx.sweep(phase=it, kernel=_lib.KERNEL_STENCIL_EXACT)
        Vk = ctx.get_value()
        slab = pr.ncells // pr.grid.n[0]
        lo, hi = 11 * slab, 13 * slab
        want, _, _, am = og.sweep_jacobi(Vk, pr.occ, g, m, pr.ctl, p, phase=6, lo=lo, hi=hi,
                                         argmin=True)
        ctx.set_value(Vk)
        _, _, gam = ctx.sweep(phase=6, kernel=_lib.KERNEL_STENCIL_EXACT, argmin=True)
        got = ctx.get_value()
    assert np.array_equal(got[lo:hi], want[lo:hi])
    assert np.array_equal(gam[lo:hi], am[lo:hi])


TIE = 1e-5  # s: best two lookaheads closer than this are a tie (argmin not compared)


def test_one_sweep_medium_slab_register_sweep(og):
    """The benchmarked sweep (k_stencil_r) on the 48x48x32x15x15x15 workload
    (125 controls) against the oracle on 12 y rows of the target's x row:
    one sweep from a structured table within FMA_SWEEP_TOL, and the argmin of
    every cell whose best two lookaheads differ by more than TIE (checked on
    a sample through the oracle's per-control lookaheads)."""
    pr = Problem("medium", seed=0)
    g, m, p = oracle_structs(og, pr)
    n = pr.grid.n
    per_x = pr.ncells // n[0]
    per_y = per_x // n[1]
    tx, ty = int(pr.seeds[0]) // per_x, (int(pr.seeds[0]) % per_x) // per_y
    y0 = min(max(ty - 6, 0), n[1] - 12)
    lo, hi = tx * per_x + y0 * per_y, tx * per_x + (y0 + 12) * per_y
    with gpu_ctx(pr) as ctx:
        ctx.set_value(init_value(pr))
        for it in range(20):
            ctx.sweep(phase=it, kernel=_lib.KERNEL_STENCIL)
        Vk = ctx.get_value()
        _, _, gam = ctx.sweep(phase=20, kernel=_lib.KERNEL_STENCIL, argmin=True)
        got = ctx.get_value()[lo:hi]
    want, _, _ = og.sweep_jacobi_slab(Vk, pr.occ, g, m, pr.ctl, p, lo, hi, phase=20)
    cap = np.float32(pr.params.cap)
    assert np.count_nonzero(want < cap) > 0.05 * (hi - lo)  # the slab carries structure
    assert np.max(np.abs(got.astype(np.float64) - want)) <= FMA_SWEEP_TOL
    rng = np.random.default_rng(1)
    cells = lo + np.flatnonzero(want < cap)
    cells = np.sort(rng.choice(cells, size=min(20000, cells.size), replace=False))
    la = og.cell_lookaheads(Vk, pr.occ, g, m, pr.ctl, p, cells).astype(np.float64)
    two = np.sort(la, axis=1)[:, :2]
    clear = (two[:, 1] - two[:, 0] > TIE) & (two[:, 0] < cap)
    assert clear.sum() > 0.5 * cells.size
    assert np.array_equal(gam[cells[clear]], np.argmin(la[clear], axis=1))


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tiny_fixed_point.npz")


@pytest.mark.parametrize("kernel", [_lib.KERNEL_STENCIL_EXACT, _lib.KERNEL_STENCIL,
                                    _lib.KERNEL_STENCIL_ROWS, _lib.KERNEL_STENCIL_GATHER])
def test_fixed_point_matches_oracle(tiny, kernel):
    """Converged tables (max-norm stop at 1e-4 s) against the oracle's Jacobi
    solve of the same inputs (tests/golden/make_golden.py): bit-identical for
    the exact stencil; for the FMA stencils, whose only difference is the
    rounding order of the interpolation sum, within FMA_FIXED_POINT_MAX
    (max) and FMA_FIXED_POINT_RMS (RMS) -- an undiscounted iteration of ~950
    sweeps random-walks per-sweep rounding noise of a few ulp; argmin >= 99.9%."""
    gold = np.load(GOLDEN)
    Vo, it_o, am_o = gold["V"], int(gold["iterations"]), gold["argmin"]
    opts = _lib.default_opts(stop_rule=_lib.STOP_MAXNORM, kernel=kernel)
    V, res = _lib.solve_value(tiny.grid.to_c(), tiny.model.to_c(), tiny.params, tiny.occ,
                              tiny.seeds, tiny.ctl, 3000, 1e-4, opts)
    err = np.abs(V.astype(np.float64) - Vo)
    msg = f"max {err.max()} rms {np.sqrt(np.mean(err ** 2))} sweeps {res.iterations} vs {it_o}"
    if kernel == _lib.KERNEL_STENCIL_EXACT:
        assert res.iterations == it_o
        assert np.array_equal(V, Vo), msg
    else:
        assert abs(res.iterations - it_o) <= 0.05 * it_o, msg
        assert err.max() <= FMA_FIXED_POINT_MAX, msg
        assert np.sqrt(np.mean(err ** 2)) <= FMA_FIXED_POINT_RMS, msg
    with gpu_ctx(tiny) as ctx:
        ctx.set_value(V)
        _, _, am_g = ctx.sweep(phase=res.iterations, kernel=kernel, argmin=True)
    free = am_o >= 0
    assert np.mean(am_g[free] == am_o[free]) >= ARGMIN_AGREE


def test_cellform_solve_bit_exact_with_reference_defaults(og, tiny):
    """The reference's default scheme (warm start, rotating scan, pattern
    search, CFL ladder, adaptive probes, Kuhn simplex) on the cell-form
    kernel: three sweeps bit-identical to the oracle's."""
    pr = tiny
    p = _lib.Params()
    C.memmove(C.byref(p), C.byref(pr.params), C.sizeof(p))
    p.ncoarse, p.rounds, p.ntau, p.cfl, p.adaptive_checks, p.simplex = 8, 2, 5, 2.0, 1, 1
    p.tau_max, p.hmax = 0.5, 0.0125
    g, m, _ = oracle_structs(og, pr)
    po = og.copy_struct(p, og.OParams)
    Vo, _, _, _ = og.solve_value(pr.occ, g, m, pr.seeds, pr.ctl, po, 3, 0.0, jacobi=True, warm=True)
    opts = _lib.default_opts(kernel=_lib.KERNEL_CELLFORM, warm_start=1)
    V, res = _lib.solve_value(pr.grid.to_c(), pr.model.to_c(), p, pr.occ, pr.seeds, pr.ctl, 3,
                              0.0, opts)
    assert res.iterations == 3
    assert np.array_equal(V, Vo), f"max |dV| {np.max(np.abs(V - Vo))}"


def test_escape_sweeps_bit_exact(og, tiny, tiny_state):
    g, m, p = oracle_structs(og, tiny)
    Vo = tiny_state.copy()
    with gpu_ctx(tiny) as ctx:
        ctx.set_value(tiny_state)
        for it in range(3):
            Vo, tot = og.sweep_escape_jacobi(Vo, tiny.occ, g, m, tiny.ctl, p, phase=it)
            d = ctx.escape_sweep(phase=it)
            assert abs(d - tot) <= 1e-9 * max(1.0, tot)
        got = ctx.get_value()
    assert np.array_equal(got, Vo)
    assert np.any(Vo < 0)


@pytest.mark.parametrize("dtype", ["u16", "u8", "f16", "f32"])
def test_encode_byte_identical(og, tiny, dtype):
    from peregrine_hjb.tables import DTYPES, escape_scale_for
    cap = float(tiny.params.cap)
    rng = np.random.default_rng(9)
    n = tiny.ncells
    V = rng.uniform(0, cap, n).astype(np.float32)
    k = rng.integers(0, 7, n)
    V[k == 0] = cap
    V[k == 1] = -rng.uniform(0, cap, np.sum(k == 1)).astype(np.float32)
    V[k == 2] = np.round(V[k == 2] * 1000) / 1000 + 0.0005  # rounding ties in the codes
    V[:4] = [np.inf, np.nan, -0.0, 0.0]
    es = escape_scale_for(dtype, cap)
    sc = DTYPES[dtype]["scale"]
    want, r, e = og.encode(V, dtype, sc, cap, es)
    with gpu_ctx(tiny) as ctx:
        ctx.set_value(V)
        got, gr, ge = ctx.encode(dtype, sc, es, 0, n)
        lo = 1000
        part, _, _ = ctx.encode(dtype, sc, es, lo, 5000)
    assert bytes(got) == bytes(want)
    assert (gr, ge) == (r, e)
    eb = DTYPES[dtype]["bytes"]
    assert bytes(part) == bytes(want[lo * eb:(lo + 5000) * eb])


def test_fp64_precision_oracle_takes_the_fp32_decisions(og, tiny, tiny_state):
    """FP64 storage runs the precision oracle: the FP32 solver's decisions
    (admissibility, successor cells and fractions) with FP64 value
    arithmetic.  One sweep from a stored FP32 table agrees with the oracle's
    FP32 sweep to FP32 rounding (no decision differs: blocked and admitted
    cells match exactly), and argmin agrees on >= 99.9 % of free cells."""
    g, m, p = oracle_structs(og, tiny)
    want, _, _, am = og.sweep_jacobi(tiny_state, tiny.occ, g, m, tiny.ctl, p, phase=4, argmin=True)
    with gpu_ctx(tiny, "fp64") as ctx:
        ctx.set_value(tiny_state)
        _, _, gam = ctx.sweep(phase=4, kernel=_lib.KERNEL_STENCIL, argmin=True)
        got = ctx.get_value()
    cap = np.float32(tiny.params.cap)
    assert np.max(np.abs(got.astype(np.float64) - want)) <= FMA_SWEEP_TOL
    free = am >= 0
    assert np.array_equal(gam < 0, am < 0)
    assert np.mean(gam[free] == am[free]) >= ARGMIN_AGREE


def test_fp64_and_16bit_storage(og, tiny):
    """The FP64 precision oracle vs FP32, and FP16/BF16 storage with FP32
    polish vs FP64, on converged tables (max-norm stop 1e-4 s)."""
    args = (tiny.grid.to_c(), tiny.model.to_c(), tiny.params, tiny.occ, tiny.seeds, tiny.ctl,
            3000, 1e-4)
    V32, _ = _lib.solve_value(*args, _lib.default_opts(stop_rule=1))
    V64, _ = _lib.solve_value(*args, _lib.default_opts(stop_rule=1, storage="fp64"))
    V16, r16 = _lib.solve_value(*args, _lib.default_opts(stop_rule=1, storage="fp16",
                                                         polish_sweeps=3000))
    Vbf, rbf = _lib.solve_value(*args, _lib.default_opts(stop_rule=1, storage="bf16",
                                                         polish_sweeps=3000))
    e64 = float(np.max(np.abs(V64.astype(np.float64) - V32)))
    # same decisions: only the value arithmetic differs, so the converged
    # tables differ by the FP32 rounding walk, not by a different model
    assert np.array_equal(V64 >= tiny.params.cap, V32 >= tiny.params.cap)
    e16 = float(np.max(np.abs(V16.astype(np.float64) - V64)))
    ebf = float(np.max(np.abs(Vbf.astype(np.float64) - V64)))
    print(f"fp32-fp64 {e64:.3g}  fp16+polish-fp64 {e16:.3g} ({r16.iterations - r16.polish_iterations}"
          f"+{r16.polish_iterations} sweeps)  bf16+polish-fp64 {ebf:.3g} "
          f"({rbf.iterations - rbf.polish_iterations}+{rbf.polish_iterations} sweeps)")
    assert e64 < 5e-3
    assert e16 <= 2e-3 and ebf <= 2e-3
    assert r16.polish_iterations >= 1


def test_minimum_time_closed_form():
    """SelfTest [1] (SelfTest.jl:90-199): the bang-bang minimum time 2*sqrt(d/a)
    of a double integrator, with the reference's three schemes on its grid."""
    from peregrine_hjb.grid import Grid6
    from peregrine_hjb.params import control_set
    from peregrine_hjb.seeds import target_cells
    g = Grid6.make((81, 5, 4, 33, 5, 5), (0, 0, -math.pi, -100, -100, -2), (200, 200, math.pi, 100, 100, 2))
    amax = 100.0
    m = _lib.Model()
    for i, v in enumerate((amax, 0, 0, 0, amax, 0, 0, 0, amax)):
        m.B[i] = v
    m.eps[0], m.eps[1], m.eps[2] = 5.0, 5.0, 0.15
    m.knee = 0.0
    occ = np.zeros(81 * 5 * 4, np.uint8)
    ttol = tuple(np.float32(g.step[k] * np.float32(0.5)) for k in range(6))
    tc = target_cells(g, (np.float32(100), np.float32(100), 0, 0, 0, 0), ttol)
    ctl = control_set(4)

    def params(**kw):
        p = _lib.Params()
        base = dict(dt=0.05, nsub=4, checks=3, adaptive_checks=1, nearest=0, cap=30.0, ntau=1,
                    tau_ratio=2.0, cfl=0.0, tau_min=0.004, tau_max=0.5, hmax=0.0125, ncoarse=0,
                    rounds=0, delta0=0.35, rk2=1, vclamp=0, simplex=1)
        base.update(kw)
        for k, v in base.items():
            setattr(p, k, v)
        return p

    def run(p, warm):
        opts = _lib.default_opts(kernel=_lib.KERNEL_CELLFORM, warm_start=int(warm))
        V, _ = _lib.solve_value(g.to_c(), m, p, occ, tc, ctl, 600, 1e-4, opts)
        return V

    legacy = run(params(checks=3, adaptive_checks=0, ntau=1, cfl=0.0, ncoarse=0, rounds=0, rk2=0), False)
    ladder = run(params(checks=2, adaptive_checks=1, ntau=4, cfl=1.0, ncoarse=0, rounds=0, rk2=1), False)
    now = run(params(checks=2, adaptive_checks=1, ntau=4, cfl=1.0, ncoarse=8, rounds=2, rk2=1), True)
    from oracle import oracle as og
    og_g = og.copy_struct(g.to_c(), og.OGrid)
    ds = (20.0, 40.0, 60.0)
    want = [2.0 * math.sqrt(d / amax) for d in ds]

    def at(V, d):
        return float(og.lib().og_interp_kuhn(V.ctypes.data, og_g, og.state(100.0 - d, 100.0, 0, 0, 0, 0),
                                             30.0, 0, None))

    gotl = [at(legacy, d) for d in ds]
    gotd = [at(ladder, d) for d in ds]
    gotn = [at(now, d) for d in ds]
    ml, md, mn = sum(gotl) / 3, sum(gotd) / 3, sum(gotn) / 3
    assert mn <= md * 1.08
    assert md <= ml * 1.02
    ex = [gotn[i] - want[i] for i in range(3)]
    slope = (ex[2] - ex[0]) / (want[2] - want[0])
    intercept = ex[0] - slope * want[0]
    assert intercept < 0.45 and slope < 0.20


def test_full_size_properties():
    """The 48x48x32x15x15x15 workload (125 controls): size-independent
    properties of a few sweeps -- monotone, bounded, seeds pinned, the
    residual equals the largest change."""
    pr = Problem("medium", seed=0)
    cap = np.float32(pr.params.cap)
    with gpu_ctx(pr) as ctx:
        opts = _lib.default_opts(stop_rule=_lib.STOP_MAXNORM)
        res = ctx.solve(pr.seeds, 3, 0.0, opts)
        V1 = ctx.get_value()
        d, dm, _ = ctx.sweep(phase=3)
        V2 = ctx.get_value()
    assert res.iterations == 3
    assert np.all(V2 <= V1) and np.all(V2 >= 0) and np.all(V2 <= cap)
    assert np.all(V2[pr.seeds] == 0)
    diff = V1.astype(np.float64) - V2.astype(np.float64)
    assert float(np.max(diff)) == dm
    assert abs(float(np.sum(diff)) - d) <= 1e-9 * max(1.0, d)
    assert np.count_nonzero(V2 < cap) > np.count_nonzero(V1 < cap) or dm == 0


def test_measured_peaks_are_plausible():
    """The on-chip probes behind the secondary rooflines: positive and below
    generous bounds for any current GPU (shared memory < 1e6 GB/s, L2 < 1e5
    GB/s, FP32 FMA < 1e3 TFLOP/s)."""
    pk = _lib.measure_peaks(0)
    assert 0 < pk["smem_gbs"] < 1e6
    assert 0 < pk["l2_gbs"] < 1e5
    assert 0 < pk["fma_tflops"] < 1e3
