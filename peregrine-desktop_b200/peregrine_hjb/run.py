"""Run driver: solve every target and write the card image.

Mirrors run_solve (solver/src/Run.jl:1539-2131): same config keys and
defaults, the same `PROGRESS {json}` phases on stdout, the same
`TABLES/T##C####.BIN`, `MANIFEST.JSON` and `MODEL.JSON` outputs.  The solve
itself goes through libperegrine_hjb.so on one GPU.
"""
from __future__ import annotations

import datetime as _dt
import hashlib
import json
import math
import os
import sys
import time

import numpy as np

from . import _lib
from .geometry import build_occupancy, wall_box
from .grid import AXES, build_grid, getc, grid_inputs
from .params import load_field, load_model, load_targets, solver_params
from .seeds import free_seed_count, seeds_for
from .tables import DTYPES, escape_codes, escape_scale_for, write_table


def progress(**kw):
    """progress (Run.jl:13-16)"""
    sys.stdout.write("PROGRESS " + json.dumps(kw) + "\n")
    sys.stdout.flush()


def filehash(path) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as fh:
        for blk in iter(lambda: fh.read(1 << 20), b""):
            h.update(blk)
    return h.hexdigest()


def _utc_now() -> str:
    t = _dt.datetime.now(_dt.timezone.utc).replace(microsecond=0, tzinfo=None)
    return t.isoformat() + "Z"


def model_json(m, reg_path, zeroed_c: bool, cfg=None) -> dict:
    """model_json (Run.jl:1278-1378): the dynamics model as the solve used
    it, in the card's over-general block form, plus the honing PID block
    (honing.py).  Refuses a model whose blocks would make the dynamics
    depend on position."""
    from .honing import honing_gains
    Am = [[float(m.A[r, c]) for c in range(3)] for r in range(3)]
    Bm = [[float(m.B[r, c]) for c in range(3)] for r in range(3)]
    Sm = [[float(m.S[r, c]) for c in range(3)] for r in range(3)]
    Dm = [[float(m.D[r, c]) for c in range(3)] for r in range(3)]
    A_s = [[0.0, 0.0, 0.0] + Am[r] for r in range(3)]
    A_ss = [[0.0, 0.0, 0.0, 0.0, 0.0, float(m.q[r])] for r in range(3)]
    A_uu = [[0.0, 0.0, 0.0] for _ in range(3)]
    A_sgn = [[0.0, 0.0, 0.0] + Sm[r] for r in range(3)]
    A_abs = [[0.0, 0.0, 0.0] + Dm[r] for r in range(3)]
    k = [float(m.c[r]) for r in range(3)]

    def nz(blk):
        return any(any(v != 0 for v in row) for row in blk)

    for nm, blk in (("A_s", A_s), ("A_ss", A_ss), ("A_sgn", A_sgn), ("A_absv", A_abs)):
        if any(v != 0 for row in blk for v in row[:3]):
            raise ValueError(f"{nm} has a non-zero x/y/h column; the dynamics must not depend "
                             "on where the robot is")
    blocks = [("A_s", nz(A_s)), ("A_u", nz(Bm)), ("A_ss", nz(A_ss)), ("A_uu", nz(A_uu)),
              ("A_sgn", nz(A_sgn)), ("A_absv", nz(A_abs)), ("k", any(v != 0 for v in k))]
    return {
        "schema_version": 2,
        "generator": "peregrine-desktop",
        "regression_sha256": filehash(reg_path),
        "equation": "a = A_s*s + A_u*u + A_ss*(s.*s) + A_uu*(u.*u) + "
                    "A_sgn*csign(s) + A_absv*(abs(s).*s) + k",
        "csign": {
            "formula": "csign(s)_i = clamp(s_i / coulomb_eps_i, -1, 1)",
            "coulomb_eps": [0.0, 0.0, 0.0] + [float(v) for v in m.eps],
            "why": "Coulomb friction is smoothed instead of using a hard sign(), which would "
                   "flip discontinuously at zero and make an integrator chatter. Use exactly "
                   "this form.",
        },
        "output": {"vector": ["a_x", "a_y", "alpha"], "units": ["cm/s^2", "cm/s^2", "rad/s^2"],
                   "frame": "robot body"},
        "state": {
            "vector": list(AXES),
            "units": ["cm", "cm", "rad", "cm/s", "cm/s", "rad/s"],
            "frame_note": "IMPORTANT: vx and vy must be rotated into the ROBOT BODY frame "
                          "before use here. The value tables index field-frame velocity, so "
                          "rotate by -h between the two. Motor forces act along the body axes, "
                          "which is why the model cannot be written with constant matrices in "
                          "the field frame. x, y and h have zero coefficients throughout.",
        },
        "control": {
            "vector": ["fwd", "strafe", "turn"],
            "note": "mecanum projection of the wheel powers; the admissible set is "
                    "|fwd| + |strafe| + |turn| <= 1",
            "saturation": {
                "knee": float(m.knee),
                "formula": "m = norm(u_raw); u = u_raw * tanh(m/knee) / (m/knee)",
                "why": "Past the knee the tyres stop delivering, so extra command buys no extra "
                       "force. APPLY THIS BEFORE A_u -- the gains were fitted against the "
                       "saturated command. The knee is always present and positive.",
            },
        },
        "A_s": A_s, "A_u": Bm, "A_ss": A_ss, "A_uu": A_uu, "A_sgn": A_sgn, "A_absv": A_abs,
        "k": k,
        "constant_zeroed": bool(zeroed_c),
        "nonzero_blocks": [b for b, f in blocks if f],
        "honing": honing_gains(m, cfg or {}),
    }


class Prepared:
    """Everything run_solve and plan build before the first sweep."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.reg_path = str(cfg["regression"])
        self.field_path = str(cfg["field"])
        self.targ_path = str(cfg["targets"])
        m, _ = load_model(self.reg_path)
        self.zero_c = bool(getc(cfg, "zero_c", True))
        self.model = m.zeroed_c() if self.zero_c else m
        self.bounds, self.polys, self.robot, _ = load_field(self.field_path)
        self.names, self.states, _ = load_targets(self.targ_path)
        gcfg = getc(cfg, "grid", {})
        self.gi = grid_inputs(cfg, self.bounds, self.robot)
        self.g = build_grid(gcfg, self.bounds, self.robot, self.gi["wall_clearance"],
                            self.gi["hsub"])
        self.cells = self.g.ncells
        self.dtype = str(getc(cfg, "dtype", "u16"))
        if self.dtype not in DTYPES:
            raise ValueError(f"unknown dtype '{self.dtype}'")
        self.scale = float(getc(cfg, "scale", DTYPES[self.dtype]["scale"]))
        self.chunk_elements = int(getc(cfg, "chunk_elements", 1 << 23))
        if self.chunk_elements <= 0 or self.chunk_elements & (self.chunk_elements - 1):
            raise ValueError("chunk_elements must be a power of two")
        self.sp = solver_params(cfg, self.g)

    def occupancy(self):
        return build_occupancy(self.g, self.polys, self.sp.margin, self.robot, self.gi["hsub"],
                               self.sp.clearance, bounds=self.bounds,
                               wall_clearance_cm=self.gi["wall_clearance"])


def check_targets(prep, occ):
    """check_targets (Advise.jl:513-570), reduced to the refusal it drives."""
    g = prep.g
    bad = []
    for name, s in zip(prep.names, prep.states):
        seeds = seeds_for(g, s, prep.sp, prep.cfg)
        if free_seed_count(g, occ, seeds) > 0:
            continue
        off = []
        for k in (0, 1, 3, 4, 5):
            hi = float(g.lo[k]) + float(g.step[k]) * (g.n[k] - 1)
            if float(s[k]) < float(g.lo[k]) - 1e-6 or float(s[k]) > hi + 1e-6:
                off.append(AXES[k])
        if off:
            span = ", ".join("%s %.1f..%.1f" % (AXES[k], float(g.lo[k]),
                                                float(g.lo[k]) + float(g.step[k]) * (g.n[k] - 1))
                             for k in (0, 1, 3, 4, 5))
            bad.append(f"  '{name}' is outside the table on {', '.join(off)} (the table spans {span})")
        else:
            why = []
            bx = wall_box(prep.bounds, prep.robot, prep.gi["wall_clearance"], float(s[2]))
            if float(s[0]) < bx[0] or float(s[0]) > bx[1] or float(s[1]) < bx[2] or float(s[1]) > bx[3]:
                why.append("the footprint crosses the field boundary")
            if not why:
                why.append("it or its heading bin is blocked by an obstacle")
            bad.append(f"  '{name}' " + "; ".join(why))
    if bad:
        raise ValueError("these targets are states the robot cannot be in, so they would seed "
                         "nothing and the whole table would come out unreachable:\n" + "\n".join(bad))


def dist_ranks():
    """(rank, world, local rank) of this process.  Under a launcher that sets
    WORLD_SIZE > 1 (torchrun) the process group is initialised here: NCCL
    when every rank has its own GPU, gloo otherwise (the ranks exchange only
    small records, never tables)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return 0, 1, 0
    import datetime

    import torch
    import torch.distributed as dist
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not dist.is_initialized():
        ngpu = torch.cuda.device_count() if torch.cuda.is_available() else 0
        backend = "nccl" if ngpu >= world else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return dist.get_rank(), dist.get_world_size(), local


def run_solve(cfg, device: int | None = None) -> dict:
    """run_solve (Run.jl:1539-2131) on the GPU.  Under torchrun the job's
    targets are shared out over the ranks (dist.assign_tables: independent
    tables, no data-path collective); each rank solves and writes its own
    targets' tables on its GPU and rank 0 writes MANIFEST.JSON and
    MODEL.JSON from every rank's records."""
    from . import dist as pdist
    rank, world, local = dist_ranks()
    if device is None:
        device = 0
        if world > 1:
            import torch
            ngpu = torch.cuda.device_count() if torch.cuda.is_available() else 1
            device = local if ngpu >= world else 0
    prep = Prepared(cfg)
    g, sp = prep.g, prep.sp
    cap = sp.cap
    out_dir = str(cfg["out_dir"])
    dtype, scale = prep.dtype, prep.scale

    do_escape = bool(getc(cfg, "escape", True))
    esc_iters = int(getc(cfg, "escape_iterations", 60))
    esc_tol = float(getc(cfg, "escape_tolerance", sp.tol))
    escape_scale = escape_scale_for(dtype, cap) if do_escape else 0.0
    ebase = int(DTYPES[dtype]["escape_base"])
    if do_escape and ebase > 0 and cap / scale >= ebase:
        raise ValueError(
            f"value_cap {cap} s at scale {scale} needs codes up to {round(cap / scale)}, which "
            f"runs into the escape band at {ebase}. Lower value_cap below "
            f"{round(ebase * scale, 2)} s, use a coarser scale, or set escape to false")
    if do_escape and escape_scale <= 0.0 and dtype in ("u8", "u16"):
        raise ValueError(f"dtype '{dtype}' has no escape band configured")
    backend = str(getc(cfg, "backend", "auto"))
    if backend not in ("auto", "cuda"):
        raise ValueError(f"backend '{backend}': this solver runs on the GPU only")
    if getc(cfg, "out_of_core", "auto") in (True, "true", "always"):
        raise ValueError("out_of_core: the tiled driver is not part of this solver; "
                         "the grid must fit in device memory")

    progress(phase="setup", cells=prep.cells, n=list(g.n), controls=sp.nctl, dtype=dtype,
             escape=do_escape, escape_scale=escape_scale, escape_base=ebase,
             escape_codes=escape_codes(dtype), bytes_per_target=prep.cells * DTYPES[dtype]["bytes"],
             iterations=sp.iters, escape_iterations=esc_iters if do_escape else 0,
             n_targets=len(prep.names))

    occ = prep.occupancy()
    blocked = int(np.count_nonzero(occ))
    progress(phase="occupancy", blocked_cells=blocked, blocked_frac=blocked / max(occ.size, 1),
             robot_vertices=0 if prep.robot is None else len(prep.robot),
             heading_substeps=prep.gi["hsub"], clearance_cm=sp.clearance,
             wall_clearance_cm=prep.gi["wall_clearance"])
    check_targets(prep, occ)
    progress(phase="backend", backend="cuda")

    tables_dir = os.path.join(out_dir, "TABLES")
    os.makedirs(tables_dir, exist_ok=True)
    entries = []
    opts = _lib.default_opts(stop_rule=sp.stop_rule, storage=sp.storage,
                             warm_start=1 if sp.warm else 0, polish_sweeps=sp.polish_sweeps)
    ntargets = len(prep.states)
    mine = pdist.assign_tables([prep.cells * sp.nctl] * ntargets, world)[rank]
    with _lib.Context(device) as ctx:
        ctx.load_problem(g.to_c(), prep.model.to_c(), sp.p, occ, sp.ctl, sp.storage)
        for ti, (name, s) in enumerate(zip(prep.names, prep.states)):
            if ti not in mine:
                continue
            seeds = seeds_for(g, s, sp, cfg)
            t0 = time.time()
            first = {"el": 0.0}

            def on_progress(it, d, dm, ti=ti, name=name, t0=t0, first=first):
                el = time.time() - t0
                if it == 1:
                    first["el"] = el
                per = (el - first["el"]) / (it - 1) if it > 1 else el
                eta = None
                if it > 1:
                    eta = max(0.0, (sp.iters - it) * per) + (ntargets - ti - 1) * sp.iters * per
                progress(phase="solve", target=ti, target_name=name, iter=it, iters=sp.iters,
                         delta=d, elapsed_s=el, sweep_s=per, eta_s=eta, maxnorm=dm)
                return False

            res = ctx.solve(seeds, sp.iters, sp.tol, opts, on_progress)
            done_iters, last_delta = res.iterations, res.last_delta
            esc_done, esc_delta = 0, 0.0
            if do_escape:
                te = time.time()

                def on_esc(it, d, dm, ti=ti, name=name, te=te):
                    progress(phase="escape", target=ti, target_name=name, iter=it,
                             iters=esc_iters, delta=d, elapsed_s=time.time() - te)
                    return False

                er = ctx.solve_escape(esc_iters, esc_tol, on_esc)
                esc_done, esc_delta = er.iterations, er.last_delta
            progress(phase="encode", target=ti, target_name=name, iters_done=done_iters,
                     delta=last_delta)
            info = write_table(tables_dir, ti, ctx, prep.cells, dtype, scale,
                               prep.chunk_elements, escape_scale)
            reached_frac = info["reached"] / info["cells"]
            escape_frac = info["escaped"] / info["cells"]
            dead = info["cells"] - info["reached"]
            esc_unr = info["escaped"] / dead if dead > 0 else 0.0
            entries.append({
                "index": ti, "name": name, "state": [float(v) for v in s],
                "file_pattern": "TABLES/T%02dC%%04d.BIN" % ti,
                "n_chunks": info["nchunks"], "bytes": info["bytes"], "sha256": info["sha256"],
                "iterations": done_iters, "final_delta": last_delta,
                "reached_frac": reached_frac, "escape_frac": escape_frac,
                "escape_of_unreached_frac": esc_unr, "escape_iterations": esc_done,
                "escape_final_delta": esc_delta,
            })
            progress(phase="target_done", target=ti, target_name=name, chunks=info["nchunks"],
                     bytes=info["bytes"], reached_frac=reached_frac, escape_frac=escape_frac,
                     escape_of_unreached_frac=esc_unr, elapsed_s=time.time() - t0)

    if world > 1:
        entries = pdist.gather_records(entries)
    if rank != 0:
        return {"targets": entries}
    r = sp.raw
    manifest = {
        "schema_version": 1,
        "generated_utc": _utc_now(),
        "generator": "peregrine-desktop",
        "regression_sha256": filehash(prep.reg_path),
        "field_sha256": filehash(prep.field_path),
        "grid": {
            "axes": list(AXES),
            "n": list(g.n),
            "min": [float(g.lo[k]) for k in range(6)],
            "max": [g.span_max(k) for k in range(6)],
            "wrap": [False, False, True, False, False, False],
            "units": ["cm", "cm", "rad", "cm/s", "cm/s", "rad/s"],
            "frame": "field",
            "frame_note": "x, y, h and the vx, vy velocity axes are all field frame; omega is "
                          "frame independent",
            "field_bounds": list(prep.bounds),
            "field_note": "grid.min/max span the positions the robot can legally occupy, which "
                          "is the field inset by the footprint plus wall_clearance_cm. Clamp x "
                          "and y into that span as section 3 of TABLE_FORMAT.md describes; the "
                          "edge cell is the nearest legal state to anything beyond it",
            "total_cells": prep.cells,
            "index_formula": "((((ix*Ny+iy)*Nh+ih)*Nvx+ivx)*Nvy+ivy)*Nw+iw",
        },
        "encoding": {
            "dtype": dtype,
            "elem_bytes": DTYPES[dtype]["bytes"],
            "scale": scale,
            "unit": "seconds",
            "unreachable": 255 if dtype == "u8" else (65535 if dtype == "u16" else "NaN"),
            "escape_base": ebase if do_escape else 0,
            "escape_codes": escape_codes(dtype) if do_escape else 0,
            "escape_scale": escape_scale if do_escape else 0.0,
            "escape_unit": "seconds",
            "escape_formula": ("raw >= escape_base -> unreachable, escape_seconds = "
                               "escape_scale * (raw - escape_base)^2") if dtype in ("u8", "u16")
            else "value < 0 -> unreachable, escape_seconds = -value",
            "escape_note": "an escape cell is UNREACHABLE and must lose every comparison against "
                           "a real route. The escape time is only for a robot already in one -- "
                           "descend it to get out, then use the table normally. See section 6 "
                           "of TABLE_FORMAT.md",
            "byte_order": "little",
            "order": "row_major_c",
            "chunk_elements": prep.chunk_elements,
            "chunk_shift": prep.chunk_elements.bit_length() - 1,
        },
        "solver": {
            "dt": r["dt"], "substeps": r["nsub"], "controls": sp.nctl, "control_level": sp.level,
            "control_set": sp.control_kind,
            "iterations_max": sp.iters, "tolerance": sp.tol, "nearest": r["nearest"],
            "control_scan": r["scan"], "refine_rounds": r["rounds"], "refine_delta": r["delta0"],
            "warm_start": sp.warm, "escape": do_escape, "escape_iterations": esc_iters,
            "escape_tolerance": esc_tol, "tau_levels": r["ntau"], "tau_ratio": r["tau_ratio"],
            "cfl": r["cfl"], "tau_min": r["tau_min"], "tau_max": r["tau_max"],
            "tau_max_auto": isinstance(getc(cfg, "tau_max", "auto"), str),
            "substep_max": r["hmax"], "adaptive_checks": r["achecks"], "rk2": r["rk2"],
            "simplex": r["simplex"],
            "interpolant": "kuhn_simplex_7pt" if r["simplex"] else "multilinear_64pt",
            "velocity_clamp": r["vclamp"],
            "integrator": "midpoint_rk2" if r["rk2"] else "semi_implicit_euler",
            "driver": "whole_grid", "tiling": None, "sweep_order": "jacobi",
            "stop_rule": "maxnorm" if sp.stop_rule == _lib.STOP_MAXNORM else "l1_quiet",
            "storage": sp.storage,
            "sweep_checks": r["checks"], "zero_c": prep.zero_c, "margin_cm": sp.margin,
            "clearance_cm": sp.clearance, "wall_clearance_cm": prep.gi["wall_clearance"],
            "value_cap_s": cap, "heading_substeps": prep.gi["hsub"],
            "robot_vertices": 0 if prep.robot is None else len(prep.robot),
            "occupancy": "per heading bin (x, y, h), obstacles and the field boundary alike",
            "resolution": {
                "xy_cm": float(min(g.step[0], g.step[1])),
                "heading_deg": math.degrees(float(g.step[2])),
                "v_cm_s": float(g.step[3]),
                "w_rad_s": float(g.step[5]),
            },
        },
        "model_file": "MODEL.JSON",
        "targets": entries,
    }
    with open(os.path.join(out_dir, "MANIFEST.JSON"), "w") as fh:
        json.dump(manifest, fh, indent=2)
    mj = model_json(prep.model, prep.reg_path, prep.zero_c, cfg)
    with open(os.path.join(out_dir, "MODEL.JSON"), "w") as fh:
        json.dump(mj, fh, indent=2)
    hn = mj["honing"]
    progress(phase="model", file="MODEL.JSON", nonzero_blocks=mj["nonzero_blocks"],
             honing_omega=hn["omega"], honing_budget_frac=hn["config"]["budget_frac"],
             honing_bound_by=hn["omega_limits"]["bound_by"])
    progress(phase="done", out_dir=out_dir, targets=len(entries))
    return manifest


# Measured sweep rates on one B200 (cell-control updates per second), the
# cost model of the `runtime` estimate: the plain scheme runs the stencil
# sweep; any other scheme the one-thread-per-cell kernel of the reference's
# cell_update.  Ceiling estimates, like the reference's (Run.jl:846-958).
RATE_STENCIL = 3.0e11
RATE_CELLFORM = 4.0e9


def _gpu_memory(device: int = 0):
    """(free, total) bytes of the device, or None without a driver."""
    try:
        import pynvml
        pynvml.nvmlInit()
        try:
            h = pynvml.nvmlDeviceGetHandleByIndex(device)
            mi = pynvml.nvmlDeviceGetMemoryInfo(h)
            return int(mi.free), int(mi.total)
        finally:
            pynvml.nvmlShutdown()
    except Exception:
        return None


def _stencil_scheme(r) -> bool:
    """Whether the position-invariant stencil sweep runs this scheme (the
    library's own test at load time)."""
    return (r["cfl"] <= 0 and r["ntau"] <= 1 and r["rounds"] <= 0 and not r["achecks"]
            and not r["nearest"] and not r["simplex"])


def plan(cfg) -> dict:
    """plan (Run.jl:699-959): what a solve of this config would build and
    cost, without solving -- the keys the wizard reads (sizes, span, the
    occupancy, per-target seeding, the device fit, the grid balance, a
    runtime ceiling).  Advice this solver has no basis for (the reference's
    resolution search and tiled-horizon scan) is reported as absent."""
    from .grid import grid_resolution
    from .seeds import free_seed_count, seeds_for

    prep = Prepared(cfg)
    g, sp = prep.g, prep.sp
    gcfg = getc(cfg, "grid", {})
    eb = DTYPES[prep.dtype]["bytes"]
    cells = prep.cells
    ntg = len(prep.names)
    elem = {"fp32": 4, "fp16": 2, "bf16": 2, "q16": 2, "fp64": 8}[sp.storage]
    occ = prep.occupancy()
    nh = g.n[2]
    per_h = [float(np.count_nonzero(occ[k::nh])) / (occ.size / nh) for k in range(nh)]
    # the device bytes of a solve: two value buffers, the warm-start policy,
    # and (plain scheme) the stencil's records and tile-order mask
    need = 2 * cells * elem + (3 * cells if sp.warm else 0)
    r = sp.raw
    stencil = _stencil_scheme(r)
    if stencil:
        planes = cells // (g.n[0] * g.n[1])
        need += planes * sp.nctl * (288 + 2 + (g.n[0] * g.n[1] + 31) // 32 * 4)
    mem = _gpu_memory()
    fits = mem is not None and need <= mem[0]
    targets = []
    for name, st in zip(prep.names, prep.states):
        seeds = seeds_for(g, st, sp, cfg)
        nfree = free_seed_count(g, occ, seeds)
        off = []
        for k in (0, 1, 3, 4, 5):
            hi = float(g.lo[k]) + float(g.step[k]) * (g.n[k] - 1)
            if float(st[k]) < float(g.lo[k]) - 1e-6 or float(st[k]) > hi + 1e-6:
                off.append(AXES[k])
        targets.append({"name": name, "ok": nfree > 0, "seed_cells": int(len(seeds)),
                        "free_seed_cells": int(nfree), "off_axes": off,
                        "blocked_by": [] if nfree > 0 or off else ["an obstacle or the wall"]})
    B = np.asarray(prep.model.B, np.float64)
    acc = max(float(np.max(np.abs(B[0]))), float(np.max(np.abs(B[1]))))
    dv = float(min(g.step[3], g.step[4]))
    cell_cm = float(min(g.step[0], g.step[1]))
    dvd = dv * dv / (2 * acc) if acc > 0 else float("nan")
    rate = RATE_STENCIL if stencil else RATE_CELLFORM
    esc = int(getc(cfg, "escape_iterations", 60)) if bool(getc(cfg, "escape", True)) else 0
    unit_s = cells * sp.nctl / rate
    blocked = float(np.count_nonzero(occ)) / max(occ.size, 1)
    runtime = {"unit": "sweep", "unit_s": unit_s, "units": sp.iters + esc,
               "escape_sweeps": esc, "escape_unit_s": unit_s * (1.0 - blocked),
               "blocked_frac": blocked, "total_s": unit_s * (sp.iters + esc) * ntg,
               "rate_cell_controls_per_s": rate,
               "rate_source": "measured on one B200: the " +
                              ("stencil sweep (plain scheme)" if stencil else
                               "cell-form sweep (the reference's cell_update)")}
    xyres = grid_resolution(gcfg)
    span_x = float(g.step[0]) * (g.n[0] - 1)
    span_y = float(g.step[1]) * (g.n[1] - 1)
    b = prep.bounds
    return {
        "cells": cells,
        "axes": list(AXES),
        "n": list(g.n),
        "bounds": {
            "field": [float(v) for v in b],
            "table_min": [float(g.lo[k]) for k in range(6)],
            "table_max": [float(g.lo[k]) + float(g.step[k]) * (g.n[k] if k == 2 else g.n[k] - 1)
                          for k in range(6)],
            "inset_cm": [float(g.lo[0]) - b[0], float(g.lo[1]) - b[1],
                         b[2] - (float(g.lo[0]) + span_x), b[3] - (float(g.lo[1]) + span_y)],
            "cells_saved_frac": 1.0 - span_x * span_y / max((b[2] - b[0]) * (b[3] - b[1]), 1e-9),
            "wall_clearance_cm": prep.gi["wall_clearance"],
            "clearance_cm": prep.gi["clearance"],
        },
        "resolution": {
            "requested": {"xy_cm": xyres[0], "heading_deg": xyres[1], "v_cm_s": xyres[2],
                          "w_rad_s": xyres[3]},
            "actual": {"xy_cm": cell_cm, "heading_deg": math.degrees(float(g.step[2])),
                       "v_cm_s": float(g.step[3]), "w_rad_s": float(g.step[5])},
            "pinned_by_n": getc(gcfg, "n", None) is not None,
        },
        "occupancy": {"blocked_frac": blocked, "blocked_cells": int(np.count_nonzero(occ)),
                      "xyh_cells": int(occ.size), "worst_heading_blocked_frac": max(per_h),
                      "best_heading_blocked_frac": min(per_h)},
        "targets": targets,
        "targets_ok": all(t["ok"] for t in targets),
        "recommend": {"size_budget_bytes": float(getc(cfg, "size_budget_bytes", 8 * 2 ** 30)),
                      "resolution": None, "in_core": None, "tau_options": [],
                      "tau_max": sp.p.tau_max, "tau_applied": sp.p.tau_max,
                      "tau_auto": isinstance(getc(cfg, "tau_max", "auto"), str),
                      "tau_reference": 0.5, "tau_pinned_waste": False, "tau_applied_cost": 0.0,
                      "tau_reason": "the grid is solved whole on the device, so there is no "
                                    "halo to trade the horizon against"},
        "dtype": prep.dtype,
        "elem_bytes": eb,
        "bytes_per_target": cells * eb,
        "n_targets": ntg,
        "bytes_total": cells * eb * ntg,
        "chunks_per_target": -(-cells // prep.chunk_elements),
        "controls": sp.nctl,
        "storage": sp.storage,
        "gpu_available": mem is not None,
        "gpu_fits": bool(fits),
        "gpu_need_gb": need / 1e9,
        "gpu_free_gb": (mem[0] / 1e9) if mem else 0.0,
        "out_of_core": {"mode": "incore" if fits or mem is None else "ooc"},
        "driver": "whole_grid",
        "grid_balance": dvd / cell_cm if acc > 0 else float("nan"),
        "dv_distance_cm": dvd,
        "max_accel_cm_s2": acc,
        "cell_cm": cell_cm,
        "cell_cm_s": dv,
        "runtime": runtime,
    }
