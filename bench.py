#!/usr/bin/env python3
"""Benchmark: Bellman cell-control updates per second of the plain FP32
value-iteration sweep on one B200 per rank.

A step is one Jacobi sweep over the whole table (every cell x every control).
Workload: 96 x 96 x 64 x 21 x 21 x 21 = 5,462,360,064 cells, 125 controls
({-1,-0.5,0,0.5,1}^3), dt 0.03 s, RK2, 8 rectangular obstacles, seed 0 (the
largest table that fits one B200 in core; `--workload medium` runs the
48 x 48 x 32 x 15^3 table) -- one table per GPU; with --gpus N every rank
solves its own independent table (different seed), so per-GPU work is fixed
(weak scaling, no data-path collective; the only collective is the max of the
timings).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`--impl reference` times the reference's CPU algorithm (the oracle port of
solve.jl's sweep, all host threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "peregrine-desktop_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "Bellman cell-control updates/s; time-to-converge vs plain FP32 at ≤2 ms max err"
UNIT = "cell-control updates/s"
WORKLOAD = "large"
KERNEL_SOURCE = os.path.join(PKG, "csrc", "pg_stencil_r.cuh")


def profile_path():
    """The committed ncu summary of the sweep kernel on this workload."""
    return os.path.join(ROOT, "profiles", f"k_stencil_r_{WORKLOAD}_fp32.md")


def kernel_source_sha(path=None):
    """SHA-256 of the sweep kernel's code: pg_stencil_r.cuh with its //
    comments, trailing blanks and blank lines removed, so that editing a
    comment does not retire a profile of the same code."""
    import hashlib
    import re
    with open(path or KERNEL_SOURCE, encoding="utf-8") as fh:
        lines = [re.sub(r"//.*$", "", ln).rstrip() for ln in fh.read().splitlines()]
    code = "\n".join(ln for ln in lines if ln)
    return hashlib.sha256(code.encode("utf-8")).hexdigest()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "of measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "of fallback (no MEASURED_PEAKS.json: an earlier copy measurement on this pool)"


def blend_tiling(n1: int, n2: int) -> tuple:
    """(tile rows, row groups) of the register-resident sweep, the library's
    rule: a block's first groups * n2 threads own one column of four window
    rows each (4 groups >= rows + 3, groups * n2 <= 512, blocks of a multiple
    of 32 threads, at least 64); per candidate -- the most rows the groups
    allow, balanced over the plane -- the work per tile cell (50 per group
    blended, 55 per group of cells shifted, 10 per idle thread) and the warps
    per SM (512 threads); the cheapest with at least 12 warps per SM wins."""
    def cand(tx):
        groups = (tx + 6) // 4
        block = 32 * ((groups * n2 + 31) // 32)
        if block > 512:
            return None
        live = (tx + 3) // 4
        block = max(64, block)
        cost = (50.0 * groups * n2 + 55.0 * live * n2 + 10.0 * (block - groups * n2)) / (tx * n2)
        return (tx, groups, cost, (512 // block) * (block // 32))
    pick = None
    groups = 1
    while groups * n2 <= 512:
        txmax = min(n1, 4 * groups - 3)
        if txmax >= 1:
            nt = -(-n1 // txmax)
            c = cand(-(-n1 // nt))
            if c and (pick is None or ((c[3] >= 12) != (pick[3] >= 12) and c[3] >= 12)
                      or ((c[3] >= 12) == (pick[3] >= 12) and c[2] < pick[2])):
                pick = c
        groups += 1
    if pick is None:
        raise ValueError(f"no register-resident tiling for {n2} columns")
    return pick[0], pick[1]


def blend_tile_rows(n1: int, n2: int) -> int:
    return blend_tiling(n1, n2)[0]


def onchip_rooflines(pr, rate_per_gpu: float, elem: int, peaks_onchip) -> dict:
    """The sweep's on-chip ceilings.  Per cell-control the register-resident
    kernel blends 16 corner values held in registers into 4 G / TX window
    values (G row groups of four rows for TX tile rows), writes them to
    shared memory as FP32, and for its four cells of one column reads five
    window rows of two values (2.5 rows per cell when the successor rows are
    consecutive), a row entry of 32 B per four cells, a column entry of 8 B
    per four cells and a warp's mask words (a broadcast); it spends
    16 (4 G / TX) + 3 FMAs plus three subtracts and an add.  (The corner
    planes are read from L2 once per group of controls, not per control.)"""
    n1, n2 = int(pr.grid.n[0]), int(pr.grid.n[1])
    tx, groups = blend_tiling(n1, n2)
    win = 4.0 * groups / tx
    del elem  # the storage type only changes the once-per-group loads
    bytes_cc = 4 * win + 10 + 8 + 2 + 4 / 32
    flops_cc = 2 * (16 * win + 3) + 4
    out = {"tile_rows": tx, "row_groups": groups, "bytes_per_update": bytes_cc,
           "flops_per_update": flops_cc}
    if peaks_onchip:
        g = rate_per_gpu * bytes_cc / 1e9
        f = rate_per_gpu * flops_cc / 1e12
        out["shared_memory"] = {"achieved": g, "peak": peaks_onchip["smem_gbs"], "unit": "GB/s",
                         "frac": g / peaks_onchip["smem_gbs"],
                         "peak_source": "measured on this GPU (pg_measure_peaks, shared-memory "
                                        "read bandwidth)"}
        out["fma"] = {"achieved": f, "peak": peaks_onchip["fma_tflops"], "unit": "TFLOP/s",
                      "frac": f / peaks_onchip["fma_tflops"],
                      "peak_source": "measured on this GPU (pg_measure_peaks, FP32 FMA)"}
        out["l2_read_gbs_measured"] = peaks_onchip["l2_gbs"]
    return out


def _profile_lines():
    p = profile_path()
    if not os.path.exists(p):
        return None
    return [ln.strip() for ln in open(p)]


def profile_current() -> bool:
    """Whether the committed profile was captured from the kernel source this
    tree builds (its `source_sha256:` line against pg_stencil_r.cuh)."""
    lines = _profile_lines()
    if not lines:
        return False
    for ln in lines:
        if ln.startswith("source_sha256:"):
            return ln.split(":", 1)[1].strip().split()[0] == kernel_source_sha()
    return False


def profiled_value(key: str):
    """A number from the committed ncu summary of the sweep kernel (a line
    `key: N ...`), or None -- also None when that profile was captured from
    another version of the kernel source, so a stale figure is never
    reported as this kernel's."""
    lines = _profile_lines()
    if not lines or not profile_current():
        return None
    for ln in lines:
        if ln.startswith(key + ":"):
            try:
                return float(ln.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def profiled_traffic():
    """DRAM bytes per launch of the sweep kernel from the committed ncu
    summary (a line `traffic_bytes_per_launch: N`), or None."""
    return profiled_value("traffic_bytes_per_launch")


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.fh = None

    def __enter__(self):
        try:
            self.fh = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.fh is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.fh.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.fh.read().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sample(pr, budget_s: float, threads: int, rank_seed: int = 0):
    """The oracle (a CPU restatement of the reference's sweep) on a bounded,
    contiguous slab of cells in the middle of the table."""
    import numpy as np
    from oracle import oracle as og
    g = og.copy_struct(pr.grid.to_c(), og.OGrid)
    m = og.copy_struct(pr.model.to_c(), og.OModel)
    p = og.copy_struct(pr.params, og.OParams)
    V = np.full(pr.ncells, np.float32(pr.params.cap), np.float32)
    V[pr.seeds] = 0.0
    mid = pr.ncells // 2
    probe = 8192 * max(1, threads)
    t0 = time.perf_counter()
    og.sweep_jacobi_slab(V, pr.occ, g, m, pr.ctl, p, mid, mid + probe, 0, threads)
    rate = probe / max(time.perf_counter() - t0, 1e-6)
    n = int(min(max(rate * budget_s, probe), pr.ncells // 4))
    t0 = time.perf_counter()
    og.sweep_jacobi_slab(V, pr.occ, g, m, pr.ctl, p, mid, mid + n, 0, threads)
    dt = time.perf_counter() - t0
    return n, dt, n * pr.nctl / dt


def problem_for_rank(rank: int):
    from peregrine_hjb.synth import Problem
    return Problem(WORKLOAD, seed=rank)


def workload_config(pr, extra=None):
    from peregrine_hjb.synth import WORKLOADS
    n = pr.grid.n
    rects = WORKLOADS[WORKLOAD]["rects"]
    cfg = {
        "workload": f"plain FP32 value iteration, {n[0]}x{n[1]}x{n[2]}x{n[3]}x{n[4]}x{n[5]} "
                    f"= {pr.ncells} cells, {pr.nctl} controls ({pr.cfg['control_set']}), "
                    f"dt {pr.cfg['dt']} s, RK2, {rects} rectangles, 64-corner multilinear, "
                    f"one table per GPU",
        "cells": pr.ncells,
        "controls": pr.nctl,
        "step": "one Jacobi sweep over every cell and control",
        "l2": f"inputs larger than L2 (V is {pr.ncells * 4 / 1e9:.3g} GB per buffer, two "
              f"buffers)",
        "kernel": "k_stencil_r<float> (register-resident blend-then-shift)",
    }
    if extra:
        cfg.update(extra)
    return cfg


def run_reference(args, rank, world):
    """--impl reference: the oracle port on all host threads, rank 0 only."""
    if rank != 0:
        return 0
    from oracle import oracle as og
    threads = og.available_threads()
    pr = problem_for_rank(0)
    per_step = []
    samples = []
    for s in range(args.warmup + args.steps):
        n, dt, rate = cpu_sample(pr, 6.0, threads)
        if s >= args.warmup:
            per_step.append(rate)
            samples.append((n, dt))
    value = statistics.mean(per_step)
    n0 = samples[0][0]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * statistics.mean(dt for _, dt in samples),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded PCG64 job in the reference's input schemas)",
        "impl": "reference",
        "config": workload_config(pr, {"kernel": "CPU restatement of the reference sweep "
                                                 "(oracle/pg_oracle.c), OpenMP"}),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{n0} contiguous cells x {pr.nctl} controls per step "
                                   f"(one Jacobi pass over a mid-table slab, about 6 s)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist
    from peregrine_hjb import _lib

    torch.cuda.set_device(local_rank)
    pr = problem_for_rank(rank)
    ctx = _lib.Context(local_rank)
    ctx.load_problem(pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.ctl, args.storage)
    opts = _lib.default_opts(stop_rule=_lib.STOP_MAXNORM, kernel=_lib.KERNEL_STENCIL,
                             storage=args.storage, polish_sweeps=0)
    # seed and take the warm-up sweeps (real Bellman updates from the seeded table)
    ctx.solve(pr.seeds, max(args.warmup, 3), 0.0, opts)

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- device-resident throughput: K sweeps, CUDA events on the launch stream
    launches0 = ctx.launch_count()
    barrier()
    torch.cuda.synchronize()
    with Clocks(local_rank) as clk:
        ms = ctx.time_sweeps(0, args.steps, _lib.KERNEL_STENCIL)
    torch.cuda.synchronize()
    barrier()
    launches = ctx.launch_count() - launches0
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    cc_per_sweep = pr.ncells * pr.nctl
    value = world * cc_per_sweep / (ms_max / 1000.0)
    if args.only_device:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
                              "workload": WORKLOAD, "storage": args.storage,
                              "gpu_launches": launches,
                              "clocks": clk.summary(), "only_device": True}), flush=True)
        ctx.close()
        return 0

    # ---- end to end through the public one-shot call, host buffers in/out
    # sweeps per end-to-end call: a real solve runs hundreds; a few keep the
    # timed calls short while the per-call load, prep and copies still count
    e2e_sweeps = 10 if pr.ncells < (1 << 30) else 2
    occ_h = torch.from_numpy(pr.occ).pin_memory()
    ctl_h = torch.from_numpy(pr.ctl).pin_memory()
    tidx_h = torch.from_numpy(pr.seeds).pin_memory()
    V_h = torch.empty(pr.ncells, dtype=torch.float32).pin_memory()
    occ_n, ctl_n, tidx_n, V_n = (x.numpy() for x in (occ_h, ctl_h, tidx_h, V_h))
    e2e_steps = max(1, min(args.steps, 3 if pr.ncells < (1 << 30) else 2))
    import ctypes as C
    lib = _lib.load_library()
    res = _lib.SolveResult()
    e2e_opts = _lib.default_opts(stop_rule=_lib.STOP_MAXNORM, kernel=_lib.KERNEL_STENCIL)
    cb = _lib.PROGRESS_CB()
    times = []
    for _ in range(e2e_steps + 1):
        barrier()
        t0 = time.perf_counter()
        rc = lib.pg_solve_value(ctx._h, C.byref(pr.grid.to_c()), C.byref(pr.model.to_c()),
                                C.byref(pr.params), occ_n.ctypes.data, tidx_n.ctypes.data,
                                tidx_n.size, ctl_n.ctypes.data, pr.nctl, e2e_sweeps, 0.0,
                                C.byref(e2e_opts), V_n.ctypes.data, C.byref(res), cb, None)
        if rc != 0:
            raise RuntimeError(lib.pg_last_error().decode())
        times.append(time.perf_counter() - t0)
    e2e_t = torch.tensor([statistics.mean(times[1:])], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_s = float(e2e_t.item())
    e2e_value = world * e2e_sweeps * cc_per_sweep / e2e_s
    h2d = pr.occ.nbytes + pr.ctl.nbytes + pr.seeds.nbytes
    d2h = pr.ncells * 4
    if not np.all(np.isfinite(V_n)):
        raise RuntimeError("non-finite values in the solved table")

    if rank != 0:
        ctx.close()
        return 0

    # ---- roofline of the dominant kernel (the stencil sweep)
    peak, peak_kind = peaks()
    alg_bytes = 2 * 4 * pr.ncells  # read V once + write V once per sweep
    achieved = alg_bytes / (ms / 1000.0) / 1e9
    traffic = profiled_traffic()
    try:
        pk = _lib.measure_peaks(local_rank)
    except Exception as exc:  # the line still reports the HBM roofline
        print(f"peak probes failed: {exc}", file=sys.stderr)
        pk = None
    onchip = onchip_rooflines(pr, cc_per_sweep / (ms / 1000.0), 4, pk)
    # the binding ceiling: instruction issue (4 warp schedulers per SM, one
    # instruction each per clock, at the SM clock sampled during the timing)
    wipu = profiled_value("warp_instructions_per_update")
    clk_mhz = (clk.summary() or {}).get("sm_mhz")
    sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
    if wipu and clk_mhz:
        issued = cc_per_sweep / (ms / 1000.0) * wipu
        peak_issue = sms * 4 * clk_mhz * 1e6
        onchip["issue"] = {"achieved": issued, "peak": peak_issue, "unit": "warp instructions/s",
                           "frac": issued / peak_issue,
                           "instructions_per_update": wipu,
                           "peak_source": f"{sms} SMs x 4 schedulers x {clk_mhz:.0f} MHz (sampled)",
                           "instructions_source": "ncu summary in profiles/"}

    # ---- CPU baseline: the oracle on the host cores, bounded sample
    from oracle import oracle as og
    threads = og.available_threads()
    n_cpu, dt_cpu, cpu_rate = cpu_sample(pr, 12.0, threads)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded PCG64 job in the reference's input schemas)",
        "config": workload_config(pr, {"parallelism": f"{world} independent tables, one per GPU"}),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "timed": "CUDA events around the sweep launches on the context stream "
                              "(sweep kernel + its one-block residual reduction)",
                     "onchip": onchip},
        "cpu_baseline": {"value": cpu_rate, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{n_cpu} contiguous cells x {pr.nctl} controls, one Jacobi "
                                   f"pass ({dt_cpu:.1f} s) of the same workload"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "step": f"one pg_solve_value call: upload occupancy/controls/seeds, "
                        f"{e2e_sweeps} sweeps, read V back to pinned host memory"},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_accuracy(args, local_rank):
    """Time-to-converge at <= 2 ms max error.  The reference answer is plain
    FP32 iterated to its own fixed point (no cell changes any more, max-norm
    stop 1e-9 s); every storage -- FP32, and FP16 / BF16 / Q16 fixed point
    followed by FP32 polish sweeps -- is solved to a ladder of max-norm stop
    tolerances, and the device time of the cheapest run within 2 ms of the
    reference is its time-to-converge.  Errors against the FP64 table
    (max-norm 1e-9 s) are reported beside them: FP64 storage runs the
    precision oracle (the FP32 solver's admissibility and successor
    decisions, FP64 interpolation, min and residual), so that difference is
    the FP32 arithmetic's, not a different model's."""
    import numpy as np
    import torch
    from peregrine_hjb import _lib

    torch.cuda.set_device(local_rank)
    pr = problem_for_rank(0)
    base = (pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.seeds, pr.ctl)

    def solve(storage, tol, polish=0):
        kw = dict(storage=storage, polish_sweeps=polish)
        opts = _lib.default_opts(stop_rule=_lib.STOP_MAXNORM, kernel=_lib.KERNEL_STENCIL, **kw)
        return _lib.solve_value(*base, 20000 if tol < 1e-8 else args.max_sweeps, tol, opts,
                                device=local_rank)

    ref32, r32 = solve("fp32", 1e-9)
    ref32 = ref32.astype(np.float64)
    reached = (ref32 > 0) & (ref32 < float(pr.params.cap) - 1e-3)
    ref64 = None
    if not args.no_fp64:
        ref64, r64 = solve("fp64", 1e-9)
        ref64 = ref64.astype(np.float64)
        d64 = np.abs(ref32 - ref64)[reached]
    target = 2e-3
    runs, ttc = {}, {}
    for name in args.storages.split(","):
        runs[name] = []
        store = name.replace("-nopolish", "")
        polish = 0 if (store == "fp32" or name.endswith("-nopolish")) else args.max_sweeps
        for tol in (float(t) for t in args.tols.split(",")):
            V, res = solve(store, tol, polish)
            V = V.astype(np.float64)
            err = np.abs(V - ref32)[reached]
            row = {"tol": tol, "sweeps": res.iterations - res.polish_iterations,
                   "polish_sweeps": res.polish_iterations, "kernel_s": res.kernel_ms / 1000.0,
                   "max_err": float(err.max()), "rms_err": float(np.sqrt(np.mean(err ** 2)))}
            if ref64 is not None:
                e64 = np.abs(V - ref64)[reached]
                row["max_err_vs_fp64"] = float(e64.max())
                row["rms_err_vs_fp64"] = float(np.sqrt(np.mean(e64 ** 2)))
            runs[name].append(row)
        ok = [r["kernel_s"] for r in runs[name] if r["max_err"] <= target]
        ttc[name] = min(ok) if ok else None
    line = {"report": "time_to_converge", "workload": WORKLOAD, "cells": pr.ncells,
            "controls": pr.nctl, "target_max_err_s": target,
            "reference": {"storage": "fp32", "stop": "max-norm < 1e-9 s (its own fixed point)",
                          "sweeps": r32.iterations, "kernel_s": r32.kernel_ms / 1000.0},
            "error_over": "reached cells (0 < V < cap)",
            "runs": runs, "time_to_converge_s": ttc}
    if ref64 is not None:
        line["fp64"] = {"stop": "max-norm < 1e-9 s", "sweeps": r64.iterations,
                        "max_diff_vs_reference": float(d64.max()),
                        "rms_diff_vs_reference": float(np.sqrt(np.mean(d64 ** 2)))}
    if ttc.get("fp32"):
        line["speedup_vs_fp32"] = {k: (ttc["fp32"] / v if v else None) for k, v in ttc.items()}
    print(json.dumps(line), flush=True)
    return 0


def _max_rms_over(V, ref, cap, device, chunk=1 << 27):
    """max and RMS of |V - ref| over the reached cells (0 < ref < cap - 1 ms)
    of two host tables, in chunks on the device."""
    import torch
    mx, ss, n = 0.0, 0.0, 0
    for i in range(0, ref.size, chunk):
        r = torch.from_numpy(ref[i:i + chunk]).to(device)
        v = torch.from_numpy(V[i:i + chunk]).to(device)
        m = (r > 0) & (r < cap - 1e-3)
        e = (v.double() - r.double()).abs()[m]
        if e.numel():
            mx = max(mx, float(e.max()))
            ss += float((e * e).sum())
            n += int(e.numel())
    return mx, math.sqrt(ss / max(n, 1)), n


def run_converge(args, local_rank):
    """Time-to-converge of plain FP32 value iteration on one table from one
    trajectory, for grids too large to solve once per stop tolerance: the
    benchmarked sweep runs from the initial table (cap everywhere, zero at
    the targets) until no cell changes by more than 1e-9 s (the table's own
    fixed point, the reference answer); at the first sweep whose max-norm
    change is within each tolerance of --tols the table is copied to host
    memory, and afterwards each copy is compared with the fixed point over
    the reached cells.  The time of a stop tolerance is the sweeps' device
    time up to that sweep; the time-to-converge is the least time whose table
    lies within 2 ms of the fixed point.  With --storages fp16, one FP16
    solve followed by FP32 polish sweeps (the library's 16-bit pattern) is
    then made at the loosest tolerance whose FP32 table met 2 ms, and
    compared with the same fixed point."""
    import numpy as np
    import torch
    from peregrine_hjb import _lib

    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    pr = problem_for_rank(0)
    cap = float(pr.params.cap)
    ladder = sorted((float(t) for t in args.tols.split(",")), reverse=True)
    snaps = []
    ctx = _lib.Context(local_rank)
    try:
        ctx.load_problem(pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.ctl, "fp32")
        opts = _lib.default_opts(stop_rule=_lib.STOP_MAXNORM, kernel=_lib.KERNEL_STENCIL)
        ctx.solve(pr.seeds, 0, 0.0, opts)  # the initial table, no sweep
        dev_s, it, k, dm, trace = 0.0, 0, 0, float("inf"), []
        while it < args.max_sweeps and dm > 1e-9:
            t0 = time.perf_counter()
            d, dm, _ = ctx.sweep(phase=it, kernel=_lib.KERNEL_STENCIL)
            dev_s += time.perf_counter() - t0
            it += 1
            if it % 25 == 0:
                trace.append([it, dm])
            while k < len(ladder) and dm <= ladder[k]:
                snaps.append({"tol": ladder[k], "sweeps": it, "sweep_s": dev_s, "V": ctx.get_value()})
                k += 1
        ref = ctx.get_value()
        ref_sweeps, ref_s = it, dev_s
    finally:
        ctx.close()
    rows = []
    for s in snaps:
        mx, rms, n = _max_rms_over(s.pop("V"), ref, cap, dev)
        s.update(max_err=mx, rms_err=rms)
        rows.append(s)
    ok = [r["sweep_s"] for r in rows if r["max_err"] <= 2e-3]
    line = {"report": "time_to_converge_trajectory", "workload": WORKLOAD, "cells": pr.ncells,
            "controls": pr.nctl, "target_max_err_s": 2e-3, "storage": "fp32",
            "kernel": "k_stencil_r (the benchmarked sweep)",
            "timing": "host clock around the synchronous per-sweep calls (the sweep on the "
                      "device plus one residual read-back per sweep)",
            "reference": {"stop": "max-norm <= 1e-9 s (its own fixed point)", "sweeps": ref_sweeps,
                          "sweep_s": ref_s},
            "error_over": "reached cells (0 < V < cap - 1 ms)", "fp32": rows,
            "maxnorm_every_25_sweeps": trace,
            "time_to_converge_s": {"fp32": min(ok) if ok else None}}
    print(json.dumps(line), flush=True)  # the FP32 record, before the longer FP16 leg
    if "fp16" in args.storages.split(",") and rows:
        # one FP16 + FP32-polish solve, at the loosest tolerance whose FP32
        # table met 2 ms (the polish has to reach the same point)
        tol = next((r["tol"] for r in rows if r["max_err"] <= 2e-3), rows[-1]["tol"])
        opts = _lib.default_opts(stop_rule=_lib.STOP_MAXNORM, kernel=_lib.KERNEL_STENCIL,
                                 storage="fp16", polish_sweeps=args.max_sweeps)
        V, res = _lib.solve_value(pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.seeds,
                                  pr.ctl, args.max_sweeps, tol, opts, device=local_rank)
        mx, rms, _ = _max_rms_over(V, ref, cap, dev)
        line["fp16"] = [{"tol": tol, "sweeps": res.iterations - res.polish_iterations,
                         "polish_sweeps": res.polish_iterations,
                         "kernel_s": res.kernel_ms / 1000.0, "max_err": mx, "rms_err": rms}]
        line["time_to_converge_s"]["fp16"] = res.kernel_ms / 1000.0 if mx <= 2e-3 else None
        print(json.dumps(line), flush=True)
    return 0


def run_ooc(args, local_rank):
    """Out-of-core rounds (pg_solve_ooc) of the workload: the table on the
    host in the store's type, updated in place tile by tile (the reference's
    store), one sweep per tile residency; the rate is cell-control updates
    per second of whole rounds, timed by the library from the first tile's
    upload to the last tile's write-back."""
    from peregrine_hjb import _lib
    pr = problem_for_rank(0)
    storage = {"fp32": _lib.STORE_F32, "fp16": _lib.STORE_F16, "bf16": _lib.STORE_BF16}[args.storage]
    opts = _lib.ooc_opts(tile_sweeps=1, jacobi=0, storage=storage,
                         kernel=_lib.KERNEL_STENCIL_ROWS)
    t0 = time.perf_counter()
    V, res = _lib.solve_ooc(pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.seeds, pr.ctl,
                            args.rounds, 0.0, opts, device=local_rank)
    wall = time.perf_counter() - t0
    upd = float(pr.ncells) * pr.nctl * res.rounds
    line = {"report": "out_of_core_rounds", "workload": WORKLOAD, "cells": pr.ncells,
            "controls": pr.nctl, "storage": args.storage,
            "store": "one host table updated in place, one sweep per tile residency",
            "sweep_kernel": "row stencil (k_stencil), decides every probe per sweep",
            "host_table_bytes": int(V.nbytes), "rounds": res.rounds,
            "tiles_per_round": res.tiles_per_round, "tile_rows": res.tile_rows,
            "halo_rows": res.halo_rows, "reach_rows": res.reach_rows,
            "elapsed_s": res.elapsed_ms / 1000.0, "kernel_s": res.kernel_ms / 1000.0,
            "updates_per_s": upd / (res.elapsed_ms / 1000.0),
            "updates_per_s_kernel_only": upd / (res.kernel_ms / 1000.0),
            "h2d_bytes": int(res.h2d_bytes), "d2h_bytes": int(res.d2h_bytes),
            "wall_s_with_host_allocation": wall, "last_maxnorm": res.last_maxnorm}
    print(json.dumps(line), flush=True)
    return 0


def run_batch(args, local_rank):
    """Batched sweeps against sequential ones: --tables tables drawn from the
    batch workload's distribution (positions 24-48, headings 16-32, velocity
    axes 9-15, 125 controls, each its own drivetrain, target and obstacles),
    FP32.  Sequential: each table alone in its own context, --steps sweeps
    timed on the device after 2 warm-up sweeps, summed over the tables.
    Batched: all tables in one batch, --steps sweeps per table in persistent
    launches captured as a CUDA graph, device time per sweep of all tables."""
    from peregrine_hjb import _lib
    from peregrine_hjb import batch as pb
    probs = pb.batch_problems(args.tables, seed=0)
    seq_ms, cells = 0.0, 0
    for pr in probs:
        with _lib.Context(local_rank) as ctx:
            ctx.load_problem(pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.ctl, "fp32")
            ctx.solve(pr.seeds, 0, 0.0, _lib.default_opts(kernel=_lib.KERNEL_STENCIL))
            seq_ms += ctx.time_sweeps(2, args.steps, _lib.KERNEL_STENCIL)
        cells += pr.ncells
    with _lib.Batch(local_rank, "fp32") as b:
        for pr in probs:
            b.add(pr.grid.to_c(), pr.model.to_c(), pr.params, pr.occ, pr.seeds, pr.ctl)
        b.solve(2, 0.0, 0, True)
        res = b.solve(args.steps, 0.0, 0, True)
    batch_ms = res.kernel_ms / max(res.sweeps, 1)
    line = {"report": "batched_sweeps", "tables": len(probs), "cells": cells,
            "controls": int(probs[0].nctl), "storage": "fp32", "sweeps_timed": int(res.sweeps),
            "sequential_ms_per_sweep_of_all_tables": seq_ms,
            "batched_ms_per_sweep_of_all_tables": batch_ms,
            "batched_vs_sequential": seq_ms / batch_ms if batch_ms > 0 else None,
            "graph": bool(res.graph)}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD,
                    help="synthetic workload (medium is the benchmark; medium_h8 is the "
                         "same planes and controls with 8 headings, for profiler captures)")
    ap.add_argument("--only-device", action="store_true",
                    help="time the device sweeps only (no end-to-end leg, no CPU baseline); "
                         "for profiler captures")
    ap.add_argument("--accuracy", action="store_true",
                    help="time-to-converge and FP32/FP64/FP16/BF16 error report instead of "
                         "the throughput line")
    ap.add_argument("--converge", action="store_true",
                    help="time-to-converge of one FP32 trajectory with snapshots at --tols "
                         "(for grids too large for --accuracy)")
    ap.add_argument("--ooc", action="store_true",
                    help="out-of-core rounds of the workload (e.g. --workload xlarge_ooc "
                         "--storage fp16) instead of the throughput line")
    ap.add_argument("--rounds", type=int, default=1, help="rounds of --ooc")
    ap.add_argument("--batch", action="store_true",
                    help="batched against sequential sweeps of --tables tables of the batch "
                         "workload's distribution")
    ap.add_argument("--tables", type=int, default=16, help="tables of --batch")
    ap.add_argument("--storages", default="fp32,fp16,bf16,q16,q16-nopolish",
                    help="storages of the accuracy report; -nopolish: no FP32 polish")
    ap.add_argument("--no-fp64", action="store_true",
                    help="accuracy report without the FP64 comparison (slow on large grids)")
    ap.add_argument("--tols", default="1e-4,3e-5,1e-5,3e-6",
                    help="max-norm stop tolerances of the accuracy report")
    ap.add_argument("--storage", default="fp32",
                    help="storage of V for --only-device timing (the benchmark line is FP32)")
    ap.add_argument("--max-sweeps", type=int, default=4000)
    args = ap.parse_args()
    globals()["WORKLOAD"] = args.workload
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.accuracy:
        return run_accuracy(args, local_rank)
    if args.converge:
        return run_converge(args, local_rank)
    if args.ooc:
        return run_ooc(args, local_rank)
    if args.batch:
        return run_batch(args, local_rank)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
