"""Seeding: target_cells (Pipeline.jl:504-536), the disk target region
(an additive job-JSON key) and the pre-flight check that a target seeds at
least one free cell (check_targets, Advise.jl:513-570)."""
from __future__ import annotations

import math

import numpy as np

f32 = np.float32


def _fwrap(c, n3):
    return f32(c - f32(np.floor(f32(c / n3)) * n3))


def target_cells(g, s, tol) -> np.ndarray:
    """0-based flat indices of the cells whose centre is within `tol` of `s`
    on every axis, or the single nearest cell (Pipeline.jl:504-536)."""
    ranges = []
    for k in range(6):
        c = f32(f32(f32(s[k]) - g.lo[k]) / g.step[k])
        if k == 2:
            c = _fwrap(c, f32(g.n[2]))
        r = f32(f32(tol[k]) / g.step[k])
        a = math.ceil(float(f32(c - r)))
        b = math.floor(float(f32(c + r)))
        if k == 2:
            ranges.append(range(a, b + 1))
        else:
            ranges.append(range(max(0, a), min(g.n[k] - 1, b) + 1))
    out = []
    seen = set()
    for i1 in ranges[0]:
        for i2 in ranges[1]:
            for i3 in ranges[2]:
                j3 = i3 % g.n[2]
                for i4 in ranges[3]:
                    for i5 in ranges[4]:
                        for i6 in ranges[5]:
                            f = int(g.flatten(i1, i2, j3, i4, i5, i6))
                            if f not in seen:
                                seen.add(f)
                                out.append(f)
    if not out:
        near = []
        for k in range(6):
            c = float(f32(f32(f32(s[k]) - g.lo[k]) / g.step[k]))
            r = int(round(c))
            near.append(r % g.n[2] if k == 2 else min(max(r, 0), g.n[k] - 1))
        out.append(int(g.flatten(*near)))
    return np.array(out, dtype=np.int64)


def region_cells(g, s, region) -> np.ndarray:
    """Seeds of a disk target region: cells whose (x, y) centre lies within
    `radius_cm` of the target, at any heading, with field speed below
    `speed_max_cm_s`, at any omega (or |omega| <= `w_max` when given).  Falls
    back to the nearest cell, like target_cells."""
    kind = str(region.get("kind", "disk")).lower()
    if kind != "disk":
        raise ValueError(f"unknown target_region kind '{kind}'")
    r = float(region.get("radius_cm", 10.0))
    smax = float(region.get("speed_max_cm_s", 20.0))
    wmax = region.get("w_max", None)
    xs = g.axis(0).astype(np.float64)
    ys = g.axis(1).astype(np.float64)
    vx = g.axis(3).astype(np.float64)
    vy = g.axis(4).astype(np.float64)
    ws = g.axis(5).astype(np.float64)
    dx = xs[:, None] - float(s[0])
    dy = ys[None, :] - float(s[1])
    xy = np.argwhere(dx * dx + dy * dy <= r * r)
    vv = np.argwhere(vx[:, None] ** 2 + vy[None, :] ** 2 < smax * smax)
    wi = np.arange(g.n[5]) if wmax is None else np.nonzero(np.abs(ws) <= float(wmax))[0]
    if len(xy) == 0 or len(vv) == 0 or len(wi) == 0:
        return target_cells(g, s, tuple(f32(g.step[k] * f32(0.5)) for k in range(6)))
    hh = np.arange(g.n[2])
    I1 = xy[:, 0][:, None, None, None]
    I2 = xy[:, 1][:, None, None, None]
    I3 = hh[None, :, None, None]
    I4 = vv[:, 0][None, None, :, None]
    I5 = vv[:, 1][None, None, :, None]
    I6 = wi[None, None, None, :]
    idx = np.asarray(g.flatten(I1, I2, I3, I4, I5, I6), dtype=np.int64)
    return np.unique(idx.reshape(-1))


def seeds_for(g, s, sp, cfg) -> np.ndarray:
    region = cfg.get("target_region") if hasattr(cfg, "get") else None
    if region:
        return region_cells(g, s, region)
    return target_cells(g, s, sp.ttol)


def free_seed_count(g, occ, seeds) -> int:
    i1, i2, i3, _, _, _ = g.unflatten(seeds)
    o = occ[(i1 * g.n[1] + i2) * g.n[2] + i3]
    return int(np.count_nonzero(o == 0))
