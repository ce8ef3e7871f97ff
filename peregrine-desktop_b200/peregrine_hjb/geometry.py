"""Field geometry and the (x, y, h) occupancy, mirroring
solver/src/Pipeline.jl:29-399.

Runs once per run on the host, in Float64 like the reference, vectorised over
cells with numpy (the reference loops cell by cell; every per-cell expression
below keeps the reference's operation order, so each cell's test rounds the
same way).
"""
from __future__ import annotations

import math

import numpy as np

EPS = np.finfo(np.float64).eps


def inpoly(px, py, poly) -> np.ndarray:
    """Ray-casting point-in-polygon (Pipeline.jl:30-44).  px, py: arrays;
    poly: (N, 2) array, or (..., N, 2) for one polygon per point."""
    poly = np.asarray(poly, dtype=np.float64)
    n = poly.shape[-2]
    inside = np.zeros(np.broadcast(px, py).shape, dtype=bool)
    j = n - 1
    for i in range(n):
        xi, yi = poly[..., i, 0], poly[..., i, 1]
        xj, yj = poly[..., j, 0], poly[..., j, 1]
        with np.errstate(divide="ignore", invalid="ignore"):
            cond = ((yi > py) != (yj > py)) & (px < (xj - xi) * (py - yi) / (yj - yi + EPS) + xi)
        inside ^= cond
        j = i
    return inside


def _d(a, b, c):
    return (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0])


def seg_cross(p1, p2, p3, p4):
    """Pipeline.jl:47-52; points are (x, y) pairs of arrays."""
    d1 = _d(p3, p4, p1)
    d2 = _d(p3, p4, p2)
    d3 = _d(p1, p2, p3)
    d4 = _d(p1, p2, p4)
    return ((d1 > 0) != (d2 > 0)) & ((d3 > 0) != (d4 > 0))


def pt_seg_dist(p, a, b):
    """Pipeline.jl:83-90"""
    abx = b[0] - a[0]
    aby = b[1] - a[1]
    L2 = abx * abx + aby * aby
    with np.errstate(divide="ignore", invalid="ignore"):
        t = np.where(L2 <= 0, 0.0, np.clip(((p[0] - a[0]) * abx + (p[1] - a[1]) * aby) / L2, 0.0, 1.0))
    dx = p[0] - (a[0] + t * abx)
    dy = p[1] - (a[1] + t * aby)
    return np.sqrt(dx * dx + dy * dy)


def seg_seg_dist(a1, a2, b1, b2):
    """Pipeline.jl:93-97"""
    d = np.minimum(np.minimum(pt_seg_dist(a1, b1, b2), pt_seg_dist(a2, b1, b2)),
                   np.minimum(pt_seg_dist(b1, a1, a2), pt_seg_dist(b2, a1, a2)))
    return np.where(seg_cross(a1, a2, b1, b2), 0.0, d)


def _pt(arr, i):
    return (arr[..., i, 0], arr[..., i, 1])


def polys_overlap(A, B):
    """Pipeline.jl:62-80.  A: (..., na, 2) per-cell polygons; B: (nb, 2)."""
    na, nb = A.shape[-2], B.shape[-2]
    hit = np.zeros(A.shape[:-2], dtype=bool)
    for i in range(na):
        hit |= inpoly(A[..., i, 0], A[..., i, 1], B)
    for j in range(nb):
        hit |= inpoly(np.full(A.shape[:-2], B[j, 0]), np.full(A.shape[:-2], B[j, 1]), A)
    for i in range(na):
        a1, a2 = _pt(A, i), _pt(A, (i + 1) % na)
        for j in range(nb):
            hit |= seg_cross(a1, a2, _pt(B, j), _pt(B, (j + 1) % nb))
    return hit


def polys_too_close(A, B, d):
    """Pipeline.jl:109-123"""
    hit = polys_overlap(A, B)
    if d <= 0:
        return hit
    na, nb = A.shape[-2], B.shape[-2]
    for i in range(na):
        a1, a2 = _pt(A, i), _pt(A, (i + 1) % na)
        for j in range(nb):
            hit |= seg_seg_dist(a1, a2, _pt(B, j), _pt(B, (j + 1) % nb)) < d
    return hit


def point_too_close(px, py, B, d):
    """Pipeline.jl:126-136"""
    hit = inpoly(px, py, B)
    if d <= 0:
        return hit
    nb = B.shape[0]
    for j in range(nb):
        hit |= pt_seg_dist((px, py), _pt(B, j), _pt(B, (j + 1) % nb)) < d
    return hit


def heading_bin_angles(nh: int, substeps: int):
    """Pipeline.jl:152-160"""
    step = 2 * math.pi / nh
    half = step / 2
    out = []
    for k in range(int(nh)):
        c = -math.pi + k * step
        out.append([c] if substeps <= 1 else
                   [c - half + 2 * half * (s - 1) / (substeps - 1) for s in range(1, int(substeps) + 1)])
    return out


def footprint_reach(robot, theta):
    """Pipeline.jl:170-181"""
    if robot is None or len(robot) < 3:
        return (0.0, 0.0, 0.0, 0.0)
    c, s = math.cos(theta), math.sin(theta)
    xlo = xhi = ylo = yhi = -math.inf
    for rx0, ry0 in robot:
        rx = c * rx0 - s * ry0
        ry = s * rx0 + c * ry0
        xlo = max(xlo, -rx)
        xhi = max(xhi, rx)
        ylo = max(ylo, -ry)
        yhi = max(yhi, ry)
    return (xlo, xhi, ylo, yhi)


def wall_box(bounds, robot, clearance, theta):
    """Pipeline.jl:199-206"""
    rxlo, rxhi, rylo, ryhi = footprint_reach(robot, theta)
    d = float(clearance)
    return (bounds[0] + d + rxlo, bounds[2] - d - rxhi, bounds[1] + d + rylo, bounds[3] - d - ryhi)


def feasible_bounds(bounds, robot, clearance, nh, substeps):
    """Pipeline.jl:227-251"""
    xlo, xhi, ylo, yhi = math.inf, -math.inf, math.inf, -math.inf
    nfeas = 0
    for angles in heading_bin_angles(nh, substeps):
        bxlo, bxhi, bylo, byhi = -math.inf, math.inf, -math.inf, math.inf
        for th in angles:
            a, b, c, d = wall_box(bounds, robot, clearance, th)
            bxlo, bxhi = max(bxlo, a), min(bxhi, b)
            bylo, byhi = max(bylo, c), min(byhi, d)
        if not (bxlo <= bxhi and bylo <= byhi):
            continue
        nfeas += 1
        xlo, xhi = min(xlo, bxlo), max(xhi, bxhi)
        ylo, yhi = min(ylo, bylo), max(yhi, byhi)
    if nfeas == 0:
        raise ValueError(
            "the robot does not fit inside the field at any heading: the field is "
            f"{round(bounds[2] - bounds[0], 1)} x {round(bounds[3] - bounds[1], 1)} cm, and the "
            f"footprint plus {clearance} cm of clearance needs more than that. Check the units "
            "on the robot polygon, or lower the clearance")
    return dict(xlo=xlo, xhi=xhi, ylo=ylo, yhi=yhi, headings=nfeas)


def build_occupancy(g, polys, margin_cm, robot=None, substeps: int = 3, clearance_cm: float = 0.0,
                    bounds=None, wall_clearance_cm=None) -> np.ndarray:
    """build_occupancy (Pipeline.jl:287-399).  Returns Nx*Ny*Nh uint8 in
    (i*Ny+j)*Nh+k order."""
    if wall_clearance_cm is None:
        wall_clearance_cm = clearance_cm
    nx, ny, nh = g.n[0], g.n[1], g.n[2]
    occ = np.zeros((nx, ny, nh), dtype=bool)
    point_robot = robot is None or len(robot) < 3
    R = None if point_robot else np.asarray(robot, dtype=np.float64)
    rad = 0.0 if point_robot else float(np.max(np.sqrt(R[:, 0] ** 2 + R[:, 1] ** 2)))
    tol = 1.0e-3
    xs = g.axis(0).astype(np.float64)
    ys = g.axis(1).astype(np.float64)
    step0, step1 = float(g.step[0]), float(g.step[1])
    lo0, lo1 = float(g.lo[0]), float(g.lo[1])
    P_list = [np.asarray(P, dtype=np.float64) for P in polys]
    for k in range(nh):
        thc = float(g.axisvalue(2, k))
        half = float(g.step[2]) / 2
        angles = [thc] if substeps <= 1 else [thc - half + 2 * half * (s - 1) / (substeps - 1)
                                               for s in range(1, substeps + 1)]
        if bounds is not None:
            for th in angles:
                bxlo, bxhi, bylo, byhi = wall_box(bounds, None if point_robot else R.tolist(),
                                                  wall_clearance_cm, th)
                rows = (xs < bxlo - tol) | (xs > bxhi + tol)
                occ[rows, :, k] = True
                cols = (ys < bylo - tol) | (ys > byhi + tol)
                occ[:, cols, k] = True
        for th in angles:
            if not point_robot:
                c, s = math.cos(th), math.sin(th)
                Rr = np.stack([c * R[:, 0] + (-s) * R[:, 1], s * R[:, 0] + c * R[:, 1]], axis=1)
            for P in P_list:
                pad = rad + margin_cm + clearance_cm
                x0 = P[:, 0].min() - pad
                x1 = P[:, 0].max() + pad
                y0 = P[:, 1].min() - pad
                y1 = P[:, 1].max() + pad
                i0 = max(0, math.floor((x0 - lo0) / step0))
                i1 = min(nx - 1, math.ceil((x1 - lo0) / step0))
                j0 = max(0, math.floor((y0 - lo1) / step1))
                j1 = min(ny - 1, math.ceil((y1 - lo1) / step1))
                if i1 < i0 or j1 < j0:
                    continue
                sub = occ[i0:i1 + 1, j0:j1 + 1, k]
                free = ~sub
                if not free.any():
                    continue
                II, JJ = np.nonzero(free)
                px = xs[i0 + II]
                py = ys[j0 + JJ]
                if point_robot:
                    hit = point_too_close(px, py, P, clearance_cm)
                else:
                    body = Rr[None, :, :] + np.stack([px, py], axis=1)[:, None, :]
                    hit = polys_too_close(body, P, clearance_cm)
                sub[II, JJ] = hit
                occ[i0:i1 + 1, j0:j1 + 1, k] = sub
    if margin_cm > 0:
        rx = max(0, math.ceil(margin_cm / step0))
        ry = max(0, math.ceil(margin_cm / step1))
        if rx > 0 or ry > 0:
            src = occ.copy()
            out = occ.copy()
            for di in range(-rx, rx + 1):
                for dj in range(-ry, ry + 1):
                    xs_src = slice(max(0, -di), min(nx, nx - di))
                    ys_src = slice(max(0, -dj), min(ny, ny - dj))
                    xs_dst = slice(max(0, di), min(nx, nx + di))
                    ys_dst = slice(max(0, dj), min(ny, ny + dj))
                    out[xs_dst, ys_dst, :] |= src[xs_src, ys_src, :]
            occ = out
    return occ.reshape(-1).astype(np.uint8)
