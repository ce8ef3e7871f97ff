"""The honing block of MODEL.JSON and the `honing` CLI mode.

Mirrors honing_gains / honing_only (solver/src/Run.jl:961-1258, 1397-1422)
and TABLE_FORMAT.md section 8.8: near the target the fitted model linearises
to a damped double integrator per body axis, dv/dt = B_eff u - Lambda v, and
three PID loops are placed on it in closed form.  The keys and the arithmetic
are the card format's (wizard/verify_tables.py re-derives every gain from the
card and fails a card that disagrees); the prose notes are this solver's own.

All arithmetic is Python float (IEEE double), as the reference's Float64.
"""
from __future__ import annotations

import math

from .grid import getc


def inv3(M):
    """3x3 inverse by cofactors; refuses a singular A_u (Run.jl:978-990)."""
    (a, b, c), (d, e, f), (g, h, i) = M
    det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g)
    if not (math.isfinite(det) and abs(det) > 1e-12):
        raise ValueError(f"A_u is singular (det = {det}); the drivetrain fit does not give the "
                         "three axes independent authority, so no controller can be derived "
                         "from it")
    return [[(e * i - f * h) / det, (c * h - b * i) / det, (b * f - c * e) / det],
            [(f * g - d * i) / det, (a * i - c * g) / det, (c * d - a * f) / det],
            [(d * h - e * g) / det, (b * g - a * h) / det, (a * e - b * d) / det]]


def _rows(M):
    return [[float(M[r][c]) for c in range(3)] for r in range(3)]


def honing_gains(m, cfg) -> dict:
    """The three honing PID controllers of drivetrain m under the config's
    honing_* keys (Run.jl:1056-1258)."""
    B, A, S = _rows(m.B), _rows(m.A), _rows(m.S)
    eps = [float(v) for v in m.eps]
    knee = float(m.knee)
    # Coulomb linearised inside its band: csign(v) = v / eps there
    Lam = [[-(A[r][c] + S[r][c] / eps[c]) for c in range(3)] for r in range(3)]

    hcm = float(getc(cfg, "honing_handoff_cm", 15.0))
    hrad = float(getc(cfg, "honing_handoff_rad", 0.25))
    hz = float(getc(cfg, "honing_loop_hz", 50.0))
    frac = float(getc(cfg, "honing_budget_frac", 0.5))
    budget = float(getc(cfg, "honing_budget", frac * knee))
    scale = float(getc(cfg, "honing_bandwidth_scale", 1.0))
    ishare = float(getc(cfg, "honing_integral_share", 0.25))
    if not (budget > 0 and frac > 0 and hz > 0 and scale > 0 and 0 < ishare < 1):
        raise ValueError(f"honing config must be positive (honing_budget={budget}, "
                         f"honing_budget_frac={frac}, honing_loop_hz={hz}, "
                         f"honing_bandwidth_scale={scale}, honing_integral_share={ishare}), "
                         "with the integral share below 1")
    if not budget <= 1:
        raise ValueError(f"honing_budget is {budget}, outside the octahedron "
                         "|fwd| + |strafe| + |turn| <= 1; the wheels would clip the command the "
                         f"gains are sized against (honing_budget_frac={frac} at a knee of {knee})")

    # the authority the tyres deliver at the design command r = budget / knee
    r_op = budget / knee
    tgain = 1.0 if r_op < 1e-6 else math.tanh(r_op) / r_op
    Binv = inv3([[tgain * B[r][c] for c in range(3)] for r in range(3)])
    lam = [Lam[i][i] for i in range(3)]
    Loff = [[0.0 if r == c else Lam[r][c] for c in range(3)] for r in range(3)]
    fcm = float(getc(cfg, "honing_fine_cm", 2.0))
    efine = [fcm, fcm, float(getc(cfg, "honing_fine_rad", 0.03))]

    def gains_at(w):
        # per channel (s + p)(s + w)^2 with p = max(lam - 2w, w): kd >= 0
        p = [max(lam[i] - 2 * w, w) for i in range(3)]
        kp = [w ** 2 + 2 * p[i] * w for i in range(3)]
        ki = [p[i] * w ** 2 for i in range(3)]
        kd = [p[i] + 2 * w - lam[i] for i in range(3)]
        Kp = [[Binv[r][c] * kp[c] for c in range(3)] for r in range(3)]
        Ki = [[Binv[r][c] * ki[c] for c in range(3)] for r in range(3)]
        Kd = [[Binv[r][c] * kd[c] - sum(Binv[r][k] * Loff[k][c] for k in range(3))
               for c in range(3)] for r in range(3)]
        return Kp, Ki, Kd, p, kd

    def prop_norm(w):
        Kp = gains_at(w)[0]
        return sum(abs(sum(Kp[r][c] * efine[c] for c in range(3))) for r in range(3))

    # the saturation bound on the bandwidth, by bisection (prop_norm grows with w)
    w_hi = 1e-3
    while prop_norm(w_hi) < budget and w_hi < 1e4:
        w_hi *= 2
    w_lo = w_hi / 2
    for _ in range(80):
        mid = 0.5 * (w_lo + w_hi)
        if prop_norm(mid) < budget:
            w_lo = mid
        else:
            w_hi = mid
    w_sat = w_lo
    w_loop = 2 * math.pi * hz / 10
    w = scale * min(w_sat, w_loop)
    if not (math.isfinite(w) and w > 0):
        raise ValueError(f"honing bandwidth came out as {w}; check honing_loop_hz, "
                         "honing_budget and honing_bandwidth_scale are positive")
    Kp, Ki, Kd, p, kd = gains_at(w)
    # anti-windup: the integral term gets at most `ishare` of the budget
    ilim = []
    for c in range(3):
        col = sum(abs(Ki[r][c]) for r in range(3))
        ilim.append(ishare * budget / (3 * col) if col > 0 else 0.0)

    return {
        "note": "PID gains for the final approach, derived in closed form from this model "
                "(no separate tuning step). The one chosen setting that matters is "
                "config.budget_frac, the share of the traction knee the approach may spend. "
                "Additive to schema 2.",
        "frame": "robot body",
        "law": "u = Kp*e + Ki*clamp(integral(e), -integral_limit, integral_limit) + "
               "Kd*d(e)/dt + u_ff",
        "error": {
            "vector": ["e_fwd", "e_strafe", "e_turn"],
            "units": ["cm", "cm", "rad"],
            "note": "e = target - current in the ROBOT BODY frame; the tables are field frame, "
                    "so rotate by -h first.",
        },
        "feedforward": {
            "formula": "u_ff = B_eff_inv*(a_ref + Lambda*v_ref)",
            "why": "Model inversion for the reference motion; optional, the gains stand alone. "
                   "Lambda already holds the linearised Coulomb term.",
        },
        "Kp": Kp, "Ki": Ki, "Kd": Kd, "B_eff_inv": Binv, "Lambda": Lam,
        "traction_gain": {
            "value": tgain,
            "why": f"B_eff = A_u * tanh(r)/r at r = budget/knee = {round(r_op, 4)}: the "
                   "authority delivered at the commanded level. B_eff_inv already contains it; "
                   "still apply the section 8.4 saturation to the final command.",
        },
        "integral_limit": {
            "value": ilim,
            "units": ["cm*s", "cm*s", "rad*s"],
            "why": f"Clamp each integrator to this before multiplying by Ki, so the integral "
                   f"term takes at most {round(ishare * 100)} percent of the command budget; "
                   "also stop integrating while the command is saturated.",
        },
        "omega": w,
        "poles": {
            "double": w,
            "third": p,
            "kd_diag": kd,
            "why": "Per axis the closed loop is (s+third)(s+omega)^2; kd is never negative.",
        },
        "omega_limits": {
            "saturation": w_sat,
            "loop_rate": w_loop,
            "bound_by": "saturation" if w_sat <= w_loop else "loop_rate",
            "why": "The smaller sets the bandwidth: `saturation` keeps Kp*e inside the budget "
                   "in the fine band, `loop_rate` keeps the poles within a tenth of the sample "
                   "rate.",
        },
        "handoff": {
            "cm": hcm, "rad": hrad,
            "note": "Where the tables hand over to this controller.",
        },
        "fine_band": {
            "cm": efine[0], "rad": efine[2],
            "why": "Inside this band the command stays within the budget.",
        },
        "config": {"loop_hz": hz, "budget": budget, "budget_frac": budget / knee,
                   "bandwidth_scale": scale, "integral_share": ishare,
                   "fine_cm": efine[0], "fine_rad": efine[2]},
        "derivation": "TABLE_FORMAT.md section 8.8",
    }


def honing_only(cfg, write_dir=None) -> dict:
    """The honing block alone, optionally rewritten into a solved run's
    MODEL.JSON (Run.jl:1397-1422): the whole file is rebuilt, and only when
    it was written from the same regression (its SHA-256)."""
    import json
    import os

    from .params import load_model
    from .run import model_json

    reg = str(cfg["regression"])
    m, _ = load_model(reg)
    zeroed = bool(getc(cfg, "zero_c", True))
    if zeroed:
        m = m.zeroed_c()
    mj = model_json(m, reg, zeroed, cfg)
    if write_dir is not None:
        path = os.path.join(str(write_dir), "MODEL.JSON")
        if not os.path.isfile(path):
            raise ValueError(f"no MODEL.JSON in {write_dir}; there is nothing to update there, "
                             "so solve the run first")
        with open(path, "r", encoding="utf-8-sig") as fh:
            old = json.load(fh)
        if str(getc(old, "regression_sha256", "")) != mj["regression_sha256"]:
            raise ValueError(f"{path} was written from a different regression than {reg}; its "
                             "tables were solved from that one, so these gains would describe "
                             "a robot the tables do not plan for")
        with open(path, "w") as fh:
            json.dump(mj, fh, indent=2)
    return mj["honing"]
