"""The honing block of MODEL.JSON and the `honing` CLI mode (host only).

Pinned to the worked example of TABLE_FORMAT.md section 8.8.6 (the block the
section 8.7 model produces at the default config) and, where the reference
tree is present, to the reference's own acceptance check, which re-derives
every gain from the card (wizard/verify_tables.py check_honing)."""
import importlib.util
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import PKG
from peregrine_hjb.honing import honing_gains, honing_only
from peregrine_hjb.params import Drivetrain
from peregrine_hjb.run import model_json
from peregrine_hjb.synth import write_job

VERIFY = "/root/reference/wizard/verify_tables.py"


def model_8_7() -> Drivetrain:
    """The section 8.7 example model (A_u, the velocity columns of A_s and
    A_sgn, coulomb_eps, knee 0.55)."""
    f = np.float32
    B = np.array([[318.44, 6.12, -4.87], [-5.33, 241.07, 3.94], [0.128, -0.061, 13.706]], f)
    A = np.array([[-2.418, 0.061, 1.472], [0.037, -3.106, -0.884], [0.0021, 0.0009, -4.233]], f)
    S = np.array([[-21.66, -0.42, 0.53], [-0.31, -27.94, -0.18], [0.004, -0.002, -1.882]], f)
    D = np.array([[-0.00417, 0.00008, 0.0312], [0.00011, -0.00583, -0.0204],
                  [0.0, 0.0, -0.2461]], f)
    return Drivetrain(B, A, np.zeros(3, f), S, D, np.zeros(3, f), np.array([5, 5, 0.15], f), 0.55)


# TABLE_FORMAT.md section 8.8.6, as printed (7 significant digits at most)
KAT = {
    "Kp": [[0.0360318, -0.0012504, 0.0381302], [0.0008021, 0.0652998, -0.0391032],
           [-0.0003329, 0.0003023, 2.4441237]],
    "Ki": [[0.0165087, -0.0005896, 0.0187047], [0.0003675, 0.0307902, -0.0191820],
           [-0.0001525, 0.0001425, 1.1989574]],
    "Kd": [[5.71816e-06, -7.74879e-05, 0.0171762], [-1.15812e-04, -2.37000e-06, -0.0089704],
           [2.28362e-04, 4.01840e-05, -0.0002003]],
    "B_eff_inv": [[0.00339581, -0.00008590, 0.00123129], [0.00007559, 0.00448599, -0.00126271],
                  [-0.00003138, 0.00002077, 0.07892471]],
    "Lambda": [[6.750000, 0.023000, -5.005333], [0.025000, 8.694000, 2.084000],
               [-0.002900, -0.000500, 16.779666]],
}


def close(got, want, rel=2e-5):
    """Equal to the printed digits: half a unit of the last printed digit of
    a 7-significant-digit number, or rel of its size."""
    return abs(got - want) <= max(rel * abs(want), 6e-8 if abs(want) < 1 else 6e-7)


def test_honing_worked_example():
    h = honing_gains(model_8_7(), {})
    for name, M in KAT.items():
        for r in range(3):
            for c in range(3):
                assert close(h[name][r][c], M[r][c]), (name, r, c, h[name][r][c], M[r][c])
    assert abs(h["traction_gain"]["value"] - 0.9242) < 5e-5
    assert close(h["omega"], 1.0148450)
    assert close(h["omega_limits"]["loop_rate"], 31.4159265)
    assert h["omega_limits"]["bound_by"] == "saturation"
    for got, want in zip(h["poles"]["third"], [4.720310, 6.664310, 14.749976]):
        assert close(got, want)
    # printed as 0.0: p + 2w - lam with p = lam - 2w, zero up to double rounding
    assert all(abs(v) < 1e-12 for v in h["poles"]["kd_diag"])
    for got, want in zip(h["integral_limit"]["value"], [1.3457636, 0.7269980, 0.0185283]):
        assert close(got, want)
    assert h["config"] == {"loop_hz": 50.0, "budget": 0.275, "budget_frac": 0.5,
                           "bandwidth_scale": 1.0, "integral_share": 0.25, "fine_cm": 2.0,
                           "fine_rad": 0.03}
    # saturation is tight: |Kp * [2, 2, 0.03]|_1 = budget
    n1 = sum(abs(sum(h["Kp"][r][c] * e for c, e in enumerate((2.0, 2.0, 0.03))))
             for r in range(3))
    assert abs(n1 - 0.275) < 1e-9


def test_honing_refusals():
    with pytest.raises(ValueError, match="outside the octahedron"):
        honing_gains(model_8_7(), {"honing_budget": 1.5})
    with pytest.raises(ValueError, match="must be positive"):
        honing_gains(model_8_7(), {"honing_integral_share": 1.0})
    m = model_8_7()
    sing = Drivetrain(np.zeros((3, 3), np.float32), m.A, m.q, m.S, m.D, m.c, m.eps, m.knee)
    with pytest.raises(ValueError, match="singular"):
        honing_gains(sing, {})


def _verify_module():
    spec = importlib.util.spec_from_file_location("verify_tables", VERIFY)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.skipif(not os.path.exists(VERIFY), reason="the reference tree is not present")
@pytest.mark.parametrize("cfg", [{}, {"honing_budget_frac": 0.9, "honing_loop_hz": 20.0},
                                 {"honing_bandwidth_scale": 0.5, "honing_integral_share": 0.1}])
def test_reference_check_honing_accepts_our_block(tmp_path, cfg):
    """The reference's acceptance tool re-derives the gains from the card's
    own matrices and compares them with ours."""
    cfgp = write_job(str(tmp_path), "tiny", seed=2)
    job = json.load(open(cfgp))
    job.update(cfg)
    from peregrine_hjb.params import load_model
    m, _ = load_model(job["regression"])
    mj = model_json(m.zeroed_c(), job["regression"], True, job)
    with open(tmp_path / "MODEL.JSON", "w") as fh:
        json.dump(mj, fh, indent=2)
    vt = _verify_module()
    fails, warns = [], []
    vt.check_honing(str(tmp_path), fails, warns)
    assert fails == [], fails
    assert warns == [], warns


def test_honing_cli(tmp_path):
    cfgp = write_job(str(tmp_path), "tiny", seed=4)
    cli = [sys.executable, os.path.join(PKG, "solve.py"), cfgp, "honing"]
    r = subprocess.run(cli, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("HONING ")]
    assert len(line) == 1
    h = json.loads(line[0][len("HONING "):])
    assert h == honing_only(json.load(open(cfgp)))
    # rewriting a run's MODEL.JSON needs one written from the same regression
    run_dir = tmp_path / "run"
    run_dir.mkdir()
    r = subprocess.run(cli + [str(run_dir)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and r.stderr.startswith("ERROR no MODEL.JSON")
    with open(run_dir / "MODEL.JSON", "w") as fh:
        json.dump({"regression_sha256": "0" * 64}, fh)
    r = subprocess.run(cli + [str(run_dir)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "different regression" in r.stderr
    from peregrine_hjb.run import filehash
    with open(run_dir / "MODEL.JSON", "w") as fh:
        json.dump({"regression_sha256": filehash(json.load(open(cfgp))["regression"])}, fh)
    r = subprocess.run(cli + [str(run_dir)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.splitlines()[-1] == "WROTE " + os.path.join(str(run_dir), "MODEL.JSON")
    assert json.load(open(run_dir / "MODEL.JSON"))["honing"] == h
