"""Command-line behaviour that needs no GPU: usage and error exits and the
plan mode (solver/solve.jl:23-61)."""
import json
import os
import subprocess
import sys

from conftest import PKG


def cli(*args):
    return subprocess.run([sys.executable, os.path.join(PKG, "solve.py"), *args],
                          capture_output=True, text=True, timeout=300)


def test_usage_exit_2():
    r = cli()
    assert r.returncode == 2 and "usage" in r.stderr


def test_missing_config_exit_2(tmp_path):
    assert cli(str(tmp_path / "nope.json")).returncode == 2


def test_bad_config_prints_error_exit_1(tmp_path):
    bad = tmp_path / "bad.json"
    bad.write_text(json.dumps({"regression": str(tmp_path / "x.toml"), "field": "f",
                               "targets": "t", "out_dir": str(tmp_path / "o")}))
    r = cli(str(bad))
    assert r.returncode == 1 and r.stderr.startswith("ERROR ")


def test_unknown_mode_exit_2(tmp_path):
    sys.path.insert(0, PKG)
    from peregrine_hjb.synth import write_job
    cfgp = write_job(str(tmp_path / "job"), "tiny", seed=1)
    assert cli(cfgp, "frobnicate").returncode == 2


def test_plan_reports_the_grid(tmp_path):
    sys.path.insert(0, PKG)
    from peregrine_hjb.synth import write_job
    cfgp = write_job(str(tmp_path / "job"), "small", seed=1)
    r = cli(cfgp, "plan")
    assert r.returncode == 0, r.stderr
    line = [l for l in r.stdout.splitlines() if l.startswith("PLAN ")][0]
    plan = json.loads(line[5:])
    assert plan["n"] == [24, 24, 16, 9, 9, 9] and plan["cells"] == 6718464
    assert plan["controls"] == 27
    # the keys the wizard reads (wizard/peregrine.py run_plan and its
    # show_* helpers), with values that follow from the job
    for k in ("bounds", "resolution", "occupancy", "targets", "targets_ok", "recommend",
              "bytes_per_target", "bytes_total", "n_targets", "chunks_per_target",
              "gpu_available", "gpu_fits", "gpu_need_gb", "gpu_free_gb", "out_of_core",
              "grid_balance", "cell_cm", "cell_cm_s", "max_accel_cm_s2", "runtime"):
        assert k in plan, k
    assert plan["bytes_per_target"] == 6718464 * 2 and plan["n_targets"] == 1
    assert plan["bytes_total"] == plan["bytes_per_target"]
    assert plan["chunks_per_target"] == 1 and plan["targets_ok"] is True
    assert plan["targets"][0]["ok"] and plan["targets"][0]["free_seed_cells"] > 0
    assert plan["out_of_core"]["mode"] in ("incore", "ooc")
    assert plan["bounds"]["table_min"][0] == 0.0
    assert abs(plan["bounds"]["table_max"][0] - 365.8) < 1e-3
    assert 0.0 < plan["occupancy"]["blocked_frac"] < 0.5
    rt = plan["runtime"]
    assert rt["unit"] == "sweep" and rt["units"] == 3000
    assert abs(rt["total_s"] - rt["unit_s"] * rt["units"]) < 1e-9
    assert plan["resolution"]["pinned_by_n"] is True


def test_missing_knee_is_refused(tmp_path):
    sys.path.insert(0, PKG)
    from peregrine_hjb.synth import write_job
    cfgp = write_job(str(tmp_path / "job"), "tiny", seed=1)
    cfg = json.load(open(cfgp))
    toml = open(cfg["regression"]).read().replace("traction_knee", "# traction_knee")
    open(cfg["regression"], "w").write(toml)
    r = cli(cfgp, "plan")
    assert r.returncode == 1 and "traction_knee" in r.stderr
