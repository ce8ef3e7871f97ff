"""End to end through the command line, the drop-in boundary the wizard
calls (solver/solve.jl:23-61): a seeded synthetic job in, a card image out,
checked against the contract of docs/TABLE_FORMAT.md the way
wizard/verify_tables.py checks a card (sizes, SHA-256, V(target) ~ 0,
field-frame velocity ordering, escape band, MODEL.JSON blocks)."""
import hashlib
import json
import math
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import PKG, gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def run_cli(cfg_path, mode="solve"):
    return subprocess.run([sys.executable, os.path.join(PKG, "solve.py"), cfg_path, mode],
                          capture_output=True, text=True, timeout=900)


def card_value(root, m, t, subs):
    n = m["grid"]["n"]
    idx = 0
    for k in range(6):
        idx = idx * n[k] + subs[k]
    enc = m["encoding"]
    ce = enc["chunk_elements"]
    path = os.path.join(root, t["file_pattern"] % (idx >> enc["chunk_shift"]))
    eb = enc["elem_bytes"]
    with open(path, "rb") as fh:
        fh.seek((idx & (ce - 1)) * eb)
        raw = fh.read(eb)
    if enc["dtype"] == "u16":
        r = int.from_bytes(raw, "little")
        if r == enc["unreachable"] or (enc["escape_codes"] and r >= enc["escape_base"]):
            return math.inf
        return r * enc["scale"]
    return float(np.frombuffer(raw, np.float32)[0])


def nearest(m, s):
    g = m["grid"]
    out = []
    for k in range(6):
        n, lo, hi = g["n"][k], g["min"][k], g["max"][k]
        if g["wrap"][k]:
            st = (hi - lo) / n
            out.append(int(round((s[k] - lo) / st)) % n)
        else:
            st = (hi - lo) / (n - 1)
            out.append(min(max(int(round((s[k] - lo) / st)), 0), n - 1))
    return out


@pytest.mark.parametrize("escape", [False, True])
def test_cli_solve_writes_a_valid_card(tmp_path, escape):
    sys.path.insert(0, PKG)
    from peregrine_hjb.synth import write_job
    cfgp = write_job(str(tmp_path / "job"), "tiny", seed=2)
    cfg = json.load(open(cfgp))
    cfg["escape"] = escape
    cfg["escape_iterations"] = 20
    json.dump(cfg, open(cfgp, "w"))
    r = run_cli(cfgp)
    assert r.returncode == 0, r.stderr[-2000:]
    phases = [json.loads(l[9:])["phase"] for l in r.stdout.splitlines() if l.startswith("PROGRESS ")]
    for ph in ("setup", "occupancy", "backend", "solve", "encode", "target_done", "model", "done"):
        assert ph in phases
    if escape:
        assert "escape" in phases
    root = cfg["out_dir"]
    m = json.load(open(os.path.join(root, "MANIFEST.JSON")))
    total = m["grid"]["total_cells"]
    assert math.prod(m["grid"]["n"]) == total
    for t in m["targets"]:
        assert t["bytes"] == total * m["encoding"]["elem_bytes"]
        assert t["n_chunks"] == -(-total // m["encoding"]["chunk_elements"])
        h = hashlib.sha256()
        for c in range(t["n_chunks"]):
            h.update(open(os.path.join(root, t["file_pattern"] % c), "rb").read())
        assert h.hexdigest() == t["sha256"]
        assert card_value(root, m, t, nearest(m, t["state"])) < 0.25
        assert t["reached_frac"] > 0.3
        if escape:
            assert m["encoding"]["escape_codes"] == 1023
    mj = json.load(open(os.path.join(root, "MODEL.JSON")))
    assert "A_u" in mj["nonzero_blocks"]
    assert mj["control"]["saturation"]["knee"] > 0
    for name in ("A_s", "A_ss", "A_sgn", "A_absv"):
        assert all(all(v == 0 for v in row[:3]) for row in mj[name])


def test_targets_shard_over_ranks(tmp_path):
    """Under torchrun the job's targets are shared out over the ranks (two
    ranks on one GPU here, gloo for the records: their solves never wait on
    each other); the card equals the single-process card byte for byte."""
    import shutil
    import socket
    sys.path.insert(0, PKG)
    from peregrine_hjb.synth import write_job
    cfgp = write_job(str(tmp_path / "job"), "tiny", seed=2)
    cfg = json.load(open(cfgp))
    tg = json.load(open(cfg["targets"]))
    first = tg["targets"][0]["state"]
    tg["targets"].append({"name": "second", "state": [first[0], first[1], 0.5, 0, 0, 0]})
    tg["targets"].append({"name": "third", "state": [first[0], first[1], -1.0, 0, 0, 0]})
    json.dump(tg, open(cfg["targets"], "w"))
    json.dump(cfg, open(cfgp, "w"))
    r = run_cli(cfgp)
    assert r.returncode == 0, r.stderr[-2000:]
    single = tmp_path / "single"
    shutil.copytree(cfg["out_dir"], single)
    shutil.rmtree(cfg["out_dir"])
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                        "--nproc-per-node", "2", "--master-addr", "127.0.0.1", "--master-port",
                        str(port), os.path.join(PKG, "solve.py"), cfgp, "solve"],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    m1 = json.load(open(single / "MANIFEST.JSON"))
    m2 = json.load(open(os.path.join(cfg["out_dir"], "MANIFEST.JSON")))
    assert [t["sha256"] for t in m1["targets"]] == [t["sha256"] for t in m2["targets"]]
    assert len(m2["targets"]) == 3
    for t in m1["targets"]:
        for c in range(t["n_chunks"]):
            a = open(single / (t["file_pattern"] % c), "rb").read()
            b = open(os.path.join(cfg["out_dir"], t["file_pattern"] % c), "rb").read()
            assert a == b
