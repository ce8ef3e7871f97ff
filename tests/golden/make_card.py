"""Generate the committed card fixture through the command line (needs the
CUDA library and a GPU).

    python tests/golden/make_card.py OUT_DIR

Writes a seeded synthetic job (the 12x12x8x5x5x5 workload, seed 2, with a
second target, the escape pass on, 5 cm obstacle and 4 cm wall clearance,
u16 tables) and runs
`solve.py <config.json> solve` on it, so OUT_DIR gets TABLES/T##C####.BIN,
MANIFEST.JSON and MODEL.JSON exactly as the wizard would receive them.  The
committed copy is tests/golden/card_tiny/; tests/test_card_fixture.py checks
it against the table format, and with the reference's acceptance tool
(wizard/verify_tables.py) where that tree is present.
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PKG = os.path.join(ROOT, "peregrine-desktop_b200")
sys.path.insert(0, PKG)

from peregrine_hjb.synth import write_job  # noqa: E402


def main(out_dir: str) -> int:
    with tempfile.TemporaryDirectory() as tmp:
        cfgp = write_job(os.path.join(tmp, "job"), "tiny", seed=2)
        cfg = json.load(open(cfgp))
        cfg["escape"] = True
        cfg["escape_iterations"] = 30
        # as the wizard writes a job: the table spans the field inset by the
        # wall clearance (no pinned bounds).  4 cm, not 5: the card's table
        # span is lo + step * (n - 1) in Float32, which for a 5 cm inset of
        # this field lands 1.8e-5 cm past the inset, and the acceptance
        # tool allows 1e-6 (the reference rounds the span identically)
        del cfg["grid"]["bounds"]
        cfg["clearance_cm"] = 5.0
        cfg["wall_clearance_cm"] = 4.0
        tg = json.load(open(cfg["targets"]))
        first = tg["targets"][0]["state"]
        # a second target 60 cm away in x, clamped into the field
        second = [min(max(first[0] + 60.0, 20.0), 345.0), first[1], 1.0, 0.0, 0.0, 0.0]
        tg["targets"].append({"name": "second", "state": second})
        json.dump(tg, open(cfg["targets"], "w"), indent=1)
        cfg["out_dir"] = os.path.join(tmp, "card")
        json.dump(cfg, open(cfgp, "w"), indent=1)
        r = subprocess.run([sys.executable, os.path.join(PKG, "solve.py"), cfgp, "solve"],
                           capture_output=True, text=True)
        sys.stdout.write(r.stdout[-2000:])
        sys.stderr.write(r.stderr[-4000:])
        if r.returncode != 0:
            return r.returncode
        if os.path.exists(out_dir):
            shutil.rmtree(out_dir)
        shutil.copytree(cfg["out_dir"], out_dir)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "card_tiny")))
