"""The committed card image (tests/golden/card_tiny, written by this
solver's command line on a B200 by tests/golden/make_card.py) against the
table format, and against the reference's own acceptance tool
(wizard/verify_tables.py, stdlib only) where the reference tree is present."""
import hashlib
import json
import math
import os
import subprocess
import sys

import pytest

CARD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "card_tiny")
VERIFY = "/root/reference/wizard/verify_tables.py"

pytestmark = pytest.mark.skipif(not os.path.exists(os.path.join(CARD, "MANIFEST.JSON")),
                                reason="no card fixture")


def test_card_sizes_and_hashes():
    m = json.load(open(os.path.join(CARD, "MANIFEST.JSON")))
    total = m["grid"]["total_cells"]
    assert math.prod(m["grid"]["n"]) == total
    assert len(m["targets"]) == 2
    for t in m["targets"]:
        assert t["bytes"] == total * m["encoding"]["elem_bytes"]
        h = hashlib.sha256()
        for c in range(t["n_chunks"]):
            h.update(open(os.path.join(CARD, t["file_pattern"] % c), "rb").read())
        assert h.hexdigest() == t["sha256"]
    mj = json.load(open(os.path.join(CARD, "MODEL.JSON")))
    assert mj["schema_version"] == 2 and "honing" in mj


@pytest.mark.skipif(not os.path.exists(VERIFY), reason="the reference tree is not present")
def test_reference_verify_tables_passes():
    r = subprocess.run([sys.executable, VERIFY, CARD], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    last = [ln for ln in r.stdout.splitlines() if ln.strip()][-1]
    assert last.strip().startswith("PASS"), last
    assert "(0 failures, 0 warnings)" in last, r.stdout[-3000:]
