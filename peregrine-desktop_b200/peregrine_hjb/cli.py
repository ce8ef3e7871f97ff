"""Command line, mirroring solver/solve.jl:23-61.

    solve.py <config.json> [plan|solve|honing [run_dir]]
    solve.py --self-test

Exit 0 on success, 1 on an error (printed as `ERROR <msg>` on stderr with a
short traceback), 2 on a usage error.
"""
from __future__ import annotations

import json
import os
import sys
import traceback


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv:
        print("usage: solve.py <config.json> [plan|solve|honing [run_dir]]", file=sys.stderr)
        print("       solve.py --self-test", file=sys.stderr)
        return 2
    if argv[0] == "--self-test":
        from .selftest import self_test
        return self_test()
    cfgpath = argv[0]
    mode = argv[1] if len(argv) >= 2 else "solve"
    try:
        with open(cfgpath, "r", encoding="utf-8-sig") as fh:
            cfg = json.load(fh)
    except FileNotFoundError:
        print(f"no such config: {cfgpath}", file=sys.stderr)
        return 2
    try:
        if mode == "plan":
            from .run import plan
            print("PLAN " + json.dumps(plan(cfg)))
        elif mode == "solve":
            from .run import run_solve
            run_solve(cfg)
        elif mode == "honing":
            from .honing import honing_only
            run_dir = argv[2] if len(argv) >= 3 else None
            h = honing_only(cfg, write_dir=run_dir)
            print("HONING " + json.dumps(h))
            if run_dir is not None:
                print("WROTE " + os.path.join(run_dir, "MODEL.JSON"))
        else:
            print(f"unknown mode '{mode}' (expected plan, solve or honing)", file=sys.stderr)
            return 2
    except Exception as e:  # the reference prints ERROR <msg> and 8 frames
        print(f"ERROR {e}", file=sys.stderr)
        for line in traceback.format_tb(e.__traceback__)[-8:]:
            print("  " + line.strip().replace("\n", " | "), file=sys.stderr)
        return 1
    sys.stdout.flush()
    return 0
