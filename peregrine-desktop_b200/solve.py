#!/usr/bin/env python3
"""CLI entry point, the counterpart of solver/solve.jl:

    python solve.py config.json [plan|solve]
    python solve.py --self-test
"""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from peregrine_hjb.cli import main  # noqa: E402

if __name__ == "__main__":
    sys.exit(main())
