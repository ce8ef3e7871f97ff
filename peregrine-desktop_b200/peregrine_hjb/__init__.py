"""peregrine_hjb -- B200-native minimum-time value-table solver.

A drop-in for the value-iteration solve of Peregrine-Desktop's
`solver/solve.jl`: the same job JSON, the same `PROGRESS` lines, the same
table bytes (docs/TABLE_FORMAT.md).  The compute path is libperegrine_hjb.so
(hand-written sm_100a CUDA) behind a C ABI; this package is the host.
"""
from ._lib import (Context, PeregrineError, default_opts, load_library, solve_value)  # noqa: F401

__all__ = ["Context", "PeregrineError", "default_opts", "load_library", "solve_value"]
