"""Table encoding and the chunked card writer, mirroring
solver/src/Pipeline.jl:620-840 and docs/TABLE_FORMAT.md §1-§6.

The per-cell encoding runs on the GPU (pg_encode, straight from the device
layout); this module only cuts chunks, names files and hashes them.
"""
from __future__ import annotations

import hashlib
import os

DTYPES = {
    "u8": dict(bytes=1, sentinel=0xFF, scale=0.025, escape_base=0x00E0),
    "u16": dict(bytes=2, sentinel=0xFFFF, scale=0.001, escape_base=0xFC00),
    "f16": dict(bytes=2, sentinel=float("nan"), scale=1.0, escape_base=0),
    "f32": dict(bytes=4, sentinel=float("nan"), scale=1.0, escape_base=0),
}


def escape_codes(dtype: str) -> int:
    """Pipeline.jl:628-630"""
    d = DTYPES[dtype]
    return 0 if d["escape_base"] == 0 else int(d["sentinel"]) - int(d["escape_base"])


def escape_scale_for(dtype: str, cap: float) -> float:
    """Pipeline.jl:651-653"""
    c = escape_codes(dtype)
    return 0.0 if c <= 1 else float(cap) / (c - 1) ** 2


def chunk_name(target_index: int, chunk: int) -> str:
    return "T%02dC%04d.BIN" % (target_index, chunk)


def write_table(dirpath, target_index: int, ctx, ncells: int, dtype: str, scale: float,
                chunk_elements: int, escape_scale: float = 0.0) -> dict:
    """write_table (Pipeline.jl:788-826): one file per chunk of
    `chunk_elements` values, SHA-256 streamed over all chunks."""
    eb = DTYPES[dtype]["bytes"]
    os.makedirs(dirpath, exist_ok=True)
    nchunks = -(-ncells // chunk_elements)
    sha = hashlib.sha256()
    reached = escaped = total = 0
    buf = None
    for ci in range(nchunks):
        lo = ci * chunk_elements
        n = min(ncells, lo + chunk_elements) - lo
        part, r, e = ctx.encode(dtype, scale, escape_scale, lo, n, buf)
        buf = part if buf is None else buf
        reached += r
        escaped += e
        data = memoryview(part)[: n * eb]
        with open(os.path.join(dirpath, chunk_name(target_index, ci)), "wb") as fh:
            fh.write(data)
        sha.update(data)
        total += n * eb
    return dict(nchunks=nchunks, bytes=total, sha256=sha.hexdigest(), reached=reached,
                escaped=escaped, cells=ncells)
