"""Shared test setup: import paths and the `gpu` marker.

`-m "not gpu"` runs the oracle against the reference's known answers, the
host-side mirrors against the oracle, and the C-ABI export check; `-m gpu`
runs the CUDA path against the oracle through the C ABI.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "peregrine-desktop_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def og():
    from oracle import oracle as og_mod
    og_mod.lib()
    return og_mod


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
