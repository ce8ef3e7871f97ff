"""bench.py's host-side helpers, no GPU: the tiling it reports matches the
library's register-resident tiling rule, the on-chip roofline model is the
one stated in its docstring, and the committed ncu summary it reads the
issue-roofline instruction count and DRAM traffic from exists and parses."""
import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("n1,n2,rows,groups", [(48, 48, 16, 5), (24, 24, 24, 7), (96, 96, 16, 5),
                                               (12, 12, 12, 4), (40, 48, 8, 3), (10, 192, 5, 2)])
def test_tile_rows_follow_the_library_rule(bench, n1, n2, rows, groups):
    # four window rows per row group: rows + 3 <= 4 groups, groups * n2 <= 512
    assert bench.blend_tiling(n1, n2) == (rows, groups)
    assert rows + 3 <= 4 * groups and groups * n2 <= 512


def test_onchip_model(bench):
    class Grid:
        n = (48, 48, 32, 15, 15, 15)

    class Pr:
        grid = Grid()

    out = bench.onchip_rooflines(Pr(), 1.0e11, 4, None)
    win = 4 * 5 / 16
    assert out["tile_rows"] == 16 and out["row_groups"] == 5
    assert abs(out["bytes_per_update"] - (4 * win + 20 + 4 / 32)) < 1e-12
    assert abs(out["flops_per_update"] - (2 * (16 * win + 3) + 4)) < 1e-12


def test_profile_figures_only_from_the_current_kernel(bench, tmp_path, monkeypatch):
    """The issue-roofline instruction count and the DRAM traffic come from
    the committed ncu summary only when it was captured from the kernel
    source this tree builds; a summary of another version gives None."""
    prof = tmp_path / "k.md"
    monkeypatch.setattr(bench, "profile_path", lambda: str(prof))
    body = "warp_instructions_per_update: 2.5\ntraffic_bytes_per_launch: 1.5e11\n"
    prof.write_text(f"source_sha256: {bench.kernel_source_sha()}\n" + body)
    assert bench.profile_current()
    assert bench.profiled_value("warp_instructions_per_update") == 2.5
    assert bench.profiled_traffic() == 1.5e11
    prof.write_text("source_sha256: " + "0" * 64 + "\n" + body)
    assert not bench.profile_current()
    assert bench.profiled_value("warp_instructions_per_update") is None
    assert bench.profiled_traffic() is None


def test_committed_profile_is_of_the_current_kernel(bench):
    """The committed summary of the benchmark workload exists, parses and
    was captured from the current kernel source."""
    assert os.path.exists(bench.profile_path()), bench.profile_path()
    assert bench.profile_current()
    wipu = bench.profiled_value("warp_instructions_per_update")
    traffic = bench.profiled_traffic()
    assert wipu is not None and 1.0 < wipu < 10.0
    assert traffic is not None and traffic > 2 * 4 * 5_462_360_064  # at least V in and out


def test_converge_error_helper_over_reached_cells(bench):
    """max / RMS |V - ref| over the reached cells (0 < ref < cap - 1 ms),
    chunked: unreached cells (ref 0 or at the cap) do not count."""
    import numpy as np
    ref = np.array([0.0, 1.0, 2.0, 30.0, 29.9995, 3.0], np.float32)
    V = np.array([5.0, 1.5, 2.0, 10.0, 1.0, 2.75], np.float32)
    mx, rms, n = bench._max_rms_over(V, ref, 30.0, "cpu", chunk=4)
    assert n == 3
    assert mx == 0.5
    assert abs(rms - np.sqrt((0.25 + 0.0 + 0.0625) / 3)) < 1e-12


def test_code_hash_ignores_comments_not_code(bench, tmp_path):
    """A profile stays the current kernel's through comment edits, and only
    through them: the hash is of the code without // comments and blank
    lines."""
    a = tmp_path / "a.cuh"
    a.write_text("// header\nint f(int x) {  // note\n    return x + 1;\n}\n")
    b = tmp_path / "b.cuh"
    b.write_text("// another header\n\nint f(int x) {\n    return x + 1;  // other note\n}\n")
    c = tmp_path / "c.cuh"
    c.write_text("int f(int x) {\n    return x + 2;\n}\n")
    assert bench.kernel_source_sha(str(a)) == bench.kernel_source_sha(str(b))
    assert bench.kernel_source_sha(str(a)) != bench.kernel_source_sha(str(c))
