"""The GPU traversal's min/max box test against the reference's compare-and-select slab test.

wf::hit_box (WVM/include/wf/bvh.hpp:64-86) keeps the compare-and-swap and ternary clamps whose NaN
behaviour decides which boxes a ray parallel to an axis enters; wf::hit_box_minmax reaches the same
boolean on fminf/fmaxf. tests/box_minmax_check.cpp compares them on the host (fminf/fmaxf return
the non-NaN operand there as on the device) over special values exhaustively per axis and by
random mixing, with contraction off as in every build of the engine.
"""
import os
import shutil
import subprocess

import pytest

from conftest import PKG_DIR, ROOT


def test_minmax_box_matches_reference_slab_test(tmp_path):
    cxx = shutil.which(os.environ.get("CXX", "g++")) or shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = tmp_path / "box_minmax_check"
    src = os.path.join(ROOT, "tests", "box_minmax_check.cpp")
    subprocess.run([cxx, "-std=c++20", "-O2", "-ffp-contract=off", "-I", os.path.join(PKG_DIR, "csrc"), src, "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    cases = int(out.stdout.split()[1])
    assert cases > 6_000_000
