"""The render server's launch planning (csrc/schedule.hpp) on the CPU: the express lane for small
jobs, large jobs in arrival order with a starvation guard, the shared (equal-slice) schedule, and
bounds / progress over random job mixes (tests/schedule_check.cpp)."""
import os
import shutil
import subprocess

import pytest

from conftest import PKG_DIR, ROOT


def test_launch_planning(tmp_path):
    cxx = shutil.which(os.environ.get("CXX", "g++")) or shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = tmp_path / "schedule_check"
    subprocess.run([cxx, "-std=c++20", "-O2", "-Wall", "-I", os.path.join(PKG_DIR, "csrc"),
                    os.path.join(ROOT, "tests", "schedule_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok ") and int(out.stdout.split()[1]) > 40000
