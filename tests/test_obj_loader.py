"""wf::load_obj edge cases (line endings, comments, slashed and many-cornered faces, error messages
with line numbers), compiled against libwf_core.so; the reference's own OBJ tests run unchanged in
tests/test_reference_host_suites.py."""
import os
import shutil
import subprocess

import pytest

from conftest import PKG_DIR, ROOT


def test_obj_loader_edge_cases(tmp_path):
    cxx = shutil.which(os.environ.get("CXX", "g++")) or shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    if not os.path.exists(os.path.join(PKG_DIR, "libwf_core.so")):
        pytest.fail("libwf_core.so is missing: build it with `make -C graphics-book-tutorials_b200`")
    exe = tmp_path / "obj_check"
    subprocess.run([cxx, "-std=c++20", "-O1", "-I", os.path.join(PKG_DIR, "csrc"),
                    os.path.join(ROOT, "tests", "obj_loader_check.cpp"), "-o", str(exe), "-L", PKG_DIR, "-lwf_core",
                    "-Wl,-rpath," + PKG_DIR], check=True)
    out = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
