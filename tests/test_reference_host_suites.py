"""The reference's own host-API test programs (WVM/tests/test_{config,report,image_io,obj,film,scene,bvh}.cpp),
compiled unchanged from the reference sources against the reference headers and linked against this
engine's host core (libwf_core.so: parse_args, report.json writer/validator, JSON, PNG/PFM/FNV,
OBJ loader, procedural scenes, finalize_scene / scene_hash / BVH build and validation, film
comparison) instead of the reference's own library. CPU only; every reference test must pass."""
import os
import re
import subprocess

import pytest

from conftest import ORACLE_DIR

SUITES = ["config", "report", "image_io", "obj", "film", "scene", "bvh"]


@pytest.mark.parametrize("suite", SUITES)
def test_reference_host_suite_passes_on_engine_core(suite):
    exe = os.path.join(ORACLE_DIR, "_ref", f"test_{suite}_core")
    if not os.path.exists(exe):
        pytest.fail(f"{exe} is missing: build it with `make -C oracle` where the reference sources exist")
    p = subprocess.run([exe], capture_output=True, text=True, timeout=300, cwd=os.path.dirname(exe))
    m = re.search(r"^(\d+) tests, (\d+) failed$", p.stdout, re.M)
    assert m, p.stdout[-2000:]
    assert int(m.group(1)) >= 15 and int(m.group(2)) == 0, p.stdout[-4000:]
    assert p.returncode == 0
