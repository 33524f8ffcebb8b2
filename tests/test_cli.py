"""`wf render` (the reference's command line, WVM/include/wf/config.hpp:30-34) on CPU: argument errors
and the refused CPU arm. Rendering through it is covered by tests/test_gpu_cli.py."""
import os
import subprocess

from conftest import PKG_DIR

WF = os.path.join(PKG_DIR, "wf")


def run(*args):
    return subprocess.run([WF, *args], capture_output=True, text=True, timeout=60)


def test_bad_flags_exit_1_with_usage():
    for args in (["render", "--bogus", "1"], ["render", "--width", "0"], ["bench"], ["render", "--spp"]):
        p = run(*args)
        assert p.returncode == 1, args
        assert "Error:" in p.stderr and "Usage: render" in p.stderr


def test_cpu_mode_is_refused_without_fallback():
    p = run("render", "--mode", "cpu", "--width", "8", "--height", "8", "--spp", "1")
    assert p.returncode == 1
    assert "GPU only" in p.stderr


def test_unknown_scene_is_an_error():
    p = run("render", "--scene", "no-such-scene", "--mode", "megakernel", "--width", "8", "--height", "8")
    assert p.returncode == 1 and "unknown scene" in p.stderr
