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


def test_batch_and_serve_reject_bad_arguments_and_job_lists(tmp_path):
    """`wf batch` / `wf serve`: argument and job-list errors exit 1 before any device work."""
    p = run("serve")
    assert p.returncode == 1 and "--jobs is required" in p.stderr and "Usage: batch" in p.stderr
    p = run("batch", "--jobs", "x.json", "--mode", "cpu")
    assert p.returncode == 1 and "--mode must be megakernel or wavefront" in p.stderr
    p = run("serve", "--jobs", "x.json", "--lambda", "fast")
    assert p.returncode == 1 and "--lambda expects a number" in p.stderr
    bad = tmp_path / "bad.json"
    bad.write_text('{"jobs": [{"scene": "cornell36", "width": 8}]}')
    p = run("batch", "--jobs", str(bad))
    assert p.returncode == 1 and "job 0 misses a field" in p.stderr
    bad.write_text('{"jobs": [{"scene": "teapot", "width": 8, "height": 8, "spp": 1, "max_depth": 8, "seed": 1,'
                   ' "cam_position": [0, 1, 5], "cam_look_at": [0, 0, 0], "cam_up": [0, 1, 0], "cam_vfov_deg": 50}]}')
    p = run("batch", "--jobs", str(bad))
    assert p.returncode == 1 and "not a benchmark generator" in p.stderr
    p = run("batch", "--jobs", str(tmp_path / "missing.json"))
    assert p.returncode == 1 and "cannot read" in p.stderr
