"""`wf render` on a B200: the reference's command line rendering through the engine. The film it
writes (PFM) and the report's pfm_hash equal the reference's own GPU megakernel on the same scene
and seed; the report validates against schema 1."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR

pytestmark = pytest.mark.gpu

WF = os.path.join(PKG_DIR, "wf")


def read_pfm(path):
    with open(path, "rb") as f:
        data = f.read()
    head = data.split(b"\n", 3)
    w, h = (int(v) for v in head[1].split())
    assert float(head[2]) < 0  # little endian
    px = np.frombuffer(head[3][: 12 * w * h], dtype="<f4").reshape(h, w, 3)
    return px[::-1].copy()  # file rows are bottom to top


@pytest.mark.parametrize("mode", ["megakernel", "wavefront"])
def test_cli_render_equals_reference_megakernel(ref, orc, tmp_path, mode):
    w, h, spp, seed = 64, 36, 4, 7
    report = tmp_path / "r.json"
    prefix = tmp_path / "img"
    p = subprocess.run([WF, "render", "--scene", "divergence", "--width", str(w), "--height", str(h), "--spp", str(spp),
                        "--seed", str(seed), "--mode", mode, "--reps", "2", "--warmup", "1", "--report", str(report),
                        "--out", str(prefix)], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    rgb = read_pfm(str(prefix) + ".pfm")
    arrays = orc.ref_make_scene("divergence", w, h)
    rrgb, _, _ = ref.ref_render_gpu(arrays, 0, spp, seed, 8)
    assert np.array_equal(rgb.view(np.uint32), rrgb.view(np.uint32))
    r = json.loads(report.read_text())
    assert r["schema_version"] == 1 and r["config"]["mode"] == mode
    assert r["outputs"]["pfm_hash"] == "%016x" % orc.fnv1a64(rrgb)
    assert r["scene"]["hash"] == "%016x" % orc.ref_scene_hash(arrays)
    assert len(r["timings_ms"]["runs"]) == 2 and r["throughput"]["samples_per_second"] > 0
    assert r["throughput"]["rays_per_second"] > 0 and r["device"]["compute_capability"] == "10.0"
    assert r["validity"] == {"nonfinite_pixels": 0, "queue_overflows": 0, "invalid_hits": 0}
    assert os.path.getsize(str(prefix) + ".png") > 0


def test_cli_renders_obj_files_and_benchmark_scenes(tmp_path):
    obj = tmp_path / "quad.obj"
    obj.write_text("v -1 -1 0\nv 1 -1 0\nv 1 1 0\nv -1 1 0\nf 1 2 3 4\n")
    for scene in (str(obj), "cornell36"):
        p = subprocess.run([WF, "render", "--scene", scene, "--width", "32", "--height", "18", "--spp", "2",
                            "--mode", "megakernel", "--report", str(tmp_path / "r.json")],
                           capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr
        r = json.loads((tmp_path / "r.json").read_text())
        assert r["scene"]["name"] == scene and len(r["scene"]["hash"]) == 16
