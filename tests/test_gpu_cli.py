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


def _small_job_list(wfb, tmp_path, n=6):
    """n jobs of the committed 64-job mix, shrunk to small films (cameras as committed)."""
    with open(os.path.join(os.path.dirname(__file__), "golden", "job_mix_64_seed1234.json")) as f:
        jobs = json.load(f)["jobs"][:n]
    sizes = [(64, 36), (40, 30), (33, 17), (96, 54), (64, 64), (17, 9)]
    for k, j in enumerate(jobs):
        j["width"], j["height"] = sizes[k % len(sizes)]
        j["spp"] = min(j["spp"], 4)
    path = tmp_path / "jobs.json"
    path.write_text(json.dumps({"jobs": jobs}))
    return path, jobs


@pytest.mark.parametrize("mode", ["megakernel", "wavefront"])
def test_cli_batch_films_equal_solo_renders(wfb, tmp_path, mode):
    """`wf batch`: every job's PFM equals the same job rendered alone through the package."""
    path, jobs = _small_job_list(wfb, tmp_path)
    out = tmp_path / "films"
    out.mkdir()
    p = subprocess.run([WF, "batch", "--jobs", str(path), "--mode", mode, "--reps", "2", "--out-dir", str(out)],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["mode"] == "batch" and line["jobs"] == len(jobs) and line["msamples_s"] > 0
    scenes = {}
    for k, j in enumerate(jobs):
        s = scenes.setdefault(j["scene"], wfb.Scene.generate(j["scene"], 64, 64, 1234, 16))
        r = wfb.GpuRenderer(s, wfb.MEGAKERNEL)
        r.set_camera(j["cam_position"], j["cam_look_at"], j["cam_up"], j["cam_vfov_deg"], j["width"], j["height"])
        want = r.render(wfb.RenderParams(spp=j["spp"], seed=j["seed"], max_depth=j["max_depth"])).rgb
        r.close()
        got = read_pfm(str(out / ("job_%03d.pfm" % k)))
        assert np.array_equal(got.view(np.uint32), np.ascontiguousarray(want, np.float32).view(np.uint32)), k
        assert line["rgb_fnv1a64"][k] == "%016x" % _fnv1a64(np.ascontiguousarray(want, np.float32).tobytes())


def _fnv1a64(data: bytes) -> int:
    h = 0xCBF29CE484222325
    for b in data:
        h = ((h ^ b) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


@pytest.mark.parametrize("plain", [False, True])
def test_cli_serve_finishes_every_job(wfb, tmp_path, plain):
    """`wf serve`: Poisson arrivals from a job list; every submitted job finishes within the drain."""
    path, _ = _small_job_list(wfb, tmp_path)
    cmd = [WF, "serve", "--jobs", str(path), "--lambda", "200", "--duration", "0.5", "--drain", "60", "--seed", "3"]
    p = subprocess.run(cmd + (["--plain"] if plain else []), capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["policy"] == ("one-job-per-launch" if plain else "continuous-batching")
    assert line["submitted"] > 20 and line["completed"] == line["submitted"] and line["incomplete"] == 0
    assert line["p99_ms"] >= line["p50_ms"] > 0 and line["msamples_s"] > 0

