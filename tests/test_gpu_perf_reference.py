"""Throughput against the reference's own GPU arms on the same B200 (same scene arrays, same BVH,
same seed), with bit-equal images. Writes the measured numbers to $WFB_PERF_OUT when set."""
import json
import os
import time

import numpy as np
import pytest

from conftest import load_engine

pytestmark = pytest.mark.gpu

CONFIGS = [
    # scene, width, height, spp  (depth 8, seed 1234)
    ("cornell36", 320, 180, 16),
    ("icospheres", 1280, 720, 64),
    ("heightfield", 1280, 720, 64),
]


@pytest.mark.parametrize("scene,w,h,spp", CONFIGS)
def test_faster_than_reference_megakernel_with_equal_image(ref, scene, w, h, spp):
    wfb = load_engine()
    sc = wfb.Scene.generate(scene, w, h, 1234, 16)
    arrays = sc.export()
    params = wfb.RenderParams(spp=spp, seed=1234, max_depth=8)
    r = wfb.GpuRenderer(sc, wfb.MEGAKERNEL)
    r.render(params)  # warm-up
    mine_ms = []
    for _ in range(3):
        st = wfb.RenderStats()
        img = r.render(params, st)
        mine_ms.append(st.render_ms)
    t0 = time.perf_counter()
    rrgb, rvar, rst = ref.ref_render_gpu(arrays, 0, spp, 1234, 8)
    ref_wall = time.perf_counter() - t0
    assert np.array_equal(img.rgb.view(np.uint32), rrgb.view(np.uint32)), "image differs from the reference megakernel"
    samples = w * h * spp
    result = {
        "scene": scene, "size": f"{w}x{h}", "spp": spp, "samples": samples,
        "engine_megakernel_ms": min(mine_ms), "engine_megakernel_msamples_s": samples / min(mine_ms) / 1e3,
        "reference_megakernel_ms": rst["render_ms"], "reference_megakernel_msamples_s": samples / rst["render_ms"] / 1e3,
        "reference_megakernel_wall_s": ref_wall,
    }
    if scene != "heightfield":
        wrgb, _, wst = ref.ref_render_gpu(arrays, 1, spp, 1234, 8)
        assert np.array_equal(wrgb.view(np.uint32), rrgb.view(np.uint32))
        result["reference_wavefront_ms"] = wst["render_ms"]
        result["reference_wavefront_msamples_s"] = samples / wst["render_ms"] / 1e3
    out = os.environ.get("WFB_PERF_OUT")
    if out:
        with open(out, "a") as f:
            f.write(json.dumps(result) + "\n")
    print(result)
    assert result["engine_megakernel_msamples_s"] > result["reference_megakernel_msamples_s"]
