"""Megakernel parity on a B200: bit-for-bit against the reference's own GPU arms (compiled for
sm_100a from the reference sources with the same float flags), statistically against the CPU
oracle, and the reference's metamorphic relations (WVM/tests/test_gpu_render.cu)."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR, load_engine, load_oracle

pytestmark = pytest.mark.gpu

with open(os.path.join(GOLDEN_DIR, "golden.json")) as _f:
    GOLDEN = json.load(_f)


def _arrays(case):
    g = GOLDEN[case]
    kind, name = g["source"].split(":")
    if kind == "engine":
        return load_engine().Scene.generate(name, g["width"], g["height"], 1234, 16).export()
    return load_oracle().ref_make_scene(name, g["width"], g["height"])


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def render(wfb, arrays, mode, spp, seed, depth, count_rays=False, **kw):
    scene = wfb.Scene.from_arrays(arrays)
    r = wfb.GpuRenderer(scene, mode)
    st = wfb.RenderStats()
    out = r.render(wfb.RenderParams(spp=spp, seed=seed, max_depth=depth, count_rays=count_rays, **kw), st)
    return out, st


@pytest.mark.parametrize("case", sorted(GOLDEN))
def test_megakernel_bitwise_equals_reference_gpu_arms(wfb, ref, case):
    g = GOLDEN[case]
    arrays = _arrays(case)
    out, st = render(wfb, arrays, wfb.MEGAKERNEL, g["spp"], g["seed"], g["max_depth"])
    for mode in (0, 1):  # reference megakernel, reference wavefront
        rrgb, rvar, _ = ref.ref_render_gpu(arrays, mode, g["spp"], g["seed"], g["max_depth"])
        diff = int((bits(out.rgb) != bits(rrgb)).sum())
        assert diff == 0, f"{case}: {diff} rgb floats differ from reference arm {mode}"
        assert np.array_equal(bits(out.lum_var), bits(rvar))
    assert st.invalid_hits == 0 and st.queue_overflows == 0
    assert np.isfinite(out.rgb).all() and float(out.rgb.sum()) > 0.0


@pytest.mark.parametrize("case", ["cornell36_64x36", "icospheres_64x36", "ref_divergence_32x18"])
def test_megakernel_agrees_with_cpu_oracle(wfb, orc, case):
    """>= 99.9% of pixels within 3 combined SE of the CPU arm, same seed (north-star criterion)."""
    g = GOLDEN[case]
    arrays = _arrays(case)
    spp = 32
    out, st = render(wfb, arrays, wfb.MEGAKERNEL, spp, g["seed"], g["max_depth"])
    rgb_s, lum, lum2, _ = orc.render_sums(arrays, spp, g["seed"], g["max_depth"], threads=8)
    crgb, cvar = orc.cpu_convention(rgb_s, lum, lum2, spp)
    cpu = wfb.RenderResult(g["width"], g["height"], spp, crgb, cvar)
    d = wfb.compare_results(cpu, out)
    assert d["frac_within_3se"] >= 0.999, d
    assert d["mean_rel"] <= 0.005, d
    assert d["nonfinite"] == 0
    # same RNG streams: the vast majority of pixels are bit-identical to the CPU arm
    same = float((bits(out.rgb) == bits(crgb)).all(axis=-1).mean())
    assert same > 0.5, same


def test_ray_counts_match_reference(wfb, ref):
    arrays = _arrays("icospheres_64x36")
    _, st = render(wfb, arrays, wfb.MEGAKERNEL, 4, 1234, 8, count_rays=True)
    _, _, rst = ref.ref_render_gpu(arrays, 0, 4, 1234, 8, count_rays=True)
    assert st.extension_rays == int(rst["extension_rays"]) > 0
    assert st.shadow_rays == int(rst["shadow_rays"]) > 0


def test_progressive_equals_one_shot(wfb):
    """run_passes(0,3) + run_passes(3,5) then download(8) == render(spp 8) (test_gpu_render.cu:259-284)."""
    arrays = _arrays("cornell36_64x36")
    scene = wfb.Scene.from_arrays(arrays)
    r = wfb.GpuRenderer(scene, wfb.MEGAKERNEL)
    p = wfb.RenderParams(spp=8, seed=3, max_depth=8)
    one = r.render(p)
    r.reset()
    r.run_passes(0, 3, p)
    r.run_passes(3, 5, p)
    prog = r.download(8)
    assert np.array_equal(bits(one.rgb), bits(prog.rgb))
    assert np.array_equal(bits(one.lum_var), bits(prog.lum_var))
    mean = r.download_mean(8)
    assert np.array_equal(bits(mean), bits(prog.rgb))


@pytest.mark.parametrize("w,h", [(1, 1), (33, 17), (31, 1), (1, 33)])
def test_odd_sizes_match_reference(wfb, ref, w, h):
    arrays = load_oracle().ref_make_scene("divergence", w, h)
    out, _ = render(wfb, arrays, wfb.MEGAKERNEL, 4, 7, 8)
    rrgb, rvar, _ = ref.ref_render_gpu(arrays, 0, 4, 7, 8)
    assert out.rgb.shape == (h, w, 3)
    assert np.array_equal(bits(out.rgb), bits(rrgb))
    assert np.array_equal(bits(out.lum_var), bits(rvar))


def test_set_camera_equals_scene_camera(wfb, ref):
    """A renderer re-aimed with set_camera renders what a scene built with that camera renders."""
    arrays = _arrays("icospheres_64x36")
    cam = dict(cam_position=[6.0, 4.0, 9.0], cam_look_at=[0.0, 0.5, 0.0], cam_up=[0.0, 1.0, 0.0], cam_vfov_deg=35.0)
    moved = dict(arrays, width=40, height=30, **cam)
    rrgb, _, _ = ref.ref_render_gpu(moved, 0, 2, 11, 8)
    r = wfb.GpuRenderer(wfb.Scene.from_arrays(arrays), wfb.MEGAKERNEL)
    r.set_camera(cam["cam_position"], cam["cam_look_at"], cam["cam_up"], cam["cam_vfov_deg"], 40, 30)
    out = r.render(wfb.RenderParams(spp=2, seed=11, max_depth=8))
    assert np.array_equal(bits(out.rgb), bits(rrgb))


def test_depth_limits_and_seeds(wfb, ref):
    arrays = _arrays("icospheres_64x36")
    for depth, seed in ((0, 1), (1, 2), (3, 99), (12, 5)):
        out, _ = render(wfb, arrays, wfb.MEGAKERNEL, 2, seed, depth)
        rrgb, _, _ = ref.ref_render_gpu(arrays, 0, 2, seed, depth)
        assert np.array_equal(bits(out.rgb), bits(rrgb)), (depth, seed)


def test_full_size_render_is_clean(wfb):
    """Benchmark scene at full resolution, 1 spp: no invalid hits, no non-finite pixels, energy > 0."""
    scene = wfb.Scene.generate("icospheres", 1280, 720, 1234, 16)
    r = wfb.GpuRenderer(scene, wfb.MEGAKERNEL)
    st = wfb.RenderStats()
    out = r.render(wfb.RenderParams(spp=1, seed=1234, max_depth=8, count_rays=True), st)
    assert st.invalid_hits == 0
    assert np.isfinite(out.rgb).all() and out.rgb.mean() > 0.0
    assert st.extension_rays >= 1280 * 720


@pytest.mark.parametrize("block,min_active,split", [(64, 1, 1), (128, 32, 1), (256, 16, 3), (128, 20, 8)])
def test_launch_configurations_give_identical_films(wfb, block, min_active, split):
    """Block size, traversal threshold and direct/split accumulation never change a bit of the film."""
    scene = wfb.Scene.generate("icospheres", 96, 54, 1234, 16)
    p = wfb.RenderParams(spp=8, seed=21, max_depth=8)
    base = wfb.GpuRenderer(scene, wfb.MEGAKERNEL).render(p)
    r = wfb.GpuRenderer(scene, wfb.MEGAKERNEL)
    r.configure(block=block, min_active=min_active, split_chunks=split)
    out = r.render(p)
    assert np.array_equal(bits(out.rgb), bits(base.rgb))
    assert np.array_equal(bits(out.lum_var), bits(base.lum_var))
