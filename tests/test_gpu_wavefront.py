"""Persistent wavefront on a B200: bit-for-bit against the reference's GPU arms and the engine's
megakernel, pool-size independence, the queue-capacity test hook (counted overflows, clean next
render; WVM/tests/catch/wavefront_failure.cu:92-134) and stage timing as pure observation."""
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


def render(wfb, scene, mode, spp, seed, depth, configure=None, **kw):
    r = wfb.GpuRenderer(scene, mode)
    if configure:
        r.configure(**configure)
    st = wfb.RenderStats()
    out = r.render(wfb.RenderParams(spp=spp, seed=seed, max_depth=depth, **kw), st)
    return out, st, r


@pytest.mark.parametrize("case", sorted(GOLDEN))
def test_wavefront_bitwise_equals_reference_arms(wfb, ref, case):
    g = GOLDEN[case]
    arrays = _arrays(case)
    out, st, _ = render(wfb, wfb.Scene.from_arrays(arrays), wfb.WAVEFRONT, g["spp"], g["seed"], g["max_depth"])
    for mode in (0, 1):
        rrgb, rvar, _ = ref.ref_render_gpu(arrays, mode, g["spp"], g["seed"], g["max_depth"])
        assert np.array_equal(bits(out.rgb), bits(rrgb)), f"{case}: differs from reference arm {mode}"
        assert np.array_equal(bits(out.lum_var), bits(rvar))
    assert st.invalid_hits == 0 and st.queue_overflows == 0


@pytest.mark.parametrize("pool", [32, 1000, 4096, 100000])
def test_pool_size_never_changes_the_film(wfb, pool):
    scene = wfb.Scene.generate("icospheres", 96, 54, 1234, 16)
    mk, _, _ = render(wfb, scene, wfb.MEGAKERNEL, 6, 9, 8)
    out, st, r = render(wfb, scene, wfb.WAVEFRONT, 6, 9, 8, configure={"paths_in_flight": pool})
    assert np.array_equal(bits(out.rgb), bits(mk.rgb))
    assert np.array_equal(bits(out.lum_var), bits(mk.lum_var))
    assert 0 < st.queue_high_water[4] <= max(pool, 32)
    assert all(0 <= v <= max(pool, 32) for v in st.queue_high_water[:4])


def test_full_resolution_matches_megakernel_and_counts(wfb):
    scene = wfb.Scene.generate("icospheres", 1280, 720, 1234, 16)
    mk, smk, _ = render(wfb, scene, wfb.MEGAKERNEL, 2, 1234, 8, count_rays=True)
    wv, swv, _ = render(wfb, scene, wfb.WAVEFRONT, 2, 1234, 8, count_rays=True)
    assert np.array_equal(bits(wv.rgb), bits(mk.rgb))
    assert swv.extension_rays == smk.extension_rays and swv.shadow_rays == smk.shadow_rays
    assert swv.invalid_hits == 0 and swv.queue_overflows == 0


def test_queue_capacity_hook_counts_overflows_and_recovers(wfb):
    """Capacity far below the paths in flight: drops are counted, nothing faults, and the next
    render without the hook is bit-exact again."""
    scene = wfb.Scene.generate("icospheres", 64, 36, 1234, 16)
    mk, _, _ = render(wfb, scene, wfb.MEGAKERNEL, 4, 5, 8)
    r = wfb.GpuRenderer(scene, wfb.WAVEFRONT)
    st = wfb.RenderStats()
    capped = r.render(wfb.RenderParams(spp=4, seed=5, max_depth=8, queue_capacity=100), st)
    assert st.queue_overflows > 0
    assert np.isfinite(capped.rgb).all()
    assert max(st.queue_high_water[:4]) <= 100
    again = r.render(wfb.RenderParams(spp=4, seed=5, max_depth=8))
    assert np.array_equal(bits(again.rgb), bits(mk.rgb))


def test_capacity_equal_to_pool_never_overflows(wfb):
    scene = wfb.Scene.generate("cornell36", 64, 36, 1234, 16)
    r = wfb.GpuRenderer(scene, wfb.WAVEFRONT)
    r.configure(paths_in_flight=2304)
    st = wfb.RenderStats()
    r.render(wfb.RenderParams(spp=4, seed=1, max_depth=8, queue_capacity=2304), st)
    assert st.queue_overflows == 0


def test_stage_timing_is_observation_only(wfb):
    scene = wfb.Scene.generate("icospheres", 128, 72, 1234, 16)
    plain, _, _ = render(wfb, scene, wfb.WAVEFRONT, 4, 3, 8)
    timed, st, _ = render(wfb, scene, wfb.WAVEFRONT, 4, 3, 8, stage_timing=True)
    assert np.array_equal(bits(plain.rgb), bits(timed.rgb))
    assert st.stages["extend"] > 0 and st.stages["shadow"] > 0 and st.stages["compact"] > 0


def test_progressive_equals_one_shot(wfb):
    scene = wfb.Scene.generate("cornell36", 64, 36, 1234, 16)
    r = wfb.GpuRenderer(scene, wfb.WAVEFRONT)
    p = wfb.RenderParams(spp=8, seed=3, max_depth=8)
    one = r.render(p)
    r.reset()
    r.run_passes(0, 3, p)
    r.run_passes(3, 5, p)
    assert np.array_equal(bits(one.rgb), bits(r.download(8).rgb))


@pytest.mark.parametrize("w,h", [(1, 1), (33, 17), (31, 1), (1, 33)])
def test_odd_sizes_match_reference(wfb, ref, w, h):
    arrays = load_oracle().ref_make_scene("divergence", w, h)
    out, _, _ = render(wfb, wfb.Scene.from_arrays(arrays), wfb.WAVEFRONT, 4, 7, 8)
    rrgb, rvar, _ = ref.ref_render_gpu(arrays, 1, 4, 7, 8)
    assert np.array_equal(bits(out.rgb), bits(rrgb))
    assert np.array_equal(bits(out.lum_var), bits(rvar))


def test_depth_zero_and_deep_paths(wfb, ref):
    arrays = _arrays("ref_furnace_32x18")
    for depth in (0, 1, 50):
        out, _, _ = render(wfb, wfb.Scene.from_arrays(arrays), wfb.WAVEFRONT, 2, 7, depth)
        rrgb, _, _ = ref.ref_render_gpu(arrays, 0, 2, 7, depth)
        assert np.array_equal(bits(out.rgb), bits(rrgb)), depth


def test_a_grid_barrier_that_cannot_complete_gives_up_and_the_next_render_is_exact(wfb):
    """Bounded device-side waits: the next launch's grid barriers wait for one CTA more than the launch
    has (nothing can complete them); with a 1 ms limit every CTA gives up, the kernel returns, the
    render reports WFB_ERR_DEVICE_WAIT, and the same renderer's next render is bit-exact (the
    reference's failure suite checks the same recovery after its queue overflows,
    WVM/tests/catch/wavefront_failure.cu:92-114)."""
    import time
    scene = wfb.Scene.generate("icospheres", 64, 36, 1234, 16)
    mk, _, _ = render(wfb, scene, wfb.MEGAKERNEL, 4, 5, 8)
    r = wfb.GpuRenderer(scene, wfb.WAVEFRONT)
    params = wfb.RenderParams(spp=4, seed=5, max_depth=8)
    assert np.array_equal(bits(r.render(params).rgb), bits(mk.rgb))
    try:
        wfb.set_bounded_wait_test(1_000_000, unsatisfiable=True)
        t0 = time.perf_counter()
        with pytest.raises(wfb.WfbError) as e:
            r.render(params)
        waited = time.perf_counter() - t0
    finally:
        wfb.set_bounded_wait_test(0)
    assert e.value.status == wfb.ERR_DEVICE_WAIT
    assert waited < 1.5, f"the failed render took {waited:.3f} s"
    again = r.render(params)
    assert np.array_equal(bits(again.rgb), bits(mk.rgb))
    assert np.array_equal(bits(again.lum_var), bits(mk.lum_var))


def test_l2_resident_pool_renders_the_same_film(wfb):
    """The largest pool that fits the device's persisting L2 set-aside runs under a persisting
    access-policy window; with or without the window, and against the megakernel, the film is
    bit-identical (residency is a cache policy, never a change of arithmetic)."""
    facts = wfb.device_facts()
    assert facts["l2_bytes"] > 0 and facts["wavefront_slot_bytes"] > 0
    paths = facts["wavefront_l2_resident_paths"]
    if facts["persisting_l2_max_bytes"] == 0 or paths < 1024:
        pytest.skip("no persisting L2 set-aside on this device")
    assert paths * facts["wavefront_slot_bytes"] <= facts["persisting_l2_max_bytes"]
    scene = wfb.Scene.generate("icospheres", 320, 180, 1234, 16)
    mk, _, _ = render(wfb, scene, wfb.MEGAKERNEL, 8, 9, 8)
    r = wfb.GpuRenderer(scene, wfb.WAVEFRONT)
    r.configure(paths_in_flight=paths)
    assert r.l2_window_bytes() > 0, "a pool that fits the set-aside gets a window by default"
    params = wfb.RenderParams(spp=8, seed=9, max_depth=8)
    st = wfb.RenderStats()
    out = r.render(params, st)
    assert np.array_equal(bits(out.rgb), bits(mk.rgb)) and np.array_equal(bits(out.lum_var), bits(mk.lum_var))
    assert st.queue_overflows == 0 and st.invalid_hits == 0
    r.set_l2_residency(0)
    assert r.l2_window_bytes() == 0
    assert np.array_equal(bits(r.render(params).rgb), bits(mk.rgb))
    big = wfb.GpuRenderer(scene, wfb.WAVEFRONT)
    big.configure(paths_in_flight=1 << 22)
    assert big.l2_window_bytes() == 0, "a pool above the set-aside gets no window unless asked"
    big.set_l2_residency(1)
    assert big.l2_window_bytes() > 0
    assert np.array_equal(bits(big.render(params).rgb), bits(mk.rgb))
    assert wfb.device_facts()["persisting_l2_set_aside_bytes"] > 0
    # the set-aside goes back once no pool holds a window: later kernels get the whole L2 again
    big.close()
    r.close()
    import gc
    gc.collect()  # renderers of earlier tests still waiting for collection may hold small windowed pools
    assert wfb.device_facts()["persisting_l2_set_aside_bytes"] == 0
