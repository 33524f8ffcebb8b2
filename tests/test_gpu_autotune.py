"""Autotuner on a B200: the tuned configuration is a valid point of the search space, the winner
is at least as fast as every measured arm, the result is cached, and a renderer with the tuning
applied renders exactly the bits of the default renderer (launch knobs never change the film)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("name,w,h", [("cornell36", 160, 90), ("icospheres", 192, 108)])
def test_autotune_picks_valid_fastest_config(wfb, name, w, h):
    scene = wfb.Scene.generate(name, w, h, 1234, 16)
    t = wfb.autotune(scene, w, h, probe_spp=2, max_depth=8, try_wavefront=True)
    assert t.mode in (wfb.MEGAKERNEL, wfb.WAVEFRONT)
    assert t.candidates >= 18 + 4 + 1 + 2 + 2  # megakernel stages 1-3; wavefront pools x caps, min_active
    assert t.megakernel_msamples_s > 0 and t.wavefront_msamples_s > 0
    assert t.msamples_s == pytest.approx(max(t.megakernel_msamples_s, t.wavefront_msamples_s), rel=1e-9)
    assert (t.mode == wfb.WAVEFRONT) == (t.wavefront_msamples_s > t.megakernel_msamples_s)
    assert (t.block, t.occupancy) in {(128, 10), (128, 8), (128, 6), (128, 0), (64, 0), (256, 0)}
    assert t.min_active in (4, 8, 12, 16, 20, 24, 28) and t.leaf_batch in (4, 8, 12, 16, 32)
    facts = wfb.device_facts()
    pools = {min(p, 64 * w * h) for p in (facts["wavefront_l2_resident_paths"], 1 << 21, 1 << 22, 1 << 23, 1 << 24)}
    assert t.paths_in_flight in pools and t.wf_min_active in (16, 20, 24) and t.wf_occupancy in (8, 10)
    mk_only = wfb.autotune(scene, w, h, probe_spp=2, max_depth=8, try_wavefront=False)
    assert mk_only.mode == wfb.MEGAKERNEL and mk_only.paths_in_flight == 0 and mk_only.wavefront_msamples_s == 0
    again = wfb.autotune(scene, w, h, probe_spp=2, max_depth=8, try_wavefront=True)
    assert again.as_dict() == t.as_dict()  # served from the cache


def test_tuned_renderer_is_bit_equal_to_default(wfb):
    w, h = 128, 72
    scene = wfb.Scene.generate("icospheres", w, h, 1234, 16)
    t = wfb.autotune(scene, w, h, probe_spp=1, max_depth=8, try_wavefront=True)
    params = wfb.RenderParams(spp=8, seed=77, max_depth=8)
    base = wfb.GpuRenderer(scene, wfb.MEGAKERNEL).render(params)
    for mode in (wfb.MEGAKERNEL, wfb.WAVEFRONT):
        r = wfb.GpuRenderer(scene, mode)
        r.apply_tuning(t)
        out = r.render(params)
        assert np.array_equal(bits(out.rgb), bits(base.rgb))
        assert np.array_equal(bits(out.lum_var), bits(base.lum_var))


def test_autotune_rejects_bad_sizes(wfb):
    scene = wfb.Scene.generate("cornell36", 32, 18, 1234, 16)
    with pytest.raises(wfb.WfbError):
        wfb.autotune(scene, 0, 18)
    with pytest.raises(wfb.WfbError):
        wfb.autotune(scene, 32, 18, probe_spp=0)
