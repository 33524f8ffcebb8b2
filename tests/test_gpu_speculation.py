"""Speculative traversal on a B200: the same film bits with it on and off, in both arms, on every golden
scene (engine and reference scenes) and on a tree that fails the nesting check. The
primitive tests are the same too (the counting megakernel reports them): speculation enters the same
leaves in the same order and only adds box steps (WVM/include/wf/bvh.hpp:91-116)."""
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


def _sums(wfb, scene, mode, spec, spp, seed, depth, count_rays=False):
    r = wfb.GpuRenderer(scene, mode)
    r.set_speculation(spec)
    r.reset()
    st = wfb.RenderStats()
    r.run_passes(0, spp, wfb.RenderParams(spp=spp, seed=seed, max_depth=depth, count_rays=count_rays), st)
    rgb, lum, lum2 = r.download_sums()
    r.close()
    return np.concatenate([rgb.ravel(), lum.ravel(), lum2.ravel()]).view(np.uint32), st


@pytest.mark.parametrize("case", sorted(GOLDEN))
@pytest.mark.parametrize("arm", ["megakernel", "wavefront"])
def test_speculation_keeps_film_bits(wfb, case, arm):
    g = GOLDEN[case]
    scene = wfb.Scene.from_arrays(_arrays(case))
    mode = wfb.MEGAKERNEL if arm == "megakernel" else wfb.WAVEFRONT
    on, _ = _sums(wfb, scene, mode, True, g["spp"], g["seed"], g["max_depth"])
    off, _ = _sums(wfb, scene, mode, False, g["spp"], g["seed"], g["max_depth"])
    assert np.array_equal(on, off), f"{case}/{arm}: {int((on != off).sum())} words differ"


@pytest.mark.parametrize("name", ["icospheres", "cornell36"])
def test_speculation_tests_the_same_primitives(wfb, name):
    scene = wfb.Scene.generate(name, 160, 90, 1234, 16)
    assert scene.boxes_nested()
    on, s_on = _sums(wfb, scene, wfb.MEGAKERNEL, True, 4, 7, 8, count_rays=True)
    off, s_off = _sums(wfb, scene, wfb.MEGAKERNEL, False, 4, 7, 8, count_rays=True)
    assert np.array_equal(on, off)
    assert s_on.prim_tests == s_off.prim_tests > 0
    assert s_on.extension_rays == s_off.extension_rays and s_on.shadow_rays == s_off.shadow_rays
    assert s_on.node_visits >= s_off.node_visits  # speculation only adds box steps


def test_tree_that_fails_the_nesting_check(wfb):
    """A child box grown past its parent's: closest-hit rays traverse without speculation (shadow rays
    still speculate), and the film matches the speculation-free render bit for bit."""
    a = wfb.Scene.generate("icospheres", 96, 54, 1234, 16).export()
    nodes = a["nodes"].copy()
    leaf = int(np.flatnonzero(nodes["prim_count"] > 0)[0])
    nodes[leaf]["hi"] = nodes[leaf]["hi"] + np.float32(1.0)  # leaks out of its parents' boxes
    scene = wfb.Scene.from_arrays(dict(a, nodes=nodes))
    assert not scene.boxes_nested()
    for mode in (wfb.MEGAKERNEL, wfb.WAVEFRONT):
        on, _ = _sums(wfb, scene, mode, True, 8, 3, 8)
        off, _ = _sums(wfb, scene, mode, False, 8, 3, 8)
        assert np.array_equal(on, off)
