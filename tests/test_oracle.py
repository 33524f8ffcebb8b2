"""The oracle is pinned before it is trusted: bit-for-bit against the reference's own CPU arm
(compiled from its sources into oracle/_ref) and against the committed golden films."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR, load_engine, load_oracle

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


@pytest.mark.parametrize("case", sorted(GOLDEN))
def test_oracle_matches_golden_film(case, orc):
    """Oracle film in the CPU-arm convention == golden film rendered by the reference CPU arm."""
    g = GOLDEN[case]
    arrays = _arrays(case)
    assert "%016x" % orc.ref_scene_hash(arrays) == g["scene_hash"] if orc.reference_available() else True
    rgb_s, lum, lum2, _ = orc.render_sums(arrays, g["spp"], g["seed"], g["max_depth"], threads=4)
    rgb, var = orc.cpu_convention(rgb_s, lum, lum2, g["spp"])
    ref = np.load(os.path.join(GOLDEN_DIR, f"golden_{case}.npz"))
    assert np.array_equal(bits(rgb), bits(ref["rgb"])), f"{case}: rgb differs from golden"
    assert np.array_equal(bits(var), bits(ref["lum_var"])), f"{case}: lum_var differs from golden"
    assert "%016x" % orc.fnv1a64(ref["rgb"]) == g["rgb_fnv1a64"]
    assert float(rgb.sum()) > 0.0


def test_oracle_matches_reference_cpu_arm_live(ref):
    """Different seed, depth and sample count than the fixtures, against the live reference build."""
    wfb = load_engine()
    arrays = wfb.Scene.generate("icospheres", 40, 24, 99, 16).export()
    for seed, depth, spp in ((5, 3, 3), (77, 12, 2)):
        rgb_s, lum, lum2, _ = ref.render_sums(arrays, spp, seed, depth, threads=3)
        rgb, var = ref.cpu_convention(rgb_s, lum, lum2, spp)
        ref_rgb, ref_var, _ = ref.ref_render_cpu(arrays, spp, seed, depth, threads=2)
        assert np.array_equal(bits(rgb), bits(ref_rgb))
        assert np.array_equal(bits(var), bits(ref_var))


def test_oracle_is_thread_count_independent(orc):
    wfb = load_engine()
    arrays = wfb.Scene.generate("cornell36", 24, 16, 1234, 16).export()
    a = orc.render_sums(arrays, 4, 1234, 8, threads=1)
    b = orc.render_sums(arrays, 4, 1234, 8, threads=7)
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(bits(x), bits(y))
    assert a[3] == b[3]


def test_oracle_progressive_equals_one_shot(orc):
    """Counter-based RNG: samples [0,2) then [2,5) accumulate to the same sums as [0,5)."""
    wfb = load_engine()
    arrays = wfb.Scene.generate("cornell36", 20, 12, 1234, 16).export()
    full = orc.render_sums(arrays, 5, 3, 8)
    h, w = 12, 20
    # The oracle API starts from zero sums, so emulate progression by summing per-sample films in order.
    parts = [orc.render_sums(arrays, 1, 3, 8, first_sample=s) for s in range(5)]
    rgb = np.zeros((h, w, 3), np.float32)
    for p in parts:
        rgb = rgb + p[0]
    assert np.array_equal(bits(rgb), bits(full[0]))


def test_traversal_matches_bruteforce(orc):
    """Stackless skip-link traversal == brute force on random rays (reference test_bvh.cpp:413-423)."""
    wfb = load_engine()
    arrays = wfb.Scene.generate("icospheres", 16, 9, 1234, 16).export()
    rng = np.random.default_rng(1)
    n = 2000
    rays = np.zeros(n, orc.RAY)
    rays["o"] = rng.uniform([-11, 0.1, -11], [11, 4, 11], (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    rays["d"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays["tmin"] = 1e-4
    rays["tmax"] = 3.402823466e38
    a = orc.intersect(arrays, rays)
    # brute force over 164k triangles: use a subset of rays to stay within seconds
    b = orc.intersect_bruteforce(arrays, rays[:64])
    assert np.array_equal(a[:64]["prim"], b["prim"])
    assert np.array_equal(a[:64]["t"].view(np.uint32), b["t"].view(np.uint32))
    assert (a["prim"] >= 0).mean() > 0.2
