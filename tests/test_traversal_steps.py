"""The device traversal steps (box_step / prim_step, compiled for the host and run in simulated
32-lane warps by wfb_test_traverse) against the oracle's preorder traversal (WVM/include/wf/bvh.hpp:
91-116), bit for bit, with speculation on and off and several round policies, on rays chosen to
break an inexact speculation: directions with zero components (+0 and -0), origins on BVH box
planes, rays through shared triangle edges and vertices, and rays that start inside geometry."""
import zlib

import numpy as np
import pytest

KNOBS = [(True, 4, 12), (True, 1, 1), (True, 8, 32), (True, 2, 4), (False, 1, 8), (False, 4, 12)]


def _scene(wfb, orc, name):
    if name in ("cornell36", "icospheres"):
        return wfb.Scene.generate(name, 16, 9, 1234, 16).export()
    return orc.ref_make_scene(name, 32, 18)


def _rays(wfb, arrays, n, seed):
    """A mix of adversarial rays for the scene's own boxes and triangles."""
    rng = np.random.default_rng(seed)
    nodes, verts, tris = arrays["nodes"], arrays["vertices"], arrays["triangles"]
    lo = nodes["lo"][0].astype(np.float64)
    hi = nodes["hi"][0].astype(np.float64)
    span = np.maximum(hi - lo, 1e-3)
    rays = np.zeros(n, wfb.RAY)
    o = rng.uniform(lo - 0.1 * span, hi + 0.1 * span, (n, 3))
    d = rng.normal(size=(n, 3))
    k = n // 6
    # 1: one or two direction components exactly +0 or -0
    for i in range(k):
        zero = rng.choice(3, size=rng.integers(1, 3), replace=False)
        d[i, zero] = 0.0
        if rng.random() < 0.5:
            d[i, zero] = -0.0
    # 2: origins on a box plane of a random node, direction parallel to that plane
    idx = rng.integers(0, len(nodes), size=k)
    for j, i in enumerate(range(k, 2 * k)):
        ax = rng.integers(0, 3)
        o[i] = rng.uniform(nodes["lo"][idx[j]], nodes["hi"][idx[j]])
        o[i, ax] = nodes["lo"][idx[j]][ax] if rng.random() < 0.5 else nodes["hi"][idx[j]][ax]
        d[i, ax] = 0.0 if rng.random() < 0.5 else -0.0
    # 3: through a shared edge's midpoint or a vertex of a triangle
    if len(tris):
        t = rng.integers(0, len(tris), size=k)
        for j, i in enumerate(range(2 * k, 3 * k)):
            a = verts[tris["i0"][t[j]]].astype(np.float64)
            b = verts[tris["i1"][t[j]]].astype(np.float64)
            target = a if rng.random() < 0.3 else 0.5 * (a + b)
            d[i] = target - o[i]
    # 4: axis-aligned directions from origins inside the scene
    for i in range(3 * k, 4 * k):
        d[i] = 0.0
        d[i, rng.integers(0, 3)] = 1.0 if rng.random() < 0.5 else -1.0
    norm = np.linalg.norm(d, axis=1, keepdims=True)
    norm[norm == 0] = 1.0
    d = d / norm
    d[np.all(d == 0, axis=1)] = (0.0, -1.0, 0.0)
    rays["o"] = o.astype(np.float32)
    # keep the signed zeros chosen above: convert component-wise
    rays["d"] = d.astype(np.float32)
    for i in range(2 * k):
        for ax in range(3):
            if d[i, ax] == 0.0:
                rays["d"][i, ax] = np.float32(np.copysign(0.0, d[i, ax]))
    rays["tmin"] = np.float32(1e-4)
    rays["tmax"] = np.float32(3.402823466e38)
    # a few finite tmax values (shadow-ray-like queries)
    rays["tmax"][5 * k:] = rng.uniform(0.1, 10.0, n - 5 * k).astype(np.float32)
    return rays


def _same(a, b):
    return (np.array_equal(a["t"].view(np.uint32), b["t"].view(np.uint32)) and np.array_equal(a["prim"], b["prim"])
            and np.array_equal(a["u"].view(np.uint32), b["u"].view(np.uint32))
            and np.array_equal(a["v"].view(np.uint32), b["v"].view(np.uint32)))


@pytest.mark.parametrize("name", ["cornell36", "icospheres", "cornell", "divergence", "trianglehv", "furnace"])
@pytest.mark.parametrize("anyhit", [False, True])
def test_traversal_steps_equal_preorder_traversal(wfb, orc, name, anyhit):
    arrays = _scene(wfb, orc, name)
    scene = wfb.Scene.from_arrays(arrays)
    assert scene.boxes_nested()
    rays = _rays(wfb, arrays, 3000, seed=zlib.crc32(f"{name}/{anyhit}".encode()))
    want = orc.intersect(arrays, rays, anyhit=anyhit)
    assert (want["prim"] >= 0).mean() > 0.05
    for spec, steps, leaf_batch in KNOBS:
        got = scene.test_traverse(rays, anyhit=anyhit, speculate=spec, box_steps=steps, leaf_batch=leaf_batch)
        bad = np.flatnonzero((got["prim"] != want["prim"]) | (got["t"].view(np.uint32) != want["t"].view(np.uint32)))
        assert _same(got, want), f"{name} anyhit={anyhit} spec={spec} steps={steps} lb={leaf_batch}: rays {bad[:8]}"


def test_traversal_steps_on_a_tree_that_fails_the_nesting_check(wfb, orc):
    """A leaf box grown out of its parents': closest-hit rays then traverse without speculation and
    still equal preorder traversal on the same (modified) tree."""
    arrays = _scene(wfb, orc, "icospheres")
    nodes = arrays["nodes"].copy()
    leaf = int(np.flatnonzero(nodes["prim_count"] > 0)[0])
    nodes[leaf]["hi"] = nodes[leaf]["hi"] + np.float32(1.0)
    arrays = dict(arrays, nodes=nodes)
    scene = wfb.Scene.from_arrays(arrays)
    assert not scene.boxes_nested()
    rays = _rays(wfb, arrays, 1500, seed=7)
    for anyhit in (False, True):
        want = orc.intersect(arrays, rays, anyhit=anyhit)
        got = scene.test_traverse(rays, anyhit=anyhit, speculate=True, box_steps=4, leaf_batch=12)
        assert _same(got, want)


def test_traverse_rejects_bad_knobs(wfb):
    scene = wfb.Scene.generate("cornell36", 16, 9, 1234, 16)
    rays = np.zeros(4, wfb.RAY)
    with pytest.raises(wfb.WfbError):
        scene.test_traverse(rays, box_steps=0)


def _coplanar_quads(wfb, seed, n_quads=200):
    """Axis-aligned quads of different extents at x = 1 (and within 1e-3 of it), in separate leaves:
    hits on one plane from many leaves, where a leaf's box test and its triangles' t round differently."""
    rng = np.random.default_rng(seed)
    base = wfb.Scene.generate("cornell36", 16, 9, 1234, 16).export()
    verts, tris = [], []
    for q in range(n_quads):
        y0, z0 = rng.uniform(-1, 0.5, 2)
        y1, z1 = y0 + rng.uniform(0.2, 1.5), z0 + rng.uniform(0.2, 1.5)
        x = np.float32(1.0) if q % 2 == 0 else np.float32(rng.uniform(0.999, 1.001))
        v = len(verts)
        verts += [(x, y0, z0), (x, y1, z0), (x, y1, z1), (x, y0, z1)]
        tris += [(v, v + 1, v + 2), (v, v + 2, v + 3)]
    t = np.zeros(len(tris), wfb.TRIANGLE)
    t["i0"], t["i1"], t["i2"] = np.array(tris).T
    arrays = dict(base, vertices=np.array(verts, np.float32), triangles=t,
                  spheres=np.zeros(0, base["spheres"].dtype), nodes=None, prim_order=None, lights=None)
    scene = wfb.Scene.from_arrays(arrays, finalize_bins=8)
    full = dict(arrays, **{k: v for k, v in scene.export().items() if k in ("nodes", "prim_order", "lights")})
    return scene, full


def test_traversal_steps_on_coplanar_quads(wfb, orc):
    """The case speculation has to get right: a leaf reached while another is pending may only be
    entered on a box test against the tmax that the pending leaf leaves. Entering it on the earlier
    (stale) test instead changes about one ray in 10^4 here -- a mistake planted in a local build was
    caught by this case -- while the held-and-retested leaf matches preorder traversal on every ray."""
    scene, arrays = _coplanar_quads(wfb, seed=1)
    assert scene.boxes_nested()
    rng = np.random.default_rng(1)
    n = 200000
    o = np.stack([rng.uniform(-3, 0.5, n), rng.uniform(-2, 2, n), rng.uniform(-2, 2, n)], 1)
    tgt = np.stack([np.ones(n), rng.uniform(-1, 2, n), rng.uniform(-1, 2, n)], 1)
    d = (tgt - o) / np.linalg.norm(tgt - o, axis=1, keepdims=True)
    rays = np.zeros(n, wfb.RAY)
    rays["o"], rays["d"] = o.astype(np.float32), d.astype(np.float32)
    rays["tmin"], rays["tmax"] = np.float32(1e-4), np.float32(3.402823466e38)
    want = orc.intersect(arrays, rays)
    assert (want["prim"] >= 0).mean() > 0.5
    for spec, steps, leaf_batch in [(True, 4, 12), (True, 1, 32), (True, 8, 32), (False, 4, 12)]:
        got = scene.test_traverse(rays, speculate=spec, box_steps=steps, leaf_batch=leaf_batch)
        assert _same(got, want), (spec, steps, leaf_batch)


@pytest.mark.parametrize("name", ["icospheres", "cornell36", "trianglehv", "divergence"])
@pytest.mark.parametrize("anyhit", [False, True])
def test_wide_model_equals_preorder_traversal(wfb, orc, name, anyhit):
    """The host model of a 4-wide traversal (grandchild boxes tested together, stacked with the tmax of
    that test, re-tested when tmax has moved) enters the reference's leaves in the reference's order:
    bit-equal hits on the adversarial rays, with far fewer dependent fetches than binary box steps."""
    arrays = _scene(wfb, orc, name)
    scene = wfb.Scene.from_arrays(arrays)
    rays = _rays(wfb, arrays, 3000, seed=zlib.crc32(f"wide/{name}/{anyhit}".encode()))
    want = orc.intersect(arrays, rays, anyhit=anyhit)
    got, counts = scene.test_traverse_wide(rays, anyhit=anyhit)
    assert _same(got, want)
    if name == "icospheres" and not anyhit:
        assert counts["fetches"] + counts["retests"] < 0.5 * counts["binary_steps"], counts


def test_wide_model_on_coplanar_quads(wfb, orc):
    scene, arrays = _coplanar_quads(wfb, seed=1)
    rng = np.random.default_rng(2)
    n = 100000
    o = np.stack([rng.uniform(-3, 0.5, n), rng.uniform(-2, 2, n), rng.uniform(-2, 2, n)], 1)
    tgt = np.stack([np.ones(n), rng.uniform(-1, 2, n), rng.uniform(-1, 2, n)], 1)
    d = (tgt - o) / np.linalg.norm(tgt - o, axis=1, keepdims=True)
    rays = np.zeros(n, wfb.RAY)
    rays["o"], rays["d"] = o.astype(np.float32), d.astype(np.float32)
    rays["tmin"], rays["tmax"] = np.float32(1e-4), np.float32(3.402823466e38)
    got, counts = scene.test_traverse_wide(rays)
    assert _same(got, orc.intersect(arrays, rays))
    assert counts["retests"] > 0  # tmax moves between a stacked test and the pop on this scene
