"""Scene model, BVH builder and hashes (CPU only)."""
import numpy as np
import pytest

from conftest import load_engine


def test_generated_scene_sizes(wfb):
    c = wfb.Scene.generate("cornell36", 32, 18).info()
    assert (c.n_triangles, c.n_spheres, c.n_lights) == (36, 0, 2)
    i = wfb.Scene.generate("icospheres", 32, 18).info()
    assert i.n_triangles == 2 + 2 + 512 * 320 and i.n_vertices == 8 + 512 * 162


@pytest.mark.slow
def test_heightfield_size(wfb):
    h = wfb.Scene.generate("heightfield", 32, 18).info()
    assert h.n_triangles == 2 * 1023 * 1023 + 2 and h.n_vertices == 1024 * 1024 + 4


def test_generators_are_deterministic(wfb):
    a = wfb.Scene.generate("icospheres", 32, 18, 1234)
    b = wfb.Scene.generate("icospheres", 32, 18, 1234)
    c = wfb.Scene.generate("icospheres", 32, 18, 4321)
    assert a.hash() == b.hash() != c.hash()
    # pinned values at the benchmark resolutions: any change to a generator shows up here
    assert wfb.Scene.generate("cornell36", 320, 180, 1234).hash() == 0xda3d860077520452
    assert wfb.Scene.generate("icospheres", 1280, 720, 1234).hash() == 0x1a1df472c06da555


@pytest.mark.parametrize("name", ["cornell36", "icospheres"])
@pytest.mark.parametrize("bins", [8, 16, 32])
def test_bvh_is_valid(wfb, name, bins):
    s = wfb.Scene.generate(name, 16, 9, 1234, bins)
    assert s.validate_bvh() == ""
    a = s.export()
    # leaves <= 4, prim_order a permutation, skip links forward
    leaves = a["nodes"][a["nodes"]["prim_count"] > 0]
    assert leaves["prim_count"].max() <= 4
    assert np.array_equal(np.sort(a["prim_order"]), np.arange(len(a["triangles"]) + len(a["spheres"])))


@pytest.mark.parametrize("name", ["cornell36", "icospheres"])
def test_8bin_builder_reproduces_reference_tree(ref, wfb, name):
    """sah_bins == 8 is the reference-compatible policy: identical nodes and prim_order bytes."""
    arrays = wfb.Scene.generate(name, 16, 9, 1234, 16).export()
    bare = dict(arrays, nodes=None, prim_order=None, lights=None)
    mine = wfb.Scene.from_arrays(bare, finalize_bins=8).export()
    nodes, order = ref.ref_build_bvh(bare)
    assert np.array_equal(mine["nodes"].view(np.uint8), nodes.view(np.uint8))
    assert np.array_equal(mine["prim_order"], order)


@pytest.mark.parametrize("name", ["cornell", "divergence", "trianglehv", "furnace"])
def test_8bin_builder_on_reference_scenes(ref, wfb, name):
    arrays = ref.ref_make_scene(name, 32, 18)
    bare = dict(arrays, nodes=None, prim_order=None, lights=None)
    mine = wfb.Scene.from_arrays(bare, finalize_bins=8).export()
    assert np.array_equal(mine["nodes"].view(np.uint8), arrays["nodes"].view(np.uint8))
    assert np.array_equal(mine["prim_order"], arrays["prim_order"])
    assert np.array_equal(mine["lights"].view(np.uint8), arrays["lights"].view(np.uint8))


@pytest.mark.parametrize("name,pin", [("cornell", 0x2ec1deb9ff15147d), ("divergence", 0x9f8c9de445c74762),
                                      ("trianglehv", 0xa489bc1b27791a9d)])
def test_scene_hash_matches_published_pins(ref, wfb, name, pin):
    """scene_hash of the reference scenes at 1280x720 equals the values in the reference's bench results."""
    arrays = ref.ref_make_scene(name, 1280, 720)
    assert ref.ref_scene_hash(arrays) == pin
    assert wfb.Scene.from_arrays(arrays).hash() == pin


def test_unfinalized_scene_is_rejected(wfb):
    arrays = wfb.Scene.generate("cornell36", 16, 9).export()
    s = wfb.Scene.from_arrays(dict(arrays, nodes=None, prim_order=None, lights=None), finalize_bins=0)
    with pytest.raises(wfb.WfbError) as e:
        wfb.GpuRenderer(s, wfb.MEGAKERNEL)
    assert e.value.status == wfb.ERR_NOT_FINALIZED


def test_invalid_scene_messages(wfb):
    arrays = wfb.Scene.generate("cornell36", 16, 9).export()
    bad = dict(arrays, nodes=None, prim_order=None, lights=None)
    t = bad["triangles"].copy()
    t["material"][0] = 99
    with pytest.raises(wfb.WfbError, match="triangle material index out of range"):
        wfb.Scene.from_arrays(dict(bad, triangles=t), finalize_bins=8)
    v = bad["vertices"].copy()
    v[0, 0] = np.inf
    with pytest.raises(wfb.WfbError, match="vertex is non-finite"):
        wfb.Scene.from_arrays(dict(bad, vertices=v), finalize_bins=8)
    with pytest.raises(wfb.WfbError, match="no primitives"):
        wfb.Scene.from_arrays(dict(bad, triangles=bad["triangles"][:0]), finalize_bins=8)


@pytest.mark.parametrize("name,bins", [("icospheres", 16), ("icospheres", 8), ("cornell36", 16)])
def test_parallel_bvh_build_is_identical_to_single_threaded(wfb, name, bins):
    """Subtrees built on many threads stitch into exactly the single-threaded tree."""
    out = {}
    for threads in (1, 3, 8):
        s = wfb.Scene.generate(name, 64, 36, 1234, 16)
        s.rebuild_bvh(bins=bins, max_leaf=4, traversal_cost=0.5, threads=threads)
        assert s.validate_bvh() == ""
        e = s.export()
        out[threads] = (e["nodes"].tobytes(), e["prim_order"].tobytes(), s.hash())
    assert out[1] == out[3] == out[8]


@pytest.mark.parametrize("name,bins", [("cornell36", 16), ("icospheres", 16), ("icospheres", 8)])
def test_bvh_boxes_nest(wfb, name, bins):
    """Speculative closest-hit traversal is exact on a nested tree; the builder's trees are nested."""
    assert wfb.Scene.generate(name, 16, 9, 1234, bins).boxes_nested()


@pytest.mark.slow
def test_heightfield_boxes_nest(wfb):
    assert wfb.Scene.generate("heightfield", 16, 9, 1234, 16).boxes_nested()


@pytest.mark.parametrize("name", ["cornell", "divergence", "trianglehv", "furnace"])
def test_reference_trees_nest(ref, wfb, name):
    assert wfb.Scene.from_arrays(ref.ref_make_scene(name, 32, 18)).boxes_nested()


def _first_internal_child(nodes):
    """(parent, child) with the child a node inside the parent's subtree."""
    for i in range(len(nodes)):
        if nodes[i]["prim_count"] == 0:
            return i, i + 1
    raise AssertionError("no internal node")


def test_boxes_nested_check_rejects_bad_trees(wfb):
    a = wfb.Scene.generate("icospheres", 16, 9, 1234, 16).export()
    assert wfb.Scene.from_arrays(a).boxes_nested()
    p, c = _first_internal_child(a["nodes"])
    # a child box reaching out of its parent's box
    bad = a["nodes"].copy()
    bad[c]["hi"][0] = np.nextafter(bad[p]["hi"][0], np.float32(np.inf))
    assert not wfb.Scene.from_arrays(dict(a, nodes=bad)).boxes_nested()
    # a leaf box shrunk by the smallest step is still nested
    ok = a["nodes"].copy()
    leaf = int(np.flatnonzero(ok["prim_count"] > 0)[0])
    ok[leaf]["hi"][0] = max(np.nextafter(ok[leaf]["hi"][0], np.float32(-np.inf)), ok[leaf]["lo"][0])
    assert wfb.Scene.from_arrays(dict(a, nodes=ok)).boxes_nested()
    # a skip link out of the parent's subtree (past the parent's own skip link)
    bad = a["nodes"].copy()
    q = next(i for i in range(len(bad)) if bad[i]["prim_count"] == 0 and 0 <= bad[i]["skip"] < len(bad) - 1)
    bad[q + 1]["skip"] = bad[q]["skip"] + 1
    assert not wfb.Scene.from_arrays(dict(a, nodes=bad)).boxes_nested()
