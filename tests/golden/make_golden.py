"""Regenerates the golden films in this directory from the REFERENCE CPU arm.

The reference implementation is compiled from its own sources by oracle/Makefile into
oracle/_ref/libwfref.so; this script renders small cases with it and stores
  * golden_<case>.npz   rgb (h, w, 3) and lum_var (h, w) in the reference CPU-arm convention,
  * golden.json         per case: scene, size, spp, seed, depth, scene_hash and FNV-1a hashes of
                        the rgb / lum_var bytes (so a mismatch is visible without numpy).
Scenes: this engine's benchmark generators (exported as reference-layout arrays, BVH built by
the engine) and the reference's own procedural scenes (make_scene). Run from the repository root:
    python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from conftest import load_engine, load_oracle  # noqa: E402

CASES = [
    # name, source, width, height, spp, seed, max_depth
    ("cornell36_64x36", "engine:cornell36", 64, 36, 8, 1234, 8),
    ("icospheres_64x36", "engine:icospheres", 64, 36, 4, 1234, 8),
    ("heightfield_48x27", "engine:heightfield", 48, 27, 2, 1234, 8),
    ("ref_cornell_32x18", "ref:cornell", 32, 18, 4, 7, 8),
    ("ref_divergence_32x18", "ref:divergence", 32, 18, 4, 7, 8),
    ("ref_trianglehv_32x18", "ref:trianglehv", 32, 18, 2, 7, 8),
    ("ref_furnace_32x18", "ref:furnace", 32, 18, 4, 7, 8),
]


def scene_arrays(source, width, height):
    kind, name = source.split(":")
    if kind == "engine":
        wfb = load_engine()
        return wfb.Scene.generate(name, width, height, 1234, 16).export()
    return load_oracle().ref_make_scene(name, width, height)


def main():
    orc = load_oracle()
    index = {}
    for case, source, w, h, spp, seed, depth in CASES:
        arrays = scene_arrays(source, w, h)
        rgb, var, _ = orc.ref_render_cpu(arrays, spp, seed, depth, threads=os.cpu_count() or 1)
        np.savez_compressed(os.path.join(HERE, f"golden_{case}.npz"), rgb=rgb, lum_var=var)
        index[case] = {
            "source": source, "width": w, "height": h, "spp": spp, "seed": seed, "max_depth": depth,
            "scene_hash": "%016x" % orc.ref_scene_hash(arrays),
            "rgb_fnv1a64": "%016x" % orc.fnv1a64(rgb), "lum_var_fnv1a64": "%016x" % orc.fnv1a64(var),
        }
        print(case, index[case])
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
