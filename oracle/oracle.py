"""ORACLE -- test infrastructure only (tests/, __graft_entry__.smoke(), bench.py's cpu_baseline leg).

ctypes access to
  * liboracle.so        the plain-C restatement of the reference path tracer (pt_oracle.c), and
  * _ref/libwfref.so    the reference implementation itself, compiled from its own sources by
                        oracle/Makefile (CPU arm, both GPU arms, BVH builder, scene generators).
Scenes are passed as the dict of numpy arrays produced by the engine's ``Scene.export()`` (the
reference byte layouts) or by ``ref_make_scene``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libwfref.so")

SPHERE = np.dtype([("center", "<f4", 3), ("radius", "<f4"), ("material", "<i4"), ("pad", "<i4", 3)])
TRIANGLE = np.dtype([("i0", "<i4"), ("i1", "<i4"), ("i2", "<i4"), ("material", "<i4")])
MATERIAL = np.dtype([("type", "<i4"), ("ior", "<f4"), ("pad0", "<f4"), ("pad1", "<f4"),
                     ("albedo", "<f4", 3), ("pad2", "<f4"), ("emission", "<f4", 3), ("pad3", "<f4")])
BVH_NODE = np.dtype([("lo", "<f4", 3), ("skip", "<i4"), ("hi", "<f4", 3), ("prim_start", "<i4"),
                     ("prim_count", "<i4"), ("pad", "<i4", 3)])
LIGHT = np.dtype([("prim", "<i4"), ("area", "<f4"), ("pad", "<f4", 2)])
RAY = np.dtype([("o", "<f4", 3), ("tmin", "<f4"), ("d", "<f4", 3), ("tmax", "<f4")])
HIT = np.dtype([("t", "<f4"), ("prim", "<i4"), ("u", "<f4"), ("v", "<f4")])

_ARRAYS = (("spheres", SPHERE), ("vertices", np.float32), ("triangles", TRIANGLE), ("materials", MATERIAL),
           ("nodes", BVH_NODE), ("prim_order", np.int32), ("lights", LIGHT))


class CScene(ctypes.Structure):
    _fields_ = [
        ("spheres", ctypes.c_void_p), ("n_spheres", ctypes.c_int),
        ("vertices", ctypes.c_void_p), ("n_vertices", ctypes.c_int),
        ("triangles", ctypes.c_void_p), ("n_triangles", ctypes.c_int),
        ("materials", ctypes.c_void_p), ("n_materials", ctypes.c_int),
        ("nodes", ctypes.c_void_p), ("n_nodes", ctypes.c_int),
        ("prim_order", ctypes.c_void_p), ("n_prim_order", ctypes.c_int),
        ("lights", ctypes.c_void_p), ("n_lights", ctypes.c_int),
        ("env", ctypes.c_float * 3),
        ("cam_position", ctypes.c_float * 3), ("cam_look_at", ctypes.c_float * 3),
        ("cam_up", ctypes.c_float * 3), ("cam_vfov_deg", ctypes.c_float),
        ("width", ctypes.c_int), ("height", ctypes.c_int),
    ]


def build(with_reference: bool = True) -> None:
    """Compiles liboracle.so and, where the reference sources exist, _ref/libwfref.so."""
    target = "all" if with_reference else "liboracle.so"
    subprocess.run(["make", "-s", "-j8", "-C", HERE, target], check=True)


def _load(path: str) -> ctypes.CDLL:
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C {HERE}`")
    return ctypes.CDLL(path)


_oracle = None
_ref = None


def oracle_lib() -> ctypes.CDLL:
    global _oracle
    if _oracle is None:
        lib = _load(ORACLE_SO)
        vp, i32 = ctypes.c_void_p, ctypes.c_int
        lib.oracle_render_sums.restype = i32
        lib.oracle_render_sums.argtypes = [ctypes.POINTER(CScene), i32, i32, ctypes.c_uint32, i32, i32, vp, vp, vp, vp]
        lib.oracle_cpu_convention.restype = None
        lib.oracle_cpu_convention.argtypes = [i32, i32, vp, vp, vp, vp, vp]
        lib.oracle_intersect_batch.restype = None
        lib.oracle_intersect_batch.argtypes = [ctypes.POINTER(CScene), vp, i32, i32, vp]
        lib.oracle_intersect_bruteforce.restype = None
        lib.oracle_intersect_bruteforce.argtypes = [ctypes.POINTER(CScene), vp, i32, vp]
        lib.oracle_fnv1a64.restype = ctypes.c_uint64
        lib.oracle_fnv1a64.argtypes = [vp, ctypes.c_size_t]
        _oracle = lib
    return _oracle


def ref_lib() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        lib = _load(REF_SO)
        vp, i32 = ctypes.c_void_p, ctypes.c_int
        lib.ref_last_error.restype = ctypes.c_char_p
        lib.ref_render_cpu.restype = i32
        lib.ref_render_cpu.argtypes = [ctypes.POINTER(CScene), i32, ctypes.c_uint32, i32, i32, vp, vp, vp]
        lib.ref_render_gpu.restype = i32
        lib.ref_render_gpu.argtypes = [ctypes.POINTER(CScene), i32, i32, ctypes.c_uint32, i32, i32, i32, vp, vp, vp]
        lib.ref_build_bvh.restype = i32
        lib.ref_build_bvh.argtypes = [ctypes.POINTER(CScene), vp, i32, vp, i32, ctypes.POINTER(i32), ctypes.POINTER(i32)]
        lib.ref_scene_hash.restype = ctypes.c_uint64
        lib.ref_scene_hash.argtypes = [ctypes.POINTER(CScene)]
        lib.ref_make_scene.restype = vp
        lib.ref_make_scene.argtypes = [ctypes.c_char_p, i32, i32]
        lib.ref_scene_counts.restype = None
        lib.ref_scene_counts.argtypes = [vp, ctypes.POINTER(i32)]
        lib.ref_scene_view.restype = None
        lib.ref_scene_view.argtypes = [vp, ctypes.POINTER(CScene)]
        lib.ref_scene_free.restype = None
        lib.ref_scene_free.argtypes = [vp]
        lib.ref_scan.restype = i32
        lib.ref_scan.argtypes = [vp, vp, i32, vp, i32]
        lib.ref_compact.restype = i32
        lib.ref_compact.argtypes = [vp, vp, vp, vp, vp, i32, i32]
        lib.ref_queue_push.restype = i32
        lib.ref_queue_push.argtypes = [vp, i32, vp, ctypes.c_uint32, vp, vp]
        _ref = lib
    return _ref


def reference_available() -> bool:
    return os.path.exists(REF_SO)


class _Packed:
    """Keeps the numpy arrays alive while the C struct points into them."""

    def __init__(self, arrays: dict):
        self.keep = []
        c = CScene()
        for key, dt in _ARRAYS:
            a = arrays.get(key)
            a = np.ascontiguousarray(a if a is not None else np.zeros(0, dt), dtype=dt)
            if key == "vertices":
                a = a.reshape(-1, 3)
            self.keep.append(a)
            setattr(c, key, a.ctypes.data if a.size else None)
            setattr(c, "n_" + key, int(a.shape[0]))
        c.env = (ctypes.c_float * 3)(*arrays["env"])
        c.cam_position = (ctypes.c_float * 3)(*arrays["cam_position"])
        c.cam_look_at = (ctypes.c_float * 3)(*arrays["cam_look_at"])
        c.cam_up = (ctypes.c_float * 3)(*arrays["cam_up"])
        c.cam_vfov_deg = float(arrays["cam_vfov_deg"])
        c.width, c.height = int(arrays["width"]), int(arrays["height"])
        self.c = c


def render_sums(arrays: dict, spp: int, seed: int, max_depth: int, threads: int = 1, first_sample: int = 0):
    """Oracle film sums (rgb (h,w,3), lum (h,w), lum2 (h,w)) and ray counts (ext, shadow)."""
    p = _Packed(arrays)
    h, w = p.c.height, p.c.width
    rgb = np.zeros((h, w, 3), np.float32)
    lum = np.zeros((h, w), np.float32)
    lum2 = np.zeros((h, w), np.float32)
    rays = np.zeros(2, np.uint64)
    rc = oracle_lib().oracle_render_sums(ctypes.byref(p.c), first_sample, spp, seed & 0xFFFFFFFF, max_depth,
                                         threads, rgb.ctypes.data, lum.ctypes.data, lum2.ctypes.data,
                                         rays.ctypes.data)
    if rc != 0:
        raise ValueError("oracle_render_sums rejected its input")
    return rgb, lum, lum2, (int(rays[0]), int(rays[1]))


def cpu_convention(rgb_sum, lum, lum2, spp: int):
    """Reference CPU-arm mean / unbiased float variance from film sums."""
    n = lum.size
    rgb = np.empty_like(rgb_sum)
    var = np.empty_like(lum)
    oracle_lib().oracle_cpu_convention(n, spp, rgb_sum.ctypes.data, lum.ctypes.data, lum2.ctypes.data,
                                       rgb.ctypes.data, var.ctypes.data)
    return rgb, var


def gpu_convention(rgb_sum, lum, lum2, spp: int):
    """Reference GPU-arm download: rgb * (1/spp) in float, population variance in double."""
    rgb = rgb_sum * np.float32(np.float32(1.0) / np.float32(spp))
    m = lum.astype(np.float64) / spp
    m2 = lum2.astype(np.float64) / spp
    var = np.maximum(0.0, m2 - m * m).astype(np.float32)
    return rgb.astype(np.float32), var


def intersect(arrays: dict, rays: np.ndarray, anyhit: bool = False) -> np.ndarray:
    p = _Packed(arrays)
    rays = np.ascontiguousarray(rays, RAY)
    hits = np.zeros(rays.shape[0], HIT)
    oracle_lib().oracle_intersect_batch(ctypes.byref(p.c), rays.ctypes.data, rays.shape[0], int(anyhit),
                                        hits.ctypes.data)
    return hits


def intersect_bruteforce(arrays: dict, rays: np.ndarray) -> np.ndarray:
    p = _Packed(arrays)
    rays = np.ascontiguousarray(rays, RAY)
    hits = np.zeros(rays.shape[0], HIT)
    oracle_lib().oracle_intersect_bruteforce(ctypes.byref(p.c), rays.ctypes.data, rays.shape[0], hits.ctypes.data)
    return hits


def fnv1a64(buf: bytes | np.ndarray) -> int:
    b = np.frombuffer(bytes(buf), np.uint8) if not isinstance(buf, np.ndarray) else buf.view(np.uint8).ravel()
    b = np.ascontiguousarray(b)
    return int(oracle_lib().oracle_fnv1a64(b.ctypes.data, b.size))


# ---- the reference implementation itself ----

def ref_render_cpu(arrays: dict, spp: int, seed: int, max_depth: int, threads: int = 0):
    p = _Packed(arrays)
    h, w = p.c.height, p.c.width
    rgb = np.zeros((h, w, 3), np.float32)
    var = np.zeros((h, w), np.float32)
    ms = ctypes.c_double(0.0)
    lib = ref_lib()
    if lib.ref_render_cpu(ctypes.byref(p.c), spp, seed & 0xFFFFFFFF, max_depth, threads, rgb.ctypes.data,
                          var.ctypes.data, ctypes.cast(ctypes.pointer(ms), ctypes.c_void_p)) != 0:
        raise RuntimeError(lib.ref_last_error().decode())
    return rgb, var, ms.value


def ref_render_gpu(arrays: dict, mode: int, spp: int, seed: int, max_depth: int, count_rays: bool = False,
                   queue_capacity: int = 0):
    p = _Packed(arrays)
    h, w = p.c.height, p.c.width
    rgb = np.zeros((h, w, 3), np.float32)
    var = np.zeros((h, w), np.float32)
    st = np.zeros(8, np.float64)
    lib = ref_lib()
    if lib.ref_render_gpu(ctypes.byref(p.c), mode, spp, seed & 0xFFFFFFFF, max_depth, int(count_rays),
                          queue_capacity, rgb.ctypes.data, var.ctypes.data, st.ctypes.data) != 0:
        raise RuntimeError(lib.ref_last_error().decode())
    keys = ("render_ms", "extension_rays", "shadow_rays", "invalid_hits", "queue_overflows", "hw0", "hw1", "hw2")
    return rgb, var, dict(zip(keys, st.tolist()))


def ref_build_bvh(arrays: dict):
    p = _Packed(arrays)
    n_prims = p.c.n_spheres + p.c.n_triangles
    nodes = np.zeros(2 * n_prims + 2, BVH_NODE)
    order = np.zeros(n_prims + 1, np.int32)
    nn, npr = ctypes.c_int(0), ctypes.c_int(0)
    lib = ref_lib()
    rc = lib.ref_build_bvh(ctypes.byref(p.c), nodes.ctypes.data, nodes.shape[0], order.ctypes.data, order.shape[0],
                           ctypes.byref(nn), ctypes.byref(npr))
    if rc != 0:
        raise RuntimeError(f"ref_build_bvh failed ({rc}): {lib.ref_last_error().decode()}")
    return nodes[: nn.value].copy(), order[: npr.value].copy()


def ref_scene_hash(arrays: dict) -> int:
    p = _Packed(arrays)
    return int(ref_lib().ref_scene_hash(ctypes.byref(p.c)))


def ref_make_scene(name: str, width: int, height: int) -> dict:
    """A reference procedural scene (cornell, divergence, trianglehv, furnace) as arrays."""
    lib = ref_lib()
    h = lib.ref_make_scene(name.encode(), width, height)
    if not h:
        raise ValueError(lib.ref_last_error().decode())
    try:
        c = CScene()
        lib.ref_scene_view(h, ctypes.byref(c))

        def grab(ptr, n, dt, shape=None):
            if n == 0:
                return np.zeros((0,) + (shape or ()), dt)
            size = n * np.dtype(dt).itemsize * (int(np.prod(shape)) if shape else 1)
            buf = (ctypes.c_char * size).from_address(ptr)
            a = np.frombuffer(bytes(buf), dt)
            return a.reshape((n,) + shape) if shape else a

        out = {
            "spheres": grab(c.spheres, c.n_spheres, SPHERE),
            "vertices": grab(c.vertices, c.n_vertices, np.float32, (3,)),
            "triangles": grab(c.triangles, c.n_triangles, TRIANGLE),
            "materials": grab(c.materials, c.n_materials, MATERIAL),
            "nodes": grab(c.nodes, c.n_nodes, BVH_NODE),
            "prim_order": grab(c.prim_order, c.n_prim_order, np.int32),
            "lights": grab(c.lights, c.n_lights, LIGHT),
            "env": list(c.env), "cam_position": list(c.cam_position), "cam_look_at": list(c.cam_look_at),
            "cam_up": list(c.cam_up), "cam_vfov_deg": c.cam_vfov_deg, "width": c.width, "height": c.height,
        }
        return out
    finally:
        lib.ref_scene_free(h)
