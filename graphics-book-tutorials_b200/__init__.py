"""Python host side of the B200 path-tracing engine (ctypes over the C ABI in include/wfb200.h).

Mirrors the reference's C++ renderer interface (WVM/include/wf/renderer.hpp:11-74 in
us-llm-engineer/graphics-book-tutorials): ``GpuRenderer(scene, mode)`` with ``render``,
``reset``, ``run_passes``, ``download``, ``download_mean``, ``device_bytes``; ``RenderParams`` and
``RenderStats`` with the reference's field names; errors are raised as ``WfbError`` carrying the
C status code (the reference raises ``std::runtime_error``).

There is no CPU fallback: importing this module requires the built ``libwfb200.so`` next to it
(``make -C graphics-book-tutorials_b200``) and every render runs the CUDA kernels.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwfb200.so")

# ---- status codes (include/wfb200.h) ----
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_CUDA = 2
ERR_OUT_OF_MEMORY = 3
ERR_NOT_FINALIZED = 4
ERR_UNSUPPORTED = 5
ERR_TIMEOUT = 6
ERR_DEVICE_WAIT = 7
ERR_INTERNAL = 8

MEGAKERNEL = 0
WAVEFRONT = 1

# ---- reference struct layouts as numpy dtypes (WVM/include/wf/scene.hpp:12-100) ----
VEC3 = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4")])
SPHERE = np.dtype([("center", "<f4", 3), ("radius", "<f4"), ("material", "<i4"), ("pad", "<i4", 3)])
TRIANGLE = np.dtype([("i0", "<i4"), ("i1", "<i4"), ("i2", "<i4"), ("material", "<i4")])
MATERIAL = np.dtype([("type", "<i4"), ("ior", "<f4"), ("pad0", "<f4"), ("pad1", "<f4"),
                     ("albedo", "<f4", 3), ("pad2", "<f4"), ("emission", "<f4", 3), ("pad3", "<f4")])
BVH_NODE = np.dtype([("lo", "<f4", 3), ("skip", "<i4"), ("hi", "<f4", 3), ("prim_start", "<i4"),
                     ("prim_count", "<i4"), ("pad", "<i4", 3)])
LIGHT = np.dtype([("prim", "<i4"), ("area", "<f4"), ("pad", "<f4", 2)])
RAY = np.dtype([("o", "<f4", 3), ("tmin", "<f4"), ("d", "<f4", 3), ("tmax", "<f4")])
HIT = np.dtype([("t", "<f4"), ("prim", "<i4"), ("u", "<f4"), ("v", "<f4")])
assert SPHERE.itemsize == 32 and MATERIAL.itemsize == 48 and BVH_NODE.itemsize == 48


class WfbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[wfb status {status}] {message}")
        self.status = status


class SceneDesc(ctypes.Structure):
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


class SceneInfo(ctypes.Structure):
    _fields_ = [
        ("n_spheres", ctypes.c_int), ("n_vertices", ctypes.c_int), ("n_triangles", ctypes.c_int),
        ("n_materials", ctypes.c_int), ("n_nodes", ctypes.c_int), ("n_prim_order", ctypes.c_int),
        ("n_lights", ctypes.c_int), ("width", ctypes.c_int), ("height", ctypes.c_int),
        ("env", ctypes.c_float * 3), ("cam_position", ctypes.c_float * 3),
        ("cam_look_at", ctypes.c_float * 3), ("cam_up", ctypes.c_float * 3),
        ("cam_vfov_deg", ctypes.c_float),
    ]


class _CRenderParams(ctypes.Structure):
    _fields_ = [("spp", ctypes.c_int), ("seed", ctypes.c_uint32), ("max_depth", ctypes.c_int),
                ("count_rays", ctypes.c_int), ("stage_timing", ctypes.c_int),
                ("queue_capacity", ctypes.c_int)]


class _CRenderStats(ctypes.Structure):
    _fields_ = [("render_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
                ("extension_rays", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64),
                ("queue_high_water", ctypes.c_int64 * 5), ("queue_overflows", ctypes.c_int64),
                ("invalid_hits", ctypes.c_int64), ("peak_vram_bytes", ctypes.c_uint64),
                ("stage_ms", ctypes.c_double * 8), ("node_visits", ctypes.c_uint64),
                ("prim_tests", ctypes.c_uint64), ("kernel_launches", ctypes.c_uint64),
                ("kernel_ms", ctypes.c_double)]


STAGE_NAMES = ("extend", "classify", "shade_lambert", "shade_metal", "shade_dielectric", "shadow",
               "compact", "other")


class _CTuneResult(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("block", ctypes.c_int), ("occupancy", ctypes.c_int),
                ("min_active", ctypes.c_int), ("leaf_batch", ctypes.c_int), ("paths_in_flight", ctypes.c_int),
                ("wf_min_active", ctypes.c_int),
                ("msamples_s", ctypes.c_double),
                ("megakernel_msamples_s", ctypes.c_double), ("wavefront_msamples_s", ctypes.c_double),
                ("candidates", ctypes.c_int), ("wf_occupancy", ctypes.c_int)]


@dataclass
class RenderParams:
    """wf::RenderParams (WVM/include/wf/renderer.hpp:11-21)."""
    spp: int = 64
    seed: int = 1234
    max_depth: int = 8
    threads: int = 0
    count_rays: bool = False
    stage_timing: bool = False
    queue_capacity: int = 0

    def _c(self) -> _CRenderParams:
        return _CRenderParams(int(self.spp), int(self.seed) & 0xFFFFFFFF, int(self.max_depth),
                              int(bool(self.count_rays)), int(bool(self.stage_timing)),
                              int(self.queue_capacity))


@dataclass
class RenderStats:
    """wf::RenderStats (WVM/include/wf/renderer.hpp:23-37)."""
    render_ms: float = 0.0
    total_ms: float = 0.0
    extension_rays: int = 0
    shadow_rays: int = 0
    queue_high_water: list = field(default_factory=lambda: [0] * 5)
    queue_overflows: int = 0
    invalid_hits: int = 0
    peak_vram_bytes: int = 0
    stages: dict = field(default_factory=dict)
    node_visits: int = 0  # megakernel with count_rays: BVH nodes visited
    prim_tests: int = 0   # megakernel with count_rays: primitive tests
    kernel_launches: int = 0  # kernels of the library launched by the call
    kernel_ms: float = 0.0    # device time of the main kernel launches alone (CUDA events)

    @classmethod
    def _from_c(cls, c: _CRenderStats) -> "RenderStats":
        return cls(c.render_ms, c.total_ms, int(c.extension_rays), int(c.shadow_rays),
                   [int(v) for v in c.queue_high_water], int(c.queue_overflows), int(c.invalid_hits),
                   int(c.peak_vram_bytes), {n: float(c.stage_ms[i]) for i, n in enumerate(STAGE_NAMES)},
                   int(c.node_visits), int(c.prim_tests), int(c.kernel_launches), float(c.kernel_ms))


@dataclass
class RenderResult:
    """wf::RenderResult (WVM/include/wf/film.hpp:11-15): rgb (h, w, 3) and lum_var (h, w)."""
    width: int
    height: int
    spp: int
    rgb: np.ndarray
    lum_var: np.ndarray


_lib = None


def _ptr(a) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libwfb200.so once; raises if it has not been built (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `make -C {_HERE}`")
    lib = ctypes.CDLL(path)
    vp, ip, i32, u32, u64 = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64
    sig = {
        "wfb_abi_version": (i32, []),
        "wfb_last_error": (ctypes.c_char_p, []),
        "wfb_device_name": (i32, [ctypes.c_char_p, i32]),
        "wfb_scene_create": (i32, [ctypes.POINTER(SceneDesc), i32, ctypes.POINTER(vp)]),
        "wfb_scene_generate": (i32, [ctypes.c_char_p, i32, i32, u32, i32, ctypes.POINTER(vp)]),
        "wfb_scene_info_get": (i32, [vp, ctypes.POINTER(SceneInfo)]),
        "wfb_scene_export": (i32, [vp, vp, vp, vp, vp, vp, vp, vp]),
        "wfb_scene_hash": (u64, [vp]),
        "wfb_scene_rebuild_bvh": (i32, [vp, i32, i32, ctypes.c_float, i32]),
        "wfb_scene_validate_bvh": (i32, [vp, ctypes.c_char_p, i32]),
        "wfb_scene_destroy": (i32, [vp]),
        "wfb_scene_device_bytes": (u64, [vp]),
        "wfb_renderer_create": (i32, [vp, i32, ctypes.POINTER(vp)]),
        "wfb_renderer_set_camera": (i32, [vp, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                          ctypes.POINTER(ctypes.c_float), ctypes.c_float, i32, i32]),
        "wfb_renderer_reset": (i32, [vp]),
        "wfb_renderer_run_passes": (i32, [vp, i32, i32, ctypes.POINTER(_CRenderParams), ctypes.POINTER(_CRenderStats)]),
        "wfb_renderer_download": (i32, [vp, i32, vp, vp]),
        "wfb_renderer_download_mean": (i32, [vp, i32, vp]),
        "wfb_renderer_download_sums": (i32, [vp, vp, vp, vp]),
        "wfb_renderer_render": (i32, [vp, ctypes.POINTER(_CRenderParams), ctypes.POINTER(_CRenderStats), vp, vp]),
        "wfb_renderer_device_bytes": (u64, [vp]),
        "wfb_renderer_configure": (i32, [vp, i32, i32, i32, i32, i32, i32, i32]),
        "wfb_renderer_set_l2_residency": (i32, [vp, i32]),
        "wfb_renderer_set_speculation": (i32, [vp, i32]),
        "wfb_scene_boxes_nested": (i32, [vp, ctypes.POINTER(ctypes.c_int)]),
        "wfb_test_traverse": (i32, [vp, vp, i32, i32, i32, i32, i32, vp]),
        "wfb_test_traverse_wide": (i32, [vp, vp, i32, i32, vp, vp]),
        "wfb_device_facts_get": (i32, [vp]),
        "wfb_renderer_l2_window_bytes": (u64, [vp]),
        "wfb_renderer_width": (i32, [vp]),
        "wfb_renderer_height": (i32, [vp]),
        "wfb_renderer_destroy": (i32, [vp]),
        "wfb_scan_workspace_create": (i32, [i32, ctypes.POINTER(vp)]),
        "wfb_scan_workspace_destroy": (i32, [vp]),
        "wfb_scan_exclusive_u32": (i32, [vp, vp, i32, vp, vp, vp]),
        "wfb_compact_u32": (i32, [vp, vp, vp, vp, vp, i32, vp, vp]),
        "wfb_test_queue_push": (i32, [vp, i32, vp, u32, vp, vp, vp]),
        "wfb_scan_workspace_check": (i32, [vp, vp]),
        "wfb_test_bounded_wait": (i32, [ctypes.c_uint64, i32]),
        "wfb_autotune": (i32, [vp, i32, i32, i32, i32, i32, ctypes.POINTER(_CTuneResult)]),
        "wfb_renderer_apply_tuning": (i32, [vp, ctypes.POINTER(_CTuneResult)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(status: int) -> None:
    if status != OK:
        raise WfbError(status, (load_library().wfb_last_error() or b"").decode())


class _CDeviceFacts(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 256), ("driver_version", ctypes.c_int), ("runtime_version", ctypes.c_int),
                ("cc_major", ctypes.c_int), ("cc_minor", ctypes.c_int), ("sm_count", ctypes.c_int),
                ("total_memory_bytes", ctypes.c_uint64), ("free_memory_bytes", ctypes.c_uint64),
                ("l2_bytes", ctypes.c_uint64), ("persisting_l2_max_bytes", ctypes.c_uint64),
                ("access_window_max_bytes", ctypes.c_uint64), ("wavefront_l2_resident_paths", ctypes.c_int),
                ("wavefront_slot_bytes", ctypes.c_int), ("persisting_l2_set_aside_bytes", ctypes.c_uint64)]


def device_facts() -> dict:
    """wf::query_cuda_device (WVM/src/gpu/gpu_renderer.cu:13-56) plus the L2 figures the wavefront uses."""
    f = _CDeviceFacts()
    _check(load_library().wfb_device_facts_get(ctypes.byref(f)))
    out = {k: getattr(f, k) for k, _ in _CDeviceFacts._fields_}
    out["name"] = f.name.decode()
    return out


def device_name() -> str:
    buf = ctypes.create_string_buffer(256)
    _check(load_library().wfb_device_name(buf, 256))
    return buf.value.decode()


class Scene:
    """A finalized scene (wf::Scene, WVM/include/wf/scene.hpp:85-100) owned by the engine."""

    def __init__(self, handle: int):
        self._h = ctypes.c_void_p(handle)

    @classmethod
    def generate(cls, name: str, width: int, height: int, seed: int = 1234, sah_bins: int = 16) -> "Scene":
        lib = load_library()
        h = ctypes.c_void_p()
        _check(lib.wfb_scene_generate(name.encode(), width, height, seed & 0xFFFFFFFF, sah_bins, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def from_arrays(cls, arrays: dict, finalize_bins: int = 0) -> "Scene":
        """arrays: dict from ``export()`` (reference dtypes) plus env/camera/width/height."""
        lib = load_library()
        keep = {}
        d = SceneDesc()
        for key, dt in (("spheres", SPHERE), ("vertices", np.float32), ("triangles", TRIANGLE),
                        ("materials", MATERIAL), ("nodes", BVH_NODE), ("prim_order", np.int32), ("lights", LIGHT)):
            a = arrays.get(key)
            a = np.ascontiguousarray(a if a is not None else np.zeros(0, dt), dtype=dt)
            if key == "vertices":
                a = a.reshape(-1, 3)
            keep[key] = a
            setattr(d, key, a.ctypes.data if a.size else None)
            setattr(d, "n_" + key, int(a.shape[0]))
        d.env = (ctypes.c_float * 3)(*arrays["env"])
        d.cam_position = (ctypes.c_float * 3)(*arrays["cam_position"])
        d.cam_look_at = (ctypes.c_float * 3)(*arrays["cam_look_at"])
        d.cam_up = (ctypes.c_float * 3)(*arrays["cam_up"])
        d.cam_vfov_deg = float(arrays["cam_vfov_deg"])
        d.width, d.height = int(arrays["width"]), int(arrays["height"])
        h = ctypes.c_void_p()
        _check(lib.wfb_scene_create(ctypes.byref(d), finalize_bins, ctypes.byref(h)))
        return cls(h.value)

    def test_traverse(self, rays: np.ndarray, anyhit: bool = False, speculate: bool = True, box_steps: int = 4,
                      leaf_batch: int = 8) -> np.ndarray:
        """Host run of the device traversal steps in simulated warps (wfb_test_traverse); rays of the
        RAY dtype, hits of the HIT dtype."""
        rays = np.ascontiguousarray(rays, RAY)
        hits = np.zeros(rays.shape[0], HIT)
        _check(load_library().wfb_test_traverse(self._h, rays.ctypes.data, int(rays.shape[0]), int(bool(anyhit)),
                                                int(bool(speculate)), int(box_steps), int(leaf_batch),
                                                hits.ctypes.data))
        return hits

    def test_traverse_wide(self, rays: np.ndarray, anyhit: bool = False):
        """Host model of a 4-wide traversal with re-tested speculation (wfb_test_traverse_wide): hits,
        and counts {fetches, pops, retests, binary_steps}."""
        rays = np.ascontiguousarray(rays, RAY)
        hits = np.zeros(rays.shape[0], HIT)
        counts = np.zeros(4, np.int64)
        _check(load_library().wfb_test_traverse_wide(self._h, rays.ctypes.data, int(rays.shape[0]), int(bool(anyhit)),
                                                     hits.ctypes.data, counts.ctypes.data))
        return hits, dict(zip(("fetches", "pops", "retests", "binary_steps"), (int(c) for c in counts)))

    def boxes_nested(self) -> bool:
        """True when the BVH's boxes nest, so closest-hit rays may traverse speculatively."""
        v = ctypes.c_int(0)
        _check(load_library().wfb_scene_boxes_nested(self._h, ctypes.byref(v)))
        return bool(v.value)

    def info(self) -> SceneInfo:
        inf = SceneInfo()
        _check(load_library().wfb_scene_info_get(self._h, ctypes.byref(inf)))
        return inf

    def export(self) -> dict:
        """Finalized host arrays in the reference layouts + env, camera and resolution."""
        inf = self.info()
        out = {
            "spheres": np.zeros(inf.n_spheres, SPHERE),
            "vertices": np.zeros((inf.n_vertices, 3), np.float32),
            "triangles": np.zeros(inf.n_triangles, TRIANGLE),
            "materials": np.zeros(inf.n_materials, MATERIAL),
            "nodes": np.zeros(inf.n_nodes, BVH_NODE),
            "prim_order": np.zeros(inf.n_prim_order, np.int32),
            "lights": np.zeros(inf.n_lights, LIGHT),
        }
        _check(load_library().wfb_scene_export(self._h, *[_ptr(out[k]) for k in (
            "spheres", "vertices", "triangles", "materials", "nodes", "prim_order", "lights")]))
        out.update(env=list(inf.env), cam_position=list(inf.cam_position), cam_look_at=list(inf.cam_look_at),
                   cam_up=list(inf.cam_up), cam_vfov_deg=inf.cam_vfov_deg, width=inf.width, height=inf.height)
        return out

    def hash(self) -> int:
        return int(load_library().wfb_scene_hash(self._h))

    def rebuild_bvh(self, bins: int = 16, max_leaf: int = 4, traversal_cost: float = 1.0, threads: int = 0) -> None:
        """Rebuilds the BVH with SAH knobs (before the first upload); see wfb_scene_rebuild_bvh."""
        _check(load_library().wfb_scene_rebuild_bvh(self._h, int(bins), int(max_leaf), float(traversal_cost),
                                                     int(threads)))

    def validate_bvh(self) -> str:
        buf = ctypes.create_string_buffer(256)
        _check(load_library().wfb_scene_validate_bvh(self._h, buf, 256))
        return buf.value.decode()

    def device_bytes(self) -> int:
        return int(load_library().wfb_scene_device_bytes(self._h))

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def close(self) -> None:
        if self._h is not None and self._h.value:
            load_library().wfb_scene_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuRenderer:
    """wf::GpuRenderer (WVM/include/wf/renderer.hpp:44-67) on this engine's sm_100a kernels."""

    def __init__(self, scene: Scene, mode: int = MEGAKERNEL):
        self._scene = scene  # keeps the scene handle alive
        h = ctypes.c_void_p()
        _check(load_library().wfb_renderer_create(scene.handle, int(mode), ctypes.byref(h)))
        self._h = h
        self.mode = mode

    @property
    def width(self) -> int:
        return int(load_library().wfb_renderer_width(self._h))

    @property
    def height(self) -> int:
        return int(load_library().wfb_renderer_height(self._h))

    def set_camera(self, position, look_at, up, vfov_deg: float, width: int, height: int) -> None:
        f3 = ctypes.c_float * 3
        _check(load_library().wfb_renderer_set_camera(self._h, f3(*position), f3(*look_at), f3(*up),
                                                       float(vfov_deg), int(width), int(height)))

    def reset(self) -> None:
        _check(load_library().wfb_renderer_reset(self._h))

    def run_passes(self, first_sample: int, count: int, params: RenderParams, stats: RenderStats | None = None):
        cs = _CRenderStats()
        _check(load_library().wfb_renderer_run_passes(self._h, first_sample, count, ctypes.byref(params._c()),
                                                       ctypes.byref(cs)))
        st = RenderStats._from_c(cs)
        if stats is not None:
            stats.__dict__.update(st.__dict__)
        return st

    def download(self, spp_done: int) -> RenderResult:
        w, h = self.width, self.height
        rgb = np.empty((h, w, 3), np.float32)
        var = np.empty((h, w), np.float32)
        _check(load_library().wfb_renderer_download(self._h, spp_done, _ptr(rgb), _ptr(var)))
        return RenderResult(w, h, spp_done, rgb, var)

    def download_mean(self, spp_done: int) -> np.ndarray:
        rgb = np.empty((self.height, self.width, 3), np.float32)
        _check(load_library().wfb_renderer_download_mean(self._h, spp_done, _ptr(rgb)))
        return rgb

    def download_sums(self):
        w, h = self.width, self.height
        rgb = np.empty((h, w, 3), np.float32)
        lum = np.empty((h, w), np.float32)
        lum2 = np.empty((h, w), np.float32)
        _check(load_library().wfb_renderer_download_sums(self._h, _ptr(rgb), _ptr(lum), _ptr(lum2)))
        return rgb, lum, lum2

    def render(self, params: RenderParams, stats: RenderStats | None = None) -> RenderResult:
        w, h = self.width, self.height
        rgb = np.empty((h, w, 3), np.float32)
        var = np.empty((h, w), np.float32)
        cs = _CRenderStats()
        _check(load_library().wfb_renderer_render(self._h, ctypes.byref(params._c()), ctypes.byref(cs),
                                                   _ptr(rgb), _ptr(var)))
        if stats is not None:
            stats.__dict__.update(RenderStats._from_c(cs).__dict__)
        return RenderResult(w, h, params.spp, rgb, var)

    def device_bytes(self) -> int:
        return int(load_library().wfb_renderer_device_bytes(self._h))

    def configure(self, block: int = -1, blocks_per_sm: int = -1, min_active: int = -1, split_chunks: int = -1,
                  paths_in_flight: int = -1, occupancy: int = -1, leaf_batch: int = -1) -> None:
        """Launch knobs (-1 keeps the current setting); see wfb_renderer_configure."""
        _check(load_library().wfb_renderer_configure(self._h, block, blocks_per_sm, min_active, split_chunks,
                                                      paths_in_flight, occupancy, leaf_batch))

    def set_l2_residency(self, mode: int) -> None:
        """Wavefront pool under a persisting L2 window: -1 when it fits the set-aside, 0 never, 1 always."""
        _check(load_library().wfb_renderer_set_l2_residency(self._h, int(mode)))

    def l2_window_bytes(self) -> int:
        return int(load_library().wfb_renderer_l2_window_bytes(self._h))

    def set_speculation(self, on: bool) -> None:
        """Speculative traversal in both arms (on by default); films are the same bits either way."""
        _check(load_library().wfb_renderer_set_speculation(self._h, int(bool(on))))

    def apply_tuning(self, tuning: "TuneResult") -> None:
        """Applies the knobs of an autotune result that belong to this renderer's arm."""
        _check(load_library().wfb_renderer_apply_tuning(self._h, ctypes.byref(tuning._c)))

    def close(self) -> None:
        if self._h is not None and self._h.value:
            load_library().wfb_renderer_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class TuneResult:
    """Outcome of :func:`autotune`: the faster arm, the best knobs of each arm, measured rates."""
    mode: int
    block: int
    occupancy: int
    min_active: int
    leaf_batch: int
    paths_in_flight: int
    wf_min_active: int
    msamples_s: float
    megakernel_msamples_s: float
    wavefront_msamples_s: float
    candidates: int
    wf_occupancy: int
    _c: _CTuneResult = field(repr=False, default=None)

    def as_dict(self) -> dict:
        return {"arm": "megakernel" if self.mode == MEGAKERNEL else "wavefront",
                "megakernel": {"block": self.block, "occupancy": self.occupancy, "min_active": self.min_active,
                               "leaf_batch": self.leaf_batch},
                "wavefront": {"paths_in_flight": self.paths_in_flight, "min_active": self.wf_min_active,
                              "occupancy": self.wf_occupancy},
                "msamples_s": round(self.msamples_s, 2),
                "megakernel_msamples_s": round(self.megakernel_msamples_s, 2),
                "wavefront_msamples_s": round(self.wavefront_msamples_s, 2), "candidates": self.candidates}


def autotune(scene: Scene, width: int, height: int, probe_spp: int = 2, max_depth: int = 8,
             try_wavefront: bool = True) -> TuneResult:
    """Measures launch configurations of both arms on the scene's camera at width x height and returns the
    fastest; cached per scene content and size inside the library (wfb_autotune)."""
    c = _CTuneResult()
    _check(load_library().wfb_autotune(scene.handle, int(width), int(height), int(probe_spp), int(max_depth),
                                       1 if try_wavefront else 0, ctypes.byref(c)))
    return TuneResult(c.mode, c.block, c.occupancy, c.min_active, c.leaf_batch, c.paths_in_flight, c.wf_min_active,
                      c.msamples_s,
                      c.megakernel_msamples_s, c.wavefront_msamples_s, c.candidates, c.wf_occupancy, c)


def compare_results(a: RenderResult, b: RenderResult) -> dict:
    """wf::compare_results (WVM/src/film.cpp:45-113): max_abs_rel, mean_rel, frac_within_3se, nonfinite."""
    if a.width != b.width or a.height != b.height:
        raise ValueError("compare_results: image dimensions mismatch")
    ra, rb = a.rgb.reshape(-1, 3), b.rgb.reshape(-1, 3)
    n = ra.shape[0]
    w = np.array([0.2126, 0.7152, 0.0722], np.float32)
    la = (np.float32(w[0]) * ra[:, 0] + np.float32(w[1]) * ra[:, 1]) + np.float32(w[2]) * ra[:, 2]
    lb = (np.float32(w[0]) * rb[:, 0] + np.float32(w[1]) * rb[:, 1]) + np.float32(w[2]) * rb[:, 2]
    fin = np.isfinite(ra) & np.isfinite(rb)
    nonfinite = int((~np.isfinite(ra)).sum() + (~np.isfinite(rb)).sum())
    denom = np.maximum(np.maximum(np.abs(ra), np.abs(rb)), np.float32(1e-6))
    rel = np.where(fin, np.abs(ra - rb) / denom, 0.0)
    sea = np.sqrt(a.lum_var.reshape(-1) / np.float32(a.spp))
    seb = np.sqrt(b.lum_var.reshape(-1) / np.float32(b.spp))
    within = np.abs(la - lb) <= np.float32(3.0) * np.sqrt(sea * sea + seb * seb)
    within &= np.isfinite(la) & np.isfinite(lb)
    mean_a, mean_b = float(la.astype(np.float64).mean()), float(lb.astype(np.float64).mean())
    mean_rel = abs(mean_a - mean_b) / mean_a if mean_a > 1e-12 else abs(mean_a - mean_b)
    return {"max_abs_rel": float(rel.max()) if n else 0.0, "mean_rel": mean_rel,
            "frac_within_3se": float(within.mean()) if n else 0.0, "nonfinite": nonfinite}


class ScanWorkspace:
    """Queue primitives on device pointers (WVM/src/gpu/queues.cuh:30-55): single-pass
    decoupled-look-back scan and stable compaction. Pointers are integers (e.g. tensor.data_ptr());
    calls are stream-ordered and return the C status (0 = OK, 1 = n > capacity)."""

    def __init__(self, capacity: int):
        h = ctypes.c_void_p()
        _check(load_library().wfb_scan_workspace_create(int(capacity), ctypes.byref(h)))
        self._h = h
        self.capacity = int(capacity)

    def scan_exclusive_u32(self, d_in: int, d_out: int, n: int, d_total: int = 0, stream: int = 0) -> int:
        return load_library().wfb_scan_exclusive_u32(d_in, d_out, n, d_total or None, self._h, stream or None)

    def compact_u32(self, d_values: int, d_flags: int, d_out: int, d_count: int, n: int, stream: int = 0) -> int:
        return load_library().wfb_compact_u32(d_values, d_flags, d_out, d_count or None, None, n, self._h,
                                              stream or None)

    def check(self, stream: int = 0) -> None:
        _check(load_library().wfb_scan_workspace_check(self._h, stream or None))

    def close(self) -> None:
        if self._h is not None and self._h.value:
            load_library().wfb_scan_workspace_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def test_queue_push(d_flags: int, n: int, d_items: int, capacity: int, d_counter: int, d_overflow: int,
                    stream: int = 0) -> int:
    """test_queue_push (WVM/src/gpu/queues.cuh:53-54) on device pointers; returns the C status."""
    return load_library().wfb_test_queue_push(d_flags, n, d_items or None, capacity & 0xFFFFFFFF, d_counter,
                                              d_overflow, stream or None)


def set_bounded_wait_test(limit_ns: int, unsatisfiable: bool = False) -> None:
    """Test hook (wfb_test_bounded_wait): limit of every bounded device-side wait (0: the 2 s default)
    and, with ``unsatisfiable``, a wait that never completes in the next wavefront launch or scan."""
    _check(load_library().wfb_test_bounded_wait(int(limit_ns), 1 if unsatisfiable else 0))


# ---------------------------------------------------------------------------------------------
# Batched rendering and the render server (no reference counterpart).

class _CJobDesc(ctypes.Structure):
    _fields_ = [("cam_position", ctypes.c_float * 3), ("cam_look_at", ctypes.c_float * 3),
                ("cam_up", ctypes.c_float * 3), ("cam_vfov_deg", ctypes.c_float), ("width", ctypes.c_int),
                ("height", ctypes.c_int), ("spp", ctypes.c_int), ("seed", ctypes.c_uint32),
                ("max_depth", ctypes.c_int)]


class _CLaunchConfig(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("use_graph", ctypes.c_int), ("block", ctypes.c_int),
                ("occupancy", ctypes.c_int), ("min_active", ctypes.c_int), ("leaf_batch", ctypes.c_int),
                ("paths_in_flight", ctypes.c_int), ("split_chunks", ctypes.c_int)]


def _launch_config(mode=0, use_graph=True, block=0, occupancy=-1, min_active=0, leaf_batch=0,
                   paths_in_flight=0, split_chunks=0) -> _CLaunchConfig:
    return _CLaunchConfig(int(mode), int(bool(use_graph)), int(block), int(occupancy), int(min_active),
                          int(leaf_batch), int(paths_in_flight), int(split_chunks))


SCHEDULES = {"express": 0, "shared": 1}  # WFB_SCHEDULE_EXPRESS, WFB_SCHEDULE_SHARED


class _CServerConfig(ctypes.Structure):
    _fields_ = [("budget_bytes", ctypes.c_uint64), ("max_jobs", ctypes.c_int), ("launch_target_ms", ctypes.c_double),
                ("fixed_slice", ctypes.c_int), ("one_job_per_launch", ctypes.c_int), ("launch", _CLaunchConfig),
                ("schedule", ctypes.c_int)]


class _CServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("cancelled", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("launches", ctypes.c_uint64), ("samples_done", ctypes.c_uint64),
                ("busy_ms", ctypes.c_double), ("wall_s", ctypes.c_double), ("p50_ms", ctypes.c_double),
                ("p95_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double), ("bytes_in_use", ctypes.c_uint64), ("peak_bytes", ctypes.c_uint64),
                ("queued", ctypes.c_int), ("active", ctypes.c_int)]


JOB_QUEUED, JOB_ACTIVE, JOB_DONE, JOB_CANCELLED, JOB_FAILED = range(5)


@dataclass
class JobDesc:
    """One render job: camera, resolution, samples, seed, depth (scene passed separately)."""
    cam_position: tuple
    cam_look_at: tuple
    cam_up: tuple = (0.0, 1.0, 0.0)
    cam_vfov_deg: float = 50.0
    width: int = 256
    height: int = 256
    spp: int = 1
    seed: int = 1
    max_depth: int = 8

    def _c(self) -> _CJobDesc:
        f3 = ctypes.c_float * 3
        return _CJobDesc(f3(*self.cam_position), f3(*self.cam_look_at), f3(*self.cam_up), float(self.cam_vfov_deg),
                         int(self.width), int(self.height), int(self.spp), int(self.seed) & 0xFFFFFFFF,
                         int(self.max_depth))


def _bind_batch_server(lib):
    vp, i32, u64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64
    jd = ctypes.POINTER(_CJobDesc)
    sig = {
        "wfb_batch_create": (i32, [i32, ctypes.POINTER(_CLaunchConfig), ctypes.POINTER(vp)]),
        "wfb_batch_add": (i32, [vp, vp, jd, ctypes.POINTER(i32)]),
        "wfb_batch_clear": (i32, [vp]),
        "wfb_batch_run": (i32, [vp, i32, ctypes.POINTER(_CRenderStats)]),
        "wfb_batch_download": (i32, [vp, i32, vp, vp]),
        "wfb_batch_download_sums": (i32, [vp, i32, vp, vp, vp]),
        "wfb_batch_destroy": (i32, [vp]),
        "wfb_server_create": (i32, [ctypes.POINTER(_CServerConfig), ctypes.POINTER(vp)]),
        "wfb_server_submit": (i32, [vp, vp, jd, ctypes.POINTER(u64)]),
        "wfb_server_poll": (i32, [vp, u64, ctypes.POINTER(i32)]),
        "wfb_server_wait": (i32, [vp, u64, i32]),
        "wfb_server_result": (i32, [vp, u64, vp, vp, ctypes.POINTER(ctypes.c_double)]),
        "wfb_server_cancel": (i32, [vp, u64]),
        "wfb_server_stats_get": (i32, [vp, ctypes.POINTER(_CServerStats)]),
        "wfb_server_reset_stats": (i32, [vp]),
        "wfb_server_destroy": (i32, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class Batch:
    """Many jobs in one persistent launch (wfb_batch_*); every job's film equals its solo render."""

    def __init__(self, max_jobs: int = 64, use_graph: bool = True, block: int = 0, min_active: int = 0,
                 mode: int = MEGAKERNEL, occupancy: int = -1, leaf_batch: int = 0, paths_in_flight: int = 0,
                 split_chunks: int = 0):
        """mode MEGAKERNEL (graph replay when use_graph) or WAVEFRONT (pool of paths_in_flight slots);
        knobs <= 0 (occupancy < 0) keep the defaults."""
        lib = _bind_batch_server(load_library())
        h = ctypes.c_void_p()
        cfg = _launch_config(mode, use_graph, block, occupancy, min_active, leaf_batch, paths_in_flight,
                             split_chunks)
        _check(lib.wfb_batch_create(int(max_jobs), ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._jobs = []
        self._scenes = []

    def add(self, scene: Scene, job: JobDesc) -> int:
        jid = ctypes.c_int()
        _check(load_library().wfb_batch_add(self._h, scene.handle, ctypes.byref(job._c()), ctypes.byref(jid)))
        self._jobs.append(job)
        self._scenes.append(scene)
        return jid.value

    def clear(self) -> None:
        _check(load_library().wfb_batch_clear(self._h))
        self._jobs.clear()
        self._scenes.clear()

    def run(self, count_rays: bool = False) -> RenderStats:
        cs = _CRenderStats()
        _check(load_library().wfb_batch_run(self._h, int(bool(count_rays)), ctypes.byref(cs)))
        return RenderStats._from_c(cs)

    def download(self, job_id: int) -> RenderResult:
        j = self._jobs[job_id]
        rgb = np.empty((j.height, j.width, 3), np.float32)
        var = np.empty((j.height, j.width), np.float32)
        _check(load_library().wfb_batch_download(self._h, job_id, _ptr(rgb), _ptr(var)))
        return RenderResult(j.width, j.height, j.spp, rgb, var)

    def download_sums(self, job_id: int):
        j = self._jobs[job_id]
        rgb = np.empty((j.height, j.width, 3), np.float32)
        lum = np.empty((j.height, j.width), np.float32)
        lum2 = np.empty((j.height, j.width), np.float32)
        _check(load_library().wfb_batch_download_sums(self._h, job_id, _ptr(rgb), _ptr(lum), _ptr(lum2)))
        return rgb, lum, lum2

    def close(self) -> None:
        if self._h is not None and self._h.value:
            load_library().wfb_batch_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching render server (wfb_server_*). Thread-safe submit/wait/result."""

    def __init__(self, budget_bytes: int = 0, max_jobs: int = 0, launch_target_ms: float = 0.0,
                 fixed_slice: int = 0, one_job_per_launch: bool = False, use_graph: bool = True, block: int = 0,
                 min_active: int = 0, mode: int = MEGAKERNEL, occupancy: int = -1, leaf_batch: int = 0,
                 paths_in_flight: int = 0, split_chunks: int = 0, schedule: str = "express"):
        lib = _bind_batch_server(load_library())
        if schedule not in SCHEDULES:
            raise ValueError(f"schedule must be one of {sorted(SCHEDULES)}")
        cfg = _CServerConfig(int(budget_bytes), int(max_jobs), float(launch_target_ms), int(fixed_slice),
                             int(bool(one_job_per_launch)),
                             _launch_config(mode, use_graph, block, occupancy, min_active, leaf_batch, paths_in_flight,
                                            split_chunks), SCHEDULES[schedule])
        h = ctypes.c_void_p()
        _check(lib.wfb_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._jobs = {}
        self._scenes = {}

    def submit(self, scene: Scene, job: JobDesc) -> int:
        t = ctypes.c_uint64()
        _check(load_library().wfb_server_submit(self._h, scene.handle, ctypes.byref(job._c()), ctypes.byref(t)))
        self._jobs[t.value] = job
        self._scenes[t.value] = scene
        return t.value

    def poll(self, ticket: int) -> int:
        st = ctypes.c_int()
        _check(load_library().wfb_server_poll(self._h, ticket, ctypes.byref(st)))
        return st.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> bool:
        rc = load_library().wfb_server_wait(self._h, ticket, int(timeout_ms))
        if rc == ERR_TIMEOUT:
            return False
        _check(rc)
        return True

    def result(self, ticket: int):
        j = self._jobs.pop(ticket)
        self._scenes.pop(ticket, None)
        rgb = np.empty((j.height, j.width, 3), np.float32)
        var = np.empty((j.height, j.width), np.float32)
        lat = ctypes.c_double()
        _check(load_library().wfb_server_result(self._h, ticket, _ptr(rgb), _ptr(var), ctypes.byref(lat)))
        return RenderResult(j.width, j.height, j.spp, rgb, var), lat.value

    def cancel(self, ticket: int) -> None:
        _check(load_library().wfb_server_cancel(self._h, ticket))

    def stats(self) -> dict:
        s = _CServerStats()
        _check(load_library().wfb_server_stats_get(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in _CServerStats._fields_}

    def reset_stats(self) -> None:
        _check(load_library().wfb_server_reset_stats(self._h))

    def close(self) -> None:
        if self._h is not None and self._h.value:
            load_library().wfb_server_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


MIX_SCENES = ("cornell36", "icospheres", "heightfield")
MIX_RESOLUTIONS = ((256, 256), (640, 360), (1280, 720), (1920, 1080))
MIX_SPP = (1, 4, 16, 64)
MIX_DEPTHS = (4, 8)


def orbit_camera(default_position, look_at, azimuth_deg: float, elevation_deg: float):
    """Camera on the orbit of the scene's default camera around its look-at point (float32)."""
    p = np.asarray(default_position, np.float32)
    t = np.asarray(look_at, np.float32)
    dist = np.float32(np.sqrt(np.float32(((p - t) ** 2).sum())))
    az, el = np.radians(np.float32(azimuth_deg)), np.radians(np.float32(elevation_deg))
    d = np.array([np.cos(el) * np.sin(az), np.sin(el), np.cos(el) * np.cos(az)], np.float32)
    return tuple(float(v) for v in (t + d * dist))


def job_mix(n: int = 64, seed: int = 1234):
    """The batched/served job distribution: n jobs with scene, resolution, spp and depth drawn
    uniformly from the sets above, seeds 1..n, orbit cameras at azimuth U(0, 360) and elevation
    U(10, 40) degrees. PRNG: numpy PCG64 seeded with `seed`; draws in this order per job: scene,
    resolution, spp, depth, azimuth, elevation. Returns a list of plain dicts."""
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n):
        scene = MIX_SCENES[int(rng.integers(len(MIX_SCENES)))]
        w, h = MIX_RESOLUTIONS[int(rng.integers(len(MIX_RESOLUTIONS)))]
        spp = MIX_SPP[int(rng.integers(len(MIX_SPP)))]
        depth = MIX_DEPTHS[int(rng.integers(len(MIX_DEPTHS)))]
        az = float(rng.uniform(0.0, 360.0))
        el = float(rng.uniform(10.0, 40.0))
        jobs.append({"scene": scene, "width": w, "height": h, "spp": spp, "max_depth": depth, "seed": i + 1,
                     "azimuth": round(az, 4), "elevation": round(el, 4)})
    return jobs


def mix_job_desc(job: dict, scene: Scene) -> JobDesc:
    """JobDesc of a job_mix entry on `scene` (orbit camera around the scene's default camera)."""
    inf = scene.info()
    pos = orbit_camera(list(inf.cam_position), list(inf.cam_look_at), job["azimuth"], job["elevation"])
    return JobDesc(cam_position=pos, cam_look_at=tuple(inf.cam_look_at), cam_up=tuple(inf.cam_up),
                   cam_vfov_deg=inf.cam_vfov_deg, width=job["width"], height=job["height"], spp=job["spp"],
                   seed=job["seed"], max_depth=job["max_depth"])
