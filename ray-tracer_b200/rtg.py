"""Python mirror of the reference renderer's interface, over the C ABI in include/rtg.h.

Names and argument meaning follow the reference's C++ API so code written against
it reads the same:

    parse_scene / load_scene / validate_scene   src/io/scene_io.cpp:380-502
    Scene.compile                                src/core/scene.cpp:31-137
    RenderSettings / RenderOptions               include/raytracer/core/scene_desc.hpp:20-35,
                                                 include/raytracer/rendering/renderer.hpp:41-44
    Renderer.render / image / stats              src/rendering/renderer.cpp:58-110
    RenderProgress                               include/raytracer/rendering/renderer.hpp:25-33

Everything runs in librtg.so (C++20 host + sm_100a kernels). This module only
marshals arguments: it has no compute path of its own and raises if the library
is missing or no GPU is present when GPU work is requested.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
import threading
from typing import Callable, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("RTG_LIBRARY") or os.path.join(_HERE, "librtg.so")  # override: another build

RTG_OK = 0
RTG_ERR_INVALID = -1
RTG_ERR_SCENE = -2
RTG_ERR_CUDA = -3
RTG_ERR_NO_DEVICE = -4
RTG_ERR_DEVICE = -5
RTG_ERR_BUSY = -6
RTG_ERR_LIMIT = -7
NOALLOC_MAX_RAYS = 262144

INTEGRATORS = {"path": 0, "direct": 1, "normals": 2}
TONE_MAPS = {"clamp": 0, "reinhard": 1, "aces": 2}


class SceneError(RuntimeError):
    """Scene JSON rejected (parse or validation); the message names the field."""


class RtgError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"rtg error {code}: {message}")
        self.code = code


class _Settings(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("max_depth", C.c_int32),
        ("rr_min_depth", C.c_int32), ("integrator", C.c_int32), ("light_sampling", C.c_int32),
        ("tone_map", C.c_int32), ("seed", C.c_uint64), ("exposure", C.c_double), ("threads", C.c_int32),
        ("tile_size", C.c_int32), ("use_bvh", C.c_int32), ("reserved", C.c_int32),
    ]


class _Options(C.Structure):
    _fields_ = [("progressive", C.c_int32), ("max_pass_spp", C.c_int32)]


class _Progress(C.Structure):
    _fields_ = [
        ("pass_", C.c_int32), ("spp_done", C.c_uint32), ("spp_target", C.c_int32), ("finished", C.c_int32),
        ("cancelled", C.c_int32), ("reserved", C.c_int32), ("elapsed_ms", C.c_double), ("rays", C.c_uint64),
    ]


class _Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "camera_samples", "rays", "shadow_rays", "rr_terminated", "invalid_samples", "passes",
        "iterations", "node_visits", "prim_tests", "sphere_tests", "extend_launches", "shadow_node_visits",
        "shadow_prim_tests", "shadow_sphere_tests", "kernel_launches")] + [
        (n, C.c_double) for n in ("elapsed_ms", "device_ms", "extend_ms", "shade_ms", "shadow_ms", "accumulate_ms",
                                  "direct_ms", "plan_ms")]


class _SceneInfo(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "primitives", "triangles", "spheres", "planes", "degenerate_skipped", "lights", "bvh_nodes",
        "bvh_leaves", "bvh_max_depth", "bvh_max_leaf", "device_bytes")] + [
        ("bvh_build_ms", C.c_double), ("bvh_sah_cost", C.c_double)]


class _SceneView(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "n_prims", "n_planes", "n_nodes", "n_order", "n_lights", "n_point_lights", "n_materials")] + [
        ("prims", C.POINTER(C.c_double)), ("planes", C.POINTER(C.c_double)), ("nodes", C.POINTER(C.c_double)),
        ("order", C.POINTER(C.c_uint32)), ("lights", C.POINTER(C.c_uint32)),
        ("point_lights", C.POINTER(C.c_double)), ("materials", C.POINTER(C.c_double)),
        ("camera", C.c_double * 19), ("background", C.c_double * 8), ("settings", _Settings),
        ("degenerate_skipped", C.c_uint64), ("bvh_max_depth", C.c_uint64), ("bvh_leaves", C.c_uint64),
        ("bvh_max_leaf", C.c_uint64), ("bvh_sah_cost", C.c_double)]


class _Tuning(C.Structure):
    _fields_ = [
        ("pool_paths", C.c_uint32), ("block", C.c_uint32), ("max_pass_samples", C.c_uint64),
        ("extend_blocks", C.c_int32), ("shade_blocks", C.c_int32), ("shadow_blocks", C.c_int32),
        ("time_kernels", C.c_int32), ("count_traversal", C.c_int32), ("backlog_pools", C.c_uint32),
        ("chained", C.c_uint32), ("serve_budget_bytes", C.c_uint64), ("serve_reserve_bytes", C.c_uint64),
        ("refine_hits", C.c_int32), ("closest_tree", C.c_int32), ("shadow_tree", C.c_int32),
        ("reserved", C.c_int32),
    ]


class _RequestEvent(C.Structure):
    _fields_ = [("request", C.c_int32), ("reserved", C.c_int32), ("progress", _Progress)]


PASS_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(_Progress))

# Every entry point declared in include/rtg.h, with its ctypes signature.
_SIGNATURES = {
    "rtg_validate": (C.c_char_p, [C.c_char_p]),
    "rtg_scene_dump": (C.c_int64, [C.c_char_p, C.c_char_p, C.c_size_t]),
    "rtg_compile": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "rtg_compile_flags": (C.c_int, [C.c_char_p, C.c_char_p, C.c_uint32, C.POINTER(C.c_void_p), C.c_char_p,
                                    C.c_size_t]),
    "rtg_host_scene_free": (None, [C.c_void_p]),
    "rtg_host_scene_view": (C.c_int, [C.c_void_p, C.POINTER(_SceneView)]),
    "rtg_context_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "rtg_context_destroy": (None, [C.c_void_p]),
    "rtg_last_error": (C.c_char_p, [C.c_void_p]),
    "rtg_device_count": (C.c_int, []),
    "rtg_scene_load_json": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.POINTER(C.c_int32)]),
    "rtg_scene_load_file": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_int32)]),
    "rtg_scene_upload": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)]),
    "rtg_scene_upload_batch": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_int32)]),
    "rtg_scene_upload_gpu_bvh": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)]),
    "rtg_scene_layout": (C.c_int64, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_uint64]),
    "rtg_host_scene_layout": (C.c_int64, [C.c_void_p, C.c_int32, C.c_void_p, C.c_uint64]),
    "rtg_scene_settings": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(_Settings)]),
    "rtg_scene_get_info": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(_SceneInfo)]),
    "rtg_scene_release": (C.c_int, [C.c_void_p, C.c_int32]),
    "rtg_render": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(_Settings), C.POINTER(_Options), PASS_FN, C.c_void_p,
                             C.POINTER(C.c_int32), C.POINTER(_Progress)]),
    "rtg_render_batch": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(_Settings),
                                   C.POINTER(_Options), C.POINTER(C.c_int32), C.POINTER(_Progress)]),
    "rtg_framebuffer_mean": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "rtg_framebuffer_moments": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                          C.POINTER(C.c_uint32)]),
    "rtg_image_rgb8": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.POINTER(C.c_uint8)]),
    "rtg_images_rgb8": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.c_double,
                                  C.POINTER(C.POINTER(C.c_uint8))]),
    "rtg_render_stats": (C.c_int, [C.c_void_p, C.POINTER(_Stats)]),
    "rtg_trace_closest": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_float), C.c_uint64, C.c_int32,
                                    C.POINTER(C.c_float), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                    C.POINTER(C.c_float)]),
    "rtg_trace_any": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_float), C.c_uint64, C.c_int32,
                                C.POINTER(C.c_uint8)]),
    "rtg_trace_closest_noalloc": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_float), C.c_uint64, C.c_int32,
                                            C.POINTER(C.c_float), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                            C.POINTER(C.c_float)]),
    "rtg_allocation_count": (C.c_uint64, []),
    "rtg_probe_read_bandwidth": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
    "rtg_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(_Tuning)]),
    "rtg_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(_Tuning)]),
    "rtg_request_submit": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(_Settings), C.POINTER(_Options), C.c_int32,
                                     C.POINTER(C.c_int32)]),
    "rtg_serve_pump": (C.c_int, [C.c_void_p, C.c_double, C.c_int32, C.POINTER(_RequestEvent), C.c_int32,
                                 C.POINTER(C.c_int32)]),
    "rtg_request_cancel": (C.c_int, [C.c_void_p, C.c_int32]),
    "rtg_request_release": (C.c_int, [C.c_void_p, C.c_int32]),
    "rtg_request_progress": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(_Progress)]),
    "rtg_request_mean": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "rtg_request_image_rgb8": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.POINTER(C.c_uint8)]),
    "rtg_serve_prepare": (C.c_int, [C.c_void_p]),
    "rtg_serve_footprint": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_int32),
                                      C.POINTER(C.c_int32)]),
    "rtg_autotune": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(_Settings), C.POINTER(_Options),
                               C.c_int32, C.POINTER(_Tuning), C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "rtg_encode_png": (C.c_int64, [C.POINTER(C.c_uint8), C.c_int32, C.c_int32, C.POINTER(C.c_uint8), C.c_size_t]),
}

_lib = None
_lib_lock = threading.Lock()


def lib() -> C.CDLL:
    """Loads librtg.so (built in tree); raises if it is missing."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C ray-tracer_b200` "
                                   "(or __graft_entry__.build())")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in _SIGNATURES.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
        return _lib


def exported_symbols() -> list[str]:
    return sorted(_SIGNATURES)


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


# ---------------------------------------------------------------------------
# Settings

@dataclasses.dataclass
class RenderSettings:
    width: int = 640
    height: int = 360
    spp: int = 64
    max_depth: int = 8
    rr_min_depth: int = 3
    integrator: str = "path"
    light_sampling: bool = True
    seed: int = 1
    tone_map: str = "aces"
    exposure: float = 1.0
    threads: int = 0
    tile_size: int = 16
    use_bvh: bool = True
    mis: bool = False  # multiple importance sampling with NEE (no reference counterpart)

    def to_c(self) -> _Settings:
        ls = (2 if self.mis else 1) if self.light_sampling else 0
        return _Settings(self.width, self.height, self.spp, self.max_depth, self.rr_min_depth,
                         INTEGRATORS[self.integrator], ls, TONE_MAPS[self.tone_map],
                         self.seed, self.exposure, self.threads, self.tile_size, int(self.use_bvh), 0)

    @staticmethod
    def from_c(c: _Settings) -> "RenderSettings":
        inv_i = {v: k for k, v in INTEGRATORS.items()}
        inv_t = {v: k for k, v in TONE_MAPS.items()}
        return RenderSettings(c.width, c.height, c.spp, c.max_depth, c.rr_min_depth, inv_i[c.integrator],
                              bool(c.light_sampling), c.seed, inv_t[c.tone_map], c.exposure, c.threads,
                              c.tile_size, bool(c.use_bvh), c.light_sampling == 2)


@dataclasses.dataclass
class RenderOptions:
    progressive: bool = True
    max_pass_spp: int = 32


@dataclasses.dataclass
class RenderProgress:
    pass_: int
    spp_done: int
    spp_target: int
    elapsed_ms: float
    rays: int
    finished: bool
    cancelled: bool

    @staticmethod
    def from_c(p: _Progress) -> "RenderProgress":
        return RenderProgress(p.pass_, p.spp_done, p.spp_target, p.elapsed_ms, p.rays, bool(p.finished),
                              bool(p.cancelled))


# ---------------------------------------------------------------------------
# Scene description (host side; no GPU needed)

def validate_scene(scene_json: str) -> str:
    """'' if the scene parses and validates, else the first problem (rt_validate)."""
    return lib().rtg_validate(scene_json.encode()).decode()


def dump_scene(scene_json: str) -> str:
    """Normalised scene JSON (scene_to_json)."""
    L = lib()
    n = L.rtg_scene_dump(scene_json.encode(), None, 0)
    if n < 0:
        raise SceneError(validate_scene(scene_json))
    buf = C.create_string_buffer(n + 1)
    L.rtg_scene_dump(scene_json.encode(), buf, n + 1)
    return buf.value.decode()


class HostScene:
    """A compiled scene on the host (Scene::compile): primitives, planes, lights, BVH."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.rtg_host_scene_free(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def view(self) -> dict:
        """The compiled scene in the reference's layout, as numpy arrays (copies)."""
        v = _SceneView()
        rc = lib().rtg_host_scene_view(self._h, C.byref(v))
        if rc != RTG_OK:
            raise RtgError(rc, "scene view failed")

        def arr(p, n, width, dtype):
            if n == 0:
                return np.zeros((0, width), dtype=dtype)
            return np.ctypeslib.as_array(p, shape=(n * width,)).reshape(n, width).astype(dtype, copy=True)

        return {
            "prims": arr(v.prims, v.n_prims, 24, np.float64),
            "planes": arr(v.planes, v.n_planes, 8, np.float64),
            "nodes": arr(v.nodes, v.n_nodes, 10, np.float64),
            "order": arr(v.order, v.n_order, 1, np.uint32).reshape(-1),
            "lights": arr(v.lights, v.n_lights, 2, np.uint32),
            "point_lights": arr(v.point_lights, v.n_point_lights, 6, np.float64),
            "materials": arr(v.materials, v.n_materials, 16, np.float64),
            "camera": np.array(v.camera[:], dtype=np.float64),
            "background": np.array(v.background[:], dtype=np.float64),
            "settings": RenderSettings.from_c(v.settings),
            "degenerate_skipped": v.degenerate_skipped,
            "bvh_max_depth": v.bvh_max_depth,
            "bvh_leaves": v.bvh_leaves,
            "bvh_max_leaf": v.bvh_max_leaf,
            "bvh_sah_cost": v.bvh_sah_cost,
        }

    def device_layout(self, part: str) -> np.ndarray:
        """One part of the device layout this scene gets at upload, computed on
        the host (no GPU); records as rows of raw words."""
        code, dtype, width = LAYOUT_PARTS[part]
        n = lib().rtg_host_scene_layout(self._h, code, None, 0)
        if n < 0:
            raise RtgError(int(n), f"no host layout for part {part}")
        out = np.zeros(n // 4, dtype=dtype)
        lib().rtg_host_scene_layout(self._h, code, out.ctypes.data_as(C.c_void_p), n)
        return out.reshape(-1, width)


COMPILE_DEFER_BVH = 1
COMPILE_AUTO_BVH = 2
# Parts of a scene's device layout (rtg_scene_layout): name -> (part, dtype, record width).
LAYOUT_PARTS = {
    "nodes": (0, np.float32, 16), "nodes4": (1, np.float32, 32), "prims": (2, np.float32, 12),
    "slot_material": (3, np.uint32, 1), "slot_normals": (4, np.float32, 12), "planes": (5, np.float32, 8),
    "materials": (6, np.float32, 16), "lights": (7, np.float32, 20), "slot_prim": (8, np.uint32, 1),
    "roots": (9, np.int32, 5), "nodes8": (10, np.uint32, 20),
}


def parse_scene(scene_json: str, base_dir: Optional[str] = None, defer_bvh=False) -> HostScene:
    """Parse + validate + compile a scene (raises SceneError with the field path).

    defer_bvh=True skips the host BVH build: uploading the scene builds it (on the
    GPU from 32,768 primitives up). defer_bvh="auto" builds small scenes' trees here
    and defers only large ones."""
    h = C.c_void_p()
    err = C.create_string_buffer(1024)
    flags = COMPILE_AUTO_BVH if defer_bvh == "auto" else (COMPILE_DEFER_BVH if defer_bvh else 0)
    rc = lib().rtg_compile_flags(scene_json.encode(), base_dir.encode() if base_dir else None,
                                 flags, C.byref(h), err, 1024)
    if rc != RTG_OK:
        raise SceneError(err.value.decode())
    return HostScene(h.value)


def load_scene(path: str) -> HostScene:
    with open(path, "r", encoding="utf-8") as f:
        text = f.read()
    return parse_scene(text, os.path.dirname(os.path.abspath(path)))


# ---------------------------------------------------------------------------
# GPU context

def device_count() -> int:
    return lib().rtg_device_count()


def allocation_count() -> int:
    """Memory allocations (device, pooled, pinned host) the library has asked
    CUDA for in this process so far."""
    return int(lib().rtg_allocation_count())


class Context:
    """One CUDA stream on one device; owns resident scenes and the wavefront pool."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        rc = lib().rtg_context_create(device, C.byref(h))
        if rc != RTG_OK:
            raise RtgError(rc, "no usable CUDA device" if rc == RTG_ERR_NO_DEVICE else "context creation failed")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().rtg_context_destroy(self._h)
            self._h = None

    def __del__(self):
        if _lib is not None:
            self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int):
        if rc != RTG_OK:
            msg = lib().rtg_last_error(self._h).decode()
            if rc == RTG_ERR_SCENE:
                raise SceneError(msg)
            raise RtgError(rc, msg)

    # scenes
    def upload(self, scene: HostScene) -> int:
        sid = C.c_int32()
        self._check(lib().rtg_scene_upload(self._h, scene.handle, C.byref(sid)))
        return sid.value

    def upload_gpu_bvh(self, scene: HostScene) -> int:
        """Uploads a host scene with its BVH built on the GPU (the same tree as the host build)."""
        sid = C.c_int32()
        self._check(lib().rtg_scene_upload_gpu_bvh(self._h, scene.handle, C.byref(sid)))
        return sid.value

    def scene_layout(self, scene_id: int, part: str) -> np.ndarray:
        """One part of a scene's device layout, read back (records as rows; raw words)."""
        code, dtype, width = LAYOUT_PARTS[part]
        n = lib().rtg_scene_layout(self._h, scene_id, code, None, 0)
        if n < 0:
            self._check(int(n))
        out = np.zeros(n // 4, dtype=dtype)
        got = lib().rtg_scene_layout(self._h, scene_id, code, out.ctypes.data_as(C.c_void_p), n)
        if got < 0:
            self._check(int(got))
        return out.reshape(-1, width)

    def upload_many(self, scenes: list[HostScene]) -> list[int]:
        """Uploads several host scenes at once (flattened in parallel)."""
        n = len(scenes)
        handles = (C.c_void_p * n)(*[s.handle for s in scenes])
        ids = (C.c_int32 * n)()
        self._check(lib().rtg_scene_upload_batch(self._h, n, handles, ids))
        return list(ids)

    def load_json(self, scene_json: str, base_dir: Optional[str] = None) -> int:
        sid = C.c_int32()
        self._check(lib().rtg_scene_load_json(self._h, scene_json.encode(),
                                              base_dir.encode() if base_dir else None, C.byref(sid)))
        return sid.value

    def release(self, scene_id: int):
        self._check(lib().rtg_scene_release(self._h, scene_id))

    def scene_settings(self, scene_id: int) -> RenderSettings:
        s = _Settings()
        self._check(lib().rtg_scene_settings(self._h, scene_id, C.byref(s)))
        return RenderSettings.from_c(s)

    def scene_info(self, scene_id: int) -> dict:
        i = _SceneInfo()
        self._check(lib().rtg_scene_get_info(self._h, scene_id, C.byref(i)))
        return {name: getattr(i, name) for name, _ in _SceneInfo._fields_}

    # tuning
    def tuning(self) -> dict:
        t = _Tuning()
        self._check(lib().rtg_get_tuning(self._h, C.byref(t)))
        return {name: getattr(t, name) for name, _ in _Tuning._fields_}

    def set_tuning(self, **kw):
        t = _Tuning()
        self._check(lib().rtg_get_tuning(self._h, C.byref(t)))
        for k, v in kw.items():
            setattr(t, k, v)
        self._check(lib().rtg_set_tuning(self._h, C.byref(t)))

    # rendering
    def render(self, scene_id: int, settings: Optional[RenderSettings] = None,
               options: Optional[RenderOptions] = None,
               on_pass: Optional[Callable[[RenderProgress], None]] = None,
               cancel: Optional[C.c_int32] = None) -> RenderProgress:
        s = settings.to_c() if settings else None
        o = _Options(int(options.progressive), options.max_pass_spp) if options else None
        cb = PASS_FN(lambda user, p: on_pass(RenderProgress.from_c(p.contents))) if on_pass else PASS_FN()
        out = _Progress()
        self._check(lib().rtg_render(self._h, scene_id, C.byref(s) if s else None, C.byref(o) if o else None, cb,
                                     None, C.byref(cancel) if cancel is not None else None, C.byref(out)))
        return RenderProgress.from_c(out)

    def render_batch(self, scene_ids: list[int], settings: list[RenderSettings],
                     options: Optional[RenderOptions] = None,
                     cancel: Optional[C.c_int32] = None) -> list[RenderProgress]:
        n = len(scene_ids)
        ids = (C.c_int32 * n)(*scene_ids)
        ss = (_Settings * n)(*[s.to_c() for s in settings])
        o = _Options(int(options.progressive), options.max_pass_spp) if options else None
        out = (_Progress * n)()
        self._check(lib().rtg_render_batch(self._h, n, ids, ss, C.byref(o) if o else None,
                                           C.byref(cancel) if cancel is not None else None, out))
        return [RenderProgress.from_c(out[j]) for j in range(n)]

    def _frame_size(self, job: int, width: int, height: int):
        return width, height

    def framebuffer_mean(self, job: int, width: int, height: int) -> np.ndarray:
        out = np.zeros((height, width, 3), dtype=np.float64)
        self._check(lib().rtg_framebuffer_mean(self._h, job, _ptr(out, C.c_double)))
        return out

    def framebuffer_moments(self, job: int, width: int, height: int):
        s = np.zeros((height, width, 4), dtype=np.float64)
        q = np.zeros((height, width, 4), dtype=np.float64)
        n = np.zeros((height, width), dtype=np.uint32)
        self._check(lib().rtg_framebuffer_moments(self._h, job, _ptr(s, C.c_double), _ptr(q, C.c_double),
                                                  _ptr(n, C.c_uint32)))
        return s[..., :3], q[..., :3], n

    def image(self, job: int, width: int, height: int, tone_map: Optional[str] = None,
              exposure: float = 1.0) -> np.ndarray:
        out = np.zeros((height, width, 3), dtype=np.uint8)
        op = -1 if tone_map is None else TONE_MAPS[tone_map]
        self._check(lib().rtg_image_rgb8(self._h, job, op, exposure, _ptr(out, C.c_uint8)))
        return out

    def images(self, jobs: Sequence[int], sizes: Sequence[tuple], tone_map: Optional[str] = None,
               exposure: float = 1.0) -> list:
        """image() of several jobs at once (one device-to-host transfer): sizes[k] is
        (width, height) of jobs[k]. The images are views into one allocation, which
        the library fills in one pass (many small arrays each fault in their own
        fresh pages: 9.1 against 5.6 ms for the 64 images of the mix)."""
        nbytes = [w * h * 3 for w, h in sizes]
        base = np.empty(sum(nbytes), dtype=np.uint8)
        outs, at = [], 0
        for (w, h), b in zip(sizes, nbytes):
            outs.append(base[at:at + b].reshape(h, w, 3))
            at += b
        n = len(outs)
        js = (C.c_int32 * n)(*[int(j) for j in jobs])
        ptrs = (C.POINTER(C.c_uint8) * n)(*[_ptr(o, C.c_uint8) for o in outs])
        op = -1 if tone_map is None else TONE_MAPS[tone_map]
        self._check(lib().rtg_images_rgb8(self._h, n, js, op, exposure, ptrs))
        return outs

    def stats(self) -> dict:
        s = _Stats()
        self._check(lib().rtg_render_stats(self._h, C.byref(s)))
        return {name: getattr(s, name) for name, _ in _Stats._fields_}

    # ray queries
    def trace_closest(self, scene_id: int, rays: np.ndarray, brute: bool = False):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = rays.shape[0]
        t = np.zeros(n, np.float32)
        prim = np.zeros(n, np.int32)
        plane = np.zeros(n, np.int32)
        bary = np.zeros((n, 2), np.float32)
        self._check(lib().rtg_trace_closest(self._h, scene_id, _ptr(rays, C.c_float), n, int(brute),
                                            _ptr(t, C.c_float), _ptr(prim, C.c_int32), _ptr(plane, C.c_int32),
                                            _ptr(bary, C.c_float)))
        return t, prim, plane, bary

    def probe_read_bandwidth(self, nbytes: int, reps: int = 8, l1: bool = False) -> float:
        """Read bandwidth (GB/s) over a buffer of nbytes on this context's GPU:
        L2 when nbytes is well under the L2 size, HBM when far above it; with l1,
        every block reads its own copy of a small buffer (aggregate L1)."""
        g = C.c_double()
        self._check(lib().rtg_probe_read_bandwidth(self._h, int(nbytes), int(reps), int(bool(l1)), C.byref(g)))
        return g.value

    def trace_closest_noalloc(self, scene_id: int, rays: np.ndarray, brute: bool = False):
        """trace_closest through the entry point that allocates no device memory
        (at most NOALLOC_MAX_RAYS rays per call)."""
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = rays.shape[0]
        t = np.zeros(n, np.float32)
        prim = np.zeros(n, np.int32)
        plane = np.zeros(n, np.int32)
        bary = np.zeros((n, 2), np.float32)
        self._check(lib().rtg_trace_closest_noalloc(self._h, scene_id, _ptr(rays, C.c_float), n, int(brute),
                                                    _ptr(t, C.c_float), _ptr(prim, C.c_int32),
                                                    _ptr(plane, C.c_int32), _ptr(bary, C.c_float)))
        return t, prim, plane, bary

    def trace_any(self, scene_id: int, rays: np.ndarray, brute: bool = False) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = rays.shape[0]
        occ = np.zeros(n, np.uint8)
        self._check(lib().rtg_trace_any(self._h, scene_id, _ptr(rays, C.c_float), n, int(brute), _ptr(occ, C.c_uint8)))
        return occ

    def autotune(self, scene_ids: list[int], settings: Optional[list[RenderSettings]] = None,
                 options: Optional[RenderOptions] = None, use_cache: bool = True) -> dict:
        """Picks pool size and block size for this batch and applies them."""
        n = len(scene_ids)
        ids = (C.c_int32 * n)(*scene_ids)
        ss = (_Settings * n)(*[s.to_c() for s in settings]) if settings else None
        o = _Options(int(options.progressive), options.max_pass_spp) if options else None
        t = _Tuning()
        rate = C.c_double()
        cached = C.c_int32()
        self._check(lib().rtg_autotune(self._h, n, ids, ss, C.byref(o) if o else None, int(use_cache), C.byref(t),
                                       C.byref(rate), C.byref(cached)))
        return {"pool_paths": t.pool_paths, "block": t.block, "probe_msamples_per_s": rate.value,
                "from_cache": bool(cached.value)}

    # serving
    def submit(self, scene_id: int, settings: Optional[RenderSettings] = None,
               options: Optional[RenderOptions] = None, priority: int = 0) -> Optional[int]:
        """Opens a request; None when admission by footprint turns it away."""
        s = settings.to_c() if settings else None
        o = _Options(int(options.progressive), options.max_pass_spp) if options else None
        rid = C.c_int32()
        rc = lib().rtg_request_submit(self._h, scene_id, C.byref(s) if s else None, C.byref(o) if o else None,
                                      priority, C.byref(rid))
        if rc == RTG_ERR_LIMIT:
            return None
        self._check(rc)
        return rid.value

    def pump(self, budget_ms: float, return_on_event: bool = False, cap: int = 256) -> list[tuple[int, RenderProgress]]:
        ev = (_RequestEvent * cap)()
        n = C.c_int32()
        self._check(lib().rtg_serve_pump(self._h, budget_ms, int(return_on_event), ev, cap, C.byref(n)))
        return [(ev[k].request, RenderProgress.from_c(ev[k].progress)) for k in range(n.value)]

    def cancel_request(self, rid: int):
        self._check(lib().rtg_request_cancel(self._h, rid))

    def release_request(self, rid: int):
        self._check(lib().rtg_request_release(self._h, rid))

    def request_progress(self, rid: int) -> RenderProgress:
        p = _Progress()
        self._check(lib().rtg_request_progress(self._h, rid, C.byref(p)))
        return RenderProgress.from_c(p)

    def request_mean(self, rid: int, width: int, height: int) -> np.ndarray:
        out = np.zeros((height, width, 3), dtype=np.float64)
        self._check(lib().rtg_request_mean(self._h, rid, _ptr(out, C.c_double)))
        return out

    def request_image(self, rid: int, width: int, height: int, tone_map: Optional[str] = None,
                      exposure: float = 1.0) -> np.ndarray:
        out = np.zeros((height, width, 3), dtype=np.uint8)
        op = -1 if tone_map is None else TONE_MAPS[tone_map]
        self._check(lib().rtg_request_image_rgb8(self._h, rid, op, exposure, _ptr(out, C.c_uint8)))
        return out

    def serve_prepare(self):
        """Maps the admission budget into the device pool up front."""
        self._check(lib().rtg_serve_prepare(self._h))

    def serve_footprint(self) -> tuple[int, int, int]:
        """(device bytes held against the admission budget, open requests, requests still rendering)."""
        b = C.c_uint64()
        n = C.c_int32()
        r = C.c_int32()
        self._check(lib().rtg_serve_footprint(self._h, C.byref(b), C.byref(n), C.byref(r)))
        return b.value, n.value, r.value


class Renderer:
    """The reference Renderer's shape (src/rendering/renderer.cpp:11-110) on one GPU scene."""

    def __init__(self, ctx: Context, scene_id: int, settings: Optional[RenderSettings] = None,
                 options: Optional[RenderOptions] = None):
        self.ctx = ctx
        self.scene_id = scene_id
        self.settings = settings or ctx.scene_settings(scene_id)
        self.options = options or RenderOptions()

    def render(self, on_pass: Optional[Callable[[RenderProgress], None]] = None,
               cancel: Optional[C.c_int32] = None) -> RenderProgress:
        return self.ctx.render(self.scene_id, self.settings, self.options, on_pass, cancel)

    def framebuffer_mean(self) -> np.ndarray:
        return self.ctx.framebuffer_mean(-1, self.settings.width, self.settings.height)

    def moments(self):
        return self.ctx.framebuffer_moments(-1, self.settings.width, self.settings.height)

    def image(self) -> np.ndarray:
        return self.ctx.image(-1, self.settings.width, self.settings.height)

    def stats(self) -> dict:
        return self.ctx.stats()


def encode_png(rgb: np.ndarray) -> bytes:
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    h, w = rgb.shape[:2]
    n = lib().rtg_encode_png(_ptr(rgb, C.c_uint8), w, h, None, 0)
    if n < 0:
        raise RtgError(int(n), "PNG encoding failed")
    out = np.zeros(n, np.uint8)
    lib().rtg_encode_png(_ptr(rgb, C.c_uint8), w, h, _ptr(out, C.c_uint8), n)
    return out.tobytes()
