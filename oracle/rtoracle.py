"""Oracle binding (test infrastructure only: imported by tests/, the smoke check
and bench.py's CPU-baseline leg, never by the product path).

Wraps oracle/librtoracle.so, the C restatement of the reference renderer's
algorithm (rtoracle.c). Scenes come in the reference's layout as the dict
returned by rtg.HostScene.view(). If the shared object is missing it is built
from rtoracle.c with gcc (present on every box of this image).
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "librtoracle.so")


class _Scene(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "n_prims", "n_planes", "n_nodes", "n_order", "n_lights", "n_point_lights", "n_materials")] + [
        ("prims", C.c_void_p), ("planes", C.c_void_p), ("nodes", C.c_void_p), ("order", C.c_void_p),
        ("lights", C.c_void_p), ("point_lights", C.c_void_p), ("materials", C.c_void_p),
        ("camera", C.c_double * 19), ("background", C.c_double * 8)] + [
        (n, C.c_int32) for n in ("width", "height", "spp", "max_depth", "rr_min_depth", "integrator",
                                 "light_sampling", "use_bvh")] + [("seed", C.c_uint64)]


_lib = None


def build() -> str:
    src = os.path.join(_HERE, "rtoracle.c")
    if (not os.path.exists(LIB)) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-std=c11", "-O2", "-fPIC", "-shared", "-fno-fast-math", "-ffp-contract=off",
                               src, "-o", LIB, "-lm"])
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.ro_rng.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, vp, C.c_int32]
        L.ro_closest.argtypes = [vp, vp, C.c_int64, C.c_int32, vp, vp, vp, vp]
        L.ro_occluded.argtypes = [vp, vp, C.c_int64, vp]
        L.ro_camera.argtypes = [vp, vp, C.c_int64, C.c_uint64, vp]
        L.ro_render_rows.argtypes = [vp, C.c_int32, C.c_int32, C.c_uint32, C.c_uint32, vp, vp, vp]
        L.ro_sample.argtypes = [vp, C.c_int32, C.c_int32, C.c_uint32, vp]
        L.ro_tone_map_srgb8.argtypes = [vp, C.c_int64, C.c_int32, C.c_double, vp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data if a.size else None


class OracleScene:
    """A compiled scene handed to the oracle (keeps its arrays alive)."""

    def __init__(self, view: dict, **overrides):
        self.arrays = {k: np.ascontiguousarray(view[k]) for k in
                       ("prims", "planes", "nodes", "order", "lights", "point_lights", "materials")}
        st = view["settings"]
        for k, v in overrides.items():
            setattr(st, k, v)
        self.settings = st
        s = _Scene()
        s.n_prims = len(self.arrays["prims"])
        s.n_planes = len(self.arrays["planes"])
        s.n_nodes = len(self.arrays["nodes"])
        s.n_order = len(self.arrays["order"])
        s.n_lights = len(self.arrays["lights"])
        s.n_point_lights = len(self.arrays["point_lights"])
        s.n_materials = len(self.arrays["materials"])
        for k in self.arrays:
            setattr(s, k, _p(self.arrays[k]))
        camera = np.array(view["camera"], dtype=np.float64)
        if "camera_override" in view:
            camera = view["camera_override"]
        s.camera[:] = list(camera)
        s.background[:] = list(view["background"])
        s.width, s.height, s.spp = st.width, st.height, st.spp
        s.max_depth, s.rr_min_depth = st.max_depth, st.rr_min_depth
        s.integrator = {"path": 0, "direct": 1, "normals": 2}[st.integrator]
        # 2: the MIS extension (the GPU's opt-in estimator), 1: the reference's NEE.
        s.light_sampling = (2 if getattr(st, "mis", False) else 1) if st.light_sampling else 0
        s.use_bvh = int(st.use_bvh)
        s.seed = st.seed
        self.c = s

    def ref(self):
        return C.byref(self.c)

    # queries
    def closest(self, rays: np.ndarray, brute: bool = False):
        rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 8)
        n = len(rays)
        t = np.zeros(n)
        prim = np.zeros(n, np.int32)
        plane = np.zeros(n, np.int32)
        gn = np.zeros((n, 3))
        lib().ro_closest(self.ref(), _p(rays), n, int(brute), _p(t), _p(prim), _p(plane), _p(gn))
        return t, prim, plane, gn

    def closest_parallel(self, rays: np.ndarray, brute: bool = False, workers: int | None = None):
        rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 8)
        workers = workers or os.cpu_count() or 1
        chunks = np.array_split(np.arange(len(rays)), workers * 4)
        outs = [None] * len(chunks)
        with cf.ThreadPoolExecutor(workers) as ex:
            futs = {ex.submit(self.closest, rays[c], brute): k for k, c in enumerate(chunks) if len(c)}
            for f in cf.as_completed(futs):
                outs[futs[f]] = f.result()
        parts = [o for o in outs if o is not None]
        return tuple(np.concatenate([p[i] for p in parts]) for i in range(4))

    def occluded(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 8)
        out = np.zeros(len(rays), np.uint8)
        lib().ro_occluded(self.ref(), _p(rays), len(rays), _p(out))
        return out

    def camera(self, pix: np.ndarray, pixel_for_rng: int = 0):
        pix = np.ascontiguousarray(pix, dtype=np.float64).reshape(-1, 4)
        out = np.zeros((len(pix), 6))
        lib().ro_camera(self.ref(), _p(pix), len(pix), pixel_for_rng, _p(out))
        return out

    def sample(self, x: int, y: int, s: int):
        out = np.zeros(3)
        lib().ro_sample(self.ref(), x, y, s, _p(out))
        return out

    def render(self, s0: int = 0, s1: int | None = None, workers: int | None = None):
        """Per-pixel (sum, sumsq) over samples [s0, s1), rows split across threads."""
        st = self.settings
        s1 = st.spp if s1 is None else s1
        W, H = st.width, st.height
        total = np.zeros((H, W, 3))
        sq = np.zeros((H, W, 3))
        stats = np.zeros(4, np.uint64)
        workers = workers or os.cpu_count() or 1
        bands = [(y, min(H, y + 1)) for y in range(0, H, 1)]

        def run(b):
            local = np.zeros(4, np.uint64)
            lib().ro_render_rows(self.ref(), b[0], b[1], s0, s1, _p(total), _p(sq), _p(local))
            return local

        with cf.ThreadPoolExecutor(workers) as ex:
            for local in ex.map(run, bands):
                stats += local
        return total, sq, {"rays": int(stats[0]), "shadow_rays": int(stats[1]), "rr_terminated": int(stats[2]),
                           "invalid_samples": int(stats[3])}


def rng_stream(seed: int, pixel: int, sample: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.uint32)
    lib().ro_rng(seed, pixel, sample, _p(out), n)
    return out


def tone_map_srgb8(rgb: np.ndarray, op: int, exposure: float) -> np.ndarray:
    rgb = np.ascontiguousarray(rgb, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(rgb.shape, np.uint8)
    lib().ro_tone_map_srgb8(_p(rgb), len(rgb), op, exposure, _p(out))
    return out
