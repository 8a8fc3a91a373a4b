"""Seeded synthetic workloads (scene JSON) for the benchmark and parity tests.

  cornell()       Cornell box, 555-unit room, 256x256, 64 spp, depth 8, path + NEE + RR, seed 1
  sphere_field()  ~480 r=0.2 spheres on a jittered 22x22 grid + 3 r=1 spheres, thin lens, 512x512x128, depth 16
  mesh_stress()   icosphere s=6 (81,920 tris) + 256x180 torus (92,160 tris), smooth normals, metal + glass,
                  emissive sphere + point light, floor + back wall, 1024x1024x64, depth 12
  batch_mix()     64 seeded scenes of uneven size/resolution/spp/depth (incl. facing mirrors)
  random_rays()   seeded fp32 rays over a scene's bounds (1% axis-parallel)

Scenes use the reference's JSON schema; the 256x180 torus needs the one schema
extension this renderer accepts ("segments_v").
"""
from __future__ import annotations

import json
import math

import numpy as np


def _quad(name, corner, u, v, mat):
    return {"type": "quad", "name": name, "corner": corner, "u": u, "v": v, "material": mat}


def cornell(width=256, height=256, spp=64, max_depth=8, seed=1) -> dict:
    S = 555.0
    return {
        "name": "Cornell box (555 units)",
        "camera": {"look_from": [278, 278, -800], "look_at": [278, 278, 0], "vfov": 40},
        "render": {"width": width, "height": height, "spp": spp, "max_depth": max_depth, "rr_min_depth": 3,
                   "integrator": "path", "light_sampling": True, "seed": seed, "tone_map": "clamp"},
        "background": {"type": "solid", "color": [0, 0, 0]},
        "materials": {
            "white": {"type": "lambertian", "albedo": [0.73, 0.73, 0.73]},
            "red": {"type": "lambertian", "albedo": [0.65, 0.05, 0.05]},
            "green": {"type": "lambertian", "albedo": [0.12, 0.45, 0.15]},
            "light": {"type": "emissive", "color": [1, 1, 1], "intensity": 15},
        },
        "objects": [
            _quad("green wall", [0, 0, 0], [0, 0, S], [0, S, 0], "green"),
            _quad("red wall", [S, 0, 0], [0, S, 0], [0, 0, S], "red"),
            _quad("floor", [0, 0, 0], [S, 0, 0], [0, 0, S], "white"),
            _quad("ceiling", [0, S, 0], [0, 0, S], [S, 0, 0], "white"),
            _quad("back wall", [0, 0, S], [S, 0, 0], [0, S, 0], "white"),
            _quad("ceiling light", [213, 554, 227], [130, 0, 0], [0, 0, 105], "light"),
            {"type": "box", "name": "tall block", "min": [265, 0, 295], "max": [430, 330, 460], "rotate_y": 15,
             "material": "white"},
            {"type": "box", "name": "short block", "min": [130, 0, 65], "max": [295, 165, 230], "rotate_y": -18,
             "material": "white"},
        ],
    }


def sphere_field(width=512, height=512, spp=128, max_depth=16, seed=7) -> dict:
    rng = np.random.default_rng(seed)
    mats = {
        "ground": {"type": "lambertian", "albedo": [0.5, 0.5, 0.5], "albedo2": [0.32, 0.36, 0.3],
                   "checker_scale": 0.5},
        "glass": {"type": "dielectric", "ior": 1.5},
        "big_diffuse": {"type": "lambertian", "albedo": [0.4, 0.2, 0.1]},
        "big_metal": {"type": "metal", "albedo": [0.7, 0.6, 0.5], "roughness": 0.0},
    }
    objs = [{"type": "plane", "name": "ground", "point": [0, 0, 0], "normal": [0, 1, 0], "material": "ground"}]
    big = [(0.0, 0.2, 0.0), (4.0, 0.2, 0.0), (-4.0, 0.2, 0.0)]
    k = 0
    for a in range(-11, 11):
        for b in range(-11, 11):
            choose = rng.random()
            jx, jz = rng.uniform(-0.35, 0.35, size=2)
            c = (a + float(jx), 0.2, b + float(jz))
            if any(math.dist(c, q) <= 0.9 for q in big):
                continue
            name = f"m{k}"
            k += 1
            if choose < 0.80:
                mats[name] = {"type": "lambertian", "albedo": [float(rng.random() * rng.random()) for _ in range(3)]}
            elif choose < 0.95:
                mats[name] = {"type": "metal", "albedo": [float(rng.uniform(0.5, 1.0)) for _ in range(3)],
                              "roughness": float(rng.uniform(0.0, 0.5))}
            else:
                name = "glass"
            objs.append({"type": "sphere", "name": f"sphere {k}", "center": list(c), "radius": 0.2,
                         "material": name})
    objs += [
        {"type": "sphere", "name": "big glass", "center": [0, 1, 0], "radius": 1.0, "material": "glass"},
        {"type": "sphere", "name": "big diffuse", "center": [-4, 1, 0], "radius": 1.0, "material": "big_diffuse"},
        {"type": "sphere", "name": "big metal", "center": [4, 1, 0], "radius": 1.0, "material": "big_metal"},
    ]
    return {
        "name": "Sphere field",
        "camera": {"look_from": [13, 2, 3], "look_at": [0, 0, 0], "vfov": 20, "aperture": 0.1, "focus_dist": 10},
        "render": {"width": width, "height": height, "spp": spp, "max_depth": max_depth, "rr_min_depth": 3,
                   "integrator": "path", "seed": 7, "tone_map": "aces"},
        "background": {"type": "gradient", "top": [0.5, 0.7, 1.0], "bottom": [1, 1, 1]},
        "materials": mats,
        "objects": objs,
    }


def mesh_stress(width=1024, height=1024, spp=64, max_depth=12, seed=3) -> dict:
    return {
        "name": "Triangle-mesh BVH stress",
        "camera": {"look_from": [0, 2.4, 7.5], "look_at": [0, 1.0, 0], "vfov": 40},
        "render": {"width": width, "height": height, "spp": spp, "max_depth": max_depth, "rr_min_depth": 3,
                   "integrator": "path", "seed": seed, "tone_map": "aces"},
        "background": {"type": "solid", "color": [0, 0, 0]},
        "materials": {
            "wall": {"type": "lambertian", "albedo": [0.7, 0.7, 0.68]},
            "rough_metal": {"type": "metal", "albedo": [0.95, 0.75, 0.35], "roughness": 0.2},
            "glass": {"type": "dielectric", "ior": 1.5, "tint": [0.95, 1.0, 0.95]},
            "lamp": {"type": "emissive", "color": [1.0, 0.9, 0.8], "intensity": 12},
        },
        "objects": [
            _quad("floor", [-6, 0, -6], [0, 0, 12], [12, 0, 0], "wall"),
            _quad("back wall", [-6, 0, -4], [12, 0, 0], [0, 8, 0], "wall"),
            {"type": "sphere", "name": "lamp", "center": [0.0, 3.4, 1.0], "radius": 0.5, "material": "lamp"},
            {"type": "mesh", "name": "icosphere", "source": "icosphere", "subdivisions": 6, "smooth": True,
             "scale": [1.2, 1.2, 1.2], "translate": [-1.6, 1.2, 0.0], "material": "rough_metal"},
            {"type": "mesh", "name": "torus", "source": "torus", "major_radius": 1.0, "minor_radius": 0.35,
             "segments": 256, "segments_v": 180, "smooth": True, "rotate_y": 20, "translate": [1.7, 0.35, 0.6],
             "material": "glass"},
        ],
        "lights": [{"type": "point", "name": "key", "position": [3, 6, 4], "intensity": [60, 60, 60]}],
    }


def random_rays(view: dict, n: int, seed: int = 11, axis_fraction: float = 0.01) -> np.ndarray:
    """n x 8 float32 rays (o, tmin, d, tmax): origins uniform over 1.5x the scene's
    bounds, directions uniform on the sphere, 1% axis-parallel."""
    rng = np.random.default_rng(seed)
    pts = []
    prims = view["prims"]
    if len(prims):
        sph = prims[prims[:, 0] == 0]
        tri = prims[prims[:, 0] == 1]
        if len(tri):
            pts.append(tri[:, 3:12].reshape(-1, 3))
        if len(sph):
            pts.append(sph[:, 3:6] + sph[:, 6:7])
            pts.append(sph[:, 3:6] - sph[:, 6:7])
    if len(view["planes"]):
        pts.append(view["planes"][:, 0:3])
    P = np.concatenate(pts) if pts else np.zeros((1, 3))
    lo, hi = P.min(0), P.max(0)
    c, h = 0.5 * (lo + hi), 0.75 * (hi - lo) + 1e-3
    o = rng.uniform(c - h, c + h, size=(n, 3))
    z = rng.uniform(-1, 1, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    r = np.sqrt(np.maximum(0, 1 - z * z))
    d = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    k = rng.random(n) < axis_fraction
    axis = rng.integers(0, 3, n)
    sign = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    ad = np.zeros((n, 3))
    ad[np.arange(n), axis] = sign
    d[k] = ad[k]
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 1e-6
    rays[:, 4:7] = d
    rays[:, 7] = np.float32(3.0e38)
    return rays


# ---------------------------------------------------------------------------
# Batched mix: 64 seeded scenes of uneven size.

RESOLUTIONS = [128, 256, 512, 1024]
SPPS = [16, 64, 256]


def _loguniform(rng, lo, hi):
    return float(np.exp(rng.uniform(np.log(lo), np.log(hi))))


def mix_scene(k: int, seed: int = 2024) -> dict:
    """Scene k of the batched mix (deterministic in (k, seed))."""
    rng = np.random.default_rng([seed, k])
    res = int(rng.choice(RESOLUTIONS))
    spp = int(rng.choice(SPPS))
    kind = int(rng.integers(0, 5))  # 0-1 spheres, 2-3 mesh, 4 facing mirrors
    mats = {
        "floor": {"type": "lambertian", "albedo": [0.6, 0.6, 0.6], "albedo2": [0.3, 0.32, 0.35],
                  "checker_scale": float(rng.uniform(0.3, 1.5))},
        "glass": {"type": "dielectric", "ior": 1.5},
        "mirror": {"type": "metal", "albedo": [0.95, 0.95, 0.95], "roughness": 0.0},
        "lamp": {"type": "emissive", "color": [1.0, 0.92, 0.85], "intensity": float(rng.uniform(4, 12))},
    }
    objs = [_quad("floor", [-8, 0, -8], [0, 0, 16], [16, 0, 0], "floor")]
    lights = []
    depth = int(rng.integers(8, 17))
    rr = 3
    if kind in (0, 1):
        n = int(round(_loguniform(rng, 10, 2000)))
        extent = max(2.0, math.sqrt(n) * 0.35)
        for i in range(n):
            name = f"s{i}"
            u = rng.random()
            if u < 0.7:
                mats[name] = {"type": "lambertian", "albedo": [float(x) for x in rng.random(3)]}
            elif u < 0.9:
                mats[name] = {"type": "metal", "albedo": [float(x) for x in rng.uniform(0.5, 1, 3)],
                              "roughness": float(rng.uniform(0, 0.5))}
            else:
                name = "glass"
            r = float(rng.uniform(0.1, 0.35))
            objs.append({"type": "sphere", "center": [float(rng.uniform(-extent, extent)), r,
                                                      float(rng.uniform(-extent, extent))],
                         "radius": r, "material": name})
        objs.append({"type": "sphere", "name": "lamp", "center": [0, extent + 2.0, 0], "radius": 1.0,
                     "material": "lamp"})
        cam = {"look_from": [extent * 1.3, extent * 0.8 + 1, extent * 1.3], "look_at": [0, 0.3, 0], "vfov": 45}
        bg = {"type": "gradient", "top": [0.5, 0.7, 1.0], "bottom": [1, 1, 1], "intensity": 0.6}
    elif kind in (2, 3):
        tris = _loguniform(rng, 1000, 200000)
        mats["body"] = {"type": "metal", "albedo": [0.9, 0.8, 0.6], "roughness": float(rng.uniform(0.05, 0.3))}
        mats["paint"] = {"type": "lambertian", "albedo": [float(x) for x in rng.uniform(0.2, 0.9, 3)]}
        if rng.random() < 0.4:
            sub = int(np.clip(round(math.log(tris / 20, 4)), 3, 6))
            mesh = {"type": "mesh", "source": "icosphere", "subdivisions": sub, "smooth": True,
                    "scale": [1.2, 1.2, 1.2], "translate": [0, 1.2, 0],
                    "material": str(rng.choice(["body", "paint", "glass"]))}
        else:
            seg = int(np.clip(round(math.sqrt(tris)), 8, 2048))
            mesh = {"type": "mesh", "source": "torus", "major_radius": 1.0, "minor_radius": 0.4,
                    "segments": seg, "smooth": True, "rotate_y": float(rng.uniform(0, 180)),
                    "translate": [0, 0.4, 0], "material": str(rng.choice(["body", "paint", "glass"]))}
        objs.append(mesh)
        objs.append({"type": "sphere", "name": "lamp", "center": [2.5, 3.5, 2.0], "radius": 0.5,
                     "material": "lamp"})
        lights.append({"type": "point", "position": [-3, 5, 3], "intensity": [30, 30, 30]})
        cam = {"look_from": [0, 2.5, 5.5], "look_at": [0, 0.8, 0], "vfov": 45}
        bg = {"type": "gradient", "top": [0.3, 0.4, 0.6], "bottom": [0.8, 0.8, 0.8], "intensity": 0.5}
    else:
        # Two facing mirrors (the reference's mirrors scene pattern): deep paths.
        depth, rr = 40, 30
        objs.append(_quad("mirror a", [-2, 0, -2], [4, 0, 0], [0, 3, 0], "mirror"))
        objs.append(_quad("mirror b", [-2, 0, 2], [0, 3, 0], [4, 0, 0], "mirror"))
        mats["orange"] = {"type": "lambertian", "albedo": [0.9, 0.5, 0.2]}
        objs.append({"type": "sphere", "center": [0, 0.5, 0], "radius": 0.5, "material": "orange"})
        objs.append({"type": "sphere", "name": "lamp", "center": [0, 2.6, 0], "radius": 0.3, "material": "lamp"})
        cam = {"look_from": [-1.2, 1.6, 1.6], "look_at": [0.6, 0.9, -1.2], "vfov": 55}
        bg = {"type": "solid", "color": [0.02, 0.02, 0.03]}
    return {
        "name": f"mix {k}",
        "camera": cam,
        "render": {"width": res, "height": res, "spp": spp, "max_depth": depth, "rr_min_depth": rr,
                   "integrator": "path", "seed": 1000 + k, "tone_map": "aces"},
        "background": bg,
        "materials": mats,
        "objects": objs,
        "lights": lights,
    }


def batch_mix(n: int = 64, seed: int = 2024) -> list[dict]:
    return [mix_scene(k, seed) for k in range(n)]


def to_json(scene: dict) -> str:
    return json.dumps(scene)
