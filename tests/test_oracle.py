"""Pins the oracle (the C restatement in oracle/rtoracle.c) to the reference:
bit-identical RNG streams, camera rays, tone mapping, ray queries and rendered
framebuffer sums against fixtures the reference produced (tests/golden/)."""
import json
import os

import numpy as np
import pytest

import rtg
import rtoracle
import workloads
from conftest import GOLDEN

CONFIGS = {"cornell": workloads.cornell, "spheres": workloads.sphere_field, "mesh": workloads.mesh_stress}


def _load(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.fixture(scope="module")
def views():
    return {k: rtg.parse_scene(json.dumps(f())).view() for k, f in CONFIGS.items()}


def test_rng_streams_bit_identical():
    g = _load("rng.npz")
    for (seed, pixel, sample), ref in zip(g["cases"], g["streams"]):
        assert np.array_equal(rtoracle.rng_stream(int(seed), int(pixel), int(sample), 64), ref)


@pytest.mark.parametrize("cfg", list(CONFIGS))
def test_camera_rays_bit_identical(cfg, views):
    g = _load(f"camera_{cfg}.npz")
    o = rtoracle.OracleScene(views[cfg])
    out = o.camera(g["pix"], int(g["pixel_for_rng"]))
    assert out.tobytes() == g["rays"].tobytes()


def test_tone_map_bit_identical():
    g = _load("tonemap.npz")
    vals = g["values"]
    rgb = np.stack([vals, vals * 0.5, -vals], 1)
    for op in range(3):
        for e, ex in enumerate(g["exposures"]):
            out = rtoracle.tone_map_srgb8(rgb, op, float(ex))
            assert np.array_equal(out, g["srgb8"][:, op, e, :]), (op, ex)


def test_tone_map_known_answers():
    one = lambda v: rtoracle.tone_map_srgb8(np.array([[v, v, v]]), 0, 1.0)[0, 0]  # noqa: E731
    assert one(0) == 0 and one(1) == 255 and one(0.5) == 188 and one(-1) == 0 and one(10) == 255
    assert rtoracle.tone_map_srgb8(np.array([[np.nan, 1, 1]]), 2, 1.0).tolist() == [[0, 0, 0]]


@pytest.mark.parametrize("cfg", list(CONFIGS))
def test_ray_queries_bit_identical(cfg, views):
    g = _load(f"rays_{cfg}.npz")
    o = rtoracle.OracleScene(views[cfg])
    rays = g["rays"].astype(np.float64)
    t, prim, plane, _ = o.closest_parallel(rays)
    assert np.array_equal(prim, g["prim"]) and np.array_equal(plane, g["is_plane"].astype(np.int32))
    assert t.tobytes() == np.where(g["hit"] == 1, g["t"], 0.0).tobytes()
    tb, pb, plb, _ = o.closest_parallel(rays, brute=True)
    assert np.array_equal(pb, g["brute_prim"]) and tb.tobytes() == np.where(g["brute_hit"] == 1, g["brute_t"], 0.0).tobytes()
    for k, tmax in enumerate(g["occluded_tmax"]):
        r = rays.copy()
        r[:, 3] = 1e-6
        r[:, 7] = tmax
        assert np.array_equal(o.occluded(r), g["occluded"][:, k].astype(np.uint8)), tmax


def test_bvh_agrees_with_brute_force_up_to_exact_ties(views):
    """The reference's own check (BVH == brute on t; ids differ only on exact ties
    such as coplanar faces)."""
    for cfg in CONFIGS:
        g = _load(f"rays_{cfg}.npz")
        assert np.array_equal(g["hit"], g["brute_hit"])
        assert np.array_equal(g["t"], g["brute_t"])


@pytest.mark.parametrize("name", ["cornell_path", "cornell_direct", "cornell_normals", "cornell_bsdf_only",
                                  "spheres_path", "spheres_brute", "mesh_path"])
def test_render_sums_bit_identical(name):
    g = _load(f"render_{name}.npz")
    scene = json.loads(str(g["scene"]))
    args = []
    if name.endswith("direct"):
        scene["render"]["integrator"] = "direct"
    if name.endswith("normals"):
        scene["render"]["integrator"] = "normals"
    if name.endswith("bsdf_only"):
        scene["render"]["light_sampling"] = False
    o = rtoracle.OracleScene(rtg.parse_scene(json.dumps(scene)).view())
    s, q, st = o.render()
    assert s.tobytes() == g["sum"].tobytes()
    assert q.tobytes() == g["sumsq"].tobytes()
    ref = json.loads(str(g["stats"]))
    assert st["rays"] == ref["rays"] and st["shadow_rays"] == ref["shadow_rays"]
    assert st["invalid_samples"] == ref["invalid_samples"] == 0


def test_oracle_invalid_sample_rule_plants_a_nan():
    """A planted NaN emitter makes every sample non-finite: all are counted invalid
    and the framebuffer stays black and finite (Renderer::render_tile's rule)."""
    scene = {"render": {"width": 4, "height": 4, "spp": 2},
             "camera": {"look_from": [0, 0, 3], "look_at": [0, 0, 0]},
             "background": {"type": "solid", "color": [0, 0, 0]},
             "materials": {"e": {"type": "emissive", "intensity": 1, "two_sided": True}},
             "objects": [{"type": "sphere", "center": [0, 0, 0], "radius": 10, "material": "e"}]}
    view = rtg.parse_scene(json.dumps(scene)).view()
    view["materials"][0, 10] = np.nan  # intensity -> NaN, in the oracle's copy only
    s, q, st = rtoracle.OracleScene(view).render()
    assert st["invalid_samples"] == 4 * 4 * 2
    assert np.isfinite(s).all() and (s == 0).all()
