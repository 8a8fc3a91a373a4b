"""BVH build on the GPU (rtg_scene_upload_gpu_bvh) against the host build.

The host build reproduces the reference's Bvh::build node for node
(tests/test_compile.py pins it with SHA-256 digests of the reference's own trees),
and flatten() derives the device layout from it. The GPU build must give the same
layout byte for byte: binary nodes, four-wide nodes, primitive slots, slot ->
primitive map and roots. The scenes cover the benchmark workloads, the batched
mix and the builder's edge cases: a single primitive, roots on either side of
the 32-primitive threshold between the level passes and the warp-built
subtrees, leaves kept by the SAH cost rule, coinciding centroids (middle
splits), the depth cap of 60, flat axis-aligned triangles, planes only, and
triangle soups.
"""
import json

import numpy as np
import pytest

import rtg
import workloads

pytestmark = pytest.mark.gpu

PARTS = ["nodes", "nodes4", "nodes8", "prims", "slot_material", "slot_normals", "planes", "materials", "lights",
         "slot_prim"]


def _scene(objects, planes=()):
    return {
        "camera": {"look_from": [0, 2, 12], "look_at": [0, 0, 0], "vfov": 40},
        "render": {"width": 48, "height": 48, "spp": 8, "max_depth": 6, "seed": 5},
        "materials": {"m": {"type": "lambertian", "albedo": [0.6, 0.5, 0.4]},
                      "lamp": {"type": "emissive", "color": [1, 1, 1], "intensity": 4}},
        "objects": list(planes) + list(objects),
        "lights": [{"type": "point", "position": [0, 6, 4], "intensity": [20, 20, 20]}],
    }


def _spheres(centres, radii=0.3, material="m"):
    radii = np.broadcast_to(np.asarray(radii, dtype=float), (len(centres),))
    return [{"type": "sphere", "center": [float(x) for x in c], "radius": float(r), "material": material}
            for c, r in zip(centres, radii)]


def _soup(n, seed, spread=4.0, size=0.3):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-spread, spread, (n, 3))
    b = a + rng.normal(0, size, (n, 3))
    c = a + rng.normal(0, size, (n, 3))
    return [{"type": "triangle", "v0": a[i].tolist(), "v1": b[i].tolist(), "v2": c[i].tolist(), "material": "m"}
            for i in range(n)]


def _flat_quads(n):
    # Axis-aligned quads: their triangles' boxes are flat, padded by the compile.
    out = []
    for i in range(n):
        x, z = float(i % 12) - 6, float(i // 12) - 6
        out.append({"type": "quad", "corner": [x, (i % 3) * 0.5, z], "u": [0.8, 0, 0], "v": [0, 0, 0.8],
                    "material": "m"})
    return out


def _chains(per_axis, cluster, rng):
    # Three chains of spheres along x, y and z at ratio 32 (so that a node's
    # largest coordinate is alone in the last bin and every other centroid falls
    # in the first), plus a cluster near the origin: every split peels one chain
    # sphere off, which drives the tree to the depth cap of 60.
    out = []
    for axis, scale in ((0, 1.0), (1, 2.0), (2, 4.0)):
        for k in range(1, per_axis + 1):
            p = [0.0, 0.0, 0.0]
            p[axis] = scale * 32.0 ** k
            out.append(p)
    return out + rng.uniform(0, 1, (cluster, 3)).tolist()


_rng = np.random.default_rng(99)
EDGE = {
    "one_sphere": _scene(_spheres([[0, 0, 0]])),
    "five_spheres": _scene(_spheres(np.arange(5)[:, None] * [1.0, 0.0, 0.0])),
    "sixteen_overlapping": _scene(_spheres(_rng.uniform(-0.01, 0.01, (16, 3)), radii=2.0)),
    "thirty_two": _scene(_spheres(_rng.uniform(-3, 3, (32, 3)))),
    "thirty_three": _scene(_spheres(_rng.uniform(-3, 3, (33, 3)))),
    "same_centre": _scene(_spheres(np.zeros((100, 3)))),
    "same_centre_radii": _scene(_spheres(np.zeros((300, 3)), radii=np.linspace(0.1, 3.0, 300))),
    "depth_cap_level_pass": _scene(_spheres(_chains(25, 40, _rng), radii=0.1)),
    "depth_cap_warp": _scene(_spheres(_chains(25, 10, _rng), radii=0.1)),
    "flat_quads": _scene(_flat_quads(144)),
    "planes_only": _scene([], planes=[{"type": "plane", "point": [0, -1, 0], "normal": [0, 1, 0], "material": "m"}]),
    "emitters_and_planes": _scene(
        _spheres(_rng.uniform(-4, 4, (200, 3)), radii=0.2) + _spheres([[0, 3, 0]], radii=0.5, material="lamp")
        + _soup(500, 3),
        planes=[{"type": "plane", "point": [0, -2, 0], "normal": [0, 1, 0], "material": "m"}]),
    "soup_10k": _scene(_soup(10_000, 1)),
    "soup_60k_clustered": _scene(_soup(60_000, 2, spread=1.0, size=0.05)),
}


def _compare(ctx, host):
    a = ctx.upload(host)
    b = ctx.upload_gpu_bvh(host)
    try:
        ra, rb = ctx.scene_layout(a, "roots")[0], ctx.scene_layout(b, "roots")[0]
        assert ra[3] == 0 and rb[3] == 1
        assert ra[:3].tolist() == rb[:3].tolist() and ra[4] == rb[4]
        for part in PARTS:
            x, y = ctx.scene_layout(a, part), ctx.scene_layout(b, part)
            assert x.shape == y.shape, (part, x.shape, y.shape)
            if x.tobytes() != y.tobytes():
                bad = np.flatnonzero((x.view(np.uint32) != y.view(np.uint32)).any(axis=1))
                raise AssertionError(f"{part}: {bad.size} of {len(x)} records differ, first {bad[:5].tolist()}")
        ia, ib = ctx.scene_info(a), ctx.scene_info(b)
        for k in ("bvh_nodes", "bvh_leaves", "bvh_max_depth", "bvh_max_leaf"):
            assert ia[k] == ib[k], (k, ia[k], ib[k])
        return ia, ib
    finally:
        ctx.release(a)
        ctx.release(b)


@pytest.mark.parametrize("name", list(EDGE))
def test_edge_case_layout_matches_host_build(ctx, name):
    _compare(ctx, rtg.parse_scene(json.dumps(EDGE[name])))


@pytest.mark.parametrize("name", ["cornell", "spheres", "mesh"])
def test_benchmark_scene_layout_matches_host_build(ctx, name):
    make = {"cornell": workloads.cornell, "spheres": workloads.sphere_field, "mesh": workloads.mesh_stress}[name]
    ia, ib = _compare(ctx, rtg.parse_scene(json.dumps(make())))
    print(f"{name}: {ia['bvh_nodes']} nodes, depth {ia['bvh_max_depth']}: host build {ia['bvh_build_ms']:.1f} ms, "
          f"GPU build {ib['bvh_build_ms']:.2f} ms")


def test_batched_mix_layouts_match_host_build(ctx):
    for k, sc in enumerate(workloads.batch_mix()):
        try:
            _compare(ctx, rtg.parse_scene(json.dumps(sc)))
        except AssertionError as e:
            raise AssertionError(f"mix scene {k}: {e}") from e


@pytest.mark.parametrize("defer", [True, "auto"])
@pytest.mark.parametrize("make,gpu", [(workloads.mesh_stress, True), (workloads.cornell, False)])
def test_deferred_compile_builds_at_upload(ctx, make, gpu, defer):
    """A scene compiled without its BVH gets it at plain upload: built on the GPU
    from 32,768 primitives up (the mesh, 174k), on the host below (Cornell, 36),
    with the same layout as the scene compiled with its tree either way. The
    automatic mode builds small trees in the compile instead."""
    text = json.dumps(make())
    deferred = rtg.parse_scene(text, defer_bvh=defer)
    assert (len(deferred.view()["nodes"]) == 0) == (defer is True or gpu)
    a = ctx.upload(rtg.parse_scene(text))
    b = ctx.upload(deferred)
    try:
        assert ctx.scene_layout(b, "roots")[0][3] == int(gpu)
        for part in PARTS:
            assert ctx.scene_layout(a, part).tobytes() == ctx.scene_layout(b, part).tobytes(), part
    finally:
        ctx.release(a)
        ctx.release(b)


def test_gpu_built_scene_renders_identically(ctx):
    """Same layout, so the same image: framebuffers are bit-identical."""
    host = rtg.parse_scene(json.dumps(workloads.cornell(width=64, height=64, spp=16)))
    a, b = ctx.upload(host), ctx.upload_gpu_bvh(host)
    try:
        for part in PARTS:
            assert ctx.scene_layout(a, part).tobytes() == ctx.scene_layout(b, part).tobytes(), part
        means = []
        for sid in (a, b):
            ctx.render(sid)
            means.append(ctx.framebuffer_mean(-1, 64, 64))
        assert np.array_equal(means[0], means[1])
    finally:
        ctx.release(a)
        ctx.release(b)


def test_ray_queries_on_a_gpu_built_scene(ctx):
    """The ray API maps slots back to primitive ids through the slot map the GPU
    build read back: closest and any hits on the GPU-built mesh equal the
    host-built scene's, ray for ray."""
    host = rtg.parse_scene(json.dumps(workloads.mesh_stress()))
    rays = workloads.random_rays(host.view(), 100_000, seed=5)
    a, b = ctx.upload(host), ctx.upload_gpu_bvh(host)
    try:
        ra, rb = ctx.trace_closest(a, rays), ctx.trace_closest(b, rays)
        for x, y in zip(ra, rb):
            assert np.array_equal(x, y)
        assert np.array_equal(ctx.trace_any(a, rays), ctx.trace_any(b, rays))
        assert (ra[1] >= 0).mean() > 0.05
    finally:
        ctx.release(a)
        ctx.release(b)


@pytest.mark.parametrize("name", ["mesh", "spheres", "depth_cap_level_pass", "emitters_and_planes"])
def test_eight_wide_layout_matches_host_build(ctx, name):
    """With an eight-wide walk selected, both builds also make the eight-wide tree
    and move the slots to its order: still byte-identical, eight-wide nodes included."""
    scene = {"mesh": workloads.mesh_stress, "spheres": workloads.sphere_field}.get(name)
    host = rtg.parse_scene(json.dumps(scene() if scene else EDGE[name]))
    ctx.set_tuning(closest_tree=8, shadow_tree=8)
    try:
        ia, _ = _compare(ctx, host)
    finally:
        ctx.set_tuning(closest_tree=2, shadow_tree=4)
