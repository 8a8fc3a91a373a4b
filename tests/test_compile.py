"""Host compile (Scene::compile + binned-SAH BVH build) is bit-identical to the
reference's on the same scene: same primitive order (= hit ids), same light
list, same tree topology and leaf contents, same double-precision boxes."""
import hashlib
import json
import os

import numpy as np
import pytest

import rtg
import workloads
from conftest import GOLDEN

KEYS = ("prims", "planes", "nodes", "order", "lights", "materials", "point_lights")


def _fixture(cfg):
    return np.load(os.path.join(GOLDEN, f"compile_{cfg}.npz"))


@pytest.mark.parametrize("cfg,make", [("cornell", workloads.cornell), ("spheres", workloads.sphere_field)])
def test_compile_bit_identical(cfg, make):
    ref = _fixture(cfg)
    v = rtg.parse_scene(json.dumps(make())).view()
    for k in KEYS:
        a, b = v[k], ref[k]
        assert a.shape == b.shape, k
        assert a.tobytes() == b.tobytes(), k
    assert v["background"].tobytes() == ref["background"].tobytes()
    meta = json.loads(str(ref["meta"]))
    assert v["bvh_max_depth"] == meta["bvh_max_depth"]
    assert v["bvh_leaves"] == meta["bvh_leaves"]
    assert v["bvh_sah_cost"] == meta["bvh_sah_cost"]


def test_mesh_compile_digests_match():
    """174k-triangle scene (icosphere s=6 + 256x180 torus): every array's SHA-256."""
    ref = _fixture("mesh")
    v = rtg.parse_scene(json.dumps(workloads.mesh_stress())).view()
    for k in KEYS:
        a = np.ascontiguousarray(v[k])
        assert tuple(a.shape) == tuple(ref[f"shape_{k}"]), k
        assert hashlib.sha256(a.tobytes()).hexdigest() == str(ref[f"sha_{k}"]), k
    meta = json.loads(str(ref["meta"]))
    assert len(v["prims"]) == meta["primitives"] == 81920 + 92160 + 5


def test_bvh_invariants():
    """Every node encloses its children / primitives and every primitive is reachable once."""
    v = rtg.parse_scene(json.dumps(workloads.sphere_field())).view()
    nodes, order, prims = v["nodes"], v["order"], v["prims"]
    seen = np.zeros(len(prims), int)
    for i, n in enumerate(nodes):
        lo, hi, first, count = n[0:3], n[3:6], int(n[6]), int(n[7])
        if count:
            for p in order[first:first + count]:
                c, r = prims[p, 3:6], prims[p, 6]
                assert (c - r >= lo - 1e-9).all() and (c + r <= hi + 1e-9).all()
                seen[p] += 1
        else:
            assert first > i
            for child in (i + 1, first):
                assert (nodes[child, 0:3] >= lo - 1e-9).all() and (nodes[child, 3:6] <= hi + 1e-9).all()
    assert (seen == 1).all()


def test_bvh_edge_cases():
    mat = '"materials": {"m": {"type": "lambertian"}}'
    # Single primitive: one leaf node.
    v = rtg.parse_scene('{' + mat + ', "objects": [{"type": "sphere", "center": [0,0,0], "material": "m"}]}').view()
    assert len(v["nodes"]) == 1 and v["nodes"][0, 7] == 1
    # 1000 identical boxes: no SAH split possible -> count split, leaves <= 4.
    objs = ",".join('{"type": "sphere", "center": [0.5,0.5,0.5], "radius": 0.5, "material": "m"}' for _ in range(1000))
    v = rtg.parse_scene('{' + mat + ', "objects": [' + objs + ']}').view()
    assert v["bvh_max_leaf"] <= 4 and sorted(v["order"]) == list(range(1000))
    # Degenerate triangles are dropped at compile time.
    scene = ('{' + mat + ', "objects": [{"type": "triangle", "v0": [0,0,0], "v1": [1,0,0], "v2": [0,1,0], "material": "m"},'
             '{"type": "mesh", "source": "icosphere", "subdivisions": 5, "scale": [1, 1e-11, 1], "material": "m"}]}')
    v = rtg.parse_scene(scene).view()
    assert v["degenerate_skipped"] > 0


def test_procedural_meshes_are_closed_and_outward():
    mat = '"materials": {"m": {"type": "lambertian"}}'
    v = rtg.parse_scene('{' + mat + ', "objects": [{"type": "mesh", "source": "icosphere", "subdivisions": 2, '
                        '"smooth": false, "material": "m"}]}').view()
    tri = v["prims"][:, 3:12].reshape(-1, 3, 3)
    assert len(tri) == 20 * 16
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    assert (np.einsum("ij,ij->i", n, tri.mean(1)) > 0).all()
    assert np.allclose(np.linalg.norm(tri, axis=2), 1)
    v = rtg.parse_scene('{' + mat + ', "objects": [{"type": "mesh", "source": "torus", "major_radius": 1, '
                        '"minor_radius": 0.3, "segments": 24, "material": "m"}]}').view()
    assert len(v["prims"]) == 24 * 12 * 2
    tri = v["prims"][:, 3:12].reshape(-1, 3, 3)
    ns = v["prims"][:, 12:21].reshape(-1, 3, 3).sum(1)
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    assert (np.einsum("ij,ij->i", n, ns) > 0).all()


def test_reference_assets_round_trip_when_present():
    """Every shipped scene parses, validates, compiles and round-trips (reads the
    reference checkout only where it exists)."""
    d = os.path.join(os.environ.get("REF_DIR", "/root/reference"), "assets", "scenes")
    if not os.path.isdir(d):
        pytest.skip("reference checkout not present")
    count = 0
    for name in sorted(os.listdir(d)):
        if not name.endswith(".json"):
            continue
        text = open(os.path.join(d, name)).read()
        assert rtg.validate_scene(text) == "", name
        dumped = rtg.dump_scene(text)
        a = rtg.parse_scene(text).view()
        b = rtg.parse_scene(dumped).view()
        assert np.array_equal(a["prims"], b["prims"]) and np.array_equal(a["nodes"], b["nodes"]), name
        count += 1
    assert count >= 8


def test_bvh_placement_flags():
    """RTG_COMPILE_DEFER_BVH leaves the tree to the upload; RTG_COMPILE_AUTO_BVH
    builds it in the compile below 32,768 primitives and defers it above. Whatever
    the compile does, the scene itself (primitives, lights, materials) is the same."""
    small = json.dumps(workloads.cornell())
    large = json.dumps(workloads.mesh_stress())
    assert len(rtg.parse_scene(small, defer_bvh=True).view()["nodes"]) == 0
    assert len(rtg.parse_scene(small, defer_bvh="auto").view()["nodes"]) > 0
    host = rtg.parse_scene(large).view()
    auto = rtg.parse_scene(large, defer_bvh="auto").view()
    assert len(host["nodes"]) > 0 and len(auto["nodes"]) == 0
    for k in ("prims", "planes", "lights", "materials", "point_lights"):
        assert np.array_equal(host[k], auto[k]), k


def test_compile_flags_are_checked():
    import ctypes as C

    h = C.c_void_p()
    err = C.create_string_buffer(256)
    text = json.dumps(workloads.cornell()).encode()
    lib = rtg.lib()
    assert lib.rtg_compile_flags(text, None, 4, C.byref(h), err, 256) == rtg.RTG_ERR_INVALID
    assert lib.rtg_compile_flags(text, None, rtg.COMPILE_DEFER_BVH | rtg.COMPILE_AUTO_BVH, C.byref(h), err,
                                 256) == rtg.RTG_ERR_INVALID
    assert lib.rtg_compile_flags(text, None, rtg.COMPILE_AUTO_BVH, C.byref(h), err, 256) == rtg.RTG_OK
    lib.rtg_host_scene_free(h)


def test_mis_setting_survives_dump_and_defaults_off():
    scene = workloads.cornell()
    assert '"mis"' not in rtg.dump_scene(json.dumps(scene))
    scene["render"]["mis"] = True
    dumped = json.loads(rtg.dump_scene(json.dumps(scene)))
    assert dumped["render"]["mis"] is True
    st = rtg.parse_scene(json.dumps(dumped)).view()["settings"]
    assert st.mis and st.light_sampling
