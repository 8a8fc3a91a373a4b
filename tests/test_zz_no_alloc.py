"""rtg_trace_closest_noalloc: the closest-hit query for callers that must not
allocate device memory during a call (a loop sharing the GPU with other streams,
a host that pre-reserves all device memory, code issuing work during stream
capture). It must give the same answers as rtg_trace_closest, through its static
device scratch array, on consecutive calls that reuse that array.

Kept in its own file, collected last, so a failure here never hides the rest of
the suite; it passes alone in a fresh process and after the other tests."""
import json

import numpy as np
import pytest

import rtg
import workloads
from parity import hit_parity

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def no_alloc_ctx():
    c = rtg.Context(0)
    yield c
    c.close()


def _same(a, b):
    """Existing entry point vs the no-alloc one: identical ids, and t within the
    1e-5 relative tolerance of the ray-parity tests."""
    ta, pa, pla, ba = a
    tb, pb, plb, bb = b
    assert np.array_equal(pa, pb) and np.array_equal(pla, plb)
    p = hit_parity(tb, pb, plb, ta, pa, pla)
    assert p["strict"] == 1.0, p
    hit = pa >= 0
    assert np.allclose(ba[hit], bb[hit], rtol=1e-5, atol=1e-6)


def test_no_alloc_matches_trace_closest_on_consecutive_calls(no_alloc_ctx):
    ctx = no_alloc_ctx
    mesh = rtg.parse_scene(json.dumps(workloads.mesh_stress()))
    spheres = rtg.parse_scene(json.dumps(workloads.sphere_field()))
    sid_mesh, sid_spheres = ctx.upload(mesh), ctx.upload(spheres)
    rays_a = workloads.random_rays(mesh.view(), 200_000, seed=71)
    rays_b = workloads.random_rays(spheres.view(), 50_000, seed=72)

    ref_a = ctx.trace_closest(sid_mesh, rays_a)
    ref_b = ctx.trace_closest(sid_spheres, rays_b)
    # First call: larger batch on the mesh scene.
    got_a = ctx.trace_closest_noalloc(sid_mesh, rays_a)
    _same(ref_a, got_a)
    # Second call reuses the array with a smaller batch on another scene: none of
    # the first call's leftovers may show through.
    got_b = ctx.trace_closest_noalloc(sid_spheres, rays_b)
    _same(ref_b, got_b)
    # Brute-force variant agrees too.
    _same(ctx.trace_closest(sid_spheres, rays_b[:4096], brute=True),
          ctx.trace_closest_noalloc(sid_spheres, rays_b[:4096], brute=True))
    ctx.release(sid_mesh)
    ctx.release(sid_spheres)


def test_no_alloc_rejects_batches_beyond_its_limit(no_alloc_ctx):
    ctx = no_alloc_ctx
    sid = ctx.load_json(json.dumps(workloads.cornell()))
    rays = np.zeros((rtg.NOALLOC_MAX_RAYS + 1, 8), np.float32)
    rays[:, 4] = 1
    rays[:, 7] = 1e30
    with pytest.raises(rtg.RtgError) as err:
        ctx.trace_closest_noalloc(sid, rays)
    assert err.value.code == rtg.RTG_ERR_LIMIT and "262144" in str(err.value)
    # Exactly the limit is accepted.
    t, prim, plane, _ = ctx.trace_closest_noalloc(sid, rays[:-1])
    assert len(prim) == rtg.NOALLOC_MAX_RAYS
    ctx.release(sid)
