"""rtg_trace_closest_noalloc: the closest-hit query for callers that must not
allocate device memory during a call (a loop sharing the GPU with other
streams, where a free would synchronise the device; a host that pre-reserves all
device memory in its own pool). It must give the same answers as
rtg_trace_closest, through its static device scratch array, on consecutive calls
that reuse that array, and it must not ask CUDA for any memory.

Kept in its own file, collected last, so a failure here never hides the rest of
the suite; it passes alone in a fresh process and after the other tests."""
import json

import numpy as np
import pytest

import rtg
import workloads
from parity import hit_parity

pytestmark = pytest.mark.gpu

# Relative distance tolerance of an fp32 hit against its double refinement, and
# the share of rays that must meet it (the ray-parity bar).
T_REL_FP32 = 1e-5
T_SHARE = 0.9999


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


def test_no_alloc_asks_cuda_for_no_memory(no_alloc_ctx):
    """The property the entry point exists for: once warm, a call makes no
    allocation at all (the library counts every cudaMalloc, pooled and pinned
    allocation it makes). rtg_trace_closest, as the control, does allocate."""
    ctx = no_alloc_ctx
    host = rtg.parse_scene(json.dumps(workloads.sphere_field()))
    sid = ctx.upload(host)
    rays = workloads.random_rays(host.view(), 100_000, seed=73)
    ref = ctx.trace_closest(sid, rays)
    ctx.trace_closest_noalloc(sid, rays)  # warm: first use on this device
    before = rtg.allocation_count()
    first = ctx.trace_closest_noalloc(sid, rays)
    second = ctx.trace_closest_noalloc(sid, rays[:5000])
    assert rtg.allocation_count() == before
    _same(ref, first)
    _same(tuple(x[:5000] for x in ref), second)
    ctx.trace_closest(sid, rays[:10])
    assert rtg.allocation_count() > before  # the counter sees rtg_trace_closest's buffers
    ctx.release(sid)


def test_no_alloc_on_a_fresh_scene_reports_the_fp32_distance(no_alloc_ctx):
    """A scene never given to rtg_trace_closest has no double-precision copy on
    the device, so the no-alloc call reports the fp32 traversal's own t: ids and
    planes exactly those of rtg_trace_closest, t within the fp32 tolerance of the
    refined distance, and equal to rtg_trace_closest's with refine_hits off."""
    ctx = no_alloc_ctx
    host = rtg.parse_scene(json.dumps(workloads.mesh_stress()))
    sid = ctx.upload(host)
    rays = workloads.random_rays(host.view(), 200_000, seed=74)
    t, prim, plane, bary = ctx.trace_closest_noalloc(sid, rays)
    rt, rprim, rplane, _ = ctx.trace_closest(sid, rays)  # uploads the double copy, refines t
    assert np.array_equal(prim, rprim) and np.array_equal(plane, rplane)
    hit = rprim >= 0
    rel = np.abs(t[hit].astype(np.float64) - rt[hit]) / np.abs(rt[hit].astype(np.float64))
    assert np.mean(rel <= T_REL_FP32) >= T_SHARE, np.quantile(rel, [0.5, 0.999, 1.0])
    ctx.set_tuning(refine_hits=0)
    try:
        raw_t, raw_prim, raw_plane, raw_bary = ctx.trace_closest(sid, rays)
    finally:
        ctx.set_tuning(refine_hits=1)
    assert np.array_equal(prim, raw_prim) and np.array_equal(plane, raw_plane)
    assert np.allclose(t, raw_t, rtol=1e-6, atol=0) and np.allclose(bary, raw_bary, rtol=1e-5, atol=1e-6)
    ctx.release(sid)


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
