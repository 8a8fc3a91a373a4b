"""Serving through the C ABI: requests share one continuous wavefront, yet each
request's framebuffer is bit-identical to rendering it alone; previews overtake
finals; cancellation, release and admission by footprint."""
import json

import numpy as np
import pytest

import rtg
import workloads

pytestmark = pytest.mark.gpu


def pump_until(ctx, done, limit_ms=60000.0):
    events = []
    waited = 0.0
    while not done(events):
        events += ctx.pump(50.0)
        waited += 50.0
        assert waited < limit_ms, "requests did not finish"
    return events


def alone(ctx, sid, st, opts):
    ctx.render(sid, st, opts)
    return ctx.framebuffer_mean(-1, st.width, st.height), ctx.image(-1, st.width, st.height)


def test_request_in_a_mix_is_bit_identical_to_rendering_it_alone(ctx):
    scenes = [workloads.cornell(width=40, height=32, spp=6), workloads.sphere_field(width=32, height=24, spp=9),
              workloads.mesh_stress(width=24, height=16, spp=5)]
    sids = [ctx.load_json(json.dumps(s)) for s in scenes]
    sts = [ctx.scene_settings(i) for i in sids]
    opts = rtg.RenderOptions(progressive=True, max_pass_spp=4)
    ref = [alone(ctx, sid, st, opts) for sid, st in zip(sids, sts)]
    # The same three, submitted together with an extra request of another seed.
    extra = rtg.RenderSettings(**{**sts[0].__dict__, "seed": 77})
    rids = [ctx.submit(sid, st, opts, priority=k % 2) for k, (sid, st) in enumerate(zip(sids, sts))]
    rx = ctx.submit(sids[0], extra, opts, priority=0)
    open_ = set(rids + [rx])
    passes = {r: [] for r in open_}

    def done(events):
        for r, p in events[len(sum(passes.values(), [])):]:
            passes[r].append(p.spp_done)
        return all(ctx.request_progress(r).finished for r in open_)

    pump_until(ctx, done)
    for k, (r, st) in enumerate(zip(rids, sts)):
        mean = ctx.request_mean(r, st.width, st.height)
        img = ctx.request_image(r, st.width, st.height)
        assert mean.tobytes() == ref[k][0].tobytes(), k
        assert img.tobytes() == ref[k][1].tobytes(), k
        # The reference's progressive schedule, reported once per pass in order.
        assert passes[r] == sorted(passes[r]) and passes[r][-1] == st.spp
    assert ctx.request_mean(rx, sts[0].width, sts[0].height).tobytes() != ref[0][0].tobytes()
    for r in open_:
        ctx.release_request(r)
    assert ctx.serve_footprint() == (0, 0, 0)
    for sid in sids:
        ctx.release(sid)


def test_scene_built_on_the_gpu_while_requests_render(ctx):
    """A cold scene arrives while a request is rendering: its BVH is built on the
    GPU (on the build stream, beside the wavefront), a preview of it is served, and
    both requests still give exactly the images they give alone."""
    busy = workloads.cornell(width=512, height=512, spp=2048)  # ~5e8 samples: still rendering
    cold = workloads.mesh_stress(width=32, height=24, spp=4)
    bs = ctx.load_json(json.dumps(busy))
    bst = ctx.scene_settings(bs)
    opts = rtg.RenderOptions(progressive=True, max_pass_spp=32)
    ref_busy = alone(ctx, bs, bst, opts)
    warm = ctx.upload(rtg.parse_scene(json.dumps(cold)))
    cst = ctx.scene_settings(warm)
    ref_cold = alone(ctx, warm, cst, opts)
    ctx.release(warm)
    rb = ctx.submit(bs, bst, opts, priority=1)
    ctx.pump(20.0)
    assert not ctx.request_progress(rb).finished
    cs = ctx.upload(rtg.parse_scene(json.dumps(cold), defer_bvh=True))
    assert ctx.scene_layout(cs, "roots")[0][3] == 1
    rc = ctx.submit(cs, cst, opts, priority=0)
    pump_until(ctx, lambda ev: ctx.request_progress(rb).finished and ctx.request_progress(rc).finished)
    assert ctx.request_mean(rb, bst.width, bst.height).tobytes() == ref_busy[0].tobytes()
    assert ctx.request_mean(rc, cst.width, cst.height).tobytes() == ref_cold[0].tobytes()
    for r in (rb, rc):
        ctx.release_request(r)
    ctx.release(bs)
    ctx.release(cs)


def test_previews_overtake_a_final_already_rendering(ctx):
    final = workloads.cornell(width=512, height=512, spp=4096)  # ~1e9 samples: renders for a while
    preview = workloads.sphere_field(width=32, height=32, spp=2)
    preview["render"]["max_depth"] = 4
    fs, ps = ctx.load_json(json.dumps(final)), ctx.load_json(json.dumps(preview))
    rf = ctx.submit(fs, None, rtg.RenderOptions(progressive=True, max_pass_spp=32), priority=1)
    ctx.pump(20.0)  # the final fills the pool
    rp = ctx.submit(ps, None, rtg.RenderOptions(progressive=False), priority=0)
    events = pump_until(ctx, lambda ev: any(r == rp and p.finished for r, p in ev))
    assert not ctx.request_progress(rf).finished
    ctx.cancel_request(rf)
    pump_until(ctx, lambda ev: ctx.serve_footprint()[2] == 0)
    for r in (rf, rp):
        ctx.release_request(r)
    assert events
    ctx.release(fs)
    ctx.release(ps)


def test_cancel_keeps_reported_passes_and_frees_the_request(ctx):
    scene = workloads.cornell(width=64, height=64, spp=100000)
    sid = ctx.load_json(json.dumps(scene))
    r = ctx.submit(sid, None, rtg.RenderOptions(progressive=True, max_pass_spp=8), priority=1)
    events = pump_until(ctx, lambda ev: len(ev) >= 3)
    with pytest.raises(rtg.RtgError) as busy:
        ctx.release_request(r)
    assert busy.value.code == rtg.RTG_ERR_BUSY
    with pytest.raises(rtg.RtgError):
        ctx.release(sid)  # the scene is in use
    ctx.cancel_request(r)
    pump_until(ctx, lambda ev: ctx.serve_footprint()[2] == 0)
    p = ctx.request_progress(r)
    assert p.cancelled and not p.finished and p.spp_done >= events[-1][1].spp_done
    mean = ctx.request_mean(r, 64, 64)
    assert np.isfinite(mean).all() and mean.mean() > 0
    ctx.release_request(r)
    assert ctx.serve_footprint() == (0, 0, 0)
    # Plain renders work again once no request is open.
    st = ctx.scene_settings(sid)
    st.spp = 2
    assert ctx.render(sid, st).finished
    ctx.release(sid)


def test_admission_by_footprint(ctx):
    scene = workloads.cornell(width=64, height=64, spp=4)
    sid = ctx.load_json(json.dumps(scene))
    t = ctx.tuning()
    one = 64 * 64 * (68 + 16) + 32  # framebuffer + first-pass radiance of one request
    ctx.set_tuning(serve_budget_bytes=one + 32, serve_reserve_bytes=0)  # room for exactly one
    try:
        a = ctx.submit(sid)
        assert a is not None
        assert ctx.submit(sid) is None  # turned away, nothing opened
        assert ctx.serve_footprint()[:2] == (one, 1)
        with pytest.raises(rtg.RtgError) as busy:
            ctx.render(sid)
        assert busy.value.code == rtg.RTG_ERR_BUSY
        pump_until(ctx, lambda ev: ctx.request_progress(a).finished)
        ctx.release_request(a)
        # The reserve keeps room for previews: priority 1 no longer fits, priority 0 does.
        ctx.set_tuning(serve_budget_bytes=one + 32, serve_reserve_bytes=64)
        assert ctx.submit(sid, priority=1) is None
        b = ctx.submit(sid, priority=0)
        assert b is not None
        pump_until(ctx, lambda ev: ctx.request_progress(b).finished)
        ctx.release_request(b)
    finally:
        ctx.set_tuning(serve_budget_bytes=t["serve_budget_bytes"], serve_reserve_bytes=t["serve_reserve_bytes"])
        ctx.release(sid)


def test_poisson_request_loop_serves_every_preview(ctx):
    import serving

    scenes = [workloads.mix_scene(k) for k in range(6)]
    sids = [ctx.load_json(json.dumps(s)) for s in scenes]
    out = serving.serve(ctx, sids, seconds=1.0, rate=100.0, preview_share=0.9, seed=5)
    pv = out["preview"]
    assert pv["count"] > 50 and pv["first_pass_on_host"] == pv["count"] == pv["finished"]
    assert 0 < pv["ttfp_ms_p50"] <= pv["ttfp_ms_p99"] < 1000
    fin = out["final"]
    assert 0 < fin["first_pass_on_host"] <= fin["admitted"] <= fin["count"]
    assert out["msamples_per_s"] > 0
    assert ctx.serve_footprint() == (0, 0, 0)
    for sid in sids:
        ctx.release(sid)


def test_poisson_loop_with_cold_scene_previews(ctx):
    """Previews of scenes that are not resident, compiled on arrival and uploaded
    with the BVH built on the GPU: every one is served, and each cold scene is
    released again when its request finishes."""
    import serving

    mix = workloads.batch_mix(8, seed=4)
    sids = [ctx.load_json(json.dumps(s)) for s in mix[:4]]
    cold = [json.dumps(s) for s in mix[4:]]
    out = serving.serve(ctx, sids, seconds=1.0, rate=100.0, preview_share=0.9, seed=11, cold_texts=cold,
                        cold_share=0.2, cold_gpu_bvh=True)
    c = out["cold_preview"]
    assert c["count"] > 5 and c["first_pass_on_host"] == c["count"] == c["finished"]
    assert out["host_calls"]["upload"]["count"] == c["count"]
    assert out["host_calls"]["release_scene"]["count"] == c["count"]
    assert out["preview"]["first_pass_on_host"] == out["preview"]["count"]
    assert ctx.serve_footprint() == (0, 0, 0)
    for sid in sids:
        ctx.release(sid)
