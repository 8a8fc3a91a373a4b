"""The autotuner: picks a valid configuration, applies it, caches it per GPU and
workload, and leaves results unchanged (the image does not depend on tuning)."""
import json

import pytest

import rtg
import workloads

pytestmark = pytest.mark.gpu


def test_autotune_applies_caches_and_keeps_images(ctx, tmp_path, monkeypatch):
    monkeypatch.setenv("RTG_TUNE_CACHE", str(tmp_path / "tuning.txt"))
    scenes = [workloads.cornell(width=48, height=40, spp=16), workloads.sphere_field(width=40, height=32, spp=16)]
    sids = [ctx.load_json(json.dumps(s)) for s in scenes]
    sts = [ctx.scene_settings(i) for i in sids]
    before = ctx.tuning()
    try:
        ctx.render_batch(sids, sts)
        ref = [ctx.framebuffer_moments(j, st.width, st.height)[0].tobytes() for j, st in enumerate(sts)]
        first = ctx.autotune(sids, sts)
        assert not first["from_cache"] and first["probe_msamples_per_s"] > 0
        assert first["pool_paths"] in (1 << 20, 1 << 21, 1 << 22, 6 << 20, 1 << 23) and first["block"] in (128, 256)
        t = ctx.tuning()
        assert (t["pool_paths"], t["block"]) == (first["pool_paths"], first["block"])
        again = ctx.autotune(sids, sts)
        assert again["from_cache"] and (again["pool_paths"], again["block"]) == (first["pool_paths"], first["block"])
        assert (tmp_path / "tuning.txt").read_text().count("\n") == 1
        ctx.render_batch(sids, sts)
        got = [ctx.framebuffer_moments(j, st.width, st.height)[0].tobytes() for j, st in enumerate(sts)]
        assert got == ref
    finally:
        ctx.set_tuning(pool_paths=before["pool_paths"], block=before["block"])
        for sid in sids:
            ctx.release(sid)
