"""The serving loop's host logic (serving.serve) on the CPU, against a simulated
context: Poisson arrivals, previews before finals, admission retries when the
footprint budget is full, cold-scene previews (compiled on worker threads,
uploaded, released when done), cancellation of finals after the window, and a
clean footprint at the end. Rendering itself is covered by the GPU tests."""
import json
import time

import pytest

import rtg
import serving
import workloads


class FakeContext:
    """Plays the serving part of rtg.Context: one pass per pump for each open
    request (previews first), passes of 1, 1, 2, 4, ... samples as the real
    progressive schedule, and a footprint budget that turns submits away."""

    def __init__(self, budget_bytes=3 * 1024 * 1024 * 70):
        self.budget = budget_bytes
        self.used = 0
        self.requests = {}
        self.scenes = {}
        self.next_id = 1
        self.prepared = False
        self.log = []

    # scenes
    def upload(self, host):
        assert isinstance(host, rtg.HostScene)
        sid = self.next_id
        self.next_id += 1
        self.scenes[sid] = host.view()["settings"]
        self.log.append(("upload", sid))
        return sid

    def release(self, sid):
        assert not any(r["scene"] == sid for r in self.requests.values()), "scene released under a request"
        del self.scenes[sid]
        self.log.append(("release", sid))

    def scene_settings(self, sid):
        s = self.scenes[sid]
        return rtg.RenderSettings(**s.__dict__)

    # serving
    def serve_prepare(self):
        self.prepared = True

    def submit(self, sid, st, opts, priority):
        assert self.prepared and sid in self.scenes
        bytes_ = st.width * st.height * 68
        if self.used + bytes_ > self.budget:
            return None
        rid = self.next_id
        self.next_id += 1
        self.used += bytes_
        self.requests[rid] = {"scene": sid, "st": st, "opts": opts, "priority": priority, "done": 0, "passes": 0,
                              "bytes": bytes_, "cancelled": False, "released": False}
        return rid

    def _progress(self, r):
        st = r["st"]
        return rtg.RenderProgress(r["passes"], r["done"], st.spp, 0.0, 0, r["done"] >= st.spp, r["cancelled"])

    def pump(self, budget_ms, return_on_event=False):
        time.sleep(0.0005)
        events = []
        for rid, r in sorted(self.requests.items(), key=lambda kv: kv[1]["priority"]):
            st = r["st"]
            if r["cancelled"] or r["done"] >= st.spp:
                continue
            k = st.spp - r["done"]
            if r["opts"].progressive:
                k = min(k, max(1, r["done"]), r["opts"].max_pass_spp)
            r["done"] += k
            r["passes"] += 1
            events.append((rid, self._progress(r)))
        return events

    def request_progress(self, rid):
        return self._progress(self.requests[rid])

    def request_image(self, rid, w, h):
        assert rid in self.requests
        return None

    def cancel_request(self, rid):
        self.requests[rid]["cancelled"] = True

    def release_request(self, rid):
        r = self.requests.pop(rid)
        self.used -= r["bytes"]

    def serve_footprint(self):
        rendering = sum(1 for r in self.requests.values() if not r["cancelled"] and r["done"] < r["st"].spp)
        return self.used, len(self.requests), rendering


@pytest.fixture(scope="module")
def mix_texts():
    return [json.dumps(s) for s in workloads.batch_mix(12, seed=9)]


def resident(ctx, texts):
    return [ctx.upload(rtg.parse_scene(t)) for t in texts]


def test_previews_all_served_and_footprint_clean(mix_texts):
    ctx = FakeContext()
    sids = resident(ctx, mix_texts[:4])
    out = serving.serve(ctx, sids, seconds=0.3, rate=400.0, preview_share=0.8, seed=3, read_images=True)
    p, f = out["preview"], out["final"]
    assert p["count"] > 50 and p["first_pass_on_host"] == p["count"] == p["finished"]
    assert f["count"] > 5 and 0 < f["admitted"] <= f["count"]
    assert out["admission_retries"] > 0  # finals waited for footprint
    assert ctx.serve_footprint() == (0, 0, 0)
    assert set(ctx.scenes) == set(sids)  # resident scenes untouched


def test_cold_previews_compile_upload_and_release(mix_texts):
    ctx = FakeContext()
    sids = resident(ctx, mix_texts[:4])
    cold = mix_texts[4:]
    out = serving.serve(ctx, sids, seconds=0.3, rate=400.0, preview_share=0.9, seed=5, cold_texts=cold,
                        cold_share=0.25, cold_gpu_bvh=True)
    c = out["cold_preview"]
    assert c["count"] > 10 and c["first_pass_on_host"] == c["count"] == c["finished"]
    # Start-up uploads each cold scene once; then one upload and one release per request.
    uploads = [e for e in ctx.log if e[0] == "upload"]
    releases = [e for e in ctx.log if e[0] == "release"]
    assert len(uploads) == len(sids) + len(cold) + c["count"]
    assert len(releases) == len(cold) + c["count"]
    assert set(ctx.scenes) == set(sids)
    phases = c["phase_ms_p50_p99"]
    assert set(phases) == {"compile", "upload", "queue", "trace", "read"}
    assert all(v[0] is not None and v[0] >= 0 for v in phases.values())
    assert ctx.serve_footprint() == (0, 0, 0)


def test_arrivals_are_seeded_and_cold_share_does_not_disturb_them():
    a = serving.poisson_arrivals([1, 2, 3], 1.0, 200.0, 0.9, seed=7)
    b = serving.poisson_arrivals([1, 2, 3], 1.0, 200.0, 0.9, seed=7)
    assert [(r.kind.name, r.scene, r.arrival) for r in a] == [(r.kind.name, r.scene, r.arrival) for r in b]
    c = serving.poisson_arrivals([1, 2, 3], 1.0, 200.0, 0.9, seed=7, cold_texts=["{}"], cold_share=0.1)
    assert any(r.kind is serving.COLD for r in c)
    assert all(r.text == "{}" for r in c if r.kind is serving.COLD)
