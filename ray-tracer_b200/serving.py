"""Request loop over resident scenes: Poisson arrivals of previews and finals,
admission by device footprint, continuous batching in one wavefront, and
time-to-first-pass (TTFP) per request.

A request's TTFP runs from its arrival time to the moment its first pass is on
the host (the pass event, then the tone-mapped image read back). Previews are
submitted at priority 0 and finals at priority 1, so previews take free path
slots first; a final's first pass is ordered ahead of other finals' later passes.

Cold previews (optional) are previews of scenes that are not resident: the scene
JSON arrives with the request, a worker thread compiles it, the serving thread
uploads it (with the BVH built on the GPU, or flattened from a host-built tree)
and submits it; the scene is released when its request finishes. Their TTFP
includes the compile and the upload. With the GPU build, scenes under 32,768
primitives still get their tree on the worker (the host is faster there).
"""
import collections
import concurrent.futures
import dataclasses
import time
from typing import Optional

import numpy as np

import rtg


@dataclasses.dataclass
class RequestKind:
    name: str
    width: int
    height: int
    spp: int
    max_depth: int
    progressive: bool
    priority: int


PREVIEW = RequestKind("preview", 128, 128, 4, 4, False, 0)
FINAL = RequestKind("final", 1024, 1024, 1024, 16, True, 1)
COLD = RequestKind("cold_preview", 128, 128, 4, 4, False, 0)


@dataclasses.dataclass
class Request:
    kind: RequestKind
    scene: int
    arrival: float                 # seconds after the loop starts
    rid: Optional[int] = None
    submitted: Optional[float] = None
    first_event: Optional[float] = None
    first_pass: Optional[float] = None
    finished: Optional[float] = None
    spp_done: int = 0
    samples: int = 0
    text: Optional[str] = None       # scene JSON of a cold preview
    future: object = None            # its compile on a worker thread
    compiled: Optional[float] = None
    uploaded: Optional[float] = None


def poisson_arrivals(scene_ids, seconds: float, rate: float, preview_share: float, seed: int, cold_texts=(),
                     cold_share: float = 0.0):
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            return out
        if cold_texts and rng.random() < cold_share:
            out.append(Request(COLD, -1, t, text=cold_texts[int(rng.integers(len(cold_texts)))]))
            continue
        kind = PREVIEW if rng.random() < preview_share else FINAL
        out.append(Request(kind, int(scene_ids[rng.integers(len(scene_ids))]), t))


def settings_for(ctx: rtg.Context, r: Request) -> rtg.RenderSettings:
    s = ctx.scene_settings(r.scene)
    s.width, s.height, s.spp, s.max_depth = r.kind.width, r.kind.height, r.kind.spp, r.kind.max_depth
    s.rr_min_depth = min(s.rr_min_depth, s.max_depth)
    return s


def serve(ctx: rtg.Context, scene_ids, seconds: float = 10.0, rate: float = 200.0, preview_share: float = 0.9,
          seed: int = 2025, read_images: bool = True, cold_texts=(), cold_share: float = 0.0,
          cold_gpu_bvh: bool = True) -> dict:
    """Runs the request loop for `seconds` of arrivals and until every preview is
    served, then cancels what is still rendering. Returns latency percentiles and
    throughput. cold_share of the arrivals are previews of the scenes in
    cold_texts (JSON), compiled and uploaded on arrival; cold_gpu_bvh builds their
    BVH on the GPU, else on the host."""
    reqs = poisson_arrivals(scene_ids, seconds, rate, preview_share, seed, cold_texts, cold_share)
    ctx.serve_prepare()  # start-up, outside the timed loop
    if cold_texts:
        # Start-up for cold scenes too: uploading each once maps the memory their
        # builds and staging need, as serve_prepare does for requests.
        for text in cold_texts:
            ctx.release(ctx.upload(rtg.parse_scene(text, None, "auto" if cold_gpu_bvh else False)))
    pending = collections.deque(reqs)
    waiting = {PREVIEW.name: collections.deque(), FINAL.name: collections.deque(), COLD.name: collections.deque()}
    compiler = concurrent.futures.ThreadPoolExecutor(max_workers=4) if cold_texts else None
    live = {}
    settings = {}
    rejected = 0
    t0 = time.perf_counter()
    calls = collections.defaultdict(lambda: [0, 0.0, 0.0, 0])  # name -> [count, total s, max s, over 20 ms]

    def now():
        return time.perf_counter() - t0

    def timed(name, fn, *args, **kw):
        c0 = time.perf_counter()
        out = fn(*args, **kw)
        dt = time.perf_counter() - c0
        rec = calls[name]
        rec[0] += 1
        rec[1] += dt
        rec[2] = max(rec[2], dt)
        rec[3] += dt > 0.02
        return out

    def admit(q) -> bool:
        """Submits the head of q; False when the footprint budget turns it away."""
        r = q[0]
        if r.kind is COLD:
            if r.scene < 0:
                if not r.future.done():
                    return False
                host, r.compiled = r.future.result()
                r.scene = timed("upload", ctx.upload, host)
                r.uploaded = now()
            st = settings_for(ctx, r)
        else:
            st = settings.get((r.scene, r.kind.name)) or settings_for(ctx, r)
            settings[(r.scene, r.kind.name)] = st
        rid = timed("submit", ctx.submit, r.scene, st,
                    rtg.RenderOptions(progressive=r.kind.progressive, max_pass_spp=32), r.kind.priority)
        if rid is None:
            return False
        r.rid, r.submitted = rid, now()
        live[rid] = r
        q.popleft()
        return True

    while True:
        t = now()
        in_window = t < seconds
        previews_open = (waiting[PREVIEW.name] or waiting[COLD.name]
                         or any(r.kind is not FINAL for r in live.values()))
        if not in_window and not pending and not previews_open:
            break
        while pending and pending[0].arrival <= t:
            r = pending.popleft()
            if r.kind is COLD:
                defer = "auto" if cold_gpu_bvh else False  # small scenes: host tree on the worker
                r.future = compiler.submit(lambda text, defer=defer: (rtg.parse_scene(text, None, defer), now()),
                                           r.text)
            waiting[r.kind.name].append(r)
        # Previews first (they may use the reserve), cold previews once compiled;
        # finals while the budget allows and only inside the arrival window.
        for name in (PREVIEW.name, COLD.name, FINAL.name):
            q = waiting[name]
            if name == FINAL.name and not in_window:
                break
            while q:
                if not admit(q):
                    if name != COLD.name or q[0].scene >= 0:
                        rejected += 1
                    break
        if not live:
            if pending:
                time.sleep(max(0.0, min(pending[0].arrival - now(), 0.002)))
            continue
        for rid, p in timed("pump", ctx.pump, 2.0, return_on_event=True):
            r = live.get(rid)
            if r is None:
                continue
            r.spp_done = p.spp_done
            if r.first_pass is None:
                r.first_event = now()
                if read_images:
                    timed("image", ctx.request_image, rid, r.kind.width, r.kind.height)
                r.first_pass = now()
            if p.finished:
                r.finished = now()
                timed("release", ctx.release_request, rid)
                if r.kind is COLD:
                    timed("release_scene", ctx.release, r.scene)
                del live[rid]
    window = now()
    # Stop what is still rendering (finals that outlast the window).
    for rid, r in list(live.items()):
        ctx.cancel_request(rid)
    while ctx.serve_footprint()[2]:
        ctx.pump(5.0)
    for rid, r in list(live.items()):
        r.spp_done = ctx.request_progress(rid).spp_done
        ctx.release_request(rid)
        if r.kind is COLD:
            ctx.release(r.scene)
    if compiler:
        compiler.shutdown()
    for r in reqs:
        r.samples = r.kind.width * r.kind.height * r.spp_done

    def pct(xs, q):
        return float(np.percentile(xs, q)) * 1e3 if xs else None

    out = {"seconds": window, "arrival_rate_per_s": rate, "requests": len(reqs), "admission_retries": rejected,
           "msamples_per_s": sum(r.samples for r in reqs) / window / 1e6,
           "host_calls": {k: {"count": v[0], "total_ms": v[1] * 1e3, "max_ms": v[2] * 1e3, "over_20ms": v[3]}
                          for k, v in calls.items()},
           "policy": "previews priority 0 (may use the reserve), finals priority 1; finals still waiting for "
                     "footprint at the end of the arrival window are not admitted; finals still rendering are "
                     "cancelled after the last preview"}
    for kind in (PREVIEW, FINAL, COLD):
        rs = [r for r in reqs if r.kind is kind]
        if kind is COLD and not rs:
            continue
        ttfp = [r.first_pass - r.arrival for r in rs if r.first_pass is not None]
        served = [r for r in rs if r.first_pass is not None]
        phases = {"queue": [r.submitted - r.arrival for r in served],
                  "trace": [r.first_event - r.submitted for r in served],
                  "read": [r.first_pass - r.first_event for r in served]}
        if kind is COLD:
            phases = {"compile": [r.compiled - r.arrival for r in served],
                      "upload": [r.uploaded - r.compiled for r in served],
                      "queue": [r.submitted - r.uploaded for r in served],
                      "trace": phases["trace"], "read": phases["read"]}
        out[kind.name] = {
            "phase_ms_p50_p99": {k: [pct(v, 50), pct(v, 99)] for k, v in phases.items()},
            "count": len(rs), "admitted": sum(1 for r in rs if r.rid is not None), "first_pass_on_host": len(ttfp),
            "finished": sum(1 for r in rs if r.finished is not None),
            "ttfp_ms_p50": pct(ttfp, 50), "ttfp_ms_p99": pct(ttfp, 99), "ttfp_ms_max": pct(ttfp, 100),
            "shape": f"{kind.width}x{kind.height}, {kind.spp} spp, depth {kind.max_depth}, "
                     f"{'progressive' if kind.progressive else 'one pass'}",
        }
    return out
