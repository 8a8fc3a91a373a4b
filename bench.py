#!/usr/bin/env python
"""Benchmark: Msamples/s of the B200 path tracer on the batched 64-scene mix.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl rtg|reference] [--workload mix|cornell|spheres|mesh]

A step renders the whole workload once (every scene to its full spp, progressive
passes as the reference renderer runs them). `value` is samples rendered by all
ranks / the slowest rank's device time (CUDA events on the render stream) with
every scene already resident in HBM; `e2e` is the same metric through the public
API with host buffers: upload of the compiled scenes, the render and the read-back
of every tone-mapped image inside the timed region. N > 1 runs N independent
replicas (one per GPU, launched with torchrun): the workload shards by scene with
no exchange step, so scaling is weak.

--impl reference times the reference's own CPU renderer (built from its sources
into oracle/_ref/; the oracle restatement if that binary is absent) on the host
cores, on a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ray-tracer_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "Msamples/s on 1 B200, batched vs plain at matched RMSE; p50/p99 preview latency"
HARNESS = os.path.join(ROOT, "oracle", "_ref", "rt_harness")
L2_BYTES = 126 * 2 ** 20


def args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["rtg", "reference"], default="rtg")
    p.add_argument("--workload", choices=["mix", "cornell", "spheres", "mesh"], default="mix")
    p.add_argument("--no-plain", action="store_true", help="skip the plain one-scene-per-launch comparison")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--single-pass", action="store_true",
                   help="render every scene in one pass (the CPU baseline's --single-pass)")
    p.add_argument("--serve-seconds", type=float, default=10.0,
                   help="length of the serving run (Poisson arrivals over 32 resident scenes of the mix)")
    p.add_argument("--no-serve", action="store_true", help="skip the serving run")
    p.add_argument("--no-cold", action="store_true",
                   help="skip the cold-scene time-to-first-pass comparison (BVH built on the host vs the GPU)")
    p.add_argument("--no-autotune", action="store_true", help="keep the default pool and block size")
    p.add_argument("--pool", type=int, default=0, help="path slots (implies --no-autotune)")
    p.add_argument("--block", type=int, default=0, help="threads per block: 64, 128, 256 (implies --no-autotune)")
    return p.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (replicas)

class Dist:
    def __init__(self, want):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            backend = "gloo"  # only barriers and one scalar max: no data-path collective
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist
        if want != self.world and self.rank == 0 and self.world > 1:
            print(f"note: --gpus {want} but WORLD_SIZE {self.world}", file=sys.stderr)

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region

class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = tempfile.mktemp(prefix="rtg_clocks_", suffix=".csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "200"], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm), "power_w_max": max(power) if power else None}


# ---------------------------------------------------------------------------
# workloads

def workload_scenes(name):
    import workloads

    if name == "mix":
        return workloads.batch_mix(), ("batched mix: 64 seeded scenes (spheres 10-2000, meshes 1k-200k tris, "
                                       "facing mirrors), resolutions 128^2-1024^2, spp 16/64/256, depth 8-40")
    make = {"cornell": workloads.cornell, "spheres": workloads.sphere_field, "mesh": workloads.mesh_stress}[name]
    desc = {"cornell": "Cornell box 555-unit room, 256x256x64 spp, depth 8, NEE + RR",
            "spheres": "sphere field ~480 spheres + plane, thin lens, 512x512x128 spp, depth 16",
            "mesh": "mesh stress 174k tris (icosphere s6 + 256x180 torus), 1024x1024x64 spp, depth 12"}[name]
    return [make()], desc


def samples_of(scenes):
    return sum(s["render"]["width"] * s["render"]["height"] * s["render"]["spp"] for s in scenes)


# ---------------------------------------------------------------------------
# CPU side: the reference renderer (oracle/_ref) or the oracle port

def cpu_render(scene: dict, spp: int) -> tuple:
    """(samples, seconds, kind, threads) for one scene at `spp` on the host cores."""
    s = json.loads(json.dumps(scene))
    s["render"]["spp"] = spp
    if os.path.exists(HARNESS):
        with tempfile.NamedTemporaryFile("w", suffix=".json", delete=False) as f:
            json.dump(s, f)
            path = f.name
        try:
            out = json.loads(subprocess.check_output([HARNESS, "bench", path, "--threads", "0"]).decode())
        finally:
            os.unlink(path)
        return out["width"] * out["height"] * out["spp"], out["elapsed_ms"] / 1e3, "reference", out["threads"]
    import rtg
    import rtoracle

    o = rtoracle.OracleScene(rtg.parse_scene(json.dumps(s)).view())
    t0 = time.perf_counter()
    o.render()
    dt = time.perf_counter() - t0
    return s["render"]["width"] * s["render"]["height"] * spp, dt, "port", os.cpu_count()


def cpu_sample(scenes, budget_s: float):
    """Renders scenes (in a fixed order, at spp/16) until the time budget is spent."""
    order = sorted(range(len(scenes)), key=lambda k: (k * 37) % len(scenes))
    samples = secs = 0.0
    used = []
    kind, threads = "reference", os.cpu_count()
    for k in order:
        spp = max(1, scenes[k]["render"]["spp"] // 16)
        n, dt, kind, threads = cpu_render(scenes[k], spp)
        samples += n
        secs += dt
        used.append(k)
        if secs >= budget_s:
            break
    return samples, secs, kind, threads, used


def run_reference(a, dist, scenes, desc):
    if dist.rank != 0:
        return
    rates = []
    kind = threads = used = None
    for step in range(a.warmup + a.steps):
        samples, secs, kind, threads, used = cpu_sample(scenes, budget_s=5.0)
        if step >= a.warmup:
            rates.append(samples / secs / 1e6)
    value = statistics.median(rates)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": dist.world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded scene generators)",
        "config": {"workload": desc, "sample": f"scenes {used} at spp/16, stock Renderer::render, threads=0"},
        "cpu_baseline": {"value": value, "unit": "Msamples/s", "cores": threads, "kind": kind,
                         "sample": f"~5 s per step of the workload: scenes {used} at spp/16"},
        "e2e": {"value": value, "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU side

def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, STREAM-style copy)"
    return 6650.0, "fallback 6.65 TB/s"


def extend_traffic(pool_paths: int, rays_per_launch: float):
    """DRAM bytes per k_extend launch from the committed ncu capture of the mix
    (profiles/k_extend_mix_dram.json, taken with a full pool), scaled to this run's
    rays per launch; None when no capture matches this pool size."""
    p = os.path.join(ROOT, "profiles", "k_extend_mix_dram.json")
    if not os.path.exists(p):
        return None, None
    d = json.load(open(p))
    if int(d.get("pool_paths", 0)) != int(pool_paths):
        return None, None
    per_ray = d["dram_bytes_per_launch"] / d["rays_per_launch"]
    return per_ray * rays_per_launch, f"ncu capture, {d['launches_captured']} launches ({os.path.basename(p)})"


def cold_scene_ttfp(ctx, named_scenes, reps=3):
    """Time to first pass for scenes that are not resident yet: scene JSON text in,
    a 128x128, 4 spp, depth 4 preview image on the host out. Two ways: the host
    compile builds the BVH and the upload flattens it (host_bvh), or the compile
    skips the BVH and the upload builds it on the GPU (gpu_bvh). Medians over
    `reps` alternating runs; the phases are compile, upload and first pass (render
    plus image read-back)."""
    import numpy as np
    import rtg

    out = {}
    for name, scene in named_scenes:
        text = json.dumps(scene)
        runs = {"host_bvh": [], "gpu_bvh": []}
        prims = None
        for _ in range(reps):
            for arm, defer in (("host_bvh", False), ("gpu_bvh", "auto")):
                t0 = time.perf_counter()
                host = rtg.parse_scene(text, defer_bvh=defer)
                t1 = time.perf_counter()
                sid = ctx.upload(host)
                t2 = time.perf_counter()
                st = ctx.scene_settings(sid)
                st.width = st.height = 128
                st.spp, st.max_depth = 4, 4
                ctx.render(sid, st, rtg.RenderOptions(progressive=False))
                ctx.image(-1, 128, 128)
                t3 = time.perf_counter()
                prims = ctx.scene_info(sid)["primitives"]
                ctx.release(sid)
                runs[arm].append((t1 - t0, t2 - t1, t3 - t2, t3 - t0))
        entry = {"primitives": prims}
        for arm, r in runs.items():
            med = np.median(np.array(r), axis=0) * 1e3
            entry[arm] = {"compile_ms": med[0], "upload_ms": med[1], "first_pass_ms": med[2], "ttfp_ms": med[3]}
        entry["speedup"] = entry["host_bvh"]["ttfp_ms"] / entry["gpu_bvh"]["ttfp_ms"]
        out[name] = entry
    return out


def run_rtg(a, dist, scenes, desc):
    import rtg

    dev = dist.local
    ctx = rtg.Context(dev)
    opts = rtg.RenderOptions(progressive=not a.single_pass, max_pass_spp=32)
    hosts = [rtg.parse_scene(json.dumps(s)) for s in scenes]
    sids = [ctx.upload(h) for h in hosts]
    settings = [ctx.scene_settings(i) for i in sids]
    scene_bytes = sum(ctx.scene_info(i)["device_bytes"] for i in sids)
    batched = len(sids) > 1
    tuned = None
    if a.pool or a.block:
        ctx.set_tuning(**({"pool_paths": a.pool} if a.pool else {}), **({"block": a.block} if a.block else {}))
    elif not a.no_autotune:
        tuned = ctx.autotune(sids, settings, opts, use_cache=True)

    def step():
        if batched:
            ctx.render_batch(sids, settings, opts)
        else:
            ctx.render(sids[0], settings[0], opts)
        return ctx.stats()

    for _ in range(a.warmup):
        step()

    # Timed region: inputs resident in HBM; device time from CUDA events.
    clocks = Clocks(dev)
    dist.barrier()
    clocks.start()
    dev_ms = 0.0
    samples = 0
    launches = 0
    for _ in range(a.steps):
        st = step()
        dev_ms += st["device_ms"]
        samples += st["camera_samples"]
        launches += st["kernel_launches"]
    dist.barrier()
    clk = clocks.stop()
    t_max = dist.max(dev_ms)
    total_samples = dist.sum(samples)
    value = total_samples / (t_max / 1e3) / 1e6

    # End to end through the public API with host buffers.
    d2h = sum(s.width * s.height * 3 for s in settings)
    for i in sids:
        ctx.release(i)
    # One untimed upload first: it maps the library's pinned staging for a whole batch.
    for i in ctx.upload_many(hosts):
        ctx.release(i)
    dist.barrier()
    t0 = time.perf_counter()
    e2e_samples = 0
    phase = {"upload_s": 0.0, "render_s": 0.0, "images_s": 0.0, "release_s": 0.0}
    for _ in range(max(1, a.steps)):
        c0 = time.perf_counter()
        ids = ctx.upload_many(hosts)
        c1 = time.perf_counter()
        if batched:
            ctx.render_batch(ids, settings, opts)
        else:
            ctx.render(ids[0], settings[0], opts)
        e2e_samples += ctx.stats()["camera_samples"]
        c2 = time.perf_counter()
        for j, s in enumerate(settings):
            ctx.image(j if batched else -1, s.width, s.height)
        c3 = time.perf_counter()
        for i in ids:
            ctx.release(i)
        c4 = time.perf_counter()
        for k, dt in zip(phase, (c1 - c0, c2 - c1, c3 - c2, c4 - c3)):
            phase[k] += dt / max(1, a.steps)
    e2e_s = dist.max(time.perf_counter() - t0)
    e2e_value = dist.sum(e2e_samples) / e2e_s / 1e6
    sids = [ctx.upload(h) for h in hosts]

    # Plain renderer on the same scenes (one scene per launch sequence).
    plain = None
    if batched and not a.no_plain:
        ctx.render(sids[0], settings[0], opts)
        p_ms = p_samples = 0.0
        for i, s in zip(sids, settings):
            ctx.render(i, s, opts)
            st = ctx.stats()
            p_ms += st["device_ms"]
            p_samples += st["camera_samples"]
        plain = {"value": p_samples / (p_ms / 1e3) / 1e6, "unit": "Msamples/s",
                 "batched_over_plain": value / dist.world / (p_samples / (p_ms / 1e3) / 1e6),
                 "rmse": "identical images (bit-identical framebuffers), so matched RMSE by construction"}

    # Roofline of the dominant kernel (closest-hit traversal + camera generation):
    # one run with per-kernel CUDA events, one with traversal counters.
    ctx.set_tuning(time_kernels=1, count_traversal=0)
    t_st = step()
    ctx.set_tuning(time_kernels=0, count_traversal=1)
    c_st = step()
    ctx.set_tuning(time_kernels=0, count_traversal=0)
    tri = c_st["prim_tests"] - c_st["sphere_tests"]
    new_paths = c_st["camera_samples"]
    cont_rays = c_st["rays"] - new_paths
    ext_bytes = (c_st["node_visits"] * 64 + tri * 48 + c_st["sphere_tests"] * 32 + cont_rays * 32
                 + c_st["rays"] * 16 + new_paths * (64 + 16))
    launches_ext = max(1, t_st["extend_launches"])
    avg_ms = t_st["extend_ms"] / launches_ext
    achieved = ext_bytes / launches_ext / (avg_ms / 1e3) / 1e9
    peak, peak_src = peaks()
    traffic, traffic_src = extend_traffic(ctx.tuning()["pool_paths"], c_st["rays"] / launches_ext)
    kernel_total = t_st["extend_ms"] + t_st["shade_ms"] + t_st["shadow_ms"] + t_st["accumulate_ms"] + t_st["plan_ms"]
    roofline = {
        "kernel": "k_extend (closest-hit BVH traversal + camera-path generation)",
        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
        "traffic": traffic, "traffic_source": traffic_src, "peak_source": peak_src,
        # The same launches measured by DRAM bytes (ncu) instead of algorithmic bytes:
        # node and primitive fetches are mostly L1/L2 hits, so this is far lower.
        "dram_achieved": traffic / (avg_ms / 1e3) / 1e9 if traffic else None,
        "dram_frac": traffic / (avg_ms / 1e3) / 1e9 / peak if traffic else None,
        "bytes_per_launch": ext_bytes / launches_ext, "avg_launch_ms": avg_ms, "launches": launches_ext,
        "share_of_kernel_time": t_st["extend_ms"] / kernel_total if kernel_total else None,
        "per_ray": {"nodes": c_st["node_visits"] / max(1, c_st["rays"]),
                    "prim_tests": c_st["prim_tests"] / max(1, c_st["rays"])},
        "kernel_ms": {k: t_st[k] for k in ("extend_ms", "shade_ms", "shadow_ms", "accumulate_ms", "plan_ms")},
    }

    # Serving: Poisson arrivals of previews and finals over 32 resident scenes.
    serve = None
    if batched and not a.no_serve and a.serve_seconds > 0:
        import serving

        serve = serving.serve(ctx, sids[:32], seconds=a.serve_seconds, rate=200.0, preview_share=0.9, seed=2025)
        serve["scenes"] = min(32, len(sids))
        # The same loop with 5% of arrivals being previews of the 32 other scenes of
        # the mix, not resident: compiled on arrival, uploaded with the BVH built on
        # the GPU or on the host.
        if len(scenes) > 32:
            cold_texts = [json.dumps(sc) for sc in scenes[32:]]
            serve["cold"] = {"share": 0.05, "scenes": len(cold_texts)}
            for arm, gpu_bvh in (("gpu_bvh", True), ("host_bvh", False)):
                r = serving.serve(ctx, sids[:32], seconds=min(5.0, a.serve_seconds), rate=200.0, preview_share=0.9,
                                  seed=2026, cold_texts=cold_texts, cold_share=0.05, cold_gpu_bvh=gpu_bvh)
                serve["cold"][arm] = {"cold_preview": r.get("cold_preview"),
                                      "preview_ttfp_ms_p50_p99": [r["preview"]["ttfp_ms_p50"],
                                                                  r["preview"]["ttfp_ms_p99"]],
                                      "msamples_per_s": r["msamples_per_s"],
                                      "upload_calls": r["host_calls"].get("upload")}

    # Scenes that are not resident: the BVH built on the host or on the GPU.
    cold = None
    if not a.no_cold:
        import workloads

        big = sorted(range(len(hosts)), key=lambda k: -len(hosts[k].view()["prims"]))[:2]
        cold = cold_scene_ttfp(ctx, [("mesh stress, 174k triangles", workloads.mesh_stress())]
                               + [(f"mix scene {k}", scenes[k]) for k in big])

    cpu = None
    if dist.rank == 0 and dist.world == 1 and not a.no_cpu_baseline:
        n, secs, kind, threads, used = cpu_sample(scenes, budget_s=15.0)
        cpu = {"value": n / secs / 1e6, "unit": "Msamples/s", "cores": threads, "kind": kind,
               "sample": f"scenes {used} of the workload at spp/16 (~15 s of CPU work), threads=0"}

    if dist.rank == 0:
        ms_per_step = t_max / a.steps
        line = {
            "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": dist.world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32 (f64 accumulation)", "data": "synthetic (seeded scene generators)",
            "config": {"workload": desc, "scenes": len(scenes), "samples_per_step": samples_of(scenes),
                       "primitives": int(sum(len(h.view()["prims"]) for h in hosts)) if len(hosts) <= 64 else None,
                       "progressive": not a.single_pass, "max_pass_spp": 32,
                       "pool_paths": ctx.tuning()["pool_paths"], "block": ctx.tuning()["block"],
                       "autotune": tuned,
                       "mode": ("batched: every scene's passes in one continuous wavefront" if batched
                                else "plain: one scene, its passes overlapping in the wavefront"),
                       "parallelism": f"replicas x{dist.world}",
                       "l2": f"inputs larger than L2: {scene_bytes / 2**20:.0f} MiB of scenes + GBs of per-pass "
                             "radiance and path state rewritten every step (L2 126 MiB)"},
            "e2e": {"value": e2e_value, "unit": "Msamples/s", "h2d_bytes_per_step": scene_bytes,
                    "d2h_bytes_per_step": d2h, "phases_per_step": phase},
            "gpu_launches": launches,
            "clocks": clk,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "plain": plain,
            "serving": serve,
            "cold_scene": cold,
            "invalid_samples": c_st["invalid_samples"],
        }
        print(json.dumps(line), flush=True)
    ctx.close()


def main():
    a = args()
    dist = Dist(a.gpus)
    scenes, desc = workload_scenes(a.workload)
    try:
        if a.impl == "reference":
            run_reference(a, dist, scenes, desc)
        else:
            run_rtg(a, dist, scenes, desc)
    finally:
        dist.barrier()
        dist.close()


if __name__ == "__main__":
    main()
