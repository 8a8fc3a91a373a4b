#!/usr/bin/env python
"""Benchmark: Msamples/s of the B200 path tracer on the batched 64-scene mix, and
on each single-scene configuration (Cornell box, sphere field, triangle mesh)
beside the reference CPU renderer.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl rtg|reference] [--workload mix|cornell|spheres|mesh]

A step renders the whole workload once (every scene to its full spp, progressive
passes as the reference renderer runs them). `value` is samples rendered by all
ranks / the slowest rank's device time (CUDA events on the render stream) with
every scene already resident in HBM; `e2e` is the same metric through the public
API with host buffers: upload of the compiled scenes, the render and the read-back
of every tone-mapped image inside the timed region.

N > 1 runs N independent replicas, one process per GPU: every rank renders the
whole workload (weak scaling) and there is no exchange step. Launched by torchrun
(RANK / WORLD_SIZE in the environment), or, when started directly with --gpus N,
bench.py starts torchrun itself.

`per_config` (and the compact `summary` that ends the line) gives, for the
Cornell box (256^2 x 64 spp, depth 8), the sphere field (512^2 x 128, depth 16)
and the 174k-triangle mesh (1024^2 x 64, depth 12): GPU Msamples/s on device
time and end to end, Mrays/s (closest-hit + shadow rays), the roofline of the
closest-hit kernel, and the reference's own CPU renderer on the same scene file:
its stock command-line renderer (`rt --threads 0 --single-pass`) for the two
scenes its JSON schema expresses, its Renderer::render through oracle/_ref's
harness for the mesh (whose 256x180 torus needs a schema extension).

--impl reference times the reference's own CPU renderer (built from its sources
into oracle/_ref/; the oracle restatement if that binary is absent) on the host
cores, on a bounded sample of the same workload.
"""
import argparse
import json
import math
import os
import re
import socket
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ray-tracer_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "Msamples/s on 1 B200, batched vs plain at matched RMSE; p50/p99 preview latency"
HARNESS = os.path.join(ROOT, "oracle", "_ref", "rt_harness")
RT_CLI = os.path.join(ROOT, "oracle", "_ref", "rt")
L2_BYTES = 126 * 2 ** 20
CONFIGS = ("cornell", "spheres", "mesh")
CONFIG_TAG = {"cornell": "C1", "spheres": "C2", "mesh": "C3"}

# Bytes one closest-hit fetch moves in the device layout (csrc/device/layout.h):
# per node visit, by the closest-hit tree in use (a binary node holds both
# children's boxes: 64 B; a compressed eight-wide node: 80 B); a primitive slot
# is three float4 rows, all fetched by every test (48 B).
NODE_BYTES = {2: 64, 8: 80}
PRIM_BYTES = 48


def args(argv=None):
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
    p.add_argument("--no-configs", action="store_true",
                   help="skip the per-configuration runs (Cornell box, sphere field, mesh)")
    p.add_argument("--no-autotune", action="store_true", help="keep the default pool and block size")
    p.add_argument("--pool", type=int, default=0, help="path slots (implies --no-autotune)")
    p.add_argument("--block", type=int, default=0, help="threads per block: 64, 128, 256 (implies --no-autotune)")
    p.add_argument("--no-probe", action="store_true",
                   help="skip the bandwidth probes (the roofline then uses the HBM figure alone)")
    p.add_argument("--closest-tree", type=int, choices=[2, 8], default=0,
                   help="closest-hit walk: 8 compressed eight-wide tree, 2 binary tree (default: the library's)")
    p.add_argument("--shadow-tree", type=int, choices=[4, 8], default=0,
                   help="any-hit walk: 4 four-wide tree, 8 compressed eight-wide tree (default: the library's)")
    return p.parse_args(argv)


def rounded(x, sig=5):
    """Floats to `sig` significant digits (keeps the one JSON line short)."""
    if isinstance(x, float):
        if not math.isfinite(x) or x == 0.0:
            return x
        return round(x, sig - 1 - int(math.floor(math.log10(abs(x)))))
    if isinstance(x, dict):
        return {k: rounded(v, sig) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [rounded(v, sig) for v in x]
    return x


# ---------------------------------------------------------------------------
# distributed plumbing (replicas)

def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def replica_command(a_gpus: int, argv) -> list:
    """torchrun command that starts `a_gpus` replicas of this benchmark."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={a_gpus}",
            "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.abspath(__file__)] + list(argv)


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
            backend = "gloo"  # only barriers and scalar reductions: no data-path collective
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist
        if want != self.world:
            raise SystemExit(f"--gpus {want} but WORLD_SIZE {self.world}: the replica count must match")

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


def timed_steps(dist, clocks, step, steps):
    """The timed region: barrier, clock sampling, `steps` calls of step() (each
    returns the render's stats), barrier. Device time is summed per rank and the
    max over ranks taken; samples are summed over ranks."""
    dist.barrier()
    if clocks:
        clocks.start()
    dev_ms = samples = rays = launches = 0.0
    for _ in range(steps):
        st = step()
        dev_ms += st["device_ms"]
        samples += st["camera_samples"]
        rays += st["rays"] + st["shadow_rays"]
        launches += st["kernel_launches"]
    dist.barrier()
    clk = clocks.stop() if clocks else None
    return {"t_max_ms": dist.max(dev_ms), "samples": dist.sum(samples), "rays": dist.sum(rays),
            "launches": int(launches), "clocks": clk}


# ---------------------------------------------------------------------------
# workloads

def workload_scenes(name):
    import workloads

    if name == "mix":
        return workloads.batch_mix(), ("batched mix: 64 seeded scenes (spheres 10-2000, meshes 1k-200k tris, "
                                       "facing mirrors), resolutions 128^2-1024^2, spp 16/64/256, depth 8-40")
    return [config_scene(name)], config_desc(name)


def config_scene(name):
    import workloads

    return {"cornell": workloads.cornell, "spheres": workloads.sphere_field, "mesh": workloads.mesh_stress}[name]()


def config_desc(name):
    return {"cornell": "C1 Cornell box 555-unit room, 256x256x64 spp, depth 8, NEE + RR",
            "spheres": "C2 sphere field ~480 spheres + plane, thin lens, 512x512x128 spp, depth 16",
            "mesh": "C3 mesh stress 174k tris (icosphere s6 + 256x180 torus), 1024x1024x64 spp, depth 12"}[name]


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


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


_RT_DONE = re.compile(r"done in ([0-9.eE+-]+) ms, (\d+) rays \(([0-9.eE+-]+) Mrays/s\)")
_RT_THREADS = re.compile(r"spp, (\d+) threads")


def cpu_config(name: str, scene: dict) -> dict:
    """The reference's CPU renderer on one whole configuration, all host cores.
    The stock CLI (`rt <scene> --threads 0 --single-pass`) where the scene file is
    in the reference's schema; its Renderer::render through the harness for the
    mesh, whose torus uses the segments_v extension."""
    w, h, spp = scene["render"]["width"], scene["render"]["height"], scene["render"]["spp"]
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "scene.json")
        with open(path, "w") as f:
            json.dump(scene, f)
        if name != "mesh" and os.path.exists(RT_CLI):
            cmd = [RT_CLI, path, "--threads", "0", "--single-pass", "-o", os.path.join(tmp, "out.ppm")]
            err = subprocess.run(cmd, capture_output=True, text=True, check=True).stderr
            m, th = _RT_DONE.search(err), _RT_THREADS.search(err)
            ms, mrays = float(m.group(1)), float(m.group(3))
            threads, tool = int(th.group(1)), "rt --threads 0 --single-pass (stock CLI, apps/rt_cli.cpp)"
        elif os.path.exists(HARNESS):
            out = json.loads(subprocess.check_output([HARNESS, "bench", path, "--threads", "0"]).decode())
            ms, mrays, threads = out["elapsed_ms"], out["mrays_per_sec"], out["threads"]
            tool = "Renderer::render single pass via oracle/_ref/rt_harness bench --threads 0"
        else:
            n, secs, _, threads = cpu_render(scene, spp)
            return {"value": n / secs / 1e6, "unit": "Msamples/s", "cores": threads, "kind": "port",
                    "sample": "whole configuration, oracle port (reference binary not built)"}
    return {"value": w * h * spp / (ms * 1e3), "unit": "Msamples/s", "mrays_per_s": mrays, "cores": threads,
            "kind": "reference", "cpu": cpu_model(), "elapsed_ms": ms, "tool": tool,
            "sample": "the whole configuration (same scene, resolution, spp and depth)"}


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
        "config": {"workload": desc, "same_config": False,
                   "sample": f"scenes {used} at spp/16 (a bounded sample of the workload: a rate, not the whole "
                             "config), stock Renderer::render via rt_harness bench, threads=0"},
        "cpu_baseline": {"value": value, "unit": "Msamples/s", "cores": threads, "kind": kind, "cpu": cpu_model(),
                         "sample": f"~5 s per step of the workload: scenes {used} at spp/16"},
        "e2e": {"value": value, "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU side: peaks and rooflines

def measured_peaks(ctx, probe=True):
    """HBM copy peak (driver-measured file, else the pool's fallback), plus the
    read bandwidths this GPU shows for an L2-resident buffer, an L1-resident one
    and an HBM-sized one (rtg_probe_read_bandwidth)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        hbm, src = float(json.load(open(p))["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, STREAM-style copy)"
    else:
        hbm, src = 6650.0, "fallback 6.65 TB/s (MEASURED_PEAKS.json absent)"
    if not probe:
        return {"hbm": hbm, "hbm_source": src, "l2": float("inf"), "l1": float("inf"), "probe": "skipped"}
    return {"hbm": hbm, "hbm_source": src,
            "l2": ctx.probe_read_bandwidth(32 << 20, reps=40),
            "l1": ctx.probe_read_bandwidth(64 << 10, reps=200, l1=True),
            "hbm_read_probe": ctx.probe_read_bandwidth(4 << 30, reps=1),
            "probe": "rtg_probe_read_bandwidth: L2 = 32 MiB buffer, L1 bypassed, x40; L1 = 64 KiB per block, "
                     "x200; HBM read = 4 GiB, x1; best of 5 launches"}


def sm_count(dev: int):
    """Streaming multiprocessors of GPU `dev` (None when it cannot be read)."""
    try:
        import torch

        return torch.cuda.get_device_properties(dev).multi_processor_count
    except Exception:
        return None


def ncu_profile(kernel: str, pool_paths: int, tree: int = 2):
    """Per-ray counters of `kernel` from the committed ncu capture of the mix
    (profiles/<kernel>_mix_*.json) at this pool size and closest-hit tree, or None."""
    for fname in sorted(os.listdir(os.path.join(ROOT, "profiles"))):
        if fname.startswith(kernel + "_mix") and fname.endswith(".json"):
            d = json.load(open(os.path.join(ROOT, "profiles", fname)))
            if int(d.get("pool_paths", 0)) != int(pool_paths) or int(d.get("closest_tree", 2)) != int(tree):
                continue
            if "dram_bytes_per_ray" not in d and d.get("rays_per_launch"):
                d["dram_bytes_per_ray"] = d["dram_bytes_per_launch"] / d["rays_per_launch"]
            d["file"] = fname
            return d
    return None


def rooflines(ctx, step, peaks, profile=True):
    """Roofline figures of the closest-hit kernel (k_extend) and the shade kernel
    (k_shade) for one step of a workload: one run with per-kernel CUDA events,
    one with traversal counters.

    k_extend is bounded at three levels; its time cannot be lower than any of
      HBM: the queue traffic that cannot stay on chip (32 B ray read per
           continuing path, 16 B hit write per ray, 64 B state + 16 B radiance
           init per new camera path) / HBM peak;
      L1:  the traversal's fetches (node bytes per visit, 48 B per primitive
           test, from device counters) / aggregate L1 read peak;
      L2:  the L2 bytes an ncu capture of the same kernel measured / L2 peak;
      issue: the warp instructions per ray that capture counted / the SM's
           peak issue rate (4 schedulers per SM, one instruction per clock each,
           at the SM clock sampled during the timed steps).
    The binding level is the `bound`; frac = that level's lower bound on the
    launch time / the measured launch time."""
    ctx.set_tuning(time_kernels=1, count_traversal=0)
    t_st = step()
    ctx.set_tuning(time_kernels=0, count_traversal=1)
    c_st = step()
    ctx.set_tuning(time_kernels=0, count_traversal=0)
    node_bytes = NODE_BYTES.get(ctx.tuning().get("closest_tree", 2), 64)
    launches = max(1, t_st["extend_launches"])
    avg_s = t_st["extend_ms"] / launches / 1e3
    rays = c_st["rays"]
    new_paths = c_st["camera_samples"]
    cont = rays - new_paths
    hbm_b = (cont * 32 + rays * 16 + new_paths * (64 + 16)) / launches
    onchip_b = (c_st["node_visits"] * node_bytes + c_st["prim_tests"] * PRIM_BYTES) / launches
    levels = {"hbm": {"bytes": hbm_b, "peak": peaks["hbm"], "unit": "GB/s"},
              "l1": {"bytes": onchip_b, "peak": peaks["l1"], "unit": "GB/s"}}
    prof = ncu_profile("k_extend", ctx.tuning()["pool_paths"], ctx.tuning().get("closest_tree", 2)) if profile else None
    rays_pl = rays / launches
    if prof and prof.get("l2_bytes_per_ray"):
        levels["l2"] = {"bytes": prof["l2_bytes_per_ray"] * rays_pl, "peak": peaks["l2"], "unit": "GB/s"}
    if prof and prof.get("warp_inst_per_ray") and peaks.get("sms") and peaks.get("sm_mhz"):
        levels["issue"] = {"bytes": prof["warp_inst_per_ray"] * rays_pl,
                           "peak": 4 * peaks["sms"] * peaks["sm_mhz"] / 1e3, "unit": "G warp instructions/s"}
    for v in levels.values():
        v["achieved"] = v["bytes"] / avg_s / 1e9
        v["frac"] = v["achieved"] / v["peak"]
    bound = max(levels, key=lambda k: levels[k]["frac"])
    traffic = prof["dram_bytes_per_ray"] * rays_pl if prof and prof.get("dram_bytes_per_ray") else None
    kernel_total = sum(t_st[k] for k in ("extend_ms", "shade_ms", "shadow_ms", "accumulate_ms", "plan_ms"))
    ext = {
        "kernel": "k_extend (closest-hit BVH traversal + camera-path generation)",
        "bound": bound, "achieved": levels[bound]["achieved"], "peak": levels[bound]["peak"],
        "unit": levels[bound]["unit"], "frac": levels[bound]["frac"], "traffic": traffic,
        "levels": {k: {"achieved": v["achieved"], "peak": v["peak"], "unit": v["unit"], "frac": v["frac"]}
                   for k, v in levels.items()},
        "dram_frac": traffic / avg_s / 1e9 / peaks["hbm"] if traffic else None,
        "avg_launch_ms": avg_s * 1e3, "launches": launches, "rays_per_launch": rays_pl,
        "share_of_kernel_time": t_st["extend_ms"] / kernel_total if kernel_total else None,
        "per_ray": {"nodes": c_st["node_visits"] / max(1, rays), "prim_tests": c_st["prim_tests"] / max(1, rays),
                    "node_bytes": node_bytes},
    }
    if prof:
        ext["ncu"] = {k: prof[k] for k in ("lanes_active", "issue_active", "l1_hit_rate", "l2_hit_rate",
                                           "warp_inst_per_ray", "thread_inst_per_ray") if k in prof}
        if prof.get("warp_inst_per_ray") and prof.get("thread_inst_per_ray"):
            # Useful share of the issue slots: lanes doing work in each issued instruction.
            ext["lane_efficiency"] = prof["thread_inst_per_ray"] / (32 * prof["warp_inst_per_ray"])
        ext["ncu"]["file"] = prof["file"]
    # k_shade streams path state: read 64 B state + 16 B hit per path, write 64 B
    # per continuing path and 48 B per shadow ray (materials and lights stay cached).
    shade_b = (rays * (64 + 16) + cont * 64 + c_st["shadow_rays"] * 48) / max(1, launches)
    shade_s = t_st["shade_ms"] / max(1, launches) / 1e3
    shade = {"kernel": "k_shade", "bound": "hbm", "achieved": shade_b / shade_s / 1e9 if shade_s else None,
             "peak": peaks["hbm"], "unit": "GB/s",
             "frac": shade_b / shade_s / 1e9 / peaks["hbm"] if shade_s else None,
             "avg_launch_ms": shade_s * 1e3}
    kernel_ms = {k: t_st[k] for k in ("extend_ms", "shade_ms", "shadow_ms", "accumulate_ms", "plan_ms")}
    return ext, shade, kernel_ms, c_st


# ---------------------------------------------------------------------------
# GPU side: workloads

class _NoDist:
    """Per-configuration runs happen on each rank alone (no cross-rank reduce)."""
    world = 1

    @staticmethod
    def barrier():
        pass

    @staticmethod
    def max(x):
        return x

    @staticmethod
    def sum(x):
        return x


def render_config(ctx, name, a, peaks):
    """One configuration rendered alone (plain renderer): device-time Msamples/s,
    Mrays/s, end to end through the public API, roofline, reference CPU. One pass
    of all samples, as the reference CLI's --single-pass run it is compared with."""
    import rtg

    scene = config_scene(name)
    host = rtg.parse_scene(json.dumps(scene))
    sid = ctx.upload(host)
    st = ctx.scene_settings(sid)
    opts = rtg.RenderOptions(progressive=False)

    def step():
        ctx.render(sid, st, opts)
        return ctx.stats()

    for _ in range(max(3, a.warmup)):
        step()
    steps = max(3, a.steps)
    t = timed_steps(_NoDist, None, step, steps)
    value = t["samples"] / (t["t_max_ms"] / 1e3) / 1e6
    ext, shade, kernel_ms, c_st = rooflines(ctx, step, peaks, profile=False)
    h2d = ctx.scene_info(sid)["device_bytes"]
    ctx.release(sid)
    # End to end: upload, render, tone-mapped image read-back, release.
    ctx.release(ctx.upload(host))
    t0 = time.perf_counter()
    e2e_samples = 0
    for _ in range(steps):
        i = ctx.upload(host)
        ctx.render(i, st, opts)
        e2e_samples += ctx.stats()["camera_samples"]
        ctx.image(-1, st.width, st.height)
        ctx.release(i)
    e2e = e2e_samples / (time.perf_counter() - t0) / 1e6
    return {"workload": config_desc(name), "passes": "single pass (as the CPU arm's --single-pass)",
            "value": value, "unit": "Msamples/s",
            "ms_per_render": t["t_max_ms"] / steps, "mrays_per_s": t["rays"] / (t["t_max_ms"] / 1e3) / 1e6,
            "e2e": {"value": e2e, "unit": "Msamples/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": st.width * st.height * 3},
            "roofline": ext, "shade_roofline": shade, "kernel_ms": kernel_ms,
            "invalid_samples": c_st["invalid_samples"]}


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
    if a.closest_tree or a.shadow_tree:
        ctx.set_tuning(**({"closest_tree": a.closest_tree} if a.closest_tree else {}),
                       **({"shadow_tree": a.shadow_tree} if a.shadow_tree else {}))
    peaks = measured_peaks(ctx, probe=not a.no_probe)
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
    t = timed_steps(dist, Clocks(dev), step, a.steps)
    t_max = t["t_max_ms"]
    value = t["samples"] / (t_max / 1e3) / 1e6
    mrays = t["rays"] / (t_max / 1e3) / 1e6

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
        if batched:
            ctx.images(range(len(settings)), [(s.width, s.height) for s in settings])
        else:
            ctx.image(-1, settings[0].width, settings[0].height)
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
        pv = p_samples / (p_ms / 1e3) / 1e6
        plain = {"value": pv, "unit": "Msamples/s", "batched_over_plain": value / dist.world / pv,
                 "target_batched_over_plain": 2.0,
                 "rmse": "identical images (bit-identical framebuffers), so matched RMSE by construction"}

    peaks["sm_mhz"] = t["clocks"].get("sm_mhz") or t["clocks"].get("sm_max_mhz")
    peaks["sms"] = sm_count(dev)
    ext, shade, kernel_ms, c_st = rooflines(ctx, step, peaks)

    # Serving: Poisson arrivals of previews and finals over 32 resident scenes.
    serve = None
    if batched and not a.no_serve and a.serve_seconds > 0:
        import serving

        serve = serving.serve(ctx, sids[:32], seconds=a.serve_seconds, rate=200.0, preview_share=0.9, seed=2025)
        serve["scenes"] = min(32, len(sids))
        # The plain renderer on the work serving spends its time on: the same 32
        # scenes, one at a time, in the final-request shape (1024^2, depth 16,
        # progressive), the first 32 samples of each.
        f_ms = f_samples = 0.0
        for i in sids[:32]:
            st = ctx.scene_settings(i)
            st.width, st.height = serving.FINAL.width, serving.FINAL.height
            st.spp, st.max_depth = 32, serving.FINAL.max_depth
            st.rr_min_depth = min(st.rr_min_depth, st.max_depth)
            ctx.render(i, st, rtg.RenderOptions(progressive=True, max_pass_spp=32))
            stt = ctx.stats()
            f_ms += stt["device_ms"]
            f_samples += stt["camera_samples"]
        serve["plain_same_shape"] = {
            "value": f_samples / (f_ms / 1e3) / 1e6, "unit": "Msamples/s",
            "workload": "the 32 served scenes one at a time, 1024^2, 32 spp, depth 16, progressive"}
        serve["served_over_plain_same_shape"] = serve["msamples_per_s"] / serve["plain_same_shape"]["value"]
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
        cpu = {"value": n / secs / 1e6, "unit": "Msamples/s", "cores": threads, "kind": kind, "cpu": cpu_model(),
               "sample": f"scenes {used} of the workload at spp/16 (~15 s of CPU work), threads=0"}

    # Each single-scene configuration, rendered alone, beside the reference CPU.
    per_config = None
    if batched and not a.no_configs:
        for i in sids:
            ctx.release(i)
        sids = []
        per_config = {}
        for name in CONFIGS:
            entry = render_config(ctx, name, a, peaks)
            if dist.rank == 0 and dist.world == 1 and not a.no_cpu_baseline:
                entry["cpu_baseline"] = cpu_config(name, config_scene(name))
                entry["over_cpu"] = entry["value"] / entry["cpu_baseline"]["value"]
                entry["e2e_over_cpu"] = entry["e2e"]["value"] / entry["cpu_baseline"]["value"]
            per_config[CONFIG_TAG[name]] = entry

    if dist.rank == 0:
        ms_per_step = t_max / a.steps
        served = serve["msamples_per_s"] if serve else None
        summary = {"mix": {"value": value, "e2e": e2e_value, "mrays_per_s": mrays,
                           "plain": plain["value"] if plain else None,
                           "batched_over_plain": plain["batched_over_plain"] if plain else None,
                           "served": served,
                           "served_over_plain_mix": served / plain["value"] if served and plain else None,
                           "served_over_plain_same_shape": serve["served_over_plain_same_shape"] if serve else None,
                           "target_2x_plain": "not met" if plain and plain["batched_over_plain"] < 2 else None,
                           "preview_p99_ms": serve["preview"]["ttfp_ms_p99"] if serve else None,
                           "cpu": cpu["value"] if cpu else None},
                   "k_extend": {"bound": ext["bound"], "frac": ext["frac"], "dram_frac": ext["dram_frac"],
                                "levels": {k: v["frac"] for k, v in ext["levels"].items()},
                                **({"lanes_active": ext["ncu"].get("lanes_active"),
                                    "issue_active": ext["ncu"].get("issue_active"),
                                    "lane_efficiency": ext.get("lane_efficiency")} if "ncu" in ext else {})},
                   "k_shade_hbm_frac": shade["frac"]}
        if per_config:
            for tag, e in per_config.items():
                summary[tag] = {"value": e["value"], "e2e": e["e2e"]["value"], "mrays_per_s": e["mrays_per_s"],
                                "cpu": e.get("cpu_baseline", {}).get("value"),
                                "cpu_cores": e.get("cpu_baseline", {}).get("cores"),
                                "over_cpu": e.get("over_cpu"), "extend_bound": e["roofline"]["bound"],
                                "extend_frac": e["roofline"]["frac"]}
        tun = ctx.tuning()
        line = {
            "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": dist.world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32 (f64 accumulation)", "data": "synthetic (seeded scene generators)",
            "mrays_per_s": mrays,
            "config": {"workload": desc, "scenes": len(scenes), "samples_per_step": samples_of(scenes),
                       "primitives": int(sum(len(h.view()["prims"]) for h in hosts)) if len(hosts) <= 64 else None,
                       "progressive": not a.single_pass, "max_pass_spp": 32,
                       "pool_paths": tun["pool_paths"], "block": tun["block"],
                       **{k: tun[k] for k in ("closest_tree", "shadow_tree") if k in tun},
                       "autotune": tuned,
                       "mode": ("batched: every scene's passes in one continuous wavefront" if batched
                                else "plain: one scene, its passes overlapping in the wavefront"),
                       "parallelism": f"replicas x{dist.world} (every rank renders the whole workload)",
                       "l2": f"inputs larger than L2: {scene_bytes / 2**20:.0f} MiB of scenes + GBs of per-pass "
                             "radiance and path state rewritten every step (L2 126 MiB)"},
            "e2e": {"value": e2e_value, "unit": "Msamples/s", "h2d_bytes_per_step": scene_bytes,
                    "d2h_bytes_per_step": d2h, "phases_per_step": phase},
            "gpu_launches": t["launches"],
            "clocks": t["clocks"],
            "roofline": ext,
            "shade_roofline": shade,
            "kernel_ms": kernel_ms,
            "peaks": peaks,
            "cpu_baseline": cpu,
            "plain": plain,
            "invalid_samples": c_st["invalid_samples"],
            "serving": serve,
            "cold_scene": cold,
            "per_config": per_config,
            "summary": summary,
        }
        print(json.dumps(rounded(line)), flush=True)
    ctx.close()


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    a = args(argv)
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # One replica per GPU: start them under torchrun rather than render on one.
        return subprocess.call(replica_command(a.gpus, argv))
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
    return 0


if __name__ == "__main__":
    sys.exit(main())
