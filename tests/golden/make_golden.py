"""Generates the golden fixtures in tests/golden/ from the reference renderer.

Runs oracle/_ref/rt_harness (the reference built from its own sources by
oracle/Makefile) on the seeded workloads and stores its outputs as .npz files:

  compile_<cfg>.npz    compiled scene arrays (cornell, spheres) / SHA-256 digests (mesh)
  rng.npz              raw PCG32 streams of Rng::for_sample
  camera_<cfg>.npz     Camera::generate rays for fixed pixel/jitter records
  tonemap.npz          tone_map + linear_to_srgb8 outputs
  render_<name>.npz    small renders: per-pixel sum, sum of squares, stats
  rays_<cfg>.npz       closest hit / brute force / occluded for 4096 seeded rays
  converged_<cfg>.npz  4096-spp mean image and a 64-spp CPU image (with moments)

Usage (needs the reference sources; run in the build container):
    make -C oracle ref && python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "ray-tracer_b200"))
import workloads  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "rt_harness")
TMP = tempfile.mkdtemp(prefix="rtg_golden_")

CONFIGS = {
    "cornell": workloads.cornell,
    "spheres": workloads.sphere_field,
    "mesh": workloads.mesh_stress,
}


def scene_file(name, scene):
    p = os.path.join(TMP, name + ".json")
    with open(p, "w") as f:
        json.dump(scene, f)
    return p


def harness(*args):
    return subprocess.check_output([HARNESS, *map(str, args)]).decode()


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def compile_fixture(cfg, scene):
    prefix = os.path.join(TMP, "c_" + cfg)
    harness("compile", scene_file("c_" + cfg, scene), prefix)
    arrs = {}
    for k, w in (("prims", 24), ("planes", 8), ("nodes", 10), ("materials", 16), ("point_lights", 6)):
        arrs[k] = np.fromfile(f"{prefix}.{k}.f64", dtype=np.float64).reshape(-1, w)
    arrs["background"] = np.fromfile(f"{prefix}.background.f64", dtype=np.float64)
    arrs["order"] = np.fromfile(f"{prefix}.pidx.u32", dtype=np.uint32)
    arrs["lights"] = np.fromfile(f"{prefix}.lights.u32", dtype=np.uint32).reshape(-1, 2)
    info = json.load(open(prefix + ".json"))
    meta = {k: info[k] for k in ("primitives", "planes", "triangles", "spheres", "degenerate_skipped", "lights",
                                 "bvh_nodes", "bvh_leaves", "bvh_max_depth", "bvh_max_leaf", "bvh_sah_cost")}
    if cfg == "mesh":
        out = {f"sha_{k}": np.array(sha(v)) for k, v in arrs.items()}
        out.update({f"shape_{k}": np.array(v.shape) for k, v in arrs.items()})
    else:
        out = dict(arrs)
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(OUT, f"compile_{cfg}.npz"), **out)


def rng_fixture():
    cases = [(1, 0, 0), (1, 2, 3), (7, 123456, 99), (2 ** 31 - 1, 1 << 20, 4095)]
    streams = [np.array(harness("rng", s, p, k, 64).split(), dtype=np.uint32) for s, p, k in cases]
    np.savez_compressed(os.path.join(OUT, "rng.npz"), cases=np.array(cases, dtype=np.uint64), streams=np.stack(streams))


def camera_fixture(cfg, scene):
    rng = np.random.default_rng(17)
    w, h = scene["render"]["width"], scene["render"]["height"]
    n = 512
    pix = np.stack([rng.integers(0, w, n), rng.integers(0, h, n), rng.random(n), rng.random(n)], 1).astype(np.float64)
    pix[:4] = [[0, 0, 0, 0], [w - 1, h - 1, 0.999, 0.999], [w // 2, h // 2, 0, 0], [w // 2, h // 2, 0.5, 0.5]]
    pf = os.path.join(TMP, f"pix_{cfg}.f64")
    pix.tofile(pf)
    of = os.path.join(TMP, f"cam_{cfg}.f64")
    harness("camera", scene_file("cam_" + cfg, scene), pf, of, 4242)
    rays = np.fromfile(of, dtype=np.float64).reshape(-1, 6)
    np.savez_compressed(os.path.join(OUT, f"camera_{cfg}.npz"), pix=pix, pixel_for_rng=np.array(4242), rays=rays)


def tonemap_fixture():
    vals = np.concatenate([np.linspace(-1, 3, 801), [0.0031308, 0.5, 1.0, 1e9, np.nan, np.inf], np.geomspace(1e-6, 1e3, 200)])
    pf = os.path.join(TMP, "tm.f64")
    vals.astype(np.float64).tofile(pf)
    of = os.path.join(TMP, "tm.u8")
    harness("tonemap", pf, of)
    out = np.fromfile(of, dtype=np.uint8).reshape(len(vals), 3, 2, 3)  # [value][op][exposure][channel]
    np.savez_compressed(os.path.join(OUT, "tonemap.npz"), values=vals, srgb8=out, exposures=np.array([1.0, 1.4]))


def render_fixture(name, scene, w, h, spp, *extra):
    scene = json.loads(json.dumps(scene))
    scene["render"].update(width=w, height=h, spp=spp)
    of = os.path.join(TMP, f"r_{name}.f64")
    stats = json.loads(harness("render", scene_file("r_" + name, scene), of, *extra))
    a = np.fromfile(of, dtype=np.float64).reshape(h, w, 6)
    np.savez_compressed(os.path.join(OUT, f"render_{name}.npz"), scene=np.array(json.dumps(scene)),
                        sum=a[..., :3], sumsq=a[..., 3:], stats=np.array(json.dumps(stats)))


def rays_fixture(cfg, scene, view_rays):
    # harness layout: o(3), d(3), tmin, tmax
    r = view_rays.astype(np.float64)
    hr = np.concatenate([r[:, 0:3], r[:, 4:7], r[:, 3:4], r[:, 7:8]], 1)
    rf = os.path.join(TMP, f"rays_{cfg}.f64")
    hr.tofile(rf)
    of = os.path.join(TMP, f"rays_{cfg}_out.f64")
    harness("rays", scene_file("rays_" + cfg, scene), rf, of)
    o = np.fromfile(of, dtype=np.float64).reshape(-1, 16)
    np.savez_compressed(os.path.join(OUT, f"rays_{cfg}.npz"), rays=view_rays.astype(np.float32),
                        hit=o[:, 0].astype(np.int8), t=o[:, 1], prim=o[:, 2].astype(np.int32),
                        is_plane=o[:, 3].astype(np.int8), gn=o[:, 4:7], front=o[:, 7].astype(np.int8),
                        brute_hit=o[:, 8].astype(np.int8), brute_t=o[:, 9], brute_prim=o[:, 10].astype(np.int32),
                        brute_plane=o[:, 11].astype(np.int8), occluded=o[:, 12:15].astype(np.int8),
                        occluded_tmax=np.array([0.5, 5.0, 50.0]), material=o[:, 15].astype(np.int32))


def converged_fixture(cfg, scene, w, h, spp_ref=4096, spp_cpu=64):
    scene = json.loads(json.dumps(scene))
    scene["render"].update(width=w, height=h)
    p = scene_file("conv_" + cfg, scene)
    out = {}
    for tag, spp, seed in (("ref", spp_ref, 9001), ("cpu", spp_cpu, scene["render"].get("seed", 1))):
        of = os.path.join(TMP, f"conv_{cfg}_{tag}.f64")
        stats = json.loads(harness("render", p, of, "--spp", spp, "--seed", seed))
        a = np.fromfile(of, dtype=np.float64).reshape(h, w, 6)
        out[f"{tag}_mean"] = (a[..., :3] / spp).astype(np.float32)
        out[f"{tag}_sumsq"] = a[..., 3:].astype(np.float32)
        out[f"{tag}_spp"] = np.array(spp)
        out[f"{tag}_seed"] = np.array(seed)
        out[f"{tag}_stats"] = np.array(json.dumps(stats))
    out["scene"] = np.array(json.dumps(scene))
    np.savez_compressed(os.path.join(OUT, f"converged_{cfg}.npz"), **out)


def main():
    import rtg  # host compile only (no GPU)

    rng_fixture()
    tonemap_fixture()
    for cfg, make in CONFIGS.items():
        scene = make()
        compile_fixture(cfg, scene)
        camera_fixture(cfg, scene)
        view = rtg.parse_scene(json.dumps(scene)).view()
        rays_fixture(cfg, scene, workloads.random_rays(view, 4096, seed=101))
        print("fixtures for", cfg, flush=True)
    render_fixture("cornell_path", workloads.cornell(), 16, 16, 8)
    render_fixture("cornell_direct", workloads.cornell(), 16, 16, 4, "--integrator", "direct")
    render_fixture("cornell_normals", workloads.cornell(), 16, 16, 2, "--integrator", "normals")
    render_fixture("cornell_bsdf_only", workloads.cornell(), 16, 16, 8, "--no-light-sampling")
    render_fixture("spheres_path", workloads.sphere_field(), 16, 16, 4)
    sb = workloads.sphere_field()
    sb["render"]["use_bvh"] = False
    render_fixture("spheres_brute", sb, 12, 12, 2)
    render_fixture("mesh_path", workloads.mesh_stress(), 12, 12, 2)
    print("render fixtures", flush=True)
    converged_fixture("cornell", workloads.cornell(), 64, 64)
    converged_fixture("spheres", workloads.sphere_field(), 64, 64)
    converged_fixture("mesh", workloads.mesh_stress(), 48, 48)
    print("converged fixtures", flush=True)


if __name__ == "__main__":
    main()
