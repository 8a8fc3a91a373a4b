"""GPU rendering through the C ABI: unbiasedness on analytic scenes, statistics
against the oracle and the reference's converged images, determinism, batched ==
plain, the progressive pass schedule and cancellation. Known answers restate the
reference's integration tests (tests/test_render.cpp:27-278)."""
import ctypes
import json
import os
import threading
import time

import numpy as np
import pytest

import rtg
import rtoracle
import workloads
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def render(ctx, scene, opts=None, on_pass=None, cancel=None):
    sid = ctx.load_json(json.dumps(scene))
    st = ctx.scene_settings(sid)
    prog = ctx.render(sid, st, opts or rtg.RenderOptions(), on_pass, cancel)
    s, q, n = ctx.framebuffer_moments(-1, st.width, st.height)
    stats = ctx.stats()
    ctx.release(sid)
    return prog, s, q, n, stats


def mean_luminance(s, n):
    return float((s[..., 1] / n).mean())


def sphere_light_over_plane(nee: bool) -> dict:
    return {"camera": {"look_from": [3, 3, 0], "look_at": [0, 0, 0], "vfov": 0.2},
            "background": {"type": "solid", "color": [0, 0, 0]},
            "render": {"width": 4, "height": 4, "spp": 4096 if nee else 65536, "max_depth": 16,
                       "light_sampling": nee},
            "materials": {"plane": {"type": "lambertian", "albedo": 0.8},
                          "glow": {"type": "emissive", "color": 1, "intensity": 4}},
            "objects": [{"type": "plane", "point": [0, 0, 0], "normal": [0, 1, 0], "material": "plane"},
                        {"type": "sphere", "center": [0, 2, 0], "radius": 0.5, "material": "glow"}]}


@pytest.mark.parametrize("nee,tol", [(True, 0.01), (False, 0.03)])
def test_sphere_light_over_plane_converges_to_analytic(ctx, nee, tol):
    # a * Le * (r/d)^2 = 0.8 * 4 * 0.25 / 4 = 0.2
    prog, s, q, n, stats = render(ctx, sphere_light_over_plane(nee))
    assert prog.finished and stats["invalid_samples"] == 0
    assert abs(mean_luminance(s, n) - 0.2) <= tol * 0.2


@pytest.mark.parametrize("nee", [True, False])
def test_ball_inside_two_sided_emitter_is_exact(ctx, nee):
    scene = {"camera": {"look_from": [0, 0, 2.5], "look_at": [0, 0, 0], "vfov": 5},
             "render": {"width": 4, "height": 4, "spp": 512, "light_sampling": nee},
             "materials": {"ball": {"type": "lambertian", "albedo": 0.6},
                           "shell": {"type": "emissive", "color": 1, "intensity": 2, "two_sided": True}},
             "objects": [{"type": "sphere", "center": [0, 0, 0], "radius": 1, "material": "ball"},
                         {"type": "sphere", "center": [0, 0, 0], "radius": 5, "material": "shell"}]}
    _, s, q, n, _ = render(ctx, scene)
    assert abs(mean_luminance(s, n) - 1.2) <= 0.01 * 1.2


def test_uniform_sky_over_diffuse_plane(ctx):
    scene = sphere_light_over_plane(True)
    scene["objects"].pop()
    scene["background"] = {"type": "solid", "color": [0.5, 0.5, 0.5]}
    scene["render"]["spp"] = 2048
    _, s, q, n, _ = render(ctx, scene)
    assert abs(mean_luminance(s, n) - 0.4) <= 0.02 * 0.4


def test_light_sampling_and_bsdf_sampling_agree(ctx):
    a = workloads.cornell(width=16, height=16, spp=1024)
    b = json.loads(json.dumps(a))
    b["render"]["light_sampling"] = False
    _, sa, _, na, _ = render(ctx, a)
    _, sb, _, nb, _ = render(ctx, b)
    la, lb = mean_luminance(sa, na), mean_luminance(sb, nb)
    assert abs(la - lb) <= 0.04 * lb, (la, lb)


def test_point_light_inverse_square_and_hard_shadow(ctx):
    """Direct integrator, one sample straight down: L = albedo/pi * I/d^2 = 2/pi."""
    scene = {"camera": {"look_from": [0, 1, 0], "look_at": [0, 0, 0], "vup": [0, 0, 1], "vfov": 0.01},
             "render": {"width": 1, "height": 1, "spp": 1, "integrator": "direct"},
             "background": {"type": "solid", "color": [0, 0, 0]},
             "materials": {"white": {"type": "lambertian", "albedo": 1}},
             "objects": [{"type": "plane", "point": [0, 0, 0], "normal": [0, 1, 0], "material": "white"}],
             "lights": [{"type": "point", "position": [0, 2, 0], "intensity": [8, 8, 8]}]}
    _, s, _, n, _ = render(ctx, scene)
    assert abs(s[0, 0, 0] - 2 / np.pi) <= 1e-4
    scene["camera"]["look_from"] = [0, 0.5, 0]
    scene["objects"].append({"type": "sphere", "center": [0, 1, 0], "radius": 0.2, "material": "white"})
    _, s, _, n, _ = render(ctx, scene)
    assert s[0, 0, 0] == 0


def test_matches_oracle_statistics_on_the_same_samples(ctx):
    scene = workloads.cornell(width=48, height=48, spp=64)
    _, s, q, n, stats = render(ctx, scene)
    o = rtoracle.OracleScene(rtg.parse_scene(json.dumps(scene)).view())
    cs, cq, cst = o.render()
    spp = 64
    for c in range(3):
        g, m = s[..., c].mean() / spp, cs[..., c].mean() / spp
        var_g = (q[..., c] / spp - (s[..., c] / spp) ** 2).sum() / spp / s[..., c].size ** 2
        var_c = (cq[..., c] / spp - (cs[..., c] / spp) ** 2).sum() / spp / cs[..., c].size ** 2
        assert abs(g - m) <= 3 * np.sqrt(var_g + var_c), (c, g, m)
    assert stats["invalid_samples"] == 0
    # Same workload: the GPU traces as many closest-hit rays as the CPU within noise.
    assert abs(stats["rays"] - cst["rays"]) <= 0.02 * cst["rays"]


@pytest.mark.parametrize("make,depth", [(workloads.cornell, 8), (workloads.sphere_field, 16),
                                        (workloads.mesh_stress, 12)])
def test_samples_match_the_oracle_one_by_one(ctx, make, depth):
    """Same RNG streams, same draws: the GPU's fp32 radiance of each sample equals
    the oracle's double radiance (the reference's path_trace restated), sample by
    sample. At 1 spp each pixel holds one sample; 1024 samples per scene. A path
    may rarely take another branch where fp32 and double round to opposite sides
    of a decision (Russian roulette against its threshold, a Fresnel draw, an edge)."""
    scene = make(width=32, height=32, spp=1, max_depth=depth)
    _, s, _, n, stats = render(ctx, scene, rtg.RenderOptions(progressive=False))
    o = rtoracle.OracleScene(rtg.parse_scene(json.dumps(scene)).view())
    cs, _, _ = o.render()
    err = np.abs(s - cs).max(axis=-1) / np.maximum(1.0, np.abs(cs).max(axis=-1))
    close = err <= 1e-3
    print(make.__name__, "samples within 1e-3:", int(close.sum()), "of", close.size, "max error", float(err.max()))
    assert close.mean() >= 0.99
    assert stats["invalid_samples"] == 0


@pytest.mark.parametrize("cfg", ["cornell", "spheres", "mesh"])
def test_rmse_against_converged_reference_matches_cpu(ctx, cfg):
    """GPU at 64 spp vs the reference's 4096-spp image: per-channel mean within 3
    sigma of the Monte Carlo error, and RMSE within 5% of the CPU image's RMSE."""
    g = np.load(os.path.join(GOLDEN, f"converged_{cfg}.npz"))
    scene = json.loads(str(g["scene"]))
    scene["render"]["spp"] = int(g["cpu_spp"])
    scene["render"]["seed"] = int(g["cpu_seed"])
    _, s, q, n, stats = render(ctx, scene, rtg.RenderOptions(progressive=False))
    spp = int(g["cpu_spp"])
    gpu = s / spp
    ref, cpu = g["ref_mean"].astype(np.float64), g["cpu_mean"].astype(np.float64)
    rs = int(g["ref_spp"])
    P = gpu[..., 0].size
    for c in range(3):
        var_g = (q[..., c] / spp - gpu[..., c] ** 2).clip(0).sum() / spp / P ** 2
        var_r = (g["ref_sumsq"][..., c] / rs - ref[..., c] ** 2).clip(0).sum() / rs / P ** 2
        assert abs(gpu[..., c].mean() - ref[..., c].mean()) <= 3 * np.sqrt(var_g + var_r) + 1e-12, c
    rmse_gpu = np.sqrt(((gpu - ref) ** 2).mean())
    rmse_cpu = np.sqrt(((cpu - ref) ** 2).mean())
    print(cfg, "rmse gpu", rmse_gpu, "cpu", rmse_cpu)
    assert abs(rmse_gpu / rmse_cpu - 1) <= 0.05
    assert stats["invalid_samples"] == 0


def test_bit_identical_across_runs_and_seeds_differ(ctx):
    scene = workloads.sphere_field(width=64, height=48, spp=8)
    a = render(ctx, scene)
    b = render(ctx, scene, rtg.RenderOptions(progressive=True, max_pass_spp=2))
    assert a[1].tobytes() == b[1].tobytes() and a[2].tobytes() == b[2].tobytes()
    scene["render"]["seed"] = 99
    c = render(ctx, scene)
    assert a[1].tobytes() != c[1].tobytes()


def test_batch_is_bit_identical_to_plain(ctx):
    scenes = [workloads.cornell(width=40, height=32, spp=6), workloads.sphere_field(width=24, height=24, spp=11),
              workloads.mesh_stress(width=16, height=20, spp=5), workloads.mix_scene(4)]
    scenes[3]["render"].update(width=20, height=20, spp=3)
    sids = [ctx.load_json(json.dumps(s)) for s in scenes]
    settings = [ctx.scene_settings(i) for i in sids]
    plain = []
    for sid, st in zip(sids, settings):
        ctx.render(sid, st)
        plain.append(ctx.framebuffer_moments(-1, st.width, st.height))
    progs = ctx.render_batch(sids, settings)
    assert all(p.finished for p in progs)
    for j, st in enumerate(settings):
        s, q, n = ctx.framebuffer_moments(j, st.width, st.height)
        assert s.tobytes() == plain[j][0].tobytes() and q.tobytes() == plain[j][1].tobytes(), j
        assert (n == st.spp).all()
    # A different batch composition leaves each job's result unchanged.
    ctx.render_batch(sids[::-1], settings[::-1])
    s, q, n = ctx.framebuffer_moments(len(sids) - 1, settings[0].width, settings[0].height)
    assert s.tobytes() == plain[0][0].tobytes()
    for sid in sids:
        ctx.release(sid)


def test_progressive_pass_schedule(ctx):
    scene = workloads.cornell(width=32, height=32, spp=20)
    seen = []

    def on_pass(p):
        seen.append(p.spp_done)
        _, _, n = ctx.framebuffer_moments(-1, 32, 32)
        assert (n == p.spp_done).all()

    prog, s, q, n, _ = render(ctx, scene, rtg.RenderOptions(progressive=True, max_pass_spp=8), on_pass)
    assert seen == [1, 2, 4, 8, 16, 20] and prog.finished and prog.pass_ == 6


def test_cancellation_stops_quickly_and_leaves_a_consistent_buffer(ctx):
    scene = workloads.cornell(width=128, height=128, spp=100000)
    flag = ctypes.c_int32(0)
    calls = []
    timer = threading.Timer(0.15, lambda: setattr(flag, "value", 1))
    t0 = time.time()
    timer.start()
    prog, s, q, n, _ = render(ctx, scene, None, lambda p: calls.append(p.spp_done), flag)
    elapsed = time.time() - t0
    timer.join()
    assert prog.cancelled and not prog.finished
    assert elapsed < 0.15 + 1.0
    assert calls and (n == prog.spp_done).all()
    assert np.isfinite(s).all()
    # The context stays usable: a small render afterwards completes.
    prog2, *_ = render(ctx, workloads.cornell(width=16, height=16, spp=4))
    assert prog2.finished and not prog2.cancelled


@pytest.mark.parametrize("integ", ["direct", "normals"])
@pytest.mark.parametrize("make", [workloads.cornell, workloads.mesh_stress])
def test_direct_and_normals_samples_match_the_oracle_one_by_one(ctx, make, integ):
    """The direct (Whitted) and normals integrators sample by sample against the
    oracle's restatement of the reference (src/rendering/integrator.cpp:141-198),
    with the same RNG streams: at 1 spp each pixel holds one sample. The mesh
    scene has a point light and an emissive sphere (cone sampling), rough metal
    (recursion with a fuzz draw) and glass (the deterministic Fresnel split).
    Normals must agree to 1e-4 except where a primary ray meets two surfaces at
    the same distance (a box edge), which decides by rounding."""
    scene = make(width=32, height=32, spp=1)
    scene["render"]["integrator"] = integ
    _, s, _, n, stats = render(ctx, scene, rtg.RenderOptions(progressive=False))
    o = rtoracle.OracleScene(rtg.parse_scene(json.dumps(scene)).view())
    cs, _, _ = o.render()
    if integ == "normals":
        close = np.abs(s - cs).max(-1) <= 1e-4
        bar = 0.998
    else:
        err = np.abs(s - cs).max(axis=-1) / np.maximum(1.0, np.abs(cs).max(axis=-1))
        close = err <= 1e-3
        bar = 0.99
    print(make.__name__, integ, "samples that agree:", int(close.sum()), "of", close.size)
    assert close.mean() >= bar
    assert stats["invalid_samples"] == 0


def test_normals_and_direct_integrators_match_oracle(ctx):
    for integ in ("normals", "direct"):
        scene = workloads.cornell(width=32, height=32, spp=4)
        scene["render"]["integrator"] = integ
        _, s, q, n, stats = render(ctx, scene)
        o = rtoracle.OracleScene(rtg.parse_scene(json.dumps(scene)).view())
        cs, cq, _ = o.render()
        gpu, cpu = s / 4, cs / 4
        if integ == "normals":
            close = np.abs(gpu - cpu).max(-1) <= 1e-4
            assert close.mean() >= 0.98, close.mean()
        else:
            assert np.allclose(gpu.mean((0, 1)), cpu.mean((0, 1)), rtol=0.02)
        assert stats["invalid_samples"] == 0


def test_image_is_the_reference_tone_map_of_the_means(ctx):
    scene = workloads.sphere_field(width=48, height=40, spp=4)
    sid = ctx.load_json(json.dumps(scene))
    st = ctx.scene_settings(sid)
    ctx.render(sid, st)
    mean = ctx.framebuffer_mean(-1, st.width, st.height)
    for tm, op in (("clamp", 0), ("reinhard", 1), ("aces", 2)):
        img = ctx.image(-1, st.width, st.height, tm, 1.3)
        ref = rtoracle.tone_map_srgb8(mean.reshape(-1, 3), op, 1.3).reshape(img.shape)
        diff = np.abs(img.astype(int) - ref.astype(int))
        assert diff.max() <= 1 and (diff > 0).mean() <= 1e-3, tm
    ctx.release(sid)


@pytest.mark.parametrize("make", [workloads.cornell, workloads.sphere_field, workloads.mesh_stress])
def test_workloads_render_with_no_invalid_samples(ctx, make):
    scene = make()
    scene["render"].update(width=64, height=64, spp=8)
    prog, s, q, n, stats = render(ctx, scene)
    assert prog.finished and stats["invalid_samples"] == 0 and np.isfinite(s).all() and s.max() > 0


def test_batch_upload_renders_like_single_uploads(ctx):
    """rtg_scene_upload_batch flattens its scenes concurrently (the largest first, each
    with its own share of threads) and stages them in pieces: every part of every
    scene's device layout is byte-identical to a single upload's, and so are renders.
    The scenes span the thread shares: 174k primitives, 82k and small ones."""
    scenes = [workloads.cornell(width=24, height=24, spp=3), workloads.mesh_stress(width=16, height=16, spp=2),
              workloads.mix_scene(5), workloads.mix_scene(1)]
    for k in (2, 3):
        scenes[k]["render"].update(width=16, height=16, spp=2)
    hosts = [rtg.parse_scene(json.dumps(s)) for s in scenes]
    single = [ctx.upload(h) for h in hosts]
    many = ctx.upload_many(hosts)
    assert len(set(single + many)) == 8
    assert ctx.scene_info(single[3])["primitives"] > 32768
    for a, b in zip(single, many):
        for part in rtg.LAYOUT_PARTS:
            assert ctx.scene_layout(a, part).tobytes() == ctx.scene_layout(b, part).tobytes(), part
        st = ctx.scene_settings(a)
        assert ctx.scene_info(a)["primitives"] == ctx.scene_info(b)["primitives"]
        ctx.render(a, st)
        ra = ctx.framebuffer_moments(-1, st.width, st.height)[0]
        ctx.render(b, st)
        rb = ctx.framebuffer_moments(-1, st.width, st.height)[0]
        assert ra.tobytes() == rb.tobytes()
    for i in single + many:
        ctx.release(i)


def _invalid_scene(kind: str, intensity: float) -> dict:
    """Every camera path ends on an emitter whose fp32 emission overflows to inf
    (intensity 1e38 times colour 10): seen directly ("inf") or through a red
    mirror ("nan": inf times the zero green and blue throughput)."""
    scene = {"camera": {"look_from": [0, 0, 0], "look_at": [0, 0, -1], "vfov": 30},
             "render": {"width": 16, "height": 12, "spp": 3, "max_depth": 4},
             "background": {"type": "solid", "color": [0, 0, 0]},
             "materials": {"hot": {"type": "emissive", "color": 10, "intensity": intensity, "two_sided": True},
                           "red_mirror": {"type": "metal", "albedo": [1, 0, 0], "roughness": 0}},
             "objects": [{"type": "sphere", "center": [0, 0, 0], "radius": 50, "material": "hot"}]}
    if kind == "nan":
        scene["objects"].append({"type": "quad", "corner": [-20, -20, -2], "u": [40, 0, 0], "v": [0, 40, 0],
                                 "material": "red_mirror"})
    return scene


@pytest.mark.parametrize("integ", ["path", "direct"])
@pytest.mark.parametrize("kind", ["inf", "nan"])
def test_invalid_samples_are_counted_and_recorded_black(ctx, kind, integ):
    """The reference's invalid-sample rule (src/rendering/renderer.cpp:39-44): a
    non-finite or negative sample is counted in invalid_samples and added as
    black, so the pixel keeps its sample count and stays finite. Here every
    sample is non-finite on the GPU, through the path and the direct integrator."""
    scene = _invalid_scene(kind, 1e38)
    scene["render"]["integrator"] = integ
    prog, s, q, n, stats = render(ctx, scene)
    w, h, spp = 16, 12, 3
    assert prog.finished
    assert stats["invalid_samples"] == w * h * spp
    assert (n == spp).all() and np.isfinite(s).all() and np.isfinite(q).all()
    assert (s == 0).all()
    # The same scene with a finite emission: no invalid sample, every pixel lit.
    prog, s, q, n, stats = render(ctx, _invalid_scene(kind, 1e30))
    assert stats["invalid_samples"] == 0 and np.isfinite(s).all() and (s[..., 0] > 0).all()


def test_eight_wide_walk_renders_the_same_samples(ctx):
    """The wavefront with the compressed eight-wide tree for closest and any hit
    gives the default walk's samples: the walks differ only in which of two
    primitives at exactly the same distance they report."""
    scene = workloads.mesh_stress(width=32, height=32, spp=1)
    opts = rtg.RenderOptions(progressive=False)
    _, s2, _, _, st2 = render(ctx, scene, opts)
    ctx.set_tuning(closest_tree=8, shadow_tree=8)
    try:
        _, s8, _, _, st8 = render(ctx, scene, opts)
    finally:
        ctx.set_tuning(closest_tree=2, shadow_tree=4)
    err = np.abs(s8 - s2).max(-1) / np.maximum(1.0, np.abs(s2).max(-1))
    assert np.mean(err <= 1e-4) >= 0.999, np.mean(err <= 1e-4)
    assert st8["invalid_samples"] == 0 and abs(st8["rays"] - st2["rays"]) <= 0.001 * st2["rays"]


def test_counting_instances_render_identical_images(ctx):
    """count_traversal switches the wavefront to kernel instances that also count
    node visits and primitive tests. The hit tests, slab set-up and camera ray have
    their rounding pinned in the source (explicit FMAs, unfused products), so those
    instances find the same hits to the bit: framebuffers identical with counting on
    and off. The batch mixes BVH scenes with a brute-force job (use_bvh false)."""
    brute = workloads.sphere_field(width=24, height=24, spp=5)
    brute["render"]["use_bvh"] = False
    scenes = [workloads.cornell(width=40, height=32, spp=6), workloads.mesh_stress(width=24, height=20, spp=4),
              brute, workloads.mix_scene(4)]
    scenes[3]["render"].update(width=20, height=20, spp=3)
    sids = [ctx.load_json(json.dumps(s)) for s in scenes]
    settings = [ctx.scene_settings(i) for i in sids]

    def run(count):
        ctx.set_tuning(count_traversal=count)
        try:
            progs = ctx.render_batch(sids, settings)
        finally:
            ctx.set_tuning(count_traversal=0)
        assert all(p.finished for p in progs)
        return ctx.stats(), [ctx.framebuffer_moments(j, s.width, s.height) for j, s in enumerate(settings)]

    st0, fb0 = run(0)
    st1, fb1 = run(1)
    for j, (a, b) in enumerate(zip(fb0, fb1)):
        assert a[0].tobytes() == b[0].tobytes() and a[1].tobytes() == b[1].tobytes(), j
    assert st0["rays"] == st1["rays"] and st0["shadow_rays"] == st1["shadow_rays"]
    assert st1["node_visits"] > 0 and st1["prim_tests"] > 0
    for sid in sids:
        ctx.release(sid)


def test_images_of_a_batch_equal_the_single_image_reads(ctx):
    """rtg_images_rgb8 (one transfer for several jobs) gives each job exactly the
    bytes rtg_image_rgb8 gives it: with every job's own tone map and exposure
    (a normals job included, shown unmapped), with an explicit operator, and for a
    subset of the jobs in another order."""
    scenes = [workloads.cornell(width=40, height=32, spp=4), workloads.sphere_field(width=24, height=20, spp=3),
              workloads.mesh_stress(width=16, height=16, spp=2)]
    scenes[1]["render"].update(tone_map="reinhard", exposure=1.5)
    scenes[2]["render"]["integrator"] = "normals"
    sids = [ctx.load_json(json.dumps(s)) for s in scenes]
    settings = [ctx.scene_settings(i) for i in sids]
    ctx.render_batch(sids, settings)
    sizes = [(s.width, s.height) for s in settings]
    for tm, ex in ((None, 1.0), ("aces", 0.7)):
        single = [ctx.image(j, w, h, tone_map=tm, exposure=ex) for j, (w, h) in enumerate(sizes)]
        many = ctx.images(range(3), sizes, tone_map=tm, exposure=ex)
        for a, b in zip(single, many):
            assert a.tobytes() == b.tobytes()
    sub = ctx.images([2, 0], [sizes[2], sizes[0]])
    assert sub[0].tobytes() == ctx.image(2, *sizes[2]).tobytes()
    assert sub[1].tobytes() == ctx.image(0, *sizes[0]).tobytes()
    assert ctx.images([], []) == []
    # A job index past the batch is an error, with either tone-map source, and the
    # context stays usable.
    for tm in (None, "clamp"):
        with pytest.raises(rtg.RtgError):
            ctx.images([0, 7], [sizes[0], (4, 4)], tone_map=tm)
    assert ctx.images([1], [sizes[1]])[0].tobytes() == ctx.image(1, *sizes[1]).tobytes()
    for sid in sids:
        ctx.release(sid)
