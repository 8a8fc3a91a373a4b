"""Multiple importance sampling (light_sampling = 2, "mis": true in the render
block): next-event estimation and BSDF sampling both count a light, each weighted
by the power heuristic against the other. The reference has no MIS (its
docs/performance.md lists it as future work), so it is checked for what it must
preserve and what it must improve:
* unbiasedness: the analytic answers of the reference's integration tests, and the
  reference's converged 4096-spp images;
* error: lower than NEE alone where area sampling is poor (points close to a
  large area light), at the same sample count.
"""
import json
import os

import numpy as np
import pytest

import rtg
import rtoracle
import workloads
from conftest import GOLDEN
from test_gpu_render import mean_luminance, render, sphere_light_over_plane

pytestmark = pytest.mark.gpu


def with_mis(scene: dict, on: bool = True) -> dict:
    out = json.loads(json.dumps(scene))
    out["render"]["light_sampling"] = True
    out["render"]["mis"] = on
    return out


def test_mis_setting_round_trips(ctx):
    sid = ctx.load_json(json.dumps(with_mis(workloads.cornell(width=8, height=8, spp=1))))
    st = ctx.scene_settings(sid)
    assert st.light_sampling and st.mis
    st.mis = False
    assert rtg.RenderSettings.from_c(st.to_c()).mis is False
    ctx.release(sid)


def test_mis_sphere_light_over_plane_converges_to_analytic(ctx):
    # a * Le * (r/d)^2 = 0.8 * 4 * 0.25 / 4 = 0.2, as with NEE alone.
    prog, s, q, n, stats = render(ctx, with_mis(sphere_light_over_plane(True)))
    assert prog.finished and stats["invalid_samples"] == 0
    assert abs(mean_luminance(s, n) - 0.2) <= 0.01 * 0.2


def test_mis_ball_inside_two_sided_emitter_is_exact(ctx):
    """Inside a sphere light NEE area-samples its surface; the weights of the two
    strategies must still sum to one: L = Le / (1 - albedo) * albedo + Le on the ball."""
    scene = {"camera": {"look_from": [0, 0, 2.5], "look_at": [0, 0, 0], "vfov": 5},
             "render": {"width": 4, "height": 4, "spp": 512, "light_sampling": True, "mis": True},
             "materials": {"ball": {"type": "lambertian", "albedo": 0.6},
                           "shell": {"type": "emissive", "color": 1, "intensity": 2, "two_sided": True}},
             "objects": [{"type": "sphere", "center": [0, 0, 0], "radius": 1, "material": "ball"},
                         {"type": "sphere", "center": [0, 0, 0], "radius": 5, "material": "shell"}]}
    _, s, q, n, _ = render(ctx, scene)
    assert abs(mean_luminance(s, n) - 1.2) <= 0.01 * 1.2


def test_mis_agrees_with_nee_on_cornell(ctx):
    a = workloads.cornell(width=16, height=16, spp=1024)
    _, sa, qa, na, _ = render(ctx, a)
    _, sb, qb, nb, stb = render(ctx, with_mis(a))
    for c in range(3):
        ma, mb = sa[..., c].mean() / 1024, sb[..., c].mean() / 1024
        va = (qa[..., c] / 1024 - (sa[..., c] / 1024) ** 2).clip(0).sum() / 1024 / sa[..., c].size ** 2
        vb = (qb[..., c] / 1024 - (sb[..., c] / 1024) ** 2).clip(0).sum() / 1024 / sb[..., c].size ** 2
        assert abs(ma - mb) <= 3.5 * np.sqrt(va + vb), (c, ma, mb)
    assert stb["invalid_samples"] == 0


@pytest.mark.parametrize("cfg", ["cornell", "mesh"])
def test_mis_against_converged_reference(ctx, cfg):
    """MIS at 64 spp against the reference's 4096-spp NEE image: means within 3
    sigma, and RMSE no worse than NEE's by more than 5%."""
    g = np.load(os.path.join(GOLDEN, f"converged_{cfg}.npz"))
    scene = json.loads(str(g["scene"]))
    spp = int(g["cpu_spp"])
    scene["render"]["spp"] = spp
    ref = g["ref_mean"].astype(np.float64)
    rs = int(g["ref_spp"])
    rmse = {}
    for on in (False, True):
        _, s, q, n, stats = render(ctx, with_mis(scene, on), rtg.RenderOptions(progressive=False))
        img = s / spp
        P = img[..., 0].size
        if on:
            for c in range(3):
                var_g = (q[..., c] / spp - img[..., c] ** 2).clip(0).sum() / spp / P ** 2
                var_r = (g["ref_sumsq"][..., c] / rs - ref[..., c] ** 2).clip(0).sum() / rs / P ** 2
                assert abs(img[..., c].mean() - ref[..., c].mean()) <= 3 * np.sqrt(var_g + var_r) + 1e-12, c
            assert stats["invalid_samples"] == 0
        rmse[on] = np.sqrt(((img - ref) ** 2).mean())
    print(cfg, "rmse nee", rmse[False], "mis", rmse[True])
    assert rmse[True] <= 1.05 * rmse[False]


def near_area_light(mode: str, spp: int) -> dict:
    """A wide emissive quad just above a diffuse floor, seen from between the two:
    for floor points under the light, area sampling's pdf (d^2 / (cos A)) swings
    by orders of magnitude, while cosine-weighted BSDF sampling is nearly ideal.
    mode: "nee", "mis" or "bsdf" (no light sampling)."""
    return {"camera": {"look_from": [0, 0.075, 1.9], "look_at": [0, 0, -2], "vfov": 40},
            "background": {"type": "solid", "color": [0, 0, 0]},
            "render": {"width": 24, "height": 24, "spp": spp, "max_depth": 2, "light_sampling": mode != "bsdf",
                       "mis": mode == "mis", "seed": 3},
            "materials": {"floor": {"type": "lambertian", "albedo": 0.7},
                          "panel": {"type": "emissive", "color": 1, "intensity": 3, "two_sided": True}},
            "objects": [{"type": "plane", "point": [0, 0, 0], "normal": [0, 1, 0], "material": "floor"},
                        {"type": "quad", "corner": [-2, 0.15, -2], "u": [4, 0, 0], "v": [0, 0, 4],
                         "material": "panel"}]}


def test_mis_reduces_error_near_a_large_area_light(ctx):
    """Ground truth from BSDF sampling alone at 4096 spp (bounded samples here, so
    its error estimate holds). At 256 spp, MIS agrees with it pixel by pixel and has
    a much lower RMSE than NEE, whose samples under the panel are heavy-tailed."""
    out = {}
    for mode, spp in (("bsdf", 4096), ("nee", 256), ("mis", 256)):
        _, s, q, n, stats = render(ctx, near_area_light(mode, spp))
        mean = s / spp
        out[mode] = (mean, (q / spp - mean ** 2).clip(0) / spp)  # mean and its variance, per pixel
        assert stats["invalid_samples"] == 0
    truth, var_t = out["bsdf"]
    mis, var_m = out["mis"]
    nee, _ = out["nee"]
    assert (np.abs(mis - truth) <= 4 * np.sqrt(var_m + var_t) + 1e-9).mean() >= 0.99
    rmse_mis = np.sqrt(((mis - truth) ** 2).mean())
    rmse_nee = np.sqrt(((nee - truth) ** 2).mean())
    print("rmse nee", rmse_nee, "mis", rmse_mis)
    assert rmse_mis <= 0.7 * rmse_nee


def _inside_shell():
    return {"camera": {"look_from": [0, 0, 2.5], "look_at": [0, 0, 0], "vfov": 40},
            "render": {"max_depth": 6},
            "materials": {"ball": {"type": "lambertian", "albedo": 0.6},
                          "shell": {"type": "emissive", "color": 1, "intensity": 2, "two_sided": True}},
            "objects": [{"type": "sphere", "center": [0, 0, 0], "radius": 1, "material": "ball"},
                        {"type": "sphere", "center": [0, 0, 0], "radius": 5, "material": "shell"}]}


@pytest.mark.parametrize("name", ["cornell", "sphere_light", "inside_shell", "mesh"])
def test_mis_samples_match_the_oracle_one_by_one(ctx, name):
    """The oracle restates the MIS weights in double (the reference has no MIS):
    with the same RNG streams, every sample's radiance matches the GPU's fp32
    value. Triangle lights (Cornell), a sphere light seen from outside (cone
    sampling), from inside (area sampling), and a point light with a sphere light
    over smooth meshes."""
    scene = {"cornell": lambda: workloads.cornell(width=32, height=32, spp=1),
             "sphere_light": lambda: sphere_light_over_plane(True),
             "inside_shell": _inside_shell,
             "mesh": lambda: workloads.mesh_stress(width=32, height=32, spp=1)}[name]()
    scene["render"].update(width=32, height=32, spp=1, light_sampling=True, mis=True)
    _, s, _, n, stats = render(ctx, scene, rtg.RenderOptions(progressive=False))
    o = rtoracle.OracleScene(rtg.parse_scene(json.dumps(scene)).view())
    assert o.c.light_sampling == 2
    cs, _, _ = o.render()
    err = np.abs(s - cs).max(axis=-1) / np.maximum(1.0, np.abs(cs).max(axis=-1))
    close = err <= 1e-3
    print(name, "samples within 1e-3:", int(close.sum()), "of", close.size, "max error", float(err.max()))
    assert close.mean() >= 0.99
    assert stats["invalid_samples"] == 0
