"""The reference's own scene assets (assets/scenes/*.json: Cornell boxes, glass and
metal, emissive glow, the direct-lit first light, materials, meshes, facing
mirrors at depth 40, soft shadows, the sphere field), rendered on the GPU at 64x36
and 64 spp against the reference renderer's images of the same scenes (fixtures
from tests/golden/make_asset_golden.py):
* no invalid samples (the reference's tests/test_render.cpp:173-193 asks the same
  of every asset);
* per-channel means within 3 sigma of the reference's converged 8192-spp image,
  with the next-event estimator and with MIS;
* RMSE against that image within 10% of the reference CPU's own 64-spp image.
"""
import json
import os

import numpy as np
import pytest

import rtg
from conftest import GOLDEN
from test_gpu_render import render

pytestmark = pytest.mark.gpu

NAMES = sorted(f[len("asset_"):-len(".npz")] for f in os.listdir(GOLDEN) if f.startswith("asset_"))


def test_all_assets_have_fixtures():
    assert len(NAMES) == 9


@pytest.mark.parametrize("mis", [False, True])
@pytest.mark.parametrize("name", NAMES)
def test_reference_asset_matches_reference_images(ctx, name, mis):
    g = np.load(os.path.join(GOLDEN, f"asset_{name}.npz"))
    scene = json.loads(str(g["scene"]))
    spp = int(g["cpu_spp"])
    scene["render"]["spp"] = spp
    scene["render"]["seed"] = int(g["cpu_seed"])
    if mis:
        scene["render"]["mis"] = True
    _, s, q, n, stats = render(ctx, scene, rtg.RenderOptions(progressive=False))
    assert stats["invalid_samples"] == 0
    gpu = s / spp
    ref = g["ref_mean"].astype(np.float64)
    rs = int(g["ref_spp"])
    P = gpu[..., 0].size
    for c in range(3):
        var_g = (q[..., c] / spp - gpu[..., c] ** 2).clip(0).sum() / spp / P ** 2
        var_r = (g["ref_sumsq"][..., c] / rs - ref[..., c] ** 2).clip(0).sum() / rs / P ** 2
        assert abs(gpu[..., c].mean() - ref[..., c].mean()) <= 3 * np.sqrt(var_g + var_r) + 1e-12, (name, c)
    if not mis:
        rmse_gpu = np.sqrt(((gpu - ref) ** 2).mean())
        rmse_cpu = np.sqrt(((g["cpu_mean"].astype(np.float64) - ref) ** 2).mean())
        print(name, "rmse gpu", rmse_gpu, "cpu", rmse_cpu)
        assert rmse_gpu <= 1.10 * rmse_cpu + 1e-9, (rmse_gpu, rmse_cpu)
