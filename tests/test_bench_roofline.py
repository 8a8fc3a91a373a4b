"""bench.py's roofline arithmetic on the CPU, with a stand-in context: the levels
of the closest-hit kernel (HBM queue bytes, L1 fetch bytes, L2 and instruction
issue from the committed counter capture), the bound, the lane efficiency and
the shade figure. No GPU: the stand-in returns fixed stats."""
import json
import os

import pytest

import bench

PROFILE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "profiles",
                       "k_extend_mix_pool8M_counters.json")


class FakeCtx:
    def __init__(self, pool, tree=2):
        self.t = {"pool_paths": pool, "closest_tree": tree, "time_kernels": 0, "count_traversal": 0}

    def set_tuning(self, **kw):
        self.t.update(kw)

    def tuning(self):
        return dict(self.t)


def fake_step(ctx):
    def step():
        st = {"extend_launches": 10, "extend_ms": 5.0, "shade_ms": 3.0, "shadow_ms": 1.5, "accumulate_ms": 0.3,
              "plan_ms": 0.1, "rays": 80_000_000, "camera_samples": 40_000_000, "node_visits": 512_000_000,
              "prim_tests": 320_000_000, "shadow_rays": 25_000_000}
        return st
    return step


PEAKS = {"hbm": 6650.0, "l1": 30000.0, "l2": 17500.0, "sms": 148, "sm_mhz": 1965.0}


def test_levels_bound_and_issue_from_the_capture():
    prof = json.load(open(PROFILE))
    ctx = FakeCtx(prof["pool_paths"])
    ext, shade, kernel_ms, _ = bench.rooflines(ctx, fake_step(ctx), PEAKS)
    avg_s = 5.0 / 10 / 1e3
    rays_pl = 8e6
    # HBM: 32 B per continuing ray read, 16 B hit per ray, 80 B per new path.
    hbm = (40e6 * 32 + 80e6 * 16 + 40e6 * 80) / 10
    assert ext["levels"]["hbm"]["achieved"] == pytest.approx(hbm / avg_s / 1e9)
    assert ext["levels"]["l1"]["achieved"] == pytest.approx((512e6 * 64 + 320e6 * 48) / 10 / avg_s / 1e9)
    assert ext["levels"]["l2"]["achieved"] == pytest.approx(prof["l2_bytes_per_ray"] * rays_pl / avg_s / 1e9)
    issue = prof["warp_inst_per_ray"] * rays_pl / avg_s / 1e9
    assert ext["levels"]["issue"]["achieved"] == pytest.approx(issue)
    assert ext["levels"]["issue"]["peak"] == pytest.approx(4 * 148 * 1965.0 / 1e3)
    assert ext["levels"]["issue"]["unit"] == "G warp instructions/s"
    fracs = {k: v["frac"] for k, v in ext["levels"].items()}
    assert ext["bound"] == max(fracs, key=fracs.get) and ext["frac"] == fracs[ext["bound"]]
    assert ext["unit"] == ext["levels"][ext["bound"]]["unit"]
    assert ext["traffic"] == pytest.approx(prof["dram_bytes_per_ray"] * rays_pl)
    assert ext["lane_efficiency"] == pytest.approx(prof["thread_inst_per_ray"] / (32 * prof["warp_inst_per_ray"]))
    # Shade: 64 B state + 16 B hit read per path, 64 B per continuing path, 48 B per shadow ray.
    sb = (80e6 * 80 + 40e6 * 64 + 25e6 * 48) / 10
    assert shade["achieved"] == pytest.approx(sb / (3.0 / 10 / 1e3) / 1e9)
    assert sum(kernel_ms.values()) == pytest.approx(9.9)


def test_no_capture_for_other_pools_or_trees():
    prof = json.load(open(PROFILE))
    for ctx in (FakeCtx(prof["pool_paths"] // 2), FakeCtx(prof["pool_paths"], tree=8)):
        ext, _, _, _ = bench.rooflines(ctx, fake_step(ctx), PEAKS)
        assert set(ext["levels"]) == {"hbm", "l1"} and ext["traffic"] is None and "ncu" not in ext


def test_issue_level_needs_the_clock():
    prof = json.load(open(PROFILE))
    ctx = FakeCtx(prof["pool_paths"])
    ext, _, _, _ = bench.rooflines(ctx, fake_step(ctx), dict(PEAKS, sm_mhz=None))
    assert "issue" not in ext["levels"] and "l2" in ext["levels"]
