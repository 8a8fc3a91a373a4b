"""Golden images of the reference's own scene assets (assets/scenes/*.json).

For every shipped scene, the reference renderer (oracle/_ref/rt_harness, built
from the reference's sources by oracle/Makefile) renders it at 64x36 twice: a
converged 8192-spp image and a 64-spp image, each with per-pixel sums of squares.
The scene is stored as its normalised JSON (the library's dump of the parsed
file) with the reduced resolution, so the fixture needs no reference checkout.

    make -C oracle ref && python tests/golden/make_asset_golden.py
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "ray-tracer_b200"))
import rtg  # noqa: E402  (host-side parse and dump only)

OUT = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "rt_harness")
ASSETS = os.path.join(os.environ.get("REF_DIR", "/root/reference"), "assets", "scenes")
W, H = 64, 36
REF_SPP, CPU_SPP, REF_SEED = 8192, 64, 9001


def render(path, spp, seed):
    of = os.path.join(tempfile.mkdtemp(prefix="rtg_assets_"), "out.f64")
    stats = json.loads(subprocess.check_output([HARNESS, "render", path, of, "--spp", str(spp),
                                                "--seed", str(seed)]).decode())
    a = np.fromfile(of, dtype=np.float64).reshape(H, W, 6)
    return a, stats


def main():
    names = sorted(f[:-5] for f in os.listdir(ASSETS) if f.endswith(".json"))
    for name in names:
        scene = json.loads(rtg.dump_scene(open(os.path.join(ASSETS, name + ".json")).read()))
        scene["render"].update(width=W, height=H)
        path = os.path.join(tempfile.mkdtemp(prefix="rtg_assets_"), name + ".json")
        with open(path, "w") as f:
            json.dump(scene, f)
        out = {"scene": np.array(json.dumps(scene))}
        seed = int(scene["render"].get("seed", 1))
        for tag, spp, s in (("ref", REF_SPP, REF_SEED), ("cpu", CPU_SPP, seed)):
            a, stats = render(path, spp, s)
            out[f"{tag}_mean"] = (a[..., :3] / spp).astype(np.float32)
            out[f"{tag}_sumsq"] = a[..., 3:].astype(np.float32)
            out[f"{tag}_spp"] = np.array(spp)
            out[f"{tag}_seed"] = np.array(s)
            out[f"{tag}_stats"] = np.array(json.dumps(stats))
        np.savez_compressed(os.path.join(OUT, f"asset_{name}.npz"), **out)
        print(name, json.loads(str(out["ref_stats"])).get("elapsed_ms"), flush=True)


if __name__ == "__main__":
    main()
