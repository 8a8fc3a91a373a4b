"""Golden data for the scene schema: what the reference's own command-line
renderer says about each scene text of a corpus.

For every case the reference's stock CLI (oracle/_ref/rt, built from the
reference sources) is run on the scene text from stdin, with --validate (the
exact error message, or "" when the scene is accepted) and, for accepted
scenes, with --dump-scene (the normalised JSON, byte for byte). The corpus
covers every typed-field error, every enumeration, every validation rule, the
"(and N more problem(s))" count, the nine shipped assets and the workloads
expressible in the reference's schema.

    python tests/golden/make_scene_schema_golden.py     # writes scene_schema.json

Needs oracle/_ref/rt (make -C oracle ref). REF_DIR locates the reference's
assets (default /root/reference).
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "ray-tracer_b200"))
import workloads  # noqa: E402

RT = os.path.join(ROOT, "oracle", "_ref", "rt")
ASSETS = os.path.join(os.environ.get("REF_DIR", "/root/reference"), "assets", "scenes")

M = '"materials": {"m": {"type": "lambertian"}}'


def obj(fields: str) -> str:
    return "{" + M + ', "objects": [{' + fields + "}]}"


def cases() -> list:
    c = []
    # Top level and record shapes.
    c += ["{}", "[]", "3", '"x"', '{"bogus": 1}', '{"name": "a", "$schema": "s", "description": "d"}',
          '{"name": 3}', '{"camera": 1}', '{"render": []}', '{"background": "x"}', '{"materials": []}',
          '{"materials": {"m": 1}}', '{"objects": {}}', '{"objects": [1]}', '{"lights": {}}', '{"lights": [3]}']
    # Typed fields.
    c += ['{"render": {"width": "a"}}', '{"render": {"width": 1.5}}', '{"render": {"width": 3e9}}',
          '{"render": {"spp": true}}', '{"render": {"light_sampling": 1}}', '{"render": {"use_bvh": "yes"}}',
          '{"render": {"exposure": "hi"}}', '{"render": {"integrator": 1}}', '{"render": {"integrator": "magic"}}',
          '{"render": {"tone_map": "filmic"}}', '{"render": {"tone_map": "reinhard", "integrator": "direct"}}',
          '{"render": {"seed": 4294967297}}', '{"render": {"seed": -5}}', '{"render": {"seed": 7.0}}',
          '{"camera": {"look_from": [1, 2]}}', '{"camera": {"look_from": [1, 2, "x"]}}',
          '{"camera": {"look_from": 5}}', '{"camera": {"vfov": "wide"}}', '{"camera": {"vup": {}}}',
          '{"background": {"type": "sky"}}', '{"background": {"type": "solid", "color": 0.25}}',
          '{"background": {"type": "solid", "top": [9, 9, 9]}}', '{"background": {"bottom": [0, 0, -1]}}',
          '{"background": {"intensity": "x"}}']
    # Render and camera rules.
    for k, v in (("width", 0), ("width", 8193), ("height", 0), ("height", 9000), ("spp", 0), ("spp", 1000001),
                 ("max_depth", 0), ("max_depth", 1001), ("rr_min_depth", -1), ("threads", -1), ("threads", 1025),
                 ("tile_size", 0), ("tile_size", 1025), ("exposure", 0), ("exposure", -1)):
        c.append(json.dumps({"render": {k: v}}))
    c += ['{"camera": {"look_from": [0, 0, 0], "look_at": [0, 0, 0]}}', '{"camera": {"vfov": 0}}',
          '{"camera": {"vfov": 180}}', '{"camera": {"aperture": -1}}', '{"camera": {"focus_dist": -2}}',
          '{"camera": {"vfov": 0, "aperture": -1, "focus_dist": -1}, "render": {"width": 0, "spp": 0}}']
    # Materials.
    c += ['{"materials": {"m": {}}}', '{"materials": {"m": {"type": 4}}}', '{"materials": {"m": {"type": "plastic"}}}',
          '{"materials": {"m": {"type": "diffuse", "albedo": [0.1, 0.2, 0.3], "albedo2": 0.5, "checker_scale": 2}}}',
          '{"materials": {"m": {"type": "lambertian", "albedo": [-1, 0, 0]}}}',
          '{"materials": {"m": {"type": "lambertian", "albedo2": [0, -1, 0]}}}',
          '{"materials": {"m": {"type": "lambertian", "checker_scale": -1}}}',
          '{"materials": {"m": {"type": "metal", "roughness": 2}}}',
          '{"materials": {"m": {"type": "metal", "roughness": -0.5, "albedo": [2, -1, 0]}}}',
          '{"materials": {"m": {"type": "glass", "ior": 0.5}}}', '{"materials": {"m": {"type": "dielectric", "ior": 5}}}',
          '{"materials": {"m": {"type": "dielectric", "tint": [-1, 1, 1]}}}',
          '{"materials": {"m": {"type": "light", "intensity": -1}}}',
          '{"materials": {"m": {"type": "emissive", "color": [1, 1, -1], "two_sided": true}}}',
          '{"materials": {"m": {"type": "emissive", "two_sided": "both"}}}',
          '{"materials": {"": {"type": "lambertian"}}}',
          '{"materials": {"m": {"type": "metal", "roughness": "x"}}}']
    # Objects.
    c += [obj('"material": "m"'), obj('"type": "sphere"'), obj('"type": 3, "material": "m"'),
          obj('"type": "cube", "material": "m"'), obj('"type": "sphere", "material": "m"'),
          obj('"type": "sphere", "center": [0, 0, 0], "material": "nope"'),
          obj('"type": "sphere", "center": [0, 0, 0], "radius": 0, "material": "m"'),
          obj('"type": "sphere", "center": [0, 0, 0], "radius": -1, "material": "nope"'),
          obj('"type": "sphere", "center": [0, 0, 0], "radius": 2, "name": 4, "material": "m"'),
          obj('"type": "sphere", "center": [0, 0, 0], "material": 5'),
          obj('"type": "plane", "normal": [0, 0, 0], "material": "m"'),
          obj('"type": "plane", "point": [0, 1, 0], "material": "m"'),
          obj('"type": "triangle", "v0": [0, 0, 0], "v1": [1, 0, 0], "material": "m"'),
          obj('"type": "triangle", "v0": [0, 0, 0], "v1": [1, 0, 0], "v2": [2, 0, 0], "material": "m"'),
          obj('"type": "quad", "corner": [0, 0, 0], "u": [1, 0, 0], "v": [2, 0, 0], "material": "m"'),
          obj('"type": "quad", "corner": [0, 0, 0], "u": [1, 0, 0], "material": "m"'),
          obj('"type": "box", "min": [0, 0, 0], "max": [1, 0, 1], "material": "m"'),
          obj('"type": "box", "min": [0, 0, 0], "material": "m"'),
          obj('"type": "box", "min": [0, 0, 0], "max": [1, 1, 1], "rotate_y": "x", "material": "m"'),
          obj('"type": "mesh", "source": "cube", "material": "m"'),
          obj('"type": "mesh", "subdivisions": 8, "material": "m"'),
          obj('"type": "mesh", "subdivisions": -1, "material": "m"'),
          obj('"type": "mesh", "subdivisions": 2.5, "material": "m"'),
          obj('"type": "mesh", "source": "torus", "segments": 2, "material": "m"'),
          obj('"type": "mesh", "source": "torus", "segments": 4096, "material": "m"'),
          obj('"type": "mesh", "source": "torus", "major_radius": 0, "material": "m"'),
          obj('"type": "mesh", "source": "torus", "minor_radius": -1, "segments": 64, "material": "m"'),
          obj('"type": "mesh", "source": "obj", "material": "m"'),
          obj('"type": "mesh", "scale": [1, 0, 1], "material": "m"'),
          obj('"type": "mesh", "scale": 0, "translate": [0, 0, 0], "smooth": 1, "material": "m"'),
          obj('"type": "mesh", "source": "torus", "major_radius": 2, "minor_radius": 0.5, "segments": 32, '
              '"smooth": false, "scale": [1, 2, 1], "rotate_y": 30, "translate": [0, 1, 0], "material": "m"'),
          obj('"type": "mesh", "source": "icosphere", "subdivisions": 2, "path": "x.obj", "material": "m"')]
    # Lights.
    c += ['{"lights": [{"type": "spot", "position": [0, 0, 0]}]}', '{"lights": [{"intensity": [1, 1, 1]}]}',
          '{"lights": [{"position": [0, 1, 0], "intensity": [-1, 0, 0]}]}',
          '{"lights": [{"position": [0, 1, 0]}, {"name": "b", "position": [1, 1, 1], "intensity": 3}]}',
          '{"lights": [{"type": 3, "position": [0, 0, 0]}]}']
    # Several problems at once: the first message and the count of the rest.
    c += ['{"render": {"width": 0, "height": 0, "spp": 0, "exposure": 0}, "camera": {"vfov": 200}, '
          '"background": {"top": [-1, 0, 0]}, "materials": {"a": {"type": "metal", "roughness": 3}}, '
          '"objects": [{"type": "sphere", "center": [0, 0, 0], "radius": -1, "material": "zz"}], '
          '"lights": [{"position": [0, 0, 0], "intensity": [-1, -1, -1]}]}',
          obj('"type": "sphere", "center": [0, 0, 0], "radius": -1, "material": "q"}, '
              '{"type": "quad", "corner": [0, 0, 0], "u": [0, 0, 0], "v": [0, 0, 0], "material": "q"')]
    # Whole scenes: workloads in the reference's schema and the shipped assets
    # (those under 16 KB of text, to keep the fixture small).
    c += [json.dumps(workloads.cornell())]
    c += [t for t in (json.dumps(workloads.mix_scene(k)) for k in range(12)) if len(t) < 16384][:3]
    if os.path.isdir(ASSETS):
        texts = [open(os.path.join(ASSETS, n)).read() for n in sorted(os.listdir(ASSETS)) if n.endswith(".json")]
        c += [t for t in texts if len(t) < 16384]
    return c


def reference(text: str) -> dict:
    v = subprocess.run([RT, "-", "--validate"], input=text, capture_output=True, text=True)
    if v.returncode == 0:
        d = subprocess.run([RT, "-", "--dump-scene"], input=text, capture_output=True, text=True, check=True)
        return {"scene": text, "error": "", "dump": d.stdout.rstrip("\n")}
    assert v.returncode == 2, (text, v.returncode, v.stderr)
    msg = v.stderr.strip()
    assert msg.startswith("error: "), msg
    return {"scene": text, "error": msg[len("error: "):], "dump": None}


def main():
    out = [reference(t) for t in cases()]
    with open(os.path.join(HERE, "scene_schema.json"), "w") as f:
        json.dump({"source": "reference rt CLI (--validate / --dump-scene) on each scene text",
                   "cases": out}, f, indent=0)
    bad = sum(1 for c in out if c["error"])
    print(f"{len(out)} cases ({bad} rejected, {len(out) - bad} accepted)")


if __name__ == "__main__":
    main()
