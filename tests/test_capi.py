"""The C-ABI library: it loads, exports every entry point include/rtg.h declares,
and its host-only paths (validation, dump, PNG) behave like the reference's."""
import os
import re

import numpy as np
import pytest

import rtg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "rtg.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rtg_[a-z0-9_]+)\s*\(", text)) - {"rtg_pass_fn"})


def test_library_exports_every_declared_symbol():
    L = rtg.lib()
    names = declared_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    # The Python mirror binds exactly the declared entry points.
    assert set(rtg.exported_symbols()) == set(names)


def test_product_path_has_no_fallback(monkeypatch):
    """Without the shared library the package refuses to work (no CPU fallback)."""
    monkeypatch.setattr(rtg, "_lib", None)
    monkeypatch.setattr(rtg, "LIB_PATH", "/nonexistent/librtg.so")
    with pytest.raises(RuntimeError, match="missing"):
        rtg.lib()


def test_validate_reports_field_paths():
    mat = '"materials": {"m": {"type": "lambertian"}}'
    cases = [
        ('{' + mat + ', "objects": [{"type": "sphere", "center": [0,0,0], "radius": -1, "material": "m"}]}',
         "objects[0].radius"),
        ('{' + mat + ', "objects": [{"type": "sphere", "center": [0,0,0], "material": "nope"}]}',
         "unknown material 'nope'"),
        ('{' + mat + ', "objects": [{"type": "cube", "material": "m"}]}', "unknown object type"),
        ('{' + mat + ', "objects": [{"type": "sphere", "center": [0,0], "material": "m"}]}', "objects[0].center"),
        ('{"render": {"width": 0}}', "render.width"),
        ('{"render": {"spp": 1.5}}', "render.spp"),
        ('{"render": {"integrator": "magic"}}', "render.integrator"),
        ('{"camera": {"look_from": [0,0,0], "look_at": [0,0,0]}}', "must differ"),
        ('{"camera": {"vfov": 180}}', "camera.vfov"),
        ('{"materials": {"g": {"type": "dielectric", "ior": 0.5}}}', "materials.g.ior"),
        ('{"materials": {"g": {"type": "metal", "roughness": 2}}}', "roughness"),
        ('{"materials": {"g": {"type": "lambertian", "albedo": [-1, 0, 0]}}}', ">= 0"),
        ('{"bogus": 1}', "unknown top-level key"),
        ('{' + mat + ', "objects": [{"type": "quad", "corner": [0,0,0], "u": [1,0,0], "v": [2,0,0], "material": "m"}]}',
         "degenerate"),
        ('{' + mat + ', "objects": [{"type": "mesh", "source": "icosphere", "subdivisions": 12, "material": "m"}]}',
         "subdivisions"),
        ("not json", "JSON parse error"),
    ]
    for text, needle in cases:
        assert needle in rtg.validate_scene(text), (text, rtg.validate_scene(text))
    ok = '{' + mat + ', "objects": [{"type": "sphere", "center": [0,0,0], "material": "m"}]}'
    assert rtg.validate_scene(ok) == ""


def test_json_errors_carry_positions():
    assert "line 1" in rtg.validate_scene('{"a": 1,}')
    assert "line 2" in rtg.validate_scene('{\n  "a" 1}')
    for bad in ["", "[", '{"a":}', "01", "1.", "-", '"abc', "[1 2]", "tru", '{"a":1}x', '"\\x"', '"\\ud800"',
                '{"a":1,"a":2}', "1e999", '"\x01"']:
        assert "JSON parse error" in rtg.validate_scene(bad), bad
    assert "nesting" in rtg.validate_scene("[" * 1000)


def test_defaults_produce_a_valid_empty_scene():
    s = rtg.parse_scene("{}")
    v = s.view()
    assert v["settings"].width == 640 and v["settings"].height == 360 and v["settings"].spp == 64
    assert len(v["prims"]) == 0 and len(v["nodes"]) == 0


def test_dump_round_trips():
    import json

    import workloads

    for scene in (workloads.cornell(), workloads.sphere_field(), workloads.mesh_stress()):
        text = json.dumps(scene)
        dumped = rtg.dump_scene(text)
        assert rtg.dump_scene(dumped) == dumped  # the normalised form is a fixed point
        a, b = rtg.parse_scene(text).view(), rtg.parse_scene(dumped).view()
        for k in ("prims", "nodes", "order", "materials", "lights"):
            assert np.array_equal(a[k], b[k]), k


def test_png_encoding():
    img = (np.arange(32 * 24 * 3) % 251).astype(np.uint8).reshape(24, 32, 3)
    png = rtg.encode_png(img)
    assert png[:4] == b"\x89PNG"
    assert int.from_bytes(png[16:20], "big") == 32 and int.from_bytes(png[20:24], "big") == 24
    import zlib

    # IDAT decodes back to the filtered scanlines.
    pos, raw = 8, b""
    while pos < len(png):
        n = int.from_bytes(png[pos:pos + 4], "big")
        kind = png[pos + 4:pos + 8]
        if kind == b"IDAT":
            raw += png[pos + 8:pos + 8 + n]
        pos += 12 + n
    rows = np.frombuffer(zlib.decompress(raw), np.uint8).reshape(24, 1 + 32 * 3)
    assert (rows[:, 0] == 0).all()
    assert np.array_equal(rows[:, 1:].reshape(24, 32, 3), img)


def test_obj_meshes_load(tmp_path):
    obj = tmp_path / "square.obj"
    obj.write_text("# square\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvn 0 0 1\nf 1//1 2//1 3//1 4//1\n")
    scene = ('{"materials": {"m": {"type": "lambertian"}}, "objects": '
             '[{"type": "mesh", "source": "obj", "path": "square.obj", "material": "m"}]}')
    v = rtg.parse_scene(scene, str(tmp_path)).view()
    assert len(v["prims"]) == 2 and (v["prims"][:, 2] == 1).all()  # fan-triangulated, smooth
    assert np.allclose(v["prims"][:, 12:15], [0, 0, 1])
    bad = tmp_path / "bad.obj"
    bad.write_text("v 0 0 0\nf 1 2 3\n")
    with pytest.raises(rtg.SceneError, match="line 2"):
        rtg.parse_scene(scene.replace("square.obj", "bad.obj"), str(tmp_path))
