"""Golden data for OBJ meshes: the reference's own Scene::compile of a corpus of
OBJ files (oracle/_ref/rt_harness compile), including the edge cases its unit
tests pin (negative indices, a two-component vertex, a two-index face; its
tests/test_geometry.cpp:150-165) and the other branches of its loader.

For each case the OBJ text is written beside a scene that places it as a mesh
(scaled, rotated and moved, smooth shading on or off); the fixture records the
compiled primitives (24 doubles each, the harness's layout) or the error
message the compile raised.

    python tests/golden/make_obj_golden.py     # writes obj_cases.json
"""
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "rt_harness")

SQUARE = "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\n"
TRI = "v 0 0 0\nv 1 0 0\nv 0 1 0\n"

CASES = {
    "square_with_normals": "# square\n" + SQUARE + "vn 0 0 1\nf 1//1 2//1 3//1 4//1\n",
    "negative_indices": TRI + "f -3 -2 -1\n",
    "two_component_vertex": "v 0 0\n",
    "two_index_face": "v 0 0 0\nv 1 0 0\nf 1 2\n",
    "index_past_end": "v 0 0 0\nf 1 2 3\n",
    "index_zero": TRI + "f 0 1 2\n",
    "negative_index_past_start": TRI + "f -4 -2 -1\n",
    "bad_corner": TRI + "f a b c\n",
    "vt_vn_corners": SQUARE + "vt 0 0\nvn 0 0 1\nf 1/1/1 2/1/1 3/1/1 4/1/1\n",
    "vt_only_corners": SQUARE + "vt 0 0\nf 1/1 2/1 3/1\n",
    "inconsistent_normals": SQUARE + "vn 0 0 1\nvn 0 1 0\nf 1//1 2//1 3//1\nf 1//2 3//1 4//1\n",
    "some_corners_without_normals": SQUARE + "vn 0 0 1\nf 1//1 2//1 3\n",
    "normal_index_out_of_range": SQUARE + "vn 0 0 1\nf 1//1 2//2 3//1\n",
    "bad_normal": TRI + "vn 0 0\nf 1 2 3\n",
    "unnormalised_and_zero_normals": TRI + "vn 0 0 5\nvn 0 0 0\nf 1//1 2//2 3//1\n",
    "pentagon_fan": "v 0 0 0\nv 2 0 0\nv 3 1 0\nv 1 2 0\nv -1 1 0\nf 1 2 3 4 5\n",
    "ignored_records": "o thing\ng group\ns 1\nusemtl red\nmtllib x.mtl\n\n   \n# comment\n" + TRI + "f 1 2 3\n",
    "crlf_and_exponents": "v 0 0 0\r\nv 1e0 0 0\r\nv 0 +1.0 -0e0\r\nf 1 2 3\r\n",
    "vertices_only": TRI,
    "faces_before_later_vertices": TRI + "f 1 2 3\nv 0 0 1\nf 1 2 4\nf -1 -2 -3\n",
}


def scene_for(obj_name: str, smooth: bool = True) -> dict:
    return {"materials": {"m": {"type": "lambertian"}},
            "objects": [{"type": "mesh", "source": "obj", "path": obj_name, "smooth": smooth,
                         "scale": [1, 2, 1], "rotate_y": 30, "translate": [1, 0, 0.5], "material": "m"}]}


def compile_reference(obj_text: str, smooth: bool) -> dict:
    with tempfile.TemporaryDirectory() as tmp:
        with open(os.path.join(tmp, "case.obj"), "w", newline="") as f:
            f.write(obj_text)
        with open(os.path.join(tmp, "scene.json"), "w") as f:
            json.dump(scene_for("case.obj", smooth), f)
        r = subprocess.run([HARNESS, "compile", os.path.join(tmp, "scene.json"), os.path.join(tmp, "out")],
                           capture_output=True, text=True)
        if r.returncode != 0:
            msg = r.stderr.strip()
            assert msg.startswith("error: "), msg
            return {"error": msg[len("error: "):]}
        prims = np.fromfile(os.path.join(tmp, "out.prims.f64"), dtype=np.float64)
        return {"error": "", "prims": prims.tolist()}


def main():
    out = []
    for name, text in CASES.items():
        for smooth in (True, False):
            out.append({"name": name, "smooth": smooth, "obj": text, **compile_reference(text, smooth)})
    with open(os.path.join(HERE, "obj_cases.json"), "w") as f:
        json.dump({"source": "reference Scene::compile via rt_harness compile", "cases": out}, f)
    print(len(out), "cases;", sum(1 for c in out if c["error"]), "rejected")


if __name__ == "__main__":
    main()
