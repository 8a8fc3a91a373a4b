"""OBJ meshes against the reference's own compile of the same files
(tests/golden/obj_cases.json, made by make_obj_golden.py): the compiled
triangles (positions, shading normals, smooth flag) bit for bit, or the same
error message, for the loader's edge cases: negative and zero indices, short
vertex and face records, v/vt/vn corner forms, inconsistent or partial normals,
polygon fans, ignored records, CRLF line ends."""
import json
import os

import numpy as np
import pytest

import rtg
from conftest import GOLDEN

CASES = json.load(open(os.path.join(GOLDEN, "obj_cases.json")))["cases"]


def _scene(smooth: bool) -> str:
    return json.dumps({"materials": {"m": {"type": "lambertian"}},
                       "objects": [{"type": "mesh", "source": "obj", "path": "case.obj", "smooth": smooth,
                                    "scale": [1, 2, 1], "rotate_y": 30, "translate": [1, 0, 0.5],
                                    "material": "m"}]})


@pytest.mark.parametrize("k", range(len(CASES)), ids=[f"{c['name']}-{'smooth' if c['smooth'] else 'flat'}"
                                                      for c in CASES])
def test_obj_compiles_like_the_reference(tmp_path, k):
    case = CASES[k]
    with open(tmp_path / "case.obj", "w", newline="") as f:
        f.write(case["obj"])
    if case["error"]:
        with pytest.raises(rtg.SceneError) as err:
            rtg.parse_scene(_scene(case["smooth"]), str(tmp_path))
        assert str(err.value) == case["error"]
        return
    prims = rtg.parse_scene(_scene(case["smooth"]), str(tmp_path)).view()["prims"]
    ref = np.array(case["prims"], np.float64).reshape(-1, 24)
    assert prims.shape == ref.shape
    assert prims.tobytes() == ref.tobytes()
