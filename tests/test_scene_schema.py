"""The scene schema against the reference's own answers (tests/golden/scene_schema.json,
made by make_scene_schema_golden.py from the reference's stock CLI): every
rejected scene gives exactly the reference's message, including the count of
further problems, and every accepted scene dumps to exactly the reference's
normalised JSON."""
import json
import os

import pytest

import rtg
from conftest import GOLDEN

CASES = json.load(open(os.path.join(GOLDEN, "scene_schema.json")))["cases"]


@pytest.mark.parametrize("k", range(len(CASES)))
def test_scene_matches_the_reference(k):
    case = CASES[k]
    assert rtg.validate_scene(case["scene"]) == case["error"]
    if not case["error"]:
        assert rtg.dump_scene(case["scene"]) == case["dump"]


def test_corpus_covers_rejections_and_acceptances():
    rejected = [c for c in CASES if c["error"]]
    assert len(rejected) >= 100 and len(CASES) - len(rejected) >= 20
    assert any("more problem(s)" in c["error"] for c in rejected)
