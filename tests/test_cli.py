"""The rtg command-line renderer: the reference CLI's flags, exit codes and
--stream protocol (apps/rt_cli.cpp:1-209) on the GPU renderer.

Exit codes: 0 done, 1 usage, 2 scene error, 3 output error, 130 cancelled.
The CPU tests stop before a GPU is needed (usage, validation, scene dumps,
scene errors); the GPU tests render and compare the files with the library's own
image of the same scene and settings.
"""
import json
import os
import subprocess

import pytest

import rtg
import workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "ray-tracer_b200", "rtg")


def run(args, stdin=None, timeout=120):
    return subprocess.run([CLI] + args, input=stdin, capture_output=True, timeout=timeout)


def cornell_text(**kw):
    return json.dumps(workloads.cornell(**kw))


@pytest.fixture
def scene_file(tmp_path):
    p = tmp_path / "cornell.json"
    p.write_text(cornell_text(width=32, height=32, spp=8))
    return p


def test_usage_errors_exit_1():
    assert run([]).returncode == 1
    r = run(["--bogus-flag", "x.json"])
    assert r.returncode == 1 and b"unknown option" in r.stderr
    r = run(["scene.json", "--spp"])
    assert r.returncode == 1 and b"missing value" in r.stderr
    r = run(["scene.json", "--spp", "many"])
    assert r.returncode == 1 and b"invalid integer" in r.stderr
    assert run(["--help"]).returncode == 0


def test_validate_reports_primitives(scene_file):
    r = run([str(scene_file), "--validate"])
    assert r.returncode == 0, r.stderr
    # 5 walls + the light: 12 triangles; 2 boxes: 24.
    assert b"scene OK: 36 primitives, 0 planes" in r.stderr
    r = run(["-", "--validate"], stdin=scene_file.read_bytes())
    assert r.returncode == 0 and b"scene OK: 36 primitives" in r.stderr


def test_dump_scene_matches_library(scene_file):
    r = run([str(scene_file), "--dump-scene"])
    assert r.returncode == 0
    assert json.loads(r.stdout) == json.loads(rtg.dump_scene(scene_file.read_text()))


def test_scene_errors_exit_2(tmp_path):
    bad = workloads.cornell()
    bad["objects"][0]["material"] = "no-such-material"
    p = tmp_path / "bad.json"
    p.write_text(json.dumps(bad))
    r = run([str(p), "--validate"])
    assert r.returncode == 2 and b"error:" in r.stderr
    r = run([str(p), "--stream"])
    assert r.returncode == 2
    line = r.stdout.decode().splitlines()[0]
    assert line.startswith("ERROR ") and "message" in json.loads(line[6:])
    assert run([str(tmp_path / "missing.json"), "--validate"]).returncode == 2
    r = run(["-", "--validate"], stdin=b"{not json")
    assert r.returncode == 2


def test_bad_integrator_is_a_scene_error(scene_file):
    r = run([str(scene_file), "--integrator", "photon"])
    assert r.returncode == 2 and b"--integrator" in r.stderr


def _library_png(text, width, height, spp):
    ctx = rtg.Context(0)
    try:
        sid = ctx.load_json(text)
        st = ctx.scene_settings(sid)
        st.width, st.height, st.spp = width, height, spp
        ctx.render(sid, st, rtg.RenderOptions(progressive=True, max_pass_spp=32))
        return rtg.encode_png(ctx.image(-1, width, height))
    finally:
        ctx.close()


def _frames(stdout: bytes):
    frames, i = [], 0
    while i < len(stdout):
        nl = stdout.index(b"\n", i)
        line = stdout[i:nl].decode()
        i = nl + 1
        if line.startswith("FRAME "):
            hdr = json.loads(line[6:])
            frames.append((hdr, stdout[i:i + hdr["bytes"]]))
            i += hdr["bytes"]
        elif line.startswith("DONE "):
            return frames, json.loads(line[5:])
        else:
            raise AssertionError(f"unexpected line {line!r}")
    raise AssertionError("no DONE line")


@pytest.mark.gpu
def test_png_matches_library_image(tmp_path, scene_file):
    out = tmp_path / "out.png"
    r = run([str(scene_file), "-o", str(out), "-q"])
    assert r.returncode == 0, r.stderr
    assert out.read_bytes() == _library_png(scene_file.read_text(), 32, 32, 8)


@pytest.mark.gpu
def test_gpu_bvh_flag_gives_the_same_image(tmp_path, scene_file):
    a, b = tmp_path / "a.png", tmp_path / "b.png"
    assert run([str(scene_file), "-o", str(a), "-q"]).returncode == 0
    r = run([str(scene_file), "-o", str(b), "-q", "--gpu-bvh"])
    assert r.returncode == 0, r.stderr
    assert a.read_bytes() == b.read_bytes()


@pytest.mark.gpu
def test_stream_protocol(tmp_path, scene_file):
    """--stream: one FRAME per progressive pass (1, 2, 4, ... spp done, then
    passes of at most --max-pass samples), PNG payloads of the announced size, and
    a DONE line with the stats; the last frame is the final image."""
    r = run([str(scene_file), "--stream", "--spp", "20", "--max-pass", "8", "-q"])
    assert r.returncode == 0, r.stderr
    frames, done = _frames(r.stdout)
    assert [h["spp_done"] for h, _ in frames] == [1, 2, 4, 8, 16, 20]
    assert [h["pass"] for h, _ in frames] == list(range(1, 7))
    assert all(png[:8] == b"\x89PNG\r\n\x1a\n" for _, png in frames)
    assert frames[-1][0]["finished"] and not done["cancelled"] and done["spp_done"] == 20
    assert done["invalid_samples"] == 0
    assert frames[-1][1] == _library_png(scene_file.read_text(), 32, 32, 20)


@pytest.mark.gpu
def test_ppm_output_and_output_errors(tmp_path, scene_file):
    out = tmp_path / "out.ppm"
    assert run([str(scene_file), "-o", str(out), "-q"]).returncode == 0
    data = out.read_bytes()
    assert data.startswith(b"P6\n32 32\n255\n") and len(data) == len(b"P6\n32 32\n255\n") + 32 * 32 * 3
    assert run([str(scene_file), "-o", str(tmp_path / "x.bmp"), "-q"]).returncode == 3
    assert run([str(scene_file), "-o", str(tmp_path / "no" / "dir.png"), "-q"]).returncode == 3


@pytest.mark.gpu
def test_mis_flag(tmp_path, scene_file):
    """--mis switches the estimator (NEE weighted against BSDF sampling): a
    different, equally valid image; with --no-light-sampling it changes nothing."""
    a, b, c, d = (tmp_path / f"{k}.png" for k in "abcd")
    assert run([str(scene_file), "-o", str(a), "-q"]).returncode == 0
    assert run([str(scene_file), "-o", str(b), "-q", "--mis"]).returncode == 0
    assert a.read_bytes() != b.read_bytes()
    assert run([str(scene_file), "-o", str(c), "-q", "--no-light-sampling"]).returncode == 0
    assert run([str(scene_file), "-o", str(d), "-q", "--no-light-sampling", "--mis"]).returncode == 0
    assert c.read_bytes() == d.read_bytes()
