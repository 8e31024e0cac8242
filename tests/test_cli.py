"""The command-line renderer (cuda-wavefront-pathtracer_b200/pt) takes the reference CLI's flags: these checks run
without a GPU and cover the refusals and the scene-file parsing that happen before any device work."""
import json
import os
import subprocess

import pytest

PT = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cuda-wavefront-pathtracer_b200", "pt")


def run(*args):
    if not os.path.exists(PT):
        pytest.skip("pt not built")
    r = subprocess.run([PT] + [str(a) for a in args], capture_output=True, text=True, timeout=60)
    return r.returncode, r.stderr


@pytest.mark.parametrize("args,msg", [
    (["--scene", "s.json", "--materials", "m.json"], "per mesh in scene files"),
    (["--loader", "assimp"], "only the built-in PLY / OBJ loader"),
    (["--light_sampling", "all"], "--light_sampling must be"),
    (["--integrator", "legacy", "--scene", "s.json"], "does not render scene files"),
    (["--bogus"], "unknown arg"),
    (["--builder", "lbvh"], "--builder must be sah or hploc"),
    (["--synthetic", "3", "--scene", "s.json"], "--synthetic and --scene cannot be combined"),
])
def test_refusals(args, msg):
    rc, err = run(*args)
    assert rc == 1 and msg in err, err


def test_scene_file_errors(tmp_path):
    """scene files are parsed (and refused where this build lacks a feature) before any device work"""
    ply = tmp_path / "q.ply"
    ply.write_text("ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\nproperty float z\n"
                   "element face 1\nproperty list uchar int vertex_indices\nend_header\n0 0 0\n1 0 0\n0 1 0\n3 0 1 2\n")
    s = tmp_path / "s.json"
    s.write_text(json.dumps({"meshes": [{"file": "q.ply"}], "instances": [{"mesh": 0, "transform": [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1]}]}))
    rc, err = run("--scene", s)
    assert rc == 1 and "transform needs 12 or 16 numbers" in err
    s.write_text(json.dumps({"meshes": [{"file": "q.ply"}], "instances": [{"mesh": 0, "transforms": [[1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], [1, 0]]}]}))
    rc, err = run("--scene", s)
    assert rc == 1 and "transforms entries need 12 or 16 numbers" in err
    s.write_text(json.dumps({"meshes": [{"file": "q.ply"}], "instances": [{"mesh": 3}]}))
    rc, err = run("--scene", s)
    assert rc == 1 and "instance mesh 3 out of range" in err
    s.write_text(json.dumps({"meshes": [{"file": "missing.ply"}], "instances": []}))
    rc, err = run("--scene", s)
    assert rc == 1 and "missing.ply" in err
    s.write_text(json.dumps({"meshes": [{"file": "q.ply", "materials": "m.json"}], "instances": [{"mesh": 0}]}))
    (tmp_path / "m.json").write_text(json.dumps({"no": []}))
    rc, err = run("--scene", s)
    assert rc == 1 and 'no "materials" array' in err
