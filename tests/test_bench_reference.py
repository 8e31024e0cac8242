"""The benchmark's reference arm builds its scene with the reference's own host code and never loads this library:
its box field, BVH buffers and frame parameters equal the library's for the same workload (so both arms render the
same frame), and the arm's process maps no libcwpb200.so."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import REF_DIR, ROOT


@pytest.fixture(scope="module")
def bench():
    sys.path.insert(0, ROOT)
    import bench as b
    if b.reference_lib() is None or not hasattr(b.reference_lib(), "ref_frame_params"):
        pytest.skip("oracle/_ref/libcwpref.so not built")
    return b


@pytest.mark.parametrize("variant", [2, 8])
def test_reference_scene_equals_library_scene(cwp, bench, variant):
    wl = dict(bench.WORKLOADS["frame256"])
    rs = bench.RefScene(bench.reference_lib(), wl, variant, w=wl["w"], h=wl["h"], bounces=wl["bounces"])
    mesh, bvh = cwp.scene(wl["scene"], variant=variant, bins=16)
    assert rs.n_tris == mesh.n_tris and rs.build_ms > 0
    assert np.array_equal(rs.nodes.view(np.uint32), bvh.nodes.view(np.uint32))
    assert np.array_equal(rs.woop.view(np.uint32), bvh.woop.view(np.uint32)) and np.array_equal(rs.tris.view(np.uint32), bvh.tris.view(np.uint32))
    p = cwp.frame_params(mesh, wl["w"], wl["h"], bounces=wl["bounces"])
    assert bytes(rs.p) == bytes(p)


def test_box_field_arrays_bit_identical(cwp):
    from importlib import import_module
    wk = import_module("cuda-wavefront-pathtracer_b200.workloads")
    for n, seed in ((1024, 1), (37, 99)):
        v, f, fm = wk.box_field_arrays(n, seed)
        a = cwp.Mesh.box_field(n, seed).arrays()
        assert np.array_equal(a[0].view(np.uint32), v.view(np.uint32)) and np.array_equal(a[1], f) and np.array_equal(a[2], fm)


def test_reference_arm_maps_no_library(bench, tmp_path):
    """The reference arm end to end on the smallest frame workload, checking /proc/self/maps at exit."""
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'frame256', '--steps', '1', '--warmup', '0', '--ref-seconds', '0.5']\n"
            "try:\n    runpy.run_path('bench.py', run_name='__main__')\n"
            "finally:\n    print('MAPS_HAS_LIB', 'libcwpb200' in open('/proc/self/maps').read())\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "MAPS_HAS_LIB False" in r.stdout and '"impl": "reference"' in r.stdout and '"unavailable"' not in r.stdout
