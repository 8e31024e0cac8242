"""The reference's procedural sphere-grid scene (scene/synthetic.cpp:6-48, the scene of its scripts/bench_synthetic.sh):
cwp_mesh_sphere_grid gives the same vertices, triangles, material ids and albedos, bit for bit, as the reference's
makeSynthetic compiled from its sources, and cwp_sphere_grid_c2w the same view as its syntheticCamera. On a GPU the
CLI renders it with bench_synthetic.sh's flags, against the reference's own CUDA build of pt."""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import REF_DIR


def ref_synthetic(ref, grid, nu, nv, gs):
    L = ref.L
    L.ref_synthetic.restype = None
    L.ref_synthetic.argtypes = [C.c_int] * 4 + [C.POINTER(C.c_long)] * 2 + [C.c_void_p] * 5
    nvx, ntr = C.c_long(), C.c_long()
    L.ref_synthetic(grid, nu, nv, gs, C.byref(nvx), C.byref(ntr), None, None, None, None, None)
    v = np.zeros((nvx.value, 3), np.float32); f = np.zeros((ntr.value, 3), np.int32)
    fm = np.zeros(ntr.value, np.int32); kd = np.zeros((5, 3), np.float32); c2w = np.zeros(16, np.float32)
    L.ref_synthetic(grid, nu, nv, gs, C.byref(nvx), C.byref(ntr), v.ctypes.data, f.ctypes.data, fm.ctypes.data, kd.ctypes.data, c2w.ctypes.data)
    return v, f, fm, kd, c2w.reshape(4, 4)


@pytest.mark.parametrize("grid,nu,nv,gs", [(1, 3, 2, 1), (2, 8, 5, 4), (7, 200, 100, 200), (5, 17, 9, 33)])
def test_sphere_grid_bit_identical(cwp, ref, grid, nu, nv, gs):
    v, f, fm, alb = cwp.Mesh.sphere_grid(grid, nu, nv, gs).arrays()
    rv, rf, rfm, rkd, rc2w = ref_synthetic(ref, grid, nu, nv, gs)
    assert len(f) == 2 * (gs * gs + grid * grid * nu * (nv - 1))
    assert v.tobytes() == rv.tobytes()
    assert np.array_equal(f, rf) and np.array_equal(fm, rfm)
    assert alb.tobytes() == rkd.tobytes()
    assert cwp.sphere_grid_c2w().tobytes() == rc2w.tobytes()


def test_sphere_grid_counts_and_refusals(cwp):
    v, f, fm, alb = cwp.Mesh.sphere_grid(7).arrays()
    assert len(f) == 2 * (200 * 200 + 49 * 200 * 99) == 2_020_400
    assert len(v) == 201 * 201 + 49 * 200 * 101 and alb.shape == (5, 3)
    assert fm.min() == 0 and fm.max() == 4 and np.all(fm[: 2 * 200 * 200] == 0)
    with pytest.raises(cwp.CwpError):
        cwp.Mesh.sphere_grid(7, nu=2)
    with pytest.raises(cwp.CwpError):
        cwp.Mesh.sphere_grid(65)


PT = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cuda-wavefront-pathtracer_b200", "pt")


@pytest.mark.gpu
def test_cli_synthetic_vs_reference_cuda(gpu, cwp, tmp_path):
    """bench_synthetic.sh's flag set (BVH2, Woop, fused trace+shade, batch 64) at a smaller grid and image: both
    builds print one JSON line per repetition for the same 'synthetic' scene, and their images agree at >= 50 dB."""
    ref_pt = os.path.join(REF_DIR, "pt")
    if not os.path.exists(ref_pt):
        pytest.skip("oracle/_ref/pt not built")
    args = ["--synthetic", "3", "--width", "160", "--height", "128", "--spp", "64", "--bounces", "4", "--variant", "bvh2",
            "--tri", "woop", "--fuse", "1", "--batch", "64", "--reps", "2"]
    out = {}
    for name, exe in (("ours", PT), ("ref", ref_pt)):
        res = subprocess.run([exe] + args + ["--out", str(tmp_path / name)], check=True, capture_output=True, text=True, timeout=600)
        lines = [json.loads(l) for l in res.stdout.splitlines() if l.startswith("{")]
        assert len(lines) == 2, res.stdout + res.stderr
        out[name] = (lines, cwp.imageio.read_pfm(str(tmp_path / name) + ".pfm"))
    (ours, a), (ref_lines, b) = out["ours"], out["ref"]
    assert a.shape == b.shape == (128, 160, 3)
    db = cwp.imageio.psnr(a, b)
    print(json.dumps({"synthetic3_psnr_vs_reference_db": db, "ours_ms": [l.get("t_frame_ms") for l in ours], "ref_ms": [l.get("t_frame_ms") for l in ref_lines]}))
    assert db >= 50.0
