"""The C ABI library: loads, exports every function include/*.h declares, validates inputs before touching a GPU,
and the Python binding declares a signature for each export."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def header_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(cwp_\w+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol(cwp):
    L = C.CDLL(cwp.LIB_PATH)
    missing = [n for n in sorted(header_functions()) if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header(cwp):
    assert header_functions() <= set(cwp.SIGNATURES), header_functions() - set(cwp.SIGNATURES)


def test_struct_layouts_match_header(cwp, tmp_path):
    """ctypes mirrors of the C structs have the C compiler's sizes and field offsets."""
    import subprocess
    structs = {"cwp_mesh_view": cwp.MeshView, "cwp_build_options": cwp.BuildOptions, "cwp_bvh_data": cwp.BvhData,
               "cwp_scene_buffers": cwp.SceneBuffers, "cwp_camera": cwp.Camera, "cwp_params": cwp.Params,
               "cwp_render_options": cwp.RenderOptions, "cwp_frame_stats": cwp.FrameStats, "cwp_renderer_info": cwp.RendererInfo}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "cwp_b200.h"', "int main(void) {"]
    for cn, py in structs.items():
        lines.append(f'printf("{cn} %zu\\n", sizeof({cn}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cn}.{fname} %zu\\n", offsetof({cn}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"; src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n") if l)
    for cn, py in structs.items():
        assert int(out[cn]) == C.sizeof(py), cn
        for fname, _ in py._fields_:
            assert int(out[f"{cn}.{fname}"]) == getattr(py, fname).offset, f"{cn}.{fname}"


def test_version_and_error_string(cwp):
    L = cwp.lib()
    assert L.cwp_version() >= 1
    h = C.c_void_p()
    rc = L.cwp_mesh_box_field(-1, 1, C.byref(h))
    assert rc == cwp.ERR_INVALID and b"out of range" in L.cwp_last_error()


def test_l2_probe_arguments_checked_before_gpu(cwp):
    L = cwp.lib(); g = C.c_double()
    for nbytes, reps in ((100, 1), ((32 << 20) + 8, 1), (1 << 30, 1), (32 << 20, 0)):
        assert L.cwp_measure_l2_read(nbytes, reps, 0, C.byref(g)) == cwp.ERR_INVALID
    assert L.cwp_measure_l2_read(32 << 20, 1, 0, None) == cwp.ERR_INVALID


def _scene_buffers(nodes, stride, tris):
    s = cwp_mod().SceneBuffers()
    s.nodes, s.n_node_float4, s.node_stride = nodes.ctypes.data, len(nodes), stride
    s.tris, s.n_tris, s.woop = tris.ctypes.data, len(tris) // 3, tris.ctypes.data
    return s


def cwp_mod():
    import importlib
    return importlib.import_module("cuda-wavefront-pathtracer_b200")


def test_malformed_nodes_rejected_before_gpu(cwp):
    """Child or leaf references outside the buffers are refused on the host (no kernel ever reads them)."""
    mesh = cwp.Mesh.box_field(16, 1)
    b = cwp.Bvh(mesh, variant=2)
    for corrupt in ("child", "leaf", "stride"):
        nodes = b.nodes.copy(); stride = 4
        meta = nodes.view(np.int32)
        if corrupt == "child":
            idx = np.nonzero((meta[3::4, 2] == 0) & (meta[3::4, 0] >= 0))[0][0]; meta[4 * idx + 3, 0] = 10 ** 6
        elif corrupt == "leaf":
            idx = np.nonzero(meta[3::4, 2] > 0)[0][0]; meta[4 * idx + 3, 0] = len(b.order) - 1; meta[4 * idx + 3, 2] = 4
        else:
            stride = 6
        s = _scene_buffers(nodes, stride, b.woop)
        h = C.c_void_p()
        rc = cwp.lib().cwp_accel_create(C.byref(s), 1, 0, C.byref(h))
        assert rc == cwp.ERR_INVALID, (corrupt, rc, cwp.lib().cwp_last_error())


def test_cwbvh_malformed_rejected(cwp):
    b = cwp.Bvh(cwp.Mesh.box_field(16, 1), variant=8)
    nodes = b.nodes.copy(); w = nodes.view(np.int32).reshape(-1, 20)
    w[0, 4] = len(w)   # child base past the end
    s = _scene_buffers(nodes, 5, b.woop); h = C.c_void_p()
    assert cwp.lib().cwp_accel_create(C.byref(s), 1, 0, C.byref(h)) == cwp.ERR_INVALID


def test_camera_look_at_matches_reference_formula(cwp):
    c = cwp.camera_look_at((0, -34, 22), (0, 0, 0), (0, 0, 1), 45.0, 512, 512)
    f = -np.array([0, -34, 22], np.float32); f /= np.linalg.norm(f)
    r = np.cross(f, [0, 0, 1]); r /= np.linalg.norm(r)
    assert np.allclose(list(c.ax), r, atol=1e-6) and np.allclose(list(c.az), -f, atol=1e-6)
    assert abs(c.fx - 256 / np.tan(np.radians(22.5))) < 1e-3 and c.px == 256 and c.w == 512


def test_filter_table_matches_reference(cwp, ref):
    """the Blackman-Harris pixel-filter inverse CDF (camera rays with --filter bh, the reference's default) is the
    reference's buildBlackmanHarrisTable output bit for bit"""
    import ctypes as C
    t = np.zeros(65, np.float32)
    ref.L.ref_bh_table.restype = None; ref.L.ref_bh_table.argtypes = [C.c_void_p, C.c_int, C.c_double]
    ref.L.ref_bh_table(t.ctypes.data, 64, 1.5)
    assert np.array_equal(np.array(list(cwp.params_defaults().ftab), np.float32).view(np.uint32), t.view(np.uint32))


def test_params_finish(cwp):
    p = cwp.params_defaults()
    assert p.seed == 1000 and p.max_b == 8
    assert abs(np.linalg.norm(list(p.sun_to)) - 1) < 1e-6
    assert abs(p.sun_cos - np.cos(np.radians(0.526 / 2))) < 1e-7
    # Blackman-Harris inverse CDF: symmetric, width 1.5 px
    t = np.array(list(p.ftab))
    assert abs(t[0] + 0.75) < 1e-6 and abs(t[-1] - 0.75) < 1e-6 and abs(t[32]) < 1e-4
