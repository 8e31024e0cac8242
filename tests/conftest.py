"""Shared fixtures: the library under test, the oracle (test infrastructure) and, where built, the reference's own
code compiled from its sources (oracle/_ref)."""
import ctypes as C
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cwp():
    return importlib.import_module("cuda-wavefront-pathtracer_b200")


def _load_oracle():
    path = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(path):
        import subprocess
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True, capture_output=True)
    L = C.CDLL(path)
    L.orc_build.restype = C.c_long
    L.orc_build.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_long, C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.orc_pack.restype = None
    L.orc_pack.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.orc_trace.restype = C.c_long
    L.orc_trace.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_render.restype = None
    L.orc_render.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    L.orc_trace_fp64.restype = C.c_long
    L.orc_trace_fp64.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_long, C.c_int, C.c_void_p, C.c_void_p]
    L.orc_trace_prec.restype = C.c_long
    L.orc_trace_prec.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_trace_inst.restype = C.c_long
    L.orc_trace_inst.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 4 + [C.c_long, C.c_void_p, C.c_void_p]
    L.orc_bsdf_eval.restype = None
    L.orc_bsdf_eval.argtypes = [C.c_void_p] * 5 + [C.c_int] + [C.c_void_p] * 3 + [C.c_long, C.c_void_p]
    L.orc_bsdf_sample.restype = None
    L.orc_bsdf_sample.argtypes = [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 6 + [C.c_long, C.c_void_p]
    L.orc_render_stats.restype = None
    L.orc_render_stats.argtypes = [C.c_int, C.c_void_p]
    L.orc_render_request.restype = C.c_long
    L.orc_render_request.argtypes = ([C.c_void_p, C.c_int, C.c_int] + [C.c_void_p] * 3 + [C.c_int] + [C.c_void_p] * 2 + [C.c_int, C.c_void_p, C.c_int, C.c_long, C.c_long, C.c_void_p, C.c_void_p]
                                     + [C.c_void_p] * 3 + [C.c_int, C.c_int] + [C.c_void_p] * 2 + [C.c_int] + [C.c_void_p] * 3 + [C.c_void_p] * 3 + [C.c_long, C.c_void_p, C.c_void_p])
    L.orc_emissive_tables.restype = C.c_long
    L.orc_emissive_tables.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_long] + [C.c_void_p] * 3
    L.orc_texture_sample.restype = None
    L.orc_texture_sample.argtypes = [C.c_void_p] * 4 + [C.c_long]
    L.orc_envmap_build.restype = None
    L.orc_envmap_build.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_half_round.restype = C.c_double
    L.orc_half_round.argtypes = [C.c_double, C.c_int]
    L.orc_rng.restype = C.c_float
    L.orc_rng.argtypes = [C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_uint]
    return L


class Oracle:
    """Thin numpy wrapper around liboracle.so."""

    def __init__(self):
        self.L = _load_oracle()
        self._ftab = None   # the pixel-filter table of camera rays (the library's, pinned to the reference's)

    def build(self, verts, faces, bins=16, leaf=4, variant=2):
        nt = len(faces)
        cap = 5 * 2 * nt + 64
        nodes = np.zeros((cap, 4), np.float32); order = np.zeros(nt, np.int32)
        md = C.c_int(); sah = C.c_double()
        v = np.ascontiguousarray(verts, np.float32); f = np.ascontiguousarray(faces, np.int32)
        n = self.L.orc_build(v.ctypes.data, f.ctypes.data, nt, bins, leaf, variant, nodes.ctypes.data, cap, order.ctypes.data, C.byref(md), C.byref(sah))
        assert n > 0
        return nodes[:n].copy(), order, md.value, sah.value

    def pack(self, verts, faces, fm, order):
        n = len(order)
        tris = np.zeros((3 * n, 4), np.float32); woop = np.zeros((3 * n, 4), np.float32)
        v = np.ascontiguousarray(verts, np.float32); f = np.ascontiguousarray(faces, np.int32); fm = np.ascontiguousarray(fm, np.int32)
        o = np.ascontiguousarray(order, np.int32)
        self.L.orc_pack(v.ctypes.data, f.ctypes.data, fm.ctypes.data, o.ctypes.data, n, tris.ctypes.data, woop.ctypes.data)
        return tris, woop

    def trace(self, variant, tri, any_hit, nodes, tv, o, d, stats=False):
        n = len(o)
        hits = np.zeros((n, 4), np.float32); occ = np.zeros(n, np.int32); st = np.zeros(2, np.int64)
        bad = self.L.orc_trace(variant, tri, 1 if any_hit else 0, np.ascontiguousarray(nodes).ctypes.data, np.ascontiguousarray(tv).ctypes.data,
                               np.ascontiguousarray(o).ctypes.data, np.ascontiguousarray(d).ctypes.data, n, hits.ctypes.data, occ.ctypes.data,
                               st.ctypes.data if stats else None)
        assert bad == 0
        res = occ if any_hit else hits
        return (res, st) if stats else res

    def trace_fp64(self, nodes, verts, o, d, any_hit=False, brute=False):
        """FP64 watertight closest (or first) hit: (t float64, leaf-order tri int32); nodes = CWBVH or brute force."""
        n = len(o); t = np.zeros(n, np.float64); tri = np.zeros(n, np.int32)
        vt = np.ascontiguousarray(verts, np.float32)
        r = self.L.orc_trace_fp64(None if brute else np.ascontiguousarray(nodes).ctypes.data, vt.ctypes.data, len(vt) // 3,
                                  np.ascontiguousarray(o).ctypes.data, np.ascontiguousarray(d).ctypes.data, n, 1 if any_hit else 0, t.ctypes.data, tri.ctypes.data)
        assert r == 0
        return t, tri

    def trace_prec(self, nodes, verts, o, d, any_hit=False, stats=False):
        """The precision form (f16 conservative slabs + watertight FP32 triangles) restated with exact f16 emulation:
        closest hits float4 (t, u, v, tri bits) or first occluders, bit for bit what the CUDA precision form returns."""
        n = len(o)
        hits = np.zeros((n, 4), np.float32); occ = np.zeros(n, np.int32); st = np.zeros(2, np.int64)
        bad = self.L.orc_trace_prec(np.ascontiguousarray(nodes).ctypes.data, np.ascontiguousarray(verts, np.float32).ctypes.data,
                                    np.ascontiguousarray(o).ctypes.data, np.ascontiguousarray(d).ctypes.data, n, 1 if any_hit else 0,
                                    hits.ctypes.data, occ.ctypes.data, st.ctypes.data if stats else None)
        assert bad == 0
        res = occ if any_hit else hits
        return (res, st) if stats else res

    def trace_inst(self, width, any_hit, blas, tris, tlas, scene_root, inst, o, d, scene_of, tlas_width=2):
        """Two-level traversal of the batched form (TLAS nodes of width 2 or 4): (hits float4 [n, 4], hit instance [n])."""
        n = len(o)
        hits = np.zeros((n, 4), np.float32); hi = np.zeros(n, np.int32)
        a = [np.ascontiguousarray(x) for x in (blas, tris, tlas)]
        sr = np.ascontiguousarray(scene_root, np.int32); ins = np.ascontiguousarray(inst, np.float32); so = np.ascontiguousarray(scene_of, np.int32)
        bad = self.L.orc_trace_inst(width, tlas_width, 1 if any_hit else 0, a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, sr.ctypes.data, len(sr),
                                    ins.ctypes.data, np.ascontiguousarray(o).ctypes.data, np.ascontiguousarray(d).ctypes.data, so.ctypes.data, n,
                                    hits.ctypes.data, hi.ctypes.data)
        assert bad == 0
        return hits, hi

    def bsdf_eval(self, mats, mat, wo, wi, eta, gd, ux, nr=None):
        """nr: an unperturbed normal per case (the bump-terminator term) or None"""
        n = len(mat); f = np.zeros((n, 3), np.float32); pdf = np.zeros(n, np.float32)
        a = [np.ascontiguousarray(x) for x in (mats, mat, wo, wi, eta, ux)]
        nr = np.ascontiguousarray(nr, np.float32) if nr is not None else None
        self.L.orc_bsdf_eval(a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, a[3].ctypes.data, a[4].ctypes.data, gd, a[5].ctypes.data, f.ctypes.data, pdf.ctypes.data, n,
                             nr.ctypes.data if nr is not None else None)
        return f, pdf

    def bsdf_sample(self, mats, mat, wo, eta, gd, ux, uvw, nr=None):
        n = len(mat); wi = np.zeros((n, 3), np.float32); w = np.zeros((n, 3), np.float32); pdf = np.zeros(n, np.float32); ok = np.zeros(n, np.int32)
        a = [np.ascontiguousarray(x) for x in (mats, mat, wo, eta, ux, uvw)]
        nr = np.ascontiguousarray(nr, np.float32) if nr is not None else None
        self.L.orc_bsdf_sample(a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, a[3].ctypes.data, gd, a[4].ctypes.data, a[5].ctypes.data,
                               wi.ctypes.data, w.ctypes.data, pdf.ctypes.data, ok.ctypes.data, n, nr.ctypes.data if nr is not None else None)
        return wi, w, pdf, ok

    def envmap_build(self, rgb, strength=1.0):
        rgb = np.ascontiguousarray(rgb, np.float32); h, w = rgb.shape[:2]
        tex = np.zeros((h, w, 4), np.float32); marg = np.zeros(h + 1, np.float32); cond = np.zeros((h, w + 1), np.float32)
        self.L.orc_envmap_build(rgb.ctypes.data, w, h, strength, tex.ctypes.data, marg.ctypes.data, cond.ctypes.data)
        return tex, marg, cond

    def emissive_tables(self, meshes, mesh_mat, mats, xforms, inst_mesh):
        """light tables of the emissive triangles of an instanced scene at one frame: (em_tris [n, 12], em_cdf [n + 1],
        mat_pdf [n_mats]); meshes: (verts, faces, face_mat, _) tuples"""
        soup, first = [], [0]
        for v, f, fm, _ in meshes:
            v = np.asarray(v, np.float32); f = np.asarray(f, np.int64)
            r = np.zeros((len(f), 12), np.float32)
            r[:, 0:3], r[:, 4:7], r[:, 8:11] = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
            r[:, 3] = np.arange(len(f), dtype=np.int32).view(np.float32)
            r[:, 7] = (np.zeros(len(f), np.int32) if fm is None else np.asarray(fm, np.int32)).view(np.float32)
            soup.append(r); first.append(first[-1] + len(f))
        soup = np.ascontiguousarray(np.concatenate(soup)); first = np.array(first, np.int32)
        mm = np.ascontiguousarray(mesh_mat, np.int32); ms = np.ascontiguousarray(mats, np.float32)
        xf = np.ascontiguousarray(xforms, np.float32).reshape(-1, 12); im = np.ascontiguousarray(inst_mesh, np.int32)
        args = (soup.ctypes.data, first.ctypes.data, len(first) - 1, mm.ctypes.data, ms.ctypes.data, len(ms), xf.ctypes.data, im.ctypes.data, len(im))
        n = self.L.orc_emissive_tables(*args, None, None, None)
        t = np.zeros((n, 12), np.float32); c = np.zeros(n + 1, np.float32); p = np.zeros(len(ms), np.float32)
        n2 = self.L.orc_emissive_tables(*args, t.ctypes.data, c.ctypes.data, p.ctypes.data)
        assert n2 == n
        return t, (c if n else np.zeros(0, np.float32)), p

    def texture_sample(self, tex, ids, uv):
        """lookups (texture id, (u, v)) -> rgba [n, 4] with the oracle's restatement of the texture unit; tex: a
        cwp_texture array"""
        ids = np.ascontiguousarray(ids, np.int32); uv = np.ascontiguousarray(uv, np.float32); out = np.zeros((len(ids), 4), np.float32)
        self.L.orc_texture_sample(C.addressof(tex), ids.ctypes.data, uv.ctypes.data, out.ctypes.data, len(ids))
        return out

    def render_request(self, req, width, blas, tris, tlas, root, inst, mats, mesh_mat, gd=1, paths=None, tlas_width=2, env=None, textures=None,
                       lights=None, normals=None):
        """A serving request on the host: (accum [w h, 4], counts [2]). env: (texels, marg, cond) of the request's
        environment map when Request.env >= 0, else None. textures: (cwp_texture array, cwp_material_textures array,
        uvs, tans or None, mesh_first) as given to the server, else None. lights: (em_tris, em_cdf, mat_pdf) of the
        request's scene at its frame (emissive_tables), else None. normals: (corner normals [n_tris, 12] in mesh
        order, mesh_first) when the batch's meshes have normals, else None."""
        n = req.cam.w * req.cam.h * req.spp
        j0, j1 = (0, n) if paths is None else paths
        acc = np.zeros((req.cam.w * req.cam.h, 4), np.float32); cnt = np.zeros(2, np.int64)
        a = [np.ascontiguousarray(x) for x in (blas, tris, tlas)]
        ins = np.ascontiguousarray(inst, np.float32); ms = np.ascontiguousarray(mats, np.float32); mm = np.ascontiguousarray(mesh_mat, np.int32)
        nr = np.ascontiguousarray(normals[0], np.float32) if normals is not None else None
        mf = np.ascontiguousarray(normals[1], np.int32) if normals is not None else None
        if self._ftab is None:
            import importlib
            self._ftab = np.array(list(importlib.import_module("cuda-wavefront-pathtracer_b200").params_defaults().ftab), np.float32)
        bad = self.L.orc_render_request(C.addressof(req), width, tlas_width, a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, int(root), ins.ctypes.data,
                                        ms.ctypes.data, len(ms), mm.ctypes.data, gd, j0, j1, acc.ctypes.data, cnt.ctypes.data,
                                        *((env[0].ctypes.data, env[1].ctypes.data, env[2].ctypes.data, env[0].shape[1], env[0].shape[0]) if env is not None
                                          else (None, None, None, 0, 0)),
                                        *((C.addressof(textures[0]), C.addressof(textures[1]), len(textures[1]), textures[2].ctypes.data,
                                           textures[3].ctypes.data if textures[3] is not None else None, textures[4].ctypes.data) if textures is not None
                                          else (None, None, 0, None, None, mf.ctypes.data if mf is not None else None)),
                                        *((lights[0].ctypes.data, lights[1].ctypes.data, lights[2].ctypes.data, len(lights[0])) if lights is not None and len(lights[0])
                                          else (None, None, None, 0)),
                                        nr.ctypes.data if nr is not None else None, self._ftab.ctypes.data)
        assert bad == 0
        return acc, cnt

    def render(self, params, variant, tri, bvh, bounces, spp, s_base=0, pix0=0, pix1=None):
        w, h = params.cam.w, params.cam.h
        acc = np.zeros((w * h, 4), np.float32); rc = np.zeros(2, np.int64)
        tv = bvh.woop if tri == 1 else bvh.tris
        alb = np.ascontiguousarray(bvh.albedo, np.float32)
        self.L.orc_render(C.addressof(params), variant, tri, bvh.nodes.ctypes.data, tv.ctypes.data, bvh.tris.ctypes.data, alb.ctypes.data,
                          bounces, spp, s_base, pix0, w * h if pix1 is None else pix1, acc.ctypes.data, rc.ctypes.data)
        return acc, rc

    def render_work(self, params, variant, tri, bvh, bounces, spp, pix0, pix1):
        """Traversal work of orc_render over pixels [pix0, pix1): (ray counts [closest, shadow], [closest node visits,
        closest triangle tests, shadow node visits, shadow triangle tests])."""
        self.L.orc_render_stats(1, None)
        _, rc = self.render(params, variant, tri, bvh, bounces, spp, 0, pix0, pix1)
        st = np.zeros(4, np.int64); self.L.orc_render_stats(0, st.ctypes.data)
        return rc, st


@pytest.fixture(scope="session")
def oracle():
    return Oracle()


class Ref:
    """The reference's own host code (oracle/_ref/libcwpref.so)."""

    def __init__(self, path):
        L = C.CDLL(path)
        L.ref_build.restype = C.c_long
        L.ref_build.argtypes = [C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_long, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.ref_xform_invert.restype = None
        L.ref_xform_invert.argtypes = [C.POINTER(C.c_float)] * 3
        L.ref_xform_animate.restype = None
        L.ref_xform_animate.argtypes = [C.POINTER(C.c_float)] * 3 + [C.c_float, C.c_float] + [C.POINTER(C.c_float)] * 2 + [C.c_int, C.POINTER(C.c_float)]
        L.ref_trace.restype = C.c_double
        L.ref_trace.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_int]
        L.ref_trace_inst.restype = C.c_double
        L.ref_trace_inst.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 4 + [C.c_long, C.c_void_p, C.c_void_p, C.c_int]
        self.L = L

    def build(self, verts, faces, fm, variant=2, leaf=4, collapse=0):
        nt = len(faces); cap = 5 * 2 * nt + 64
        nodes = np.zeros((cap, 4), np.float32); order = np.zeros(nt, np.int32)
        tris = np.zeros((3 * nt, 4), np.float32); woop = np.zeros((3 * nt, 4), np.float32)
        md = C.c_int(); sah = C.c_double(); ms = C.c_double()
        v = np.ascontiguousarray(verts, np.float32); f = np.ascontiguousarray(faces, np.int32); m = np.ascontiguousarray(fm, np.int32)
        n = self.L.ref_build(v.ctypes.data, len(v), f.ctypes.data, m.ctypes.data, nt, variant, leaf, collapse, nodes.ctypes.data, cap,
                             order.ctypes.data, tris.ctypes.data, woop.ctypes.data, C.byref(md), C.byref(sah), C.byref(ms))
        assert n > 0
        return dict(nodes=nodes[:n].copy(), order=order, tris=tris, woop=woop, max_depth=md.value, sah=sah.value)

    def trace_inst(self, width, any_hit, blas, tris, tlas, scene_root, inst, o, d, scene_of, threads=0):
        """The reference's travInst (Moller-Trumbore leaves) over a scene-tagged batch: (hits, hit instance)."""
        n = len(o)
        hits = np.zeros((n, 4), np.float32); hi = np.zeros(n, np.int32)
        a = [np.ascontiguousarray(x) for x in (blas, tris, tlas)]
        sr = np.ascontiguousarray(scene_root, np.int32); ins = np.ascontiguousarray(inst, np.float32); so = np.ascontiguousarray(scene_of, np.int32)
        self.L.ref_trace_inst(width, 1 if any_hit else 0, 0, a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, sr.ctypes.data, len(sr), ins.ctypes.data,
                              np.ascontiguousarray(o).ctypes.data, np.ascontiguousarray(d).ctypes.data, so.ctypes.data, n, hits.ctypes.data, hi.ctypes.data, threads)
        return hits, hi

    def trace(self, variant, tri, any_hit, nodes, tv, o, d, threads=0):
        n = len(o)
        hits = np.zeros((n, 4), np.float32); occ = np.zeros(n, np.int32)
        self.L.ref_trace(variant, 1 if any_hit else 0, tri, np.ascontiguousarray(nodes).ctypes.data, np.ascontiguousarray(tv).ctypes.data,
                         np.ascontiguousarray(o).ctypes.data, np.ascontiguousarray(d).ctypes.data, n, hits.ctypes.data, occ.ctypes.data, threads)
        return occ if any_hit else hits


@pytest.fixture(scope="session")
def ref():
    path = os.path.join(REF_DIR, "libcwpref.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built (needs the reference sources; see oracle/Makefile)")
    return Ref(path)


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA GPU")
    import torch
    torch.cuda.init()
    return torch


from importlib import import_module as _im
_pc = _im("cuda-wavefront-pathtracer_b200.precision_check")
classify_vs_fp64, wt32, edge_excess, explain_differences = _pc.classify_vs_fp64, _pc.wt32, _pc.edge_excess, _pc.explain_differences


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def tie_or_equal(h_a, h_b, rel=1e-6):
    """Per-ray classification of two closest-hit float4 arrays: (same id, tie, lost). A tie is two hits whose
    distances agree within rel * t; lost is hit vs miss or different hits at different distances."""
    ia, ib = h_a[:, 3].view(np.int32), h_b[:, 3].view(np.int32)
    same = ia == ib
    both = (ia >= 0) & (ib >= 0)
    ta, tb = h_a[:, 0].astype(np.float64), h_b[:, 0].astype(np.float64)
    tie = ~same & both & (np.abs(ta - tb) <= rel * np.maximum(np.abs(ta), np.abs(tb)))
    lost = ~same & ~tie
    return same, tie, lost
