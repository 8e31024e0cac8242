"""Precision form, host side: the FP64 watertight oracle traversing the CWBVH finds exactly the closest hits that
brute force over every triangle finds (so the conservative double-precision box test loses nothing)."""
import numpy as np
import pytest

from conftest import golden


def test_fp64_bvh_equals_brute_force_fixture(cwp, oracle):
    g = golden("boxes64.npz")
    mesh = cwp.Mesh.from_arrays(g["verts"], g["faces"], g["face_mat"])
    bvh = cwp.Bvh(mesh, variant=8, bins=16)
    t1, i1 = oracle.trace_fp64(bvh.nodes, bvh.verts, g["rays_o"], g["rays_d"])
    t2, i2 = oracle.trace_fp64(None, bvh.verts, g["rays_o"], g["rays_d"], brute=True)
    assert np.array_equal(i1, i2) and np.array_equal(t1, t2)
    o1 = oracle.trace_fp64(bvh.nodes, bvh.verts, g["rays_o"], g["rays_d"], any_hit=True)[1]
    assert np.array_equal(o1 >= 0, i2 >= 0)


def test_fp64_bvh_equals_brute_force_12k(cwp, oracle):
    mesh, bvh = cwp.scene("boxes12k", variant=8, bins=32)
    p = cwp.frame_params(mesh, 256, 256)
    o, d = cwp.incoherent_rays(2000, p, bvh.tris, lambda o, d: oracle.trace(8, 1, False, bvh.nodes, bvh.woop, o, d), seed=3)
    t1, i1 = oracle.trace_fp64(bvh.nodes, bvh.verts, o, d)
    t2, i2 = oracle.trace_fp64(None, bvh.verts, o, d, brute=True)
    assert np.array_equal(i1, i2) and np.array_equal(t1, t2)


def test_exact_corner_buffer(cwp):
    mesh, bvh = cwp.scene("boxes12k", variant=8, bins=32)
    v, f, _, _ = mesh.arrays()
    want = v[f[bvh.order]].reshape(-1, 3)
    assert np.array_equal(bvh.verts[:, :3], want) and np.all(bvh.verts[:, 3] == 0)
