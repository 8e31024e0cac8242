"""Batched form, host side: instance transforms against the reference's own invertXform / instanceXform (fixtures
made by its code), the oracle's BVH4 traversal against the reference's, and the oracle's two-level traversal against
single-level traversal and brute force."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden, tie_or_equal


def test_xform_invert_matches_reference(cwp):
    g = golden("instances.npz")
    for m, inv, det in zip(g["mats"], g["inv"], g["det_sign"]):
        got, sg = cwp.xform_invert(m)
        assert np.array_equal(got.view(np.uint32), inv.view(np.uint32)) and sg == det


def test_xform_animate_matches_reference(cwp):
    g = golden("instances.npz")
    for i in range(len(g["desc_angle"])):
        for j, f in enumerate(g["frames"]):
            m = cwp.xform_animate(0, int(f), translate=g["desc_translate"][i], axis=g["desc_axis"][i], angle_deg=float(g["desc_angle"][i]),
                                  scale=g["desc_scale"][i], translate_per_frame=g["desc_translate_vel"][i],
                                  angle_deg_per_frame=float(g["desc_angle_vel"][i]), scale_per_frame=g["desc_scale_vel"][i])
            assert np.array_equal(m.view(np.uint32), g["anim"][i, j].view(np.uint32)), (i, f)


def test_instance_record(cwp):
    m = cwp.xform_animate(0, 0, translate=(1, 2, 3), axis=(0, 1, 0), angle_deg=30, scale=(2, 2, 2))
    rec = cwp.instances([m], [3])[0]
    assert C.sizeof(cwp.Instance) == 112 and rec.mesh == 3 and rec.root == -1 and rec.det_sign == 1.0
    fwd = np.array(rec.fwd).reshape(3, 4); inv = np.array(rec.inv).reshape(3, 4)
    A = np.vstack([fwd, [0, 0, 0, 1]]); B = np.vstack([inv, [0, 0, 0, 1]])
    assert np.allclose(A @ B, np.eye(4), atol=1e-6)
    with pytest.raises(cwp.CwpError):
        cwp.instances([m], [-1])


def test_oracle_bvh4_matches_reference_traversal(oracle):
    g, h = golden("boxes64.npz"), golden("instances.npz")
    for tri, tv in ((1, h["bvh4_woop"]), (0, h["bvh4_tris"])):
        got = oracle.trace(4, tri, False, g["bvh4_nodes"], tv, g["rays_o"], g["rays_d"])
        same, tie, lost = tie_or_equal(got, h[f"bvh4_t{tri}_closest"])
        assert not lost.any() and tie.sum() <= 2
        occ = oracle.trace(4, tri, True, g["bvh4_nodes"], tv, g["rays_o"], g["rays_d"])
        assert np.array_equal(occ >= 0, h[f"bvh4_t{tri}_any"] >= 0)


def _single_instance_tlas(inst):
    """TLAS of one instance: a root whose first child is the instance leaf (a box covering everything) and whose
    second child is empty."""
    E = 3e37
    lo, hi = [-1e30] * 3, [1e30] * 3
    t = np.zeros((4, 4), np.float32)
    t[0] = [lo[0], hi[0], lo[1], hi[1]]; t[1] = [E, E, E, E]; t[2] = [lo[2], hi[2], E, E]
    t[3] = np.array([0, -1, 1, 0], np.int32).view(np.float32)
    return t


@pytest.mark.parametrize("width", [2, 4, 8])
def test_oracle_two_level_single_instance(cwp, oracle, width):
    """One instance under a one-node TLAS: identity gives the single-level result bit for bit; a rigid motion gives
    the brute-force closest hits of the moved triangles."""
    g = golden("boxes64.npz")
    mesh = cwp.Mesh.from_arrays(g["verts"], g["faces"], g["face_mat"])
    bvh = cwp.Bvh(mesh, variant=width, bins=16, leaf=4 if width != 8 else 1)
    o, d = g["rays_o"], g["rays_d"]
    ident = np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], np.float32)
    rec = np.frombuffer(bytes(cwp.instances([ident], [0])), np.float32).reshape(1, 28).copy()
    rec[0, 24] = np.array([0], np.int32).view(np.float32)[0]   # root node of the BLAS
    tlas = _single_instance_tlas(rec)
    h, hi = oracle.trace_inst(width, False, bvh.nodes, bvh.tris, tlas, np.array([0], np.int32), rec, o, d, np.zeros(len(o), np.int32))
    ref = oracle.trace(width, 0, False, bvh.nodes, bvh.tris, o, d)
    assert np.array_equal(h.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(hi, np.where(ref[:, 3].view(np.int32) >= 0, 0, -1))
    # moved: world triangles = fwd(object triangles); compare distances with a float64 brute force in world space
    m = cwp.xform_animate(0, 0, translate=(3, -2, 1), axis=(1, 2, 3), angle_deg=40, scale=(1, 1, 1))
    rec = np.frombuffer(bytes(cwp.instances([m], [0])), np.float32).reshape(1, 28).copy()
    rec[0, 24] = np.array([0], np.int32).view(np.float32)[0]
    h, hi = oracle.trace_inst(width, False, bvh.nodes, bvh.tris, tlas, np.array([0], np.int32), rec, o, d, np.zeros(len(o), np.int32))
    A = m.reshape(3, 4).astype(np.float64)
    v = g["verts"][g["faces"]].astype(np.float64) @ A[:, :3].T + A[:, 3]
    t_bf = _brute_force(o[:, :3].astype(np.float64), d[:, :3].astype(np.float64), v)
    hit = np.isfinite(t_bf)
    ih = h[:, 3].view(np.int32)
    assert np.array_equal(ih >= 0, hit) or np.sum((ih >= 0) != hit) <= 2   # grazing edge rays may differ
    both = hit & (ih >= 0)
    assert np.allclose(h[both, 0], t_bf[both], rtol=1e-4, atol=1e-4)


def _brute_force(o, d, v):
    """closest t of rays (o, d) against triangles v [m, 3, 3] in float64 (inf on a miss)"""
    e1 = v[:, 1] - v[:, 0]; e2 = v[:, 2] - v[:, 0]
    best = np.full(len(o), np.inf)
    for k in range(len(v)):
        p = np.cross(d, e2[k]); det = p @ e1[k]
        ok = np.abs(det) > 1e-14
        inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
        s = o - v[k, 0]; u = (s * p).sum(1) * inv
        q = np.cross(s, e1[k]); w = (d * q).sum(1) * inv; t = (q @ e2[k]) * inv
        good = ok & (u >= 0) & (w >= 0) & (u + w <= 1) & (t > 0)
        best = np.where(good & (t < best), t, best)
    return best
