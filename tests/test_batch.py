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


def _tlas2_from_boxes(cwp, lo, hi):
    """host BVH2 over instance boxes (leaf = one instance; references are instance indices)"""
    n = len(lo)
    V = np.concatenate([np.stack([lo[i], hi[i], lo[i]]) for i in range(n)]).astype(np.float32)
    tb = cwp.Bvh(cwp.Mesh.from_arrays(V, np.arange(3 * n, dtype=np.int32).reshape(n, 3)), variant=2, bins=32, leaf=1)
    t = tb.nodes.copy(); tv = t.view(np.int32)
    for r in range(3, len(t), 4):
        for j in (0, 1):
            if tv[r, 2 + j] > 0:
                tv[r, j] = tb.order[tv[r, j]]
    return t


def tlas4_from_tlas2(t2):
    """The width-4 TLAS of a BVH2 TLAS, node for node: node i's children are the grandchildren of BVH2 node i (a child
    that is an instance stays one child). The GPU writes its width-4 TLAS by the same rule from the H-PLOC tree."""
    E = np.float32(3.4e38)
    n = len(t2) // 4
    B = t2.reshape(n, 4, 4); iv = t2.view(np.int32).reshape(n, 4, 4)
    child = lambda i, j: (iv[i, 3, j], iv[i, 3, 2 + j],
                          (B[i, j, 0], B[i, j, 2], B[i, 2, 2 * j]), (B[i, j, 1], B[i, j, 3], B[i, 2, 2 * j + 1]))
    out = np.zeros((n, 8, 4), np.float32); ov = out.view(np.int32)
    for i in range(n):
        kids = []
        for j in (0, 1):
            c, k, lo, hi = child(i, j)
            if c < 0:
                continue
            if k > 0:
                kids.append((c, 1, lo, hi))
            else:
                for jj in (0, 1):
                    g, kg, glo, ghi = child(c, jj)
                    if g >= 0:
                        kids.append((g, 1 if kg > 0 else 0, glo, ghi))
        for s in range(4):
            if s < len(kids):
                c, k, lo, hi = kids[s]
                ov[i, 6, s], ov[i, 7, s] = c, k
                for a in range(3):
                    out[i, 2 * a, s], out[i, 2 * a + 1, s] = lo[a], hi[a]
            else:
                ov[i, 6, s], ov[i, 7, s] = -1, 0
                for a in range(3):
                    out[i, 2 * a, s], out[i, 2 * a + 1, s] = E, E
    return out.reshape(8 * n, 4)


def test_oracle_tlas4_matches_tlas2(cwp, oracle):
    """The oracle's two-level traversal over a width-4 TLAS (grandchildren of a BVH2 TLAS) finds the same closest
    hits and occlusion as over the BVH2 TLAS itself: 40 instances of a box field, rigid motions, random rays."""
    g = golden("boxes64.npz")
    mesh = cwp.Mesh.from_arrays(g["verts"], g["faces"], g["face_mat"])
    bvh = cwp.Bvh(mesh, variant=8, bins=16, leaf=1)
    rng = np.random.default_rng(5)
    v = g["verts"].astype(np.float64); blo, bhi = v.min(0), v.max(0)
    recs, lo, hi = [], [], []
    for i in range(40):
        m = cwp.xform_animate(0, 0, translate=tuple(rng.uniform(-60, 60, 3)), axis=tuple(rng.normal(size=3)), angle_deg=float(rng.uniform(0, 360)))
        r = np.frombuffer(bytes(cwp.instances([m], [0])), np.float32).reshape(28).copy()
        r[24] = np.array([0], np.int32).view(np.float32)[0]
        recs.append(r)
        A = m.reshape(3, 4).astype(np.float64)
        cs = np.array([[x, y, z] for x in (blo[0], bhi[0]) for y in (blo[1], bhi[1]) for z in (blo[2], bhi[2])]) @ A[:, :3].T + A[:, 3]
        lo.append(cs.min(0) - 1e-3); hi.append(cs.max(0) + 1e-3)
    rec = np.array(recs, np.float32)
    t2 = _tlas2_from_boxes(cwp, np.array(lo, np.float32), np.array(hi, np.float32))
    t4 = tlas4_from_tlas2(t2)
    o = np.zeros((3000, 4), np.float32); d = np.zeros((3000, 4), np.float32)
    o[:, :3] = rng.uniform(-90, 90, (3000, 3)); dd = rng.normal(size=(3000, 3)); d[:, :3] = dd / np.linalg.norm(dd, axis=1, keepdims=True)
    d[:, 3] = 1e30
    sc = np.zeros(3000, np.int32); root = np.array([0], np.int32)
    for any_hit in (False, True):
        h2, i2 = oracle.trace_inst(8, any_hit, bvh.nodes, bvh.tris, t2, root, rec, o, d, sc, tlas_width=2)
        h4, i4 = oracle.trace_inst(8, any_hit, bvh.nodes, bvh.tris, t4, root, rec, o, d, sc, tlas_width=4)
        if any_hit:
            assert np.array_equal(i2 >= 0, i4 >= 0)
        else:
            assert (i2 >= 0).mean() > 0.1
            same = (i2 == i4) & (h2[:, 3].view(np.int32) == h4[:, 3].view(np.int32))
            assert np.array_equal(h2[:, 0].view(np.uint32), h4[:, 0].view(np.uint32))   # closest t never depends on the order
            assert same.mean() > 0.999
