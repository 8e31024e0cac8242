"""Precision form, host side: the FP64 watertight oracle traversing the CWBVH finds exactly the closest hits that
brute force over every triangle finds (so the conservative double-precision box test loses nothing)."""
import numpy as np
import pytest

from conftest import classify_vs_fp64, edge_excess, golden, wt32


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


def test_half_rounding_emulation(oracle):
    """The oracle's f16 rounding (to nearest even, down, up) agrees with numpy's float16 conversion and brackets every
    value between adjacent halves, across normal, subnormal and overflowing magnitudes."""
    rng = np.random.default_rng(2)
    xs = np.concatenate([rng.normal(size=4000) * 10.0 ** rng.integers(-9, 6, 4000), [0.0, 65504.0, 65519.9, 65520.0, 7e4, -7e4, 2 ** -24, 3 * 2 ** -26, 1025.5, 1026.5]])
    hr = oracle.L.orc_half_round
    with np.errstate(over="ignore"):
        for x in xs:
            rn, rd, ru = hr(float(x), 0), hr(float(x), -1), hr(float(x), 1)
            assert rn == float(np.float16(x)) or (np.isinf(rn) and np.isinf(np.float16(x))), x
            assert rd <= x <= ru, x
            for r in (rd, ru):
                assert np.isinf(r) or float(np.float16(r)) == r, x
            if rd != ru and np.isfinite(rd) and np.isfinite(ru):
                assert np.nextafter(np.float16(rd), np.float16(np.inf)) == np.float16(ru), x


def test_precision_restatement_against_fp64_12k(cwp, oracle):
    """The precision form restated on the host (f16 conservative slabs, watertight FP32 triangles): no hit the FP64
    oracle finds is lost, different triangles only at equal distance, t within 1e-6 of max(t, scene extent), and
    the conservative box test costs at most 1.5x the plain form's node visits."""
    mesh, bvh = cwp.scene("boxes12k", variant=8, bins=32)
    p = cwp.frame_params(mesh, 256, 256)
    o, d = cwp.incoherent_rays(20000, p, bvh.tris, lambda o, d: oracle.trace(8, 1, False, bvh.nodes, bvh.woop, o, d), seed=29)
    h, st = oracle.trace_prec(bvh.nodes, bvh.verts, o, d, stats=True)
    _, st_plain = oracle.trace(8, 1, False, bvh.nodes, bvh.woop, o, d, stats=True)
    t64, i64 = oracle.trace_fp64(bvh.nodes, bvh.verts, o, d)
    ext = float(np.ptp(mesh.arrays()[0], axis=0).max())
    c = classify_vs_fp64(h, t64, i64, ext, o=o, d=d, verts=bvh.verts)
    assert c["lost"] == 0 and c["max_t_error"] <= 1e-6, c
    ih = h[:, 3].view(np.int32); k = ih >= 0
    acc, t32 = wt32(o[k], d[k], bvh.verts, ih[k])   # the numpy mirror of the FP32 triangle test agrees bit for bit
    assert acc.all() and np.array_equal(t32, h[k, 0])
    ex = c["extra_mask"]
    assert np.all(edge_excess(o[ex], d[ex], bvh.verts, h[ex, 3].view(np.int32)) <= 1.0)
    assert st[0] <= 1.5 * st_plain[0]
    occ = oracle.trace_prec(bvh.nodes, bvh.verts, o, d, any_hit=True)
    assert np.all(occ[i64 >= 0] >= 0)


def test_precision_restatement_corners_and_edges(cwp, oracle):
    """Rays aimed exactly at corners and edge midpoints: the conservative FP32 edge test never loses a hit that the
    FP64 oracle finds; the hits FP64 does not report lie within the edge bound of the reported triangle."""
    mesh, bvh = cwp.scene("boxes12k", variant=8, bins=32)
    v, f, _, _ = mesh.arrays()
    rng = np.random.default_rng(5)
    tri = v[f[rng.choice(len(f), 4000)]]
    targets = np.concatenate([tri[:, 0], 0.5 * (tri[:, 0] + tri[:, 1]), 0.5 * (tri[:, 1] + tri[:, 2])]).astype(np.float32)
    dirs = rng.normal(size=targets.shape).astype(np.float32); dirs[:, 2] = -np.abs(dirs[:, 2]) - 0.2
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    o = np.zeros((len(targets), 4), np.float32); o[:, :3] = targets - 30.0 * dirs
    d = np.zeros((len(targets), 4), np.float32); d[:, :3] = dirs; d[:, 3] = 1e30
    t64, i64 = oracle.trace_fp64(bvh.nodes, bvh.verts, o, d)
    h = oracle.trace_prec(bvh.nodes, bvh.verts, o, d)
    c = classify_vs_fp64(h, t64, i64, float(np.ptp(v, axis=0).max()), o=o, d=d, verts=bvh.verts)
    assert c["lost"] == 0, c
    ex = c["extra_mask"]
    assert np.all(edge_excess(o[ex], d[ex], bvh.verts, h[ex, 3].view(np.int32)) <= 1.0)


def test_explain_differences_classes():
    """The FP64 classification of disagreeing rays (used against the reference's fast-math device traversal): one
    unit triangle in the plane z = 0 and a second one behind it at z = -1, rays straight down."""
    from conftest import explain_differences
    verts = np.zeros((6, 4), np.float32)
    verts[0, :3], verts[1, :3], verts[2, :3] = (0, 0, 0), (1, 0, 0), (0, 1, 0)
    verts[3, :3], verts[4, :3], verts[5, :3] = (-5, -5, -1), (5, -5, -1), (0, 5, -1)
    xy = np.array([[0.25, 0.25], [0.25, 0.25], [0.5, 0.5 + 1e-9], [0.25, 0.25], [0.25, 0.25]], np.float32)
    o = np.zeros((len(xy), 4), np.float32); o[:, :2] = xy; o[:, 2] = 1
    d = np.zeros((len(xy), 4), np.float32); d[:, 2] = -1; d[:, 3] = 1e30

    def hits(tri, t):
        h = np.zeros((len(tri), 4), np.float32); h[:, 0] = t; h[:, 3] = np.asarray(tri, np.int32).view(np.float32)
        return h
    ours = hits([0, 0, 1, 1, 0], [1, 1, 2, 2, 1])
    other = hits([0, 1, 0, 0, -1], [1, 2, 1, 1, 1e30])
    c, rows = explain_differences(o, d, verts, ours, other)
    cls = [r["class"] for r in rows]
    # ray 1: ours inside and closer; ray 2: the other's triangle within 1e-9 of the edge u + v = 1; ray 3: the other
    # reports the closer triangle, well inside it, and ours the farther one; ray 4: the other misses a hit inside
    assert cls == ["ours_exact", "graze", "unexplained", "ours_exact"] and c["differ"] == 4
    occ_o, occ_x = np.array([0, -1, -1, 0, 0], np.int32), np.array([0, 0, 0, -1, 0], np.int32)
    c, rows = explain_differences(o, d, verts, occ_o, occ_x, any_hit=True)
    # ray 1: the other's occluder is inside (we missed it); ray 2: near the edge; ray 3: ours inside
    assert [r["class"] for r in rows] == ["unexplained", "graze", "ours_exact"]


def _key(t, slot):
    """the closest-hit kernel's shared-test key (trace.cu wt_key): the float order of t in the high 32 bits, the slot
    in the low ones"""
    u = int(np.float32(t).view(np.uint32))
    hi = (~u & 0xFFFFFFFF) if u & 0x80000000 else (u | 0x80000000)
    return (hi << 32) | slot


def test_shared_triangle_tests_keep_the_sequential_hit():
    """A model of the precision form's shared triangle tests: a ray's pending triangles (slot order) are tested in
    rounds of up to 32 against the interval the previous round left, and the smallest (t, slot) key of each round's
    hits wins. That is the hit one-by-one testing keeps (a later triangle replaces the hit only when strictly closer),
    over random distances with repeats (ties), negative t, misses and lists longer than a round."""
    rng = np.random.default_rng(3)
    for trial in range(4000):
        n = int(rng.integers(1, 80))
        tmin = float(np.float32(rng.choice([0.0, -0.5, 1e-4])))
        tmax = float(np.float32(rng.choice([1e30, 5.0, 2.0])))
        pool = np.float32(rng.uniform(-1.0, 6.0, 6))            # few distinct values: many exact ties
        t = np.float32(rng.choice(pool, n))
        hit = rng.random(n) < 0.6                                 # the watertight test's verdict on the triangle
        # sequential: one test at a time, strict tmin < t < hitT
        hitT, win = tmax, -1
        for i in range(n):
            if hit[i] and tmin < t[i] < hitT:
                hitT, win = float(t[i]), i
        # shared: rounds of 32 slots, each tested against the interval the previous rounds left
        hitT2, win2 = tmax, -1
        # the slot offset within the warp differs from the ray's own index by the lanes before it: keep a random base
        first = int(rng.integers(0, 32))
        for base in range(0, first + n, 32):
            best = None
            for s in range(max(base, first), min(base + 32, first + n)):
                i = s - first
                if hit[i] and tmin < t[i] < hitT2:
                    k = _key(t[i], s)
                    best = k if best is None else min(best, k)
            if best is not None:
                win2 = (best & 0xFFFFFFFF) - first
                hitT2 = float(t[win2])
        assert (win, hitT) == (win2, hitT2), (trial, win, win2, hitT, hitT2)
