"""Host BVH construction of the library (C ABI cwp_bvh_build) against the reference's encodings: byte-identical
node arrays, leaf orders, packed triangles and Woop rows; independence of the thread count; the 32-bin build
against the oracle; edge cases."""
import numpy as np
import pytest

from conftest import golden


@pytest.fixture(scope="module")
def g():
    return golden("boxes64.npz")


def _mesh(cwp, g):
    return cwp.Mesh.from_arrays(g["verts"], g["faces"], g["face_mat"])


@pytest.mark.parametrize("name,variant,collapse", [("bvh2", 2, 0), ("bvh4", 4, 0), ("bvh8g", 8, 1), ("cwbvh", 8, 0)])
def test_build_matches_reference_fixture(cwp, g, name, variant, collapse):
    b = cwp.Bvh(_mesh(cwp, g), variant=variant, bins=16, leaf=4, collapse=collapse)
    assert np.array_equal(b.nodes.view(np.uint32), g[f"{name}_nodes"].view(np.uint32))
    assert np.array_equal(b.order, g[f"{name}_order"])
    if f"{name}_tris" in g:
        assert np.array_equal(b.tris.view(np.uint32), g[f"{name}_tris"].view(np.uint32))
        assert np.array_equal(b.woop.view(np.uint32), g[f"{name}_woop"].view(np.uint32))


def test_box_field_sizes(cwp):
    assert cwp.Mesh.box_field(1024, 1).n_tris == 12290
    assert cwp.Mesh.box_field(9750, 1).n_tris == 117002


def test_box_field_deterministic(cwp):
    a = cwp.Mesh.box_field(100, 3).arrays()[0]; b = cwp.Mesh.box_field(100, 3).arrays()[0]; c = cwp.Mesh.box_field(100, 4).arrays()[0]
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert a[:, 2].min() == 0.0 and a[:, 2].max() <= 3.0 + 1e-6   # boxes rest on the ground (z up)
    assert np.abs(a[:, :2]).max() <= 20.0 + 3.0


@pytest.mark.parametrize("variant", [2, 4, 8])
def test_build_thread_count_independent(cwp, variant):
    mesh = cwp.Mesh.box_field(3000, 2)
    a = cwp.Bvh(mesh, variant=variant, bins=32, threads=1)
    b = cwp.Bvh(mesh, variant=variant, bins=32, threads=0)
    c = cwp.Bvh(mesh, variant=variant, bins=32, threads=3)
    for x in (b, c):
        assert np.array_equal(a.nodes.view(np.uint32), x.nodes.view(np.uint32)) and np.array_equal(a.order, x.order)


@pytest.mark.parametrize("bins", [16, 32, 7])
def test_build_matches_oracle_any_bins(cwp, oracle, bins):
    mesh = cwp.Mesh.box_field(1024, 1)
    v, f, fm, _ = mesh.arrays()
    for variant in (2, 8):
        b = cwp.Bvh(mesh, variant=variant, bins=bins, leaf=4)
        nodes, order, depth, _ = oracle.build(v, f, bins=bins, leaf=4, variant=variant)
        assert np.array_equal(b.nodes.view(np.uint32), nodes.view(np.uint32))
        assert np.array_equal(b.order, order)
        tris, woop = oracle.pack(v, f, fm, order)
        assert np.array_equal(b.woop.view(np.uint32), woop.view(np.uint32))


@pytest.mark.parametrize("variant,collapse", [(2, 0), (4, 0), (8, 0), (8, 1)])
def test_build_matches_reference_code_117k(cwp, ref, variant, collapse):
    mesh = cwp.Mesh.box_field(9750, 1)
    v, f, fm, _ = mesh.arrays()
    b = cwp.Bvh(mesh, variant=variant, bins=16, leaf=4, collapse=collapse)
    r = ref.build(v, f, fm, variant=variant, leaf=4, collapse=collapse)
    assert np.array_equal(b.nodes.view(np.uint32), r["nodes"].view(np.uint32))
    assert np.array_equal(b.order, r["order"])
    assert np.array_equal(b.woop.view(np.uint32), r["woop"].view(np.uint32))
    assert b.max_depth == r["max_depth"]
    assert abs(b.sah - r["sah"]) <= 1e-9 * abs(r["sah"])


def test_single_triangle_root_leaf(cwp, ref):
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32); f = np.array([[0, 1, 2]], np.int32); fm = np.zeros(1, np.int32)
    mesh = cwp.Mesh.from_arrays(v, f, fm)
    for variant, collapse in ((2, 0), (4, 0), (8, 0), (8, 1)):
        b = cwp.Bvh(mesh, variant=variant, collapse=collapse)
        r = ref.build(v, f, fm, variant=variant, leaf=4, collapse=collapse)
        assert np.array_equal(b.nodes.view(np.uint32), r["nodes"].view(np.uint32)), variant


def test_coincident_centroids(cwp, ref):
    # 40 copies of the same triangle: every axis of the centroid box is degenerate -> median splits
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32); f = np.tile(np.array([[0, 1, 2]], np.int32), (40, 1)); fm = np.zeros(40, np.int32)
    mesh = cwp.Mesh.from_arrays(v, f, fm)
    for variant in (2, 8):
        b = cwp.Bvh(mesh, variant=variant)
        r = ref.build(v, f, fm, variant=variant, leaf=4)
        assert np.array_equal(b.nodes.view(np.uint32), r["nodes"].view(np.uint32))
        assert np.array_equal(b.order, r["order"])


def test_invalid_inputs(cwp):
    with pytest.raises(cwp.CwpError):
        cwp.Mesh.from_arrays(np.zeros((3, 3), np.float32), np.array([[0, 1, 5]], np.int32))
    empty = cwp.Mesh.from_arrays(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32))
    with pytest.raises(cwp.CwpError):
        cwp.Bvh(empty)
    mesh = cwp.Mesh.box_field(4, 1)
    for kw in (dict(variant=3), dict(bins=1), dict(leaf=0), dict(collapse=2)):
        with pytest.raises(cwp.CwpError) as e:
            cwp.Bvh(mesh, **kw)
        assert e.value.code == cwp.ERR_INVALID


@pytest.mark.parametrize("variant", [2, 4, 8])
def test_spatial_splits_same_hits_fewer_visits(cwp, oracle, variant):
    """SBVH (spatial splits): every triangle is referenced, the tree does not depend on the thread count, and the
    oracle traversal finds the same closest triangle (original id) at the same distance as over the binned-SAH tree,
    visiting fewer nodes."""
    mesh = cwp.Mesh.box_field(600, 1)
    leaf = 1 if variant == 8 else 4
    b0 = cwp.Bvh(mesh, variant=variant, bins=32, leaf=leaf)
    b1 = cwp.Bvh(mesh, variant=variant, bins=32, leaf=leaf, spatial=1e-5)
    b1s = cwp.Bvh(mesh, variant=variant, bins=32, leaf=leaf, spatial=1e-5, threads=1)
    assert np.array_equal(b1.nodes.view(np.uint32), b1s.nodes.view(np.uint32)) and np.array_equal(b1.order, b1s.order)
    assert set(b1.order.tolist()) == set(range(mesh.n_tris)) and len(b1.order) > mesh.n_tris
    p = cwp.frame_params(mesh, 128, 128)
    o, d = cwp.incoherent_rays(4000, p, b0.tris, lambda o, d: oracle.trace(variant, 1, False, b0.nodes, b0.woop, o, d), seed=2)
    h0, s0 = oracle.trace(variant, 1, False, b0.nodes, b0.woop, o, d, stats=True)
    h1, s1 = oracle.trace(variant, 1, False, b1.nodes, b1.woop, o, d, stats=True)
    i0, i1 = h0[:, 3].view(np.int32), h1[:, 3].view(np.int32)
    id0 = np.where(i0 >= 0, b0.tris[3 * np.maximum(i0, 0), 3].view(np.int32), -1)
    id1 = np.where(i1 >= 0, b1.tris[3 * np.maximum(i1, 0), 3].view(np.int32), -1)
    same = id0 == id1
    tie = ~same & (i0 >= 0) & (i1 >= 0) & (np.abs(h0[:, 0] - h1[:, 0]) <= 1e-6 * np.abs(h0[:, 0]))
    assert np.all(same | tie) and np.array_equal(h0[same, 0], h1[same, 0])
    assert s1[0] < s0[0]
    occ0 = oracle.trace(variant, 1, True, b0.nodes, b0.woop, o, d); occ1 = oracle.trace(variant, 1, True, b1.nodes, b1.woop, o, d)
    assert np.array_equal(occ0 >= 0, occ1 >= 0)


def test_frame_work_counters(cwp, oracle):
    """The oracle's frame counters (the on-chip roofline's algorithmic bytes) count the same rays as the frame and do
    not change its image; the spatial-split tree needs fewer node visits per closest ray for the same frame."""
    mesh = cwp.Mesh.box_field(300, 1)
    p = cwp.frame_params(mesh, 32, 32, bounces=2)
    b0 = cwp.Bvh(mesh, variant=8, bins=32, leaf=1)
    b1 = cwp.Bvh(mesh, variant=8, bins=32, leaf=1, spatial=1e-3)
    acc, rc = oracle.render(p, 8, 1, b0, 2, 4, 0, 0, 1024)
    rc0, st0 = oracle.render_work(p, 8, 1, b0, 2, 4, 0, 1024)
    assert np.array_equal(rc, rc0) and rc0[0] > 0 and rc0[1] > 0
    assert np.all(st0 > 0) and st0[0] >= rc0[0] and st0[2] >= rc0[1]   # at least the root per ray
    acc2, _ = oracle.render(p, 8, 1, b0, 2, 4, 0, 0, 1024)            # counters off again: same image
    assert np.array_equal(acc, acc2)
    rc1, st1 = oracle.render_work(p, 8, 1, b1, 2, 4, 0, 1024)
    assert st1[0] / rc1[0] < st0[0] / rc0[0]
