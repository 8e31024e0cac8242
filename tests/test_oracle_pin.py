"""Pins the oracle (oracle/oracle.c) to the reference: the committed fixtures the reference's own code produced
(tests/golden/boxes64.npz) and, where oracle/_ref is built, the reference's code run here on larger inputs."""
import numpy as np
import pytest

from conftest import golden, tie_or_equal


@pytest.fixture(scope="module")
def g():
    return golden("boxes64.npz")


def test_oracle_bvh2_matches_reference_fixture(oracle, g):
    nodes, order, depth, _ = oracle.build(g["verts"], g["faces"], bins=16, leaf=4, variant=2)
    assert np.array_equal(nodes.view(np.uint32), g["bvh2_nodes"].view(np.uint32))
    assert np.array_equal(order, g["bvh2_order"])


def test_oracle_cwbvh_matches_reference_fixture(oracle, g):
    nodes, order, depth, _ = oracle.build(g["verts"], g["faces"], bins=16, leaf=4, variant=8)
    assert np.array_equal(nodes.view(np.uint32), g["cwbvh_nodes"].view(np.uint32))
    assert np.array_equal(order, g["cwbvh_order"])


def test_oracle_packing_matches_reference_fixture(oracle, g):
    for name in ("bvh2", "cwbvh"):
        tris, woop = oracle.pack(g["verts"], g["faces"], g["face_mat"], g[f"{name}_order"])
        assert np.array_equal(tris.view(np.uint32), g[f"{name}_tris"].view(np.uint32))
        assert np.array_equal(woop.view(np.uint32), g[f"{name}_woop"].view(np.uint32))


@pytest.mark.parametrize("name,variant", [("bvh2", 2), ("cwbvh", 8)])
@pytest.mark.parametrize("tri", [1, 0])
def test_oracle_traversal_matches_reference_fixture(oracle, g, name, variant, tri):
    tv = g[f"{name}_woop"] if tri else g[f"{name}_tris"]
    o, d = g["rays_o"], g["rays_d"]
    hits = oracle.trace(variant, tri, False, g[f"{name}_nodes"], tv, o, d)
    same, tie, lost = tie_or_equal(hits, g[f"{name}_t{tri}_closest"])
    # the oracle fuses multiply-adds where the reference's host build rounds twice: only exact ties may differ
    assert lost.sum() == 0, f"{lost.sum()} rays differ beyond a tie"
    assert same.mean() > 0.999
    occ = oracle.trace(variant, tri, True, g[f"{name}_nodes"], tv, o, d)
    ref_occ = g[f"{name}_t{tri}_any"]
    assert np.array_equal(occ >= 0, ref_occ >= 0), "occluded / unoccluded differs"


def test_oracle_rng_known_values(oracle):
    # the stateless hash is a pure function of (pixel, sample, depth, dim, seed); spot values fixed by core/rng.h
    vals = [oracle.L.orc_rng(p, s, dp, dm, 1000) for p, s, dp, dm in ((0, 0, 0, 0), (1, 2, 3, 4), (123456, 255, 5, 7))]
    assert all(0.0 <= x < 1.0 for x in vals)
    assert len(set(vals)) == 3
    # 24-bit resolution
    assert all(abs(x * 16777216 - round(x * 16777216)) < 1e-3 for x in vals)


@pytest.mark.parametrize("boxes", [256, 1024])
def test_oracle_build_matches_reference_code(oracle, ref, cwp, boxes):
    v, f, fm, _ = cwp.Mesh.box_field(boxes, 1).arrays()
    for variant in (2, 8):
        r = ref.build(v, f, fm, variant=variant, leaf=4)
        nodes, order, depth, _ = oracle.build(v, f, bins=16, leaf=4, variant=variant)
        assert np.array_equal(nodes.view(np.uint32), r["nodes"].view(np.uint32))
        assert np.array_equal(order, r["order"])
        assert depth == r["max_depth"]


def test_oracle_traversal_matches_reference_code(oracle, ref, cwp):
    mesh = cwp.Mesh.box_field(1024, 1)
    v, f, fm, _ = mesh.arrays()
    p = cwp.frame_params(mesh, 128, 128)
    for variant in (2, 8):
        r = ref.build(v, f, fm, variant=variant, leaf=4)
        o, d = cwp.incoherent_rays(20000, p, r["tris"], lambda o, d: ref.trace(variant, 1, False, r["nodes"], r["woop"], o, d), seed=9)
        for tri, tv in ((1, r["woop"]), (0, r["tris"])):
            same, tie, lost = tie_or_equal(oracle.trace(variant, tri, False, r["nodes"], tv, o, d), ref.trace(variant, tri, False, r["nodes"], tv, o, d))
            assert lost.sum() <= 2, (variant, tri, lost.sum())
            assert same.mean() > 0.999
