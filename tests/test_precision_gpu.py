"""Precision form on the GPU (config 1's 12,290-triangle scene): f16x2 conservative slab tests over the CWBVH's 8-bit
child boxes plus the watertight FP32 triangle test. Checked against the FP64 oracle on the GPU (itself bit-identical
to the oracle's host restatement): no lost hits, ties only among equal distances, t within 1e-6 of max(t, scene extent)
(FP32 cancellation on large triangles near the origin bounds t absolutely, not relatively); an adversarial batch
aimed at shared edges and corners finds no gap, and every hit that FP64 does not report lies within the conservative
FP32 edge bound of the reported triangle. The CUDA precision form also returns, bit for bit, what the oracle's
exact-f16 restatement of it returns."""
import numpy as np
import pytest

from conftest import classify_vs_fp64, edge_excess

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run(torch, acc, o, d, any_hit=False):
    to, td = dev(torch, o), dev(torch, d); n = len(o)
    if any_hit:
        out = torch.empty(n, dtype=torch.int32, device="cuda"); acc.trace_any(to.data_ptr(), td.data_ptr(), out.data_ptr(), n)
    else:
        out = torch.empty((n, 4), dtype=torch.float32, device="cuda"); acc.trace_closest(to.data_ptr(), td.data_ptr(), out.data_ptr(), n)
    torch.cuda.synchronize(); acc.status()
    return out.cpu().numpy()


def run64(torch, acc, o, d, any_hit=False):
    to, td = dev(torch, o), dev(torch, d); n = len(o)
    t = torch.empty(n, dtype=torch.float64, device="cuda"); tri = torch.empty(n, dtype=torch.int32, device="cuda")
    acc.trace_fp64(to.data_ptr(), td.data_ptr(), t.data_ptr(), tri.data_ptr(), n, any_hit=any_hit)
    torch.cuda.synchronize(); acc.status()
    return t.cpu().numpy(), tri.cpu().numpy()


def extent(mesh):
    return float(np.ptp(mesh.arrays()[0], axis=0).max())


@pytest.fixture(scope="module")
def scene12k(cwp):
    return cwp.scene("boxes12k", variant=8, bins=32)


def test_fp64_gpu_matches_host_oracle(gpu, cwp, oracle, scene12k):
    mesh, bvh = scene12k
    acc = cwp.Accel(bvh, tri=1)
    p = cwp.frame_params(mesh, 256, 256)
    o, d = cwp.incoherent_rays(20000, p, bvh.tris, lambda o, d: run(gpu, acc, o, d), seed=13)
    t, i = run64(gpu, acc, o, d)
    th, ih = oracle.trace_fp64(bvh.nodes, bvh.verts, o, d)
    assert np.array_equal(i, ih) and np.array_equal(t, th)


def test_precision_form_loses_no_hit_1m(gpu, cwp, scene12k):
    mesh, bvh = scene12k
    acc = cwp.Accel(bvh, tri=1)
    p = cwp.frame_params(mesh, 256, 256)
    o, d = cwp.incoherent_rays(1 << 20, p, bvh.tris, lambda o, d: run(gpu, acc, o, d), seed=17)
    t64, i64 = run64(gpu, acc, o, d)
    acc.set_precision(1)
    h = run(gpu, acc, o, d)
    c = classify_vs_fp64(h, t64, i64, extent(mesh), o=o, d=d, verts=bvh.verts)
    assert c["lost"] == 0, c
    assert c["tie"] + c["extra"] <= 1e-4 * len(o), c
    assert c["max_t_error"] <= 1e-6, c
    ex = c["extra_mask"]
    assert np.all(edge_excess(o[ex], d[ex], bvh.verts, h[ex, 3].view(np.int32)) <= 1.0)
    occ = run(gpu, acc, o, d, any_hit=True)
    _, o64 = run64(gpu, acc, o, d, any_hit=True)
    assert np.all(occ[o64 >= 0] >= 0)                      # no occluder lost
    extra = (occ >= 0) & (o64 < 0)                         # occluders within the edge bound of a silhouette
    assert np.all(edge_excess(o[extra], d[extra], bvh.verts, occ[extra]) <= 1.0)


def test_watertight_on_shared_edges_and_corners(gpu, cwp, scene12k):
    """Rays from above aimed exactly at corner positions and edge midpoints of the mesh: the precision form hits
    whenever the FP64 oracle does (no ray slips between neighbouring triangles)."""
    mesh, bvh = scene12k
    v, f, _, _ = mesh.arrays()
    rng = np.random.default_rng(5)
    pick = rng.choice(len(f), 20000)
    tri = v[f[pick]]
    targets = np.concatenate([tri[:, 0], 0.5 * (tri[:, 0] + tri[:, 1]), 0.5 * (tri[:, 1] + tri[:, 2])]).astype(np.float32)
    dirs = rng.normal(size=targets.shape).astype(np.float32); dirs[:, 2] = -np.abs(dirs[:, 2]) - 0.2
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    o = np.zeros((len(targets), 4), np.float32); o[:, :3] = targets - 30.0 * dirs
    d = np.zeros((len(targets), 4), np.float32); d[:, :3] = dirs; d[:, 3] = 1e30
    acc = cwp.Accel(bvh, tri=1)
    t64, i64 = run64(gpu, acc, o, d)
    acc.set_precision(1)
    h = run(gpu, acc, o, d)
    c = classify_vs_fp64(h, t64, i64, extent(mesh), o=o, d=d, verts=bvh.verts)
    assert c["lost"] == 0, c
    # silhouette rays that FP64 passes just outside a corner may hit within the conservative edge bound
    ex = c["extra_mask"]
    assert np.all(edge_excess(o[ex], d[ex], bvh.verts, h[ex, 3].view(np.int32)) <= 1.0)


def test_precision_form_matches_host_restatement(gpu, cwp, oracle, scene12k):
    """Every f16 slab test and FP32 triangle test on the GPU rounds exactly as the oracle's restatement: closest hits
    (t, u, v, triangle) and first occluders identical bit for bit."""
    mesh, bvh = scene12k
    acc = cwp.Accel(bvh, tri=1)
    p = cwp.frame_params(mesh, 256, 256)
    o, d = cwp.incoherent_rays(40000, p, bvh.tris, lambda o, d: run(gpu, acc, o, d), seed=31)
    acc.set_precision(1)
    for trav in (1, 2):   # refill kernel and one ray per thread
        acc.set_traversal(trav)
        h = run(gpu, acc, o, d)
        assert np.array_equal(h.view(np.uint32), oracle.trace_prec(bvh.nodes, bvh.verts, o, d).view(np.uint32))
        assert np.array_equal(run(gpu, acc, o, d, any_hit=True), oracle.trace_prec(bvh.nodes, bvh.verts, o, d, any_hit=True))


def test_precision_form_matches_host_restatement_signed_interval(gpu, cwp, oracle, scene12k):
    """The closest-hit kernel ranks a warp's shared triangle tests by (t, slot) on the float order of t: rays whose
    interval starts behind the origin (tmin = -0.5, so hits at negative t count) and ends short (tmax = 5) still give
    the oracle's restatement bit for bit, through the refill kernel and one ray per thread."""
    mesh, bvh = scene12k
    acc = cwp.Accel(bvh, tri=1)
    p = cwp.frame_params(mesh, 256, 256)
    o, d = cwp.incoherent_rays(40000, p, bvh.tris, lambda o, d: run(gpu, acc, o, d), seed=37)
    o[:, 3] = -0.5; d[:, 3] = 5.0
    acc.set_precision(1)
    want_h = oracle.trace_prec(bvh.nodes, bvh.verts, o, d)
    want_o = oracle.trace_prec(bvh.nodes, bvh.verts, o, d, any_hit=True)
    assert (want_h[:, 0] < 0).sum() > 100   # the batch does hit behind its origins
    for trav in (1, 2):
        acc.set_traversal(trav)
        assert np.array_equal(run(gpu, acc, o, d).view(np.uint32), want_h.view(np.uint32))
        assert np.array_equal(run(gpu, acc, o, d, any_hit=True), want_o)


def test_precision_requires_cwbvh_and_corners(gpu, cwp):
    _, b2 = cwp.scene("boxes12k", variant=2, bins=16)
    acc = cwp.Accel(b2, tri=1)
    with pytest.raises(cwp.CwpError):
        acc.set_precision(1)
