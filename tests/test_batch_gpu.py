"""Batched form on the GPU: the segmented H-PLOC build of many meshes in one launch (every triangle placed exactly
once per layout, boxes that contain their children), the two-level persistent traversal against the oracle's
restatement on the very buffers the GPU built (bit for bit, every width, closest and any-hit, scene-tagged queue),
agreement across widths and tunings, per-frame TLAS rebuilds, and the autotuner."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def batch_case(gpu, cwp):
    meshes, xf, mesh_of, first = cwp.batch_scenes(n_scenes=6, seed=3, tris=(200, 20000), instances=(1, 60), blas_per_scene=(1, 3))
    first = np.concatenate([first[:3], [first[2]], first[3:]]).astype(np.int32)   # an empty scene (index 2) in the middle
    b = cwp.Batch(meshes)
    inst = cwp.instances(xf, mesh_of)
    b.set_scenes(inst, first)
    o, d, sc = cwp.batch_rays(xf, first, 3000, seed=4)
    sc[::97] = 99   # rays with an unknown scene id miss
    return meshes, xf, mesh_of, first, b, o, d, sc


def trace(gpu, b, o, d, sc, any_hit=False):
    n = len(o)
    hits = gpu.empty((n, 4), dtype=gpu.float32, device="cuda"); hi = gpu.empty(n, dtype=gpu.int32, device="cuda")
    to, td, ts = dev(gpu, o), dev(gpu, d), dev(gpu, sc)
    b.trace(to.data_ptr(), td.data_ptr(), ts.data_ptr(), hits.data_ptr(), hi.data_ptr(), n, any_hit=any_hit)
    gpu.cuda.synchronize(); b.status()
    return hits.cpu().numpy(), hi.cpu().numpy()


def test_build_places_every_triangle_once(gpu, cwp, batch_case):
    meshes, xf, mesh_of, first, b, *_ = batch_case
    info = b.info()
    assert info.blas_hploc_launches == 1 and info.n_blas == len(meshes) and info.blas_build_ms > 0
    ntri = [m.n_tris for m in meshes]; off = np.concatenate([[0], np.cumsum(ntri)])
    for w in (2, 4, 8):
        nodes, tris = b.download(w)
        assert info.node_bytes[{2: 0, 4: 1, 8: 2}[w]] == nodes.nbytes
        ids = tris[0::3, 3].view(np.int32)
        # every mesh's local ids appear exactly once (triangles of one mesh may sit anywhere in the array)
        assert np.array_equal(np.sort(ids), np.sort(np.concatenate([np.arange(n) for n in ntri])))
        # corners reproduce the input triangles: v0 and v0 + e1 / e2 against each mesh's faces
        assert np.all(np.isfinite(tris))


def test_binary_and_wide_boxes_contain_triangles(gpu, cwp, batch_case):
    """Every leaf triangle lies inside the box its parent stores for it (BVH2 / BVH4 exact boxes; CWBVH quantised
    planes rounded outward)."""
    meshes, xf, mesh_of, first, b, *_ = batch_case
    for w in (2, 4):
        nodes, tris = b.download(w)
        st = 4 if w == 2 else 8
        N = nodes.reshape(-1, st, 4)
        v0 = tris[0::3, :3]; v1 = v0 + tris[1::3, :3]; v2 = v0 + tris[2::3, :3]
        tlo = np.minimum(np.minimum(v0, v1), v2); thi = np.maximum(np.maximum(v0, v1), v2)
        for node in N:
            if w == 2:
                boxes = [((node[0, 0], node[0, 2], node[2, 0]), (node[0, 1], node[0, 3], node[2, 1])), ((node[1, 0], node[1, 2], node[2, 2]), (node[1, 1], node[1, 3], node[2, 3]))]
                c = node[3].view(np.int32); refs = [(c[0], c[2]), (c[1], c[3])]
            else:
                boxes = [((node[0, j], node[2, j], node[4, j]), (node[1, j], node[3, j], node[5, j])) for j in range(4)]
                refs = [(node[6].view(np.int32)[j], node[7].view(np.int32)[j]) for j in range(4)]
            for (lo, hi), (c, k) in zip(boxes, refs):
                if k > 0:
                    assert np.all(tlo[c:c + k] >= np.array(lo) - 1e-6) and np.all(thi[c:c + k] <= np.array(hi) + 1e-6)


@pytest.mark.parametrize("tlas_width", [2, 4])
@pytest.mark.parametrize("width", [2, 4, 8])
def test_two_level_trace_matches_oracle(gpu, cwp, oracle, batch_case, width, tlas_width):
    meshes, xf, mesh_of, first, b, o, d, sc = batch_case
    b.set_tuning(block=128, width=width, fetch=8, smem_stack=0)
    b.set_tlas_width(tlas_width)
    nodes, tris = b.download(width)
    tlas, roots, inst = b.download_tlas(len(first) - 1, len(mesh_of))
    assert roots[2] == -1 and len(tlas) == (8 if tlas_width == 4 else 4) * len(mesh_of)
    for any_hit in (False, True):
        h, hi = trace(gpu, b, o, d, sc, any_hit)
        ho, hio = oracle.trace_inst(width, any_hit, nodes, tris, tlas, roots, inst, o, d, sc, tlas_width=tlas_width)
        if any_hit:
            assert np.array_equal(hi, hio) and np.array_equal(h[:, 3].view(np.int32), ho[:, 3].view(np.int32))
        else:
            assert np.array_equal(h.view(np.uint32), ho.view(np.uint32)) and np.array_equal(hi, hio)
    assert np.all(hi[sc == 99] == -1) and np.all(hi[sc == 2] == -1)
    assert (hi >= 0).mean() > 0.05   # the batch does hit geometry
    b.set_tlas_width(4)


@pytest.mark.parametrize("width", [2, 4, 8])
def test_two_level_trace_matches_reference_travinst(gpu, cwp, ref, batch_case, width):
    """The reference's own two-level traversal (travInst, compiled from its sources for the host) over the buffers the
    GPU built: the same closest hit (instance, triangle) on every ray up to exact-distance ties (the reference
    enters a TLAS leaf's instances as soon as its node is visited, this traversal when the leaf comes up in
    nearer-first order; box bottoms are coplanar with the ground, so rays from below meet many exact ties), and the
    same occlusion."""
    meshes, xf, mesh_of, first, b, o, d, sc = batch_case
    b.set_tuning(block=128, width=width, fetch=8, smem_stack=0)
    nodes, tris = b.download(width)
    h, hi = trace(gpu, b, o, d, sc)                           # the default width-4 TLAS
    b.set_tlas_width(2)                                       # the reference's travInst reads a BVH2 TLAS
    tlas, roots, inst = b.download_tlas(len(first) - 1, len(mesh_of))
    b.set_tlas_width(4)
    hr, hir = ref.trace_inst(width, False, nodes, tris, tlas, roots, inst, o, d, sc)
    tri, trr = h[:, 3].view(np.int32), hr[:, 3].view(np.int32)
    same = (tri == trr) & (hi == hir)
    tie = ~same & (tri >= 0) & (trr >= 0) & (np.abs(h[:, 0].astype(np.float64) - hr[:, 0]) <= 1e-6 * np.abs(hr[:, 0].astype(np.float64)))
    assert np.all(same | tie) and tie.mean() < 0.02
    _, oi = trace(gpu, b, o, d, sc, any_hit=True)
    _, oir = ref.trace_inst(width, True, nodes, tris, tlas, roots, inst, o, d, sc)
    assert np.array_equal(oi >= 0, oir >= 0)


def test_widths_and_tunings_agree(gpu, cwp, batch_case):
    """All widths, block sizes, fetch sizes and stack placements report the same closest hit (instance, mesh-local
    triangle id, t) up to exact-distance ties."""
    meshes, xf, mesh_of, first, b, o, d, sc = batch_case
    base = None
    for t in ((128, 8, 12, 0), (64, 2, 1, 1), (256, 4, 32, 0), (512, 8, 4, 1), (128, 4, 8, 1), (256, 2, 16, 0)):
        b.set_tuning(*t)
        h, hi = trace(gpu, b, o, d, sc)
        _, tris = b.download(t[1])
        tri = h[:, 3].view(np.int32)
        key = np.where(tri >= 0, tris[3 * np.maximum(tri, 0), 3].view(np.int32), -1)
        cur = (h[:, 0].astype(np.float64), hi, key)
        if base is None:
            base = cur; continue
        same = (cur[1] == base[1]) & (cur[2] == base[2])
        tie = ~same & (cur[1] >= 0) & (base[1] >= 0) & (np.abs(cur[0] - base[0]) <= 1e-6 * np.abs(base[0]))
        assert np.all(same | tie), t
        assert np.array_equal(cur[1] >= 0, base[1] >= 0)


def test_tlas_rebuild_per_frame(gpu, cwp, oracle, batch_case):
    meshes, xf, mesh_of, first, b, o, d, sc = batch_case
    moved = xf.copy().reshape(-1, 3, 4); moved[:, :, 3] += np.float32(1.5)
    b.set_scenes(cwp.instances(moved.reshape(-1, 12), mesh_of), first)
    b.set_tuning(128, 8, 12, 0)
    h, hi = trace(gpu, b, o, d, sc)
    nodes, tris = b.download(8)
    tlas, roots, inst = b.download_tlas(len(first) - 1, len(mesh_of))
    ho, hio = oracle.trace_inst(8, False, nodes, tris, tlas, roots, inst, o, d, sc, tlas_width=b.tlas_width)
    assert np.array_equal(h.view(np.uint32), ho.view(np.uint32)) and np.array_equal(hi, hio)
    assert b.info().tlas_build_ms > 0
    b.set_scenes(cwp.instances(xf, mesh_of), first)


def test_autotune_picks_a_valid_tuning(gpu, cwp, batch_case):
    meshes, xf, mesh_of, first, b, o, d, sc = batch_case
    n = len(o)
    hits = gpu.empty((n, 4), dtype=gpu.float32, device="cuda"); hi = gpu.empty(n, dtype=gpu.int32, device="cuda")
    to, td, ts = dev(gpu, o), dev(gpu, d), dev(gpu, sc)
    t = b.autotune(to.data_ptr(), td.data_ptr(), ts.data_ptr(), hits.data_ptr(), hi.data_ptr(), n)
    assert t.block in (64, 128, 256, 512) and t.width in (2, 4, 8) and 1 <= t.fetch <= 32 and t.smem_stack in (0, 1) and t.ms > 0
    cur = b.tuning()
    assert (cur.block, cur.width, cur.fetch, cur.smem_stack) == (t.block, t.width, t.fetch, t.smem_stack)


def test_bad_arguments(gpu, cwp, batch_case):
    meshes, xf, mesh_of, first, b, *_ = batch_case
    with pytest.raises(cwp.CwpError):
        b.set_tuning(block=100)
    with pytest.raises(cwp.CwpError):
        b.set_tuning(width=3)
    with pytest.raises(cwp.CwpError):
        b.set_scenes(cwp.instances(xf[:1], [len(meshes)]), [0, 1])


@pytest.mark.parametrize("spatial", [0.0, 1e-5])
def test_host_built_blas_match_oracle(gpu, cwp, oracle, spatial):
    """Resident scenes built on the host (binned SAH or SBVH, SAH-collapsed CWBVH), concatenated with per-layout mesh
    roots: the persistent two-level launch returns the oracle's hits bit for bit at every width, and the same
    closest hits (instance, mesh-local triangle, t) as the GPU-built BLAS up to ties."""
    meshes, xf, mesh_of, first = cwp.batch_scenes(n_scenes=4, seed=8, tris=(200, 6000), instances=(1, 40), blas_per_scene=(1, 3))
    o, d, sc = cwp.batch_rays(xf, first, 2000, seed=6)
    inst = cwp.instances(xf, mesh_of)
    hb = cwp.Batch(meshes, builder=1, spatial=spatial); hb.set_scenes(inst, first)
    gb = cwp.Batch(meshes); gb.set_scenes(inst, first)
    for width in (2, 4, 8):
        hb.set_tuning(128, width, 8, 0)
        h, hi = trace(gpu, hb, o, d, sc)
        nodes, tris = hb.download(width)
        tlas, roots, ins = hb.download_tlas(len(first) - 1, len(mesh_of))
        ho, hio = oracle.trace_inst(width, False, nodes, tris, tlas, roots, ins, o, d, sc, tlas_width=hb.tlas_width)
        assert np.array_equal(h.view(np.uint32), ho.view(np.uint32)) and np.array_equal(hi, hio)
        gb.set_tuning(128, width, 8, 0)
        g, gi = trace(gpu, gb, o, d, sc)
        _, gtris = gb.download(width)
        ka = np.where(h[:, 3].view(np.int32) >= 0, tris[3 * np.maximum(h[:, 3].view(np.int32), 0), 3].view(np.int32), -1)
        kb = np.where(g[:, 3].view(np.int32) >= 0, gtris[3 * np.maximum(g[:, 3].view(np.int32), 0), 3].view(np.int32), -1)
        same = (ka == kb) & (hi == gi)
        tie = ~same & (hi >= 0) & (gi >= 0) & (np.abs(h[:, 0].astype(np.float64) - g[:, 0]) <= 1e-6 * np.abs(g[:, 0].astype(np.float64)))
        assert np.all(same | tie) and tie.mean() < 0.02


def test_degenerate_segments(gpu, cwp, oracle):
    """One-triangle and two-triangle meshes (a segment whose root is a leaf), scenes with 0, 1 and 2 instances (an
    empty TLAS, the one-instance wrapper node), a zero-length trace: every width returns the oracle's hits."""
    tri1 = (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]], np.int32), np.zeros(1, np.int32), None)
    quad = (np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2], [0, 2, 3]], np.int32), np.zeros(2, np.int32), None)
    box = cwp.Mesh.box_field(3, 4)
    b = cwp.Batch([tri1, quad, box])
    I = np.eye(3, 4, dtype=np.float32).reshape(12)
    shift = I.copy(); shift[3] = 2.0
    xf = np.stack([I, I, shift, I]).astype(np.float32); mesh_of = np.array([0, 1, 0, 2], np.int32)
    first = np.array([0, 0, 1, 3, 4], np.int32)   # scene 0 empty, 1: one instance, 2: two, 3: one box field
    b.set_scenes(cwp.instances(xf, mesh_of), first)
    rng = np.random.default_rng(1)
    n = 4000
    o = np.zeros((n, 4), np.float32); o[:, :3] = rng.uniform(-3, 4, (n, 3)); o[:, 2] = 5.0
    d = np.zeros((n, 4), np.float32); v = rng.normal(size=(n, 3)); v[:, 2] = -np.abs(v[:, 2]) - 1.0; d[:, :3] = v / np.linalg.norm(v, axis=1, keepdims=True); d[:, 3] = 1e30
    sc = rng.integers(0, 4, n).astype(np.int32)
    for width, tw in ((2, 4), (4, 2), (8, 4), (8, 2)):
        b.set_tuning(64, width, 1, 1)
        b.set_tlas_width(tw)
        h, hi = trace(gpu, b, o, d, sc)
        nodes, tris = b.download(width)
        tlas, roots, ins = b.download_tlas(4, 4)
        ho, hio = oracle.trace_inst(width, False, nodes, tris, tlas, roots, ins, o, d, sc, tlas_width=tw)
        assert np.array_equal(h.view(np.uint32), ho.view(np.uint32)) and np.array_equal(hi, hio)
        assert np.all(hi[sc == 0] == -1) and (hi[sc == 1] >= 0).any() and (hi[sc == 2] >= 0).any()
    b.trace(0, 0, 0, 0, 0, 0)   # n = 0: nothing to do, no error


def test_incremental_scene_updates_match_packed(gpu, cwp):
    """Fixed per-scene regions updated a few scenes at a time trace exactly like the packed form built over the same
    instances (hits bit for bit, instance indices moved into the scene's region); scenes left out of an update keep
    their TLAS; an emptied scene's rays miss."""
    meshes, xf, mesh_of, first = cwp.batch_scenes(n_scenes=3, seed=7, tris=(200, 5000), instances=(1, 40), blas_per_scene=(1, 3))
    first = np.asarray(first, np.int32)
    inst = cwp.instances(xf, mesh_of)
    b = cwp.Batch(meshes)
    b.set_scenes(inst, first)
    o, d, sc = cwp.batch_rays(xf, first, 2000, seed=8)
    sc[::50] = 3   # a scene that is empty (incremental) or absent (packed): misses either way
    packed, pinst = trace(gpu, b, o, d, sc)
    assert (pinst >= 0).any()

    def part(scenes):
        lst = [inst[i] for s in scenes for i in range(first[s], first[s + 1])]
        return (cwp.Instance * len(lst))(*lst), [int(first[s + 1] - first[s]) for s in scenes]

    def region(pi, cap):
        s = np.searchsorted(first, np.maximum(pi, 0), side="right") - 1
        return np.where(pi >= 0, s * cap + (pi - first[s]), -1)

    cap = int(np.diff(first).max()) + 3
    b.reserve_scenes(4, cap)
    h0, _ = trace(gpu, b, o, d, sc)
    assert np.all(h0[:, 3].view(np.int32) == -1)   # every scene empty
    arr, cnt = part([2, 0]); b.update_scenes([2, 0], arr, cnt)
    arr, cnt = part([1]); b.update_scenes([1], arr, cnt)   # scenes 0 and 2 untouched
    h1, i1 = trace(gpu, b, o, d, sc)
    assert np.array_equal(h1.view(np.uint32), packed.view(np.uint32)) and np.array_equal(i1, region(pinst, cap))
    assert b.info().n_instances == 4 * cap
    b.update_scenes([0], None, [0])   # scene 0 emptied
    h2, i2 = trace(gpu, b, o, d, sc)
    assert np.all(h2[sc == 0, 3].view(np.int32) == -1)
    keep = sc != 0
    assert np.array_equal(h2[keep].view(np.uint32), packed[keep].view(np.uint32))
    with pytest.raises(Exception):
        b.update_scenes([1, 1], None, [0, 0])   # listed twice
    with pytest.raises(Exception):
        arr, cnt = part([1]); b.update_scenes([4], arr, cnt)   # out of range
