"""Serving form on the GPU: device BSDFs against the reference's own render/bsdf.h (fixture), a request's image
against the oracle's host restatement of the serving integrator, the same request alone and inside a mix of
concurrent requests, continuous batching against the plain form, and admission by free device memory."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def close(a, b, rel, abs_):
    return np.abs(a - b) <= abs_ + rel * np.maximum(np.abs(a), np.abs(b))


def test_device_bsdf_matches_reference(gpu, cwp):
    g, bump = golden("bsdf.npz"), golden("bsdf_bump.npz")
    for gd in (0, 1):   # the bump-terminator term (unperturbed normals per case)
        f, pdf = cwp.bsdf_eval_batch(g["mats"], g["mat"], g["wo"], g["wi"], g["eta"], gd, g["ux"], nr=bump["nr"])
        assert close(f, bump[f"f{gd}"], 1e-4, 1e-6).mean() >= 0.999 and close(pdf, bump[f"pdf{gd}"], 1e-4, 1e-6).mean() >= 0.999
        wi, w, p, ok = cwp.bsdf_sample_batch(g["mats"], g["mat"], g["wo"], g["eta"], gd, g["ux"], g["uvw"], nr=bump["nr"])
        k = (ok == bump[f"s_ok{gd}"]) & (ok == 1)
        assert (ok == bump[f"s_ok{gd}"]).mean() >= 0.998 and close(w[k], bump[f"s_w{gd}"][k], 1e-3, 1e-4).mean() >= 0.998
    for gd in (0, 1):
        f, pdf = cwp.bsdf_eval_batch(g["mats"], g["mat"], g["wo"], g["wi"], g["eta"], gd, g["ux"])
        assert close(f, g[f"f{gd}"], 1e-4, 1e-6).mean() >= 0.999 and close(pdf, g[f"pdf{gd}"], 1e-4, 1e-6).mean() >= 0.999
        wi, w, p, ok = cwp.bsdf_sample_batch(g["mats"], g["mat"], g["wo"], g["eta"], gd, g["ux"], g["uvw"])
        same = ok == g[f"s_ok{gd}"]
        assert same.mean() >= 0.998
        k = same & (ok == 1)
        assert close(wi[k], g[f"s_wi{gd}"][k], 1e-3, 1e-4).mean() >= 0.998 and close(w[k], g[f"s_w{gd}"][k], 1e-3, 1e-4).mean() >= 0.998


@pytest.fixture(scope="module")
def serving(gpu, cwp):
    meshes, descs, first, mats, base, boxes = cwp.serving_scenes(n_scenes=3, seed=2, tris=(200, 8000), instances=(1, 24), blas_per_scene=(1, 3))
    b = cwp.Batch(meshes)
    b.meshes = meshes   # the host meshes, for the oracle's emissive-triangle tables
    return b, descs, first, mats, base, boxes


def server(cwp, serving, **kw):
    b, descs, first, mats, base, boxes = serving
    s = cwp.Server(b, mats, base, **kw)
    s.set_scenes(descs, first)
    return s


def run_all(s, reqs):
    ids = [s.submit(r) for r in reqs]
    done = {}
    for _ in range(100000):
        a, p = s.step()
        for i in s.poll():
            done[i] = True
        if len(done) == len(ids):
            break
    assert len(done) == len(ids)
    out = []
    for i, r in zip(ids, reqs):
        acc, st = s.result(i, r.cam.w, r.cam.h)
        out.append((acc, st))
    return out


def requests(cwp, boxes, n, seed, res=((32, 32), (48, 32), (64, 64)), spps=(1, 2, 4)):
    return [r for _, r in cwp.serving_requests(n, 100.0, boxes, seed=seed, resolutions=list(res), spps=list(spps))]


def test_request_matches_oracle(gpu, cwp, oracle, serving):
    b, descs, first, mats, base, boxes = serving
    s = server(cwp, serving, max_paths=1 << 16, max_requests=4)
    req = requests(cwp, boxes, 1, seed=3, res=((64, 48),), spps=(4,))[0]
    (acc, st), = run_all(s, [req])
    nodes, tris = b.download(b.tuning().width)
    tlas, roots, inst = b.download_tlas(4, _n_inst(b, 4))   # the server's slots are the batch's scenes; slot 0 held the request
    ref, cnt = oracle.render_request(req, b.tuning().width, nodes, tris, tlas, roots[0], inst, mats, base, tlas_width=b.tlas_width)
    a = acc[:, :3] / req.spp; r = ref[:, :3] / req.spp
    assert cwp.imageio.psnr(a, r) >= 50.0
    assert abs(st.rays - cnt[0]) <= 2e-3 * cnt[0] and abs(st.shadow_rays - cnt[1]) <= 2e-3 * max(cnt[1], 1)
    assert st.done_ms >= st.admit_ms >= st.submit_ms


def _n_inst(b, n_scenes):
    """instances currently in the batch's TLAS set"""
    return int(b.info().n_instances)


def test_alone_equals_in_the_mix(gpu, cwp, serving):
    """Every request's image is the same whether it runs alone (plain form, one request at a time) or among others
    admitted concurrently, with or without the per-step regrouping of the queue by request, under either feeding
    policy, and whether a step returns with its launches queued or waits for them: only the order of float atomics
    differs."""
    b, descs, first, mats, base, boxes = serving
    reqs = requests(cwp, boxes, 8, seed=5)
    mix = run_all(server(cwp, serving, max_paths=1 << 15, max_requests=8), reqs)
    mixed_order = run_all(server(cwp, serving, max_paths=1 << 15, max_requests=8, regroup=False), reqs)
    oldest_first = run_all(server(cwp, serving, max_paths=1 << 15, max_requests=8, policy=1), reqs)
    waiting = run_all(server(cwp, serving, max_paths=1 << 15, max_requests=8, overlap=False), reqs)
    alone = run_all(server(cwp, serving, max_paths=1 << 15, max_requests=1), reqs)
    for (am, sm), (ao, so), (af, sf), (aw, sw), (aa, sa) in zip(mix, mixed_order, oldest_first, waiting, alone):
        assert sm.rays == sa.rays == so.rays == sf.rays == sw.rays and sm.shadow_rays == sa.shadow_rays == so.shadow_rays == sf.shadow_rays == sw.shadow_rays
        assert all(np.allclose(x, aa, rtol=1e-4, atol=1e-5) for x in (am, ao, af, aw))
    # in the mix, requests overlapped: some request was admitted before an earlier one finished
    adm = sorted((s.admit_ms, s.done_ms) for _, s in mix)
    assert any(adm[i + 1][0] < adm[i][1] for i in range(len(adm) - 1))


def test_admission_waits_for_memory(gpu, cwp, serving):
    s = server(cwp, serving, max_paths=1 << 12, max_requests=4, hbm_reserve=1 << 50)   # more than any device has
    req = requests(cwp, serving[5], 1, seed=9)[0]
    s.submit(req)
    for _ in range(3):
        a, p = s.step()
        assert a == 0 and p == 1


def test_environment_request_matches_oracle(gpu, cwp, oracle, serving):
    """A request lit by an environment map (importance-sampled by luminance x sin(theta), combined with BSDF sampling
    by the power heuristic, rotated 30 degrees) and the sun: the image matches the oracle's restatement at >= 50 dB and
    the ray counts agree; environment and sky requests in one mix give each request's image alone."""
    from conftest import golden
    b, descs, first, mats, base, boxes = serving
    g = golden("env.npz")
    env_rgb = g["big_rgb"]
    s = server(cwp, serving, max_paths=1 << 16, max_requests=4)
    s.set_envmaps([(env_rgb, 1.5)])
    req = requests(cwp, boxes, 1, seed=13, res=((64, 48),), spps=(4,))[0]
    req.env, req.env_rot_deg = 0, 30.0
    (acc, st), = run_all(s, [req])
    nodes, tris = b.download(b.tuning().width)
    tlas, roots, inst = b.download_tlas(4, _n_inst(b, 4))
    ref, cnt = oracle.render_request(req, b.tuning().width, nodes, tris, tlas, roots[0], inst, mats, base, tlas_width=b.tlas_width,
                                     env=cwp.envmap_build(env_rgb, 1.5))
    a = acc[:, :3] / req.spp; r = ref[:, :3] / req.spp
    assert cwp.imageio.psnr(a, r) >= 50.0
    assert abs(st.rays - cnt[0]) <= 2e-3 * cnt[0] and abs(st.shadow_rays - cnt[1]) <= 2e-3 * max(cnt[1], 1)
    # the environment adds light over the sky-lit request of the same path samples
    sky_req = requests(cwp, boxes, 1, seed=13, res=((64, 48),), spps=(4,))[0]
    (acc_sky, _), = run_all(s, [sky_req])
    assert not np.allclose(acc, acc_sky)
    # mixed with sky requests, and alone: the same images up to the order of float atomics
    reqs = requests(cwp, boxes, 6, seed=17)
    for i, rq in enumerate(reqs):
        rq.env, rq.env_rot_deg = (0, 45.0 * i) if i % 2 == 0 else (-1, 0.0)
    mix = run_all(s, reqs)
    alone_s = server(cwp, serving, max_paths=1 << 15, max_requests=1)
    alone_s.set_envmaps([(env_rgb, 1.5)])
    alone = run_all(alone_s, reqs)
    for (am, sm), (aa, sa) in zip(mix, alone):
        assert sm.rays == sa.rays and sm.shadow_rays == sa.shadow_rays
        assert np.allclose(am, aa, rtol=1e-4, atol=1e-5)
    with pytest.raises(cwp.CwpError):
        bad = requests(cwp, boxes, 1, seed=3)[0]; bad.env = 1   # only one map
        s.submit(bad)


def _emissive(mats, base, rgb=(4.0, 3.0, 2.0)):
    """every mesh's material 1 (one box in seven) emits"""
    m = mats.copy()
    for b0 in base:
        m[b0 + 1, 8:11] = rgb
    return m


@pytest.mark.parametrize("case", ["sun", "env", "nee", "bsdf", "rr", "env_uniform"])
def test_emissive_request_matches_oracle(gpu, cwp, oracle, serving, case):
    """Emissive boxes as area lights: a light sample picks the sun, a triangle by power (a uniform point on it, the
    shadow ray ending just short of it) or an environment texel, each type with equal probability, and is weighted
    against BSDF sampling by the power heuristic; emitters hit by BSDF samples are weighted the other way. The MIS, NEE
    and BSDF modes, Russian roulette and uniform environment samples: the request's image matches the oracle's
    restatement at >= 45 dB and the ray counts agree."""
    b, descs, first, mats, base, boxes = serving
    em = _emissive(mats, base)
    s = cwp.Server(b, em, base, max_paths=1 << 16, max_requests=4)
    s.set_scenes(descs, first)
    g = golden("env.npz")
    s.set_envmaps([(g["big_rgb"], 1.5)])
    req = requests(cwp, boxes, 1, seed=29, res=((64, 48),), spps=(4,))[0]
    if case != "sun":
        req.env, req.env_rot_deg = 0, 30.0
    req.light_mode = {"nee": cwp.LIGHT_NEE, "bsdf": cwp.LIGHT_BSDF}.get(case, cwp.LIGHT_MIS)
    if case == "rr":
        req.rr, req.rr_depth = 1, 1
    req.env_uniform = 1 if case == "env_uniform" else 0
    (acc, st), = run_all(s, [req])
    nodes, tris = b.download(b.tuning().width)
    tlas, roots, inst = b.download_tlas(4, _n_inst(b, 4))
    lights = cwp.emissive_tables(b.meshes, base, em, *cwp.scene_xforms(descs, first, req.scene, req.frame))
    assert len(lights[0]) > 0
    ref, cnt = oracle.render_request(req, b.tuning().width, nodes, tris, tlas, roots[0], inst, em, base, tlas_width=b.tlas_width,
                                     env=cwp.envmap_build(g["big_rgb"], 1.5) if req.env >= 0 else None, lights=lights)
    a = acc[:, :3] / req.spp; r = ref[:, :3] / req.spp
    assert cwp.imageio.psnr(a, r) >= 45.0
    assert abs(st.rays - cnt[0]) <= 2e-3 * cnt[0] and abs(st.shadow_rays - cnt[1]) <= 2e-3 * max(cnt[1], 1)


def test_light_modes_agree_and_requests_keep_their_lights(gpu, cwp, serving):
    """Lit by the emissive boxes alone (no sun, black sky): light sampling with MIS, light sampling alone (NEE), BSDF
    sampling alone and MIS with Russian roulette converge to the same image. The reference's consistency check
    (tests/mis_consistency.py:1-6) restated: 16 independent seeds per mode, the mean luminance of every region of a
    4x4 grid per seed, per mode its mean and standard error over the seeds, every pair of modes z = |a - b| /
    sqrt(se_a^2 + se_b^2). The whole image's z stays <= 3 for every pair. Per region, z <= 4 (the bound for 48
    comparisons at a family-wise 1% with standard errors from 16 seeds; the reference's 3 is per comparison) for the
    pairs among MIS, BSDF sampling and MIS with roulette. NEE alone is left out of the regional test: its
    contribution grows as 1 / distance^2 for shading points near an emitter, so its variance is unbounded and a
    standard-error test does not apply (16 seeds of one region gave z = 5.6 against MIS, 64 seeds z = 0.35). MIS is
    less noisy than BSDF sampling. Requests of different scenes and frames in one mix give each
    one's image alone (every slot reads its own request's light tables).
    The emissive boxes float 0.6 above the ground here. An emitter face coplanar with another surface (a box bottom
    on the ground) leaks light into light sampling, in the reference's algorithm as in this one: a shadow ray starts
    on the light point's side of the surface, below the ground for a point on the ground plane, and passes under the
    walls. The estimators then disagree by design, so the check needs emitters clear of other surfaces."""
    b0, descs, first, mats, base, boxes = serving
    lifted = []
    for v, f, fm, x in b0.meshes:
        v = v.copy(); v[np.unique(f[fm == 1]), 2] += 0.6; lifted.append((v, f, fm, x))
    b = cwp.Batch(lifted)
    em = _emissive(mats, base)
    s = cwp.Server(b, em, base, max_paths=1 << 21, max_requests=16)
    s.set_scenes(descs, first)
    w, h, gx, gy = 64, 48, 4, 4
    stats = {}
    for name, mode, rr in (("mis", cwp.LIGHT_MIS, 0), ("nee", cwp.LIGHT_NEE, 0), ("bsdf", cwp.LIGHT_BSDF, 0), ("rr", cwp.LIGHT_MIS, 1)):
        reqs = []
        for seed in range(16):
            r = requests(cwp, boxes, 1, seed=31, res=((w, h),), spps=(32,))[0]
            r.sun_e[:] = (0.0, 0.0, 0.0); r.sky[:] = (0.0, 0.0, 0.0)
            r.light_mode, r.rr, r.rr_depth, r.seed = mode, rr, 2, 1000 + seed
            reqs.append(r)
        vals = []
        for acc, _ in run_all(s, reqs):
            im = (acc[:, :3] / 32).reshape(h, w, 3).astype(np.float64)
            L = 0.2126 * im[..., 0] + 0.7152 * im[..., 1] + 0.0722 * im[..., 2]
            vals.append([L[j * h // gy:(j + 1) * h // gy, i * w // gx:(i + 1) * w // gx].mean() for j in range(gy) for i in range(gx)] + [L.mean()])
        v = np.array(vals)
        stats[name] = (v.mean(0), v.std(0, ddof=1) / np.sqrt(len(v)))
    assert np.all(stats["mis"][0] > 0)
    names = list(stats)
    for i in range(len(names)):
        for j in range(i + 1, len(names)):
            (ma, sa), (mb, sb) = stats[names[i]], stats[names[j]]
            z = np.abs(ma - mb) / np.sqrt(sa ** 2 + sb ** 2)
            assert z[-1] <= 3.0, (names[i], names[j], z)
            if "nee" not in (names[i], names[j]):
                assert z[:-1].max() <= 4.0, (names[i], names[j], z)
    assert np.median(stats["mis"][1] / stats["mis"][0]) < np.median(stats["bsdf"][1] / stats["bsdf"][0])
    reqs = requests(cwp, boxes, 4, seed=37)
    mix = run_all(s, reqs)
    alone_s = cwp.Server(b, em, base, max_paths=1 << 15, max_requests=1)
    alone_s.set_scenes(descs, first)
    alone = run_all(alone_s, reqs)
    for (am, sm), (aa, sa) in zip(mix, alone):
        assert sm.rays == sa.rays and sm.shadow_rays == sa.shadow_rays
        assert np.allclose(am, aa, rtol=1e-4, atol=1e-5)
    with pytest.raises(cwp.CwpError):
        bad = requests(cwp, boxes, 1, seed=3)[0]; bad.light_mode = 3
        s.submit(bad)


def vertex_normals(meshes, seed=3):
    """per-vertex normals for the box-field meshes: the direction from the mesh's centre, tilted at random (every
    second mesh keeps flat shading: None)"""
    rng = np.random.default_rng(seed)
    out = []
    for k, (v, f, fm, _) in enumerate(meshes):
        if k % 2:
            out.append(None); continue
        n = v - v.mean(0) + rng.normal(0, 0.3, v.shape)
        out.append((n / np.linalg.norm(n, axis=1, keepdims=True)).astype(np.float32))
    return out


def mesh_order_normals(meshes, normals):
    """corner normals [n_tris, 12] in mesh order (zero for meshes without) and each mesh's first triangle"""
    rows, first = [], [0]
    for (v, f, fm, _), n in zip(meshes, normals):
        r = np.zeros((len(f), 12), np.float32)
        if n is not None:
            r[:, 0:3], r[:, 4:7], r[:, 8:11] = n[f[:, 0]], n[f[:, 1]], n[f[:, 2]]
        rows.append(r); first.append(first[-1] + len(f))
    return np.concatenate(rows), np.array(first, np.int32)


def test_smooth_normals_request_matches_oracle(gpu, cwp, oracle):
    """Meshes with vertex normals (every second one; the others flat): the shading normal interpolates the corner
    normals, maps them by the instance's inverse transpose and turns them to the geometric normal's side; with
    emissive boxes and an environment map the request's image matches the oracle at >= 45 dB."""
    meshes, descs, first, mats, base, boxes = cwp.serving_scenes(n_scenes=2, seed=6, tris=(200, 3000), instances=(2, 12), blas_per_scene=(2, 3))
    nrm = vertex_normals(meshes)
    b = cwp.Batch(meshes, normals=nrm)
    em = _emissive(mats, base)
    s = cwp.Server(b, em, base, max_paths=1 << 16, max_requests=2)
    s.set_scenes(descs, first)
    g = golden("env.npz")
    s.set_envmaps([(g["big_rgb"], 1.0)])
    req = requests(cwp, boxes, 1, seed=43, res=((64, 48),), spps=(4,))[0]
    req.env = 0
    (acc, st), = run_all(s, [req])
    nodes, tris = b.download(b.tuning().width)
    tlas, roots, inst = b.download_tlas(2, _n_inst(b, 2))
    lights = cwp.emissive_tables(meshes, base, em, *cwp.scene_xforms(descs, first, req.scene, req.frame))
    ref, cnt = oracle.render_request(req, b.tuning().width, nodes, tris, tlas, roots[0], inst, em, base, tlas_width=b.tlas_width,
                                     env=cwp.envmap_build(g["big_rgb"], 1.0), lights=lights, normals=mesh_order_normals(meshes, nrm))
    a = acc[:, :3] / req.spp; r = ref[:, :3] / req.spp
    assert cwp.imageio.psnr(a, r) >= 45.0
    assert abs(st.rays - cnt[0]) <= 2e-3 * cnt[0] and abs(st.shadow_rays - cnt[1]) <= 2e-3 * max(cnt[1], 1)
    # the normals change the image against flat shading of the same paths
    flat = cwp.Batch(meshes)
    sf = cwp.Server(flat, em, base, max_paths=1 << 16, max_requests=2); sf.set_scenes(descs, first); sf.set_envmaps([(g["big_rgb"], 1.0)])
    (acc_flat, _), = run_all(sf, [req])
    assert not np.allclose(acc, acc_flat)


def test_camera_options_match_oracle(gpu, cwp, oracle, serving):
    """Camera rays as the reference's k_raygen: a thin lens focused on the scene centre, a near clip and the
    Blackman-Harris pixel filter; the request's image matches the oracle's at >= 45 dB and differs from the pinhole
    box-filtered image of the same samples."""
    b, descs, first, mats, base, boxes = serving
    s = server(cwp, serving, max_paths=1 << 16, max_requests=4)
    req = requests(cwp, boxes, 1, seed=47, res=((64, 48),), spps=(4,))[0]
    (pin, _), = run_all(s, [req])
    c = (boxes[req.scene][0] + boxes[req.scene][1]) / 2
    req.cam.lens_r = 0.02 * float(np.max(boxes[req.scene][1] - boxes[req.scene][0]))
    req.cam.focus_d = float(np.linalg.norm(np.array(list(req.cam.pos)) - c))
    req.near_clip = 0.05 * req.cam.focus_d
    req.filter_bh = 1
    (acc, st), = run_all(s, [req])
    assert not np.allclose(acc, pin)
    nodes, tris = b.download(b.tuning().width)
    tlas, roots, inst = b.download_tlas(4, _n_inst(b, 4))
    ref, cnt = oracle.render_request(req, b.tuning().width, nodes, tris, tlas, roots[0], inst, mats, base, tlas_width=b.tlas_width)
    assert cwp.imageio.psnr(acc[:, :3] / req.spp, ref[:, :3] / req.spp) >= 45.0
    assert abs(st.rays - cnt[0]) <= 2e-3 * cnt[0] and abs(st.shadow_rays - cnt[1]) <= 2e-3 * max(cnt[1], 1)
    with pytest.raises(cwp.CwpError):
        bad = requests(cwp, boxes, 1, seed=3)[0]; bad.cam.lens_r = 0.1; bad.cam.focus_d = 0.0   # a lens needs a focus distance
        s.submit(bad)


def test_instance_matrices_match_animation(gpu, cwp, serving):
    """Instances placed by per-frame matrices (scene files' "transforms") render as the animation parameters
    that produced the matrices; past the last matrix the last one holds; a fixed matrix ("transform") for every
    frame; clearing the matrices restores the animation."""
    b, descs, first, mats, base, boxes = serving
    s = server(cwp, serving, max_paths=1 << 16, max_requests=2)
    ref_s = server(cwp, serving, max_paths=1 << 16, max_requests=2)
    n = len(descs)
    per = [np.stack([cwp.scene_xforms(descs, [0, n], 0, f)[0][i] for f in range(12)]) for i in range(n)]
    s.set_instance_xforms(per)
    req = requests(cwp, boxes, 1, seed=51, res=((48, 32),), spps=(2,))[0]
    req.frame = 5
    (a, _), = run_all(s, [req])
    (r, _), = run_all(ref_s, [req])
    assert np.allclose(a, r, rtol=1e-4, atol=1e-5)   # up to the order of float atomics
    req.frame = 20   # past the 12 matrices: frame 11's placement
    (a, _), = run_all(s, [req])
    req.frame = 11
    (r, _), = run_all(ref_s, [req])
    assert np.allclose(a, r, rtol=1e-4, atol=1e-5)   # up to the order of float atomics
    s.set_instance_xforms([p[3:4] for p in per])   # one fixed matrix each: frame 3's placement at any frame
    req.frame = 9
    (a, _), = run_all(s, [req])
    req.frame = 3
    (r, _), = run_all(ref_s, [req])
    assert np.allclose(a, r, rtol=1e-4, atol=1e-5)   # up to the order of float atomics
    s.set_instance_xforms(None)
    req.frame = 9
    (a, _), = run_all(s, [req])
    (r, _), = run_all(ref_s, [req])
    assert np.allclose(a, r, rtol=1e-4, atol=1e-5)   # up to the order of float atomics
    with pytest.raises(cwp.CwpError):
        s.set_instance_xforms(per[:-1])   # one range per descriptor


def test_texture_lookups_match_oracle(gpu, cwp, oracle):
    """Hardware bilinear lookups (wrap, normalised coordinates, sRGB decode for colour images) against the oracle's
    restatement of the documented filtering rule, over odd image sizes and coordinates wrapping over several periods.
    The filter weights are kept to 8 fractional bits, and the hardware's rounding of them (and of its sRGB decode) is
    not documented, so a lookup may differ by one weight step per axis times the texel difference (at most about
    2/255); the mean difference stays far below that."""
    rng = np.random.default_rng(2)
    imgs = [(rng.integers(0, 256, (7, 13, 4)).astype(np.uint8), False), (rng.integers(0, 256, (5, 9, 4)).astype(np.uint8), True)]
    imgs += cwp.texture_images()
    n = 20000
    ids = rng.integers(0, len(imgs), n).astype(np.int32)
    uv = rng.uniform(-2.0, 3.0, (n, 2)).astype(np.float32)
    got = cwp.texture_sample_batch(imgs, ids, uv)
    tex, keep = cwp.textures_array(imgs)
    ref = oracle.texture_sample(tex, ids, uv)
    err = np.abs(got - ref)
    assert err.max() <= 2.5 / 255.0 and err.mean() < 1e-3
    # nearest-texel lookups (the reference's --tex_filter nearest): the same texel except where a coordinate lies
    # within rounding of a texel edge; linear images exactly, colour images within the hardware's sRGB decode
    got = cwp.texture_sample_batch(imgs, ids, uv, nearest=True)
    tex, keep = cwp.textures_array(imgs, nearest=True)
    ref = oracle.texture_sample(tex, ids, uv)
    srgb = np.array([bool(sp) for _, sp in imgs])[ids]
    err = np.abs(got - ref).max(axis=1)
    assert (err[~srgb] <= 1e-6).mean() >= 0.999 and (err[srgb] <= 2.5 / 255.0).mean() >= 0.999


def test_textured_request_matches_oracle(gpu, cwp, oracle, serving):
    """Materials with base-colour, metallic/roughness, normal and emission images on box-field uvs (the emissive
    material is light-sampled, its image scaling the sampled radiance): the request's image matches the oracle's at
    >= 45 dB (the texture unit's filtering is restated, not bit-identical) with the same ray counts within 0.5%, and
    differs from the untextured image. With bump-terminator shadowing on the normal-mapped materials it matches again
    and differs from the image without."""
    b, descs, first, mats, base, boxes = serving
    meshes = cwp.serving_scenes(n_scenes=3, seed=2, tris=(200, 8000), instances=(1, 24), blas_per_scene=(1, 3))[0]   # the fixture's meshes
    uvs, tans = cwp.planar_uvs(meshes)
    imgs = cwp.texture_images()
    nm = len(mats)
    binds = [dict() for _ in range(nm)]
    for m in range(nm):
        if m % 4 == 0: binds[m] = dict(base_color=0)
        elif m % 4 == 1: binds[m] = dict(base_color=0, metallic=1, roughness=1, normal=2, normal_scale=0.8)
        elif m % 4 == 2: binds[m] = dict(normal=2, roughness=1)
    mats_e = np.array(mats, np.float32).copy()
    for b0 in base:   # every mesh's material 1 emits through image 3
        binds[b0 + 1] = dict(emission=3, base_color=0); mats_e[b0 + 1, 8:11] = 2.0
    mt = cwp.material_textures(binds)
    s = cwp.Server(b, mats_e, base, max_paths=1 << 16, max_requests=4)
    s.set_scenes(descs, first)
    req = requests(cwp, boxes, 1, seed=23, res=((64, 48),), spps=(4,))[0]
    (plain_acc, _), = run_all(s, [req])
    s.set_textures(imgs, mt, uvs, tans)
    (acc, st), = run_all(s, [req])
    assert not np.allclose(acc, plain_acc)
    nodes, tris = b.download(b.tuning().width)
    tlas, roots, inst = b.download_tlas(4, _n_inst(b, 4))
    tex, keep = cwp.textures_array(imgs)
    mesh_first = np.concatenate([[0], np.cumsum([len(f) for _, f, _, _ in meshes])]).astype(np.int32)
    lights = cwp.emissive_tables(meshes, base, mats_e, *cwp.scene_xforms(descs, first, req.scene, req.frame))
    assert len(lights[0]) > 0
    ref, cnt = oracle.render_request(req, b.tuning().width, nodes, tris, tlas, roots[0], inst, mats_e, base, tlas_width=b.tlas_width,
                                     textures=(tex, mt, uvs, tans, mesh_first), lights=lights)
    a = acc[:, :3] / req.spp; r = ref[:, :3] / req.spp
    assert cwp.imageio.psnr(a, r) >= 45.0
    assert abs(st.rays - cnt[0]) <= 5e-3 * cnt[0] and abs(st.shadow_rays - cnt[1]) <= 5e-3 * max(cnt[1], 1)
    req.bump_shadow = 1
    (acc_b, st_b), = run_all(s, [req])
    assert not np.allclose(acc_b, acc)
    tlas, roots, inst = b.download_tlas(4, _n_inst(b, 4))
    ref_b, cnt_b = oracle.render_request(req, b.tuning().width, nodes, tris, tlas, roots[0], inst, mats_e, base, tlas_width=b.tlas_width,
                                         textures=(tex, mt, uvs, tans, mesh_first), lights=lights)
    assert cwp.imageio.psnr(acc_b[:, :3] / req.spp, ref_b[:, :3] / req.spp) >= 45.0
    assert abs(st_b.rays - cnt_b[0]) <= 5e-3 * cnt_b[0]
    with pytest.raises(cwp.CwpError):
        s.set_textures(imgs, cwp.material_textures([dict(base_color=9)]), uvs)   # texture id out of range
