"""The benchmark frame (117,002-triangle box field, 512 x 512, 256 spp, depth 4) rendered by the reference's own CUDA
build (oracle/_ref/pt, compiled from its sources for sm_100 with its own flags) and by this library on the same B200:
images agree at >= 50 dB PSNR in tone-mapped sRGB, and both frame rates are recorded (printed, and written as JSON to
$CWP_RESULTS_DIR/vs_reference_cuda.json when that variable is set)."""
import json
import os
import subprocess

import pytest

from conftest import REF_DIR

pytestmark = pytest.mark.gpu


def run_ref_pt(cwp, mesh, p, tmp, w, h, spp, batch, variant, reps=2):
    pt = os.path.join(REF_DIR, "pt")
    args = cwp.reference_inputs(mesh, p, str(tmp), w, h, spp, batch, variant=variant)
    out = str(tmp / f"ref_{variant}")
    res = subprocess.run([pt] + args + ["--out", out, "--reps", str(reps)], check=True, capture_output=True, text=True, timeout=600)
    lines = [json.loads(l) for l in res.stdout.splitlines() if l.startswith("{")]
    return lines, cwp.imageio.read_pfm(out + ".pfm")


# (layout, SAH bins, spatial-split overlap threshold) of this library's trees per resolution: the binned-SAH trees at
# the reference's 16 bins and BASELINE's 32, and the SBVH-built CWBVH at 128 bins that the benchmark renders
TREES = {(512, 512): ((2, 16, 0.0), (8, 32, 0.0), (2, 32, 0.0), (8, 128, 1e-3)),
         (1280, 720): ((8, 32, 0.0), (8, 128, 1e-3))}


@pytest.mark.parametrize("w,h", [(512, 512), (1280, 720)])
def test_benchmark_frame_vs_reference_cuda(gpu, cwp, tmp_path, w, h):
    """Config 2's frame at both of its resolutions, 256 spp, depth 4: every tree of TREES renders within 50 dB of
    the reference's own CUDA build (render/wavefront.cu:684-741 over accel/traverse.cuh:112-152)."""
    if not os.path.exists(os.path.join(REF_DIR, "pt")):
        pytest.skip("oracle/_ref/pt not built")
    spp, batch = 256, 256
    mesh, bvh16 = cwp.scene("boxes117k", variant=2, bins=16)
    p = cwp.frame_params(mesh, w, h)
    record = {"scene": "boxes117k", "w": w, "h": h, "spp": spp, "batch": batch}
    ref_img = None
    for rv in ("bvh2", "bvh8"):
        lines, img = run_ref_pt(cwp, mesh, p, tmp_path, w, h, spp, batch, rv)
        ref_img = img if ref_img is None else ref_img
        best = min(lines, key=lambda l: l["t_frame_ms"])
        record[f"reference_{rv}"] = {k: best[k] for k in ("t_frame_ms", "rays_total", "rays_closest", "rays_shadow", "mrays_s_e2e", "gpu")}
    for variant, bins, spatial in TREES[(w, h)]:
        _, bvh = cwp.scene("boxes117k", variant=variant, bins=bins, spatial=spatial)
        r = cwp.Renderer(); r.init(p, bvh, variant=variant, batch=batch, bounces=4)
        r.render(spp)   # warm-up (graph capture)
        times = []
        for _ in range(3):
            st = r.render(spp); times.append(st.frame_ms)
        img = cwp.imageio.accum_to_image(r.read_accum(), w, h, spp)
        db = cwp.imageio.psnr(img, ref_img)
        key = f"ours_v{variant}_b{bins}" + ("_sbvh" if spatial else "")
        record[key] = {"t_frame_ms": min(times), "rays_total": st.rays + st.shadow_rays, "psnr_vs_reference_db": db,
                       "grays_s": (st.rays + st.shadow_rays) / min(times) / 1e6}
        r.close()
        assert db >= 50.0, (variant, bins, spatial, db)
    ref_best = min(record["reference_bvh2"]["t_frame_ms"], record["reference_bvh8"]["t_frame_ms"])
    ours_best = min(v["t_frame_ms"] for k, v in record.items() if k.startswith("ours_"))
    record["speedup_vs_reference_best"] = ref_best / ours_best
    print(json.dumps(record))
    d = os.environ.get("CWP_RESULTS_DIR")
    if d:
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, f"vs_reference_cuda_{w}x{h}.json"), "w") as f:
            json.dump(record, f, indent=1)


# ---------------- the serving integrator against the reference's full integrator on an instanced scene ----------------

def _write_ply(path, v, f, fm, n=None):
    """binary PLY with a per-face material_index and optional vertex normals, as the reference's loader reads it
    (io/mesh_loader.cpp:100-146)"""
    import numpy as np
    v = np.ascontiguousarray(v, "<f4"); f = np.asarray(f, np.int32); fm = np.asarray(fm, np.int32)
    if n is not None:
        v = np.ascontiguousarray(np.concatenate([v, np.asarray(n, "<f4")], 1))
    rec = np.zeros(len(f), dtype=[("n", "u1"), ("i", "<i4", 3), ("m", "<i4")])
    rec["n"] = 3; rec["i"] = f; rec["m"] = fm
    hdr = ("ply\nformat binary_little_endian 1.0\nelement vertex %d\nproperty float x\nproperty float y\nproperty float z\n" % len(v)
           + ("property float nx\nproperty float ny\nproperty float nz\n" if n is not None else "")
           + "element face %d\nproperty list uchar int vertex_indices\nproperty int material_index\nend_header\n" % len(f))
    with open(path, "wb") as fp:
        fp.write(hdr.encode()); fp.write(v.tobytes()); fp.write(rec.tobytes())


def _fl(x):
    import numpy as np
    return float(np.float32(x))


def write_reference_scene(tmp, meshes, descs, first, mats, base, frames, normals=None):
    """scene file (scene/instances.cpp:19-47) with one PLY and one materials file (io/scene_files.cpp:28-55) per mesh;
    the float values are written so that they parse back to the same floats"""
    import numpy as np
    mesh_entries = []
    for k, (v, f, fm, _) in enumerate(meshes):
        _write_ply(tmp / f"m{k}.ply", v, f, fm, normals[k] if normals is not None else None)
        n = (base[k + 1] if k + 1 < len(base) else len(mats)) - base[k]
        ms = []
        for m in mats[base[k]:base[k] + n]:
            em = m[8:11]
            ms.append({"base_color": [_fl(x) for x in m[0:3]], "metallic": _fl(m[3]), "specular_color": [_fl(x) for x in m[4:7]],
                       "roughness": _fl(m[7]), "ior": _fl(m[11]), "specular_weight": _fl(m[12]), "transmission": _fl(m[13]),
                       "emission_color": [_fl(x) for x in em] if np.any(em > 0) else [1.0, 1.0, 1.0],
                       "emission_strength": 1.0 if np.any(em > 0) else 0.0})
        with open(tmp / f"m{k}_mats.json", "w") as fp:
            json.dump({"materials": ms}, fp)
        mesh_entries.append({"file": f"m{k}.ply", "materials": f"m{k}_mats.json"})
    inst = []
    for i in range(int(first[0]), int(first[1])):
        d = descs[i]
        inst.append({"mesh": int(d.mesh), "translate": [_fl(x) for x in d.translate], "translate_per_frame": [_fl(x) for x in d.translate_per_frame],
                     "axis": [_fl(x) for x in d.axis], "angle_deg": _fl(d.angle_deg), "angle_deg_per_frame": _fl(d.angle_deg_per_frame),
                     "scale": [_fl(x) for x in d.scale], "scale_per_frame": [_fl(x) for x in d.scale_per_frame]})
    path = tmp / "scene.json"
    with open(path, "w") as fp:
        json.dump({"frames": frames, "meshes": mesh_entries, "instances": inst}, fp)
    return str(path)


def reference_eps(cwp, meshes, descs, first, scale=1e-4):
    """the reference's ray offset for a scene file: scale x the largest extent of the frame-0 world box over every
    instance's vertices (app/scene_setup.cpp:107, 153-155, 183), in float"""
    import numpy as np
    xf, im = cwp.scene_xforms(descs, first, 0, 0)
    lo = np.full(3, np.inf, np.float32); hi = np.full(3, -np.inf, np.float32)
    for m, k in zip(xf, im):
        v = np.asarray(meshes[k][0], np.float32)
        w = np.stack([m[4 * r] * v[:, 0] + m[4 * r + 1] * v[:, 1] + m[4 * r + 2] * v[:, 2] + m[4 * r + 3] for r in range(3)], 1)
        lo = np.minimum(lo, w.min(0)); hi = np.maximum(hi, w.max(0))
    return float(np.float32(scale) * np.max(hi - lo))


@pytest.mark.parametrize("case", ["sun", "sun_env", "nee_rr", "smooth"])
def test_serving_vs_reference_full_integrator(gpu, cwp, tmp_path, case):
    """An animated instanced scene with emissive boxes, rendered by the reference's own CUDA build (oracle/_ref/pt,
    scene-file mode: its full integrator over its TLAS/BLAS) and by a serving request of the same frame, camera,
    lights and seed. The sample streams are the same; the reference's fast-math build rounds differently, so paths
    decorrelate after a bounce and the agreement is Monte Carlo-limited. The bound: the two images differ less than
    two of this library's own renders with independent seeds do (PSNR in tone-mapped sRGB). Cases: sun and sky; with
    an environment map; NEE-only light sampling with Russian roulette; vertex normals on every second mesh. The first
    uses the Blackman-Harris pixel filter (the reference's default), the others the box filter."""
    import numpy as np
    from conftest import golden
    pt = os.path.join(REF_DIR, "pt")
    if not os.path.exists(pt):
        pytest.skip("oracle/_ref/pt not built")
    meshes, descs, first, mats, base, boxes = cwp.serving_scenes(n_scenes=1, seed=5, tris=(500, 4000), instances=(6, 16), blas_per_scene=(2, 3))
    mats = mats.copy()
    for b0 in base:
        mats[b0 + 1, 8:11] = (4.0, 3.0, 2.0)
    w, h, spp, depth = 96, 64, 256, 4
    (_, req), = cwp.serving_requests(1, 100.0, boxes, seed=41, resolutions=[(w, h)], spps=[spp], max_depth=depth, frames=30)
    req.eps = reference_eps(cwp, meshes, descs, first)
    nrm = None
    if case == "smooth":
        rng = np.random.default_rng(3)
        nrm = []
        for k, (v, f, fm, _) in enumerate(meshes):
            n = v - v.mean(0) + rng.normal(0, 0.3, v.shape)
            nrm.append(None if k % 2 else (n / np.linalg.norm(n, axis=1, keepdims=True)).astype(np.float32))
        # the reference gives every mesh normals once one has them (zeros elsewhere: flat shading there too)
        nrm_file = [n if n is not None else np.zeros((len(m[0]), 3), np.float32) for n, m in zip(nrm, meshes)]
    scene = write_reference_scene(tmp_path, meshes, descs, first, mats, base, frames=30, normals=nrm_file if nrm is not None else None)
    c = req.cam
    c2w = [c.ax[0], c.ay[0], c.az[0], c.pos[0], c.ax[1], c.ay[1], c.az[1], c.pos[1], c.ax[2], c.ay[2], c.az[2], c.pos[2], 0, 0, 0, 1]
    with open(tmp_path / "camera.json", "w") as fp:
        fp.write('{"c2w_blender_zup": [' + ", ".join("%.9g" % x for x in c2w) + "]}\n")
    W = cwp.workloads
    with open(tmp_path / "lighting.json", "w") as fp:
        json.dump({"sun_dir_to_light_world_zup": list(W.SUN_TO), "sun_irradiance_W_m2": W.SUN_E, "sun_angle_rad": W.SUN_ANGLE_RAD,
                   "sky_radiance_rgb_linear": list(W.SKY)}, fp)
    args = [pt, "--scene", scene, "--frame_start", str(req.frame), "--frames", "1", "--camera", str(tmp_path / "camera.json"),
            "--lighting", str(tmp_path / "lighting.json"), "--filter", "bh" if case == "sun" else "box", "--hfov", str(W.HFOV), "--width", str(w), "--height", str(h),
            "--spp", str(spp), "--batch", "64", "--bounces", str(depth), "--seed", str(req.seed), "--variant", "bvh2", "--warm", "0",
            "--out", str(tmp_path / "ref")]
    req.filter_bh = 1 if case == "sun" else 0   # the reference's default pixel filter in one case
    b = cwp.Batch(meshes, normals=nrm)
    s = cwp.Server(b, mats, base, max_paths=1 << 20, max_requests=2)
    s.set_scenes(descs, first)
    if case == "sun_env":
        g = golden("env.npz")
        (tmp_path / "env.hdr").write_bytes(g["big_hdr"].tobytes())
        args += ["--env", str(tmp_path / "env.hdr"), "--env_strength", "1.5", "--env_rot", "30"]
        s.set_envmaps([(g["big_rgb"], 1.5)])
        req.env, req.env_rot_deg = 0, 30.0
    if case == "nee_rr":
        args += ["--light_sampling", "nee", "--rr", "1", "--rr_depth", "2"]
        req.light_mode, req.rr, req.rr_depth = cwp.LIGHT_NEE, 1, 2
    subprocess.run(args, check=True, capture_output=True, text=True, timeout=600)
    ref = cwp.imageio.read_pfm(str(tmp_path / "ref.pfm"))

    def render(seed):
        import ctypes as C
        r = cwp.Request(); C.memmove(C.addressof(r), C.addressof(req), C.sizeof(r)); r.seed = seed
        i = s.submit(r)
        while True:
            s.step()
            if i in s.poll():
                break
        acc, _ = s.result(i, w, h)
        return cwp.imageio.accum_to_image(acc, w, h, spp)
    ours = render(req.seed)
    other = render(req.seed + 7919)
    db, floor = cwp.imageio.psnr(ours, ref), cwp.imageio.psnr(ours, other)
    print(json.dumps({"case": case, "psnr_vs_reference_db": db, "psnr_independent_seeds_db": floor}))
    assert db >= floor, (db, floor)


def test_cli_scene_file_vs_reference(gpu, cwp, tmp_path):
    """This library's command-line renderer and the reference's, on the same scene file, camera, lighting file and
    environment map (emissive boxes, animated instances, frame 7, Blackman-Harris filter, both CLIs' defaults
    otherwise): the images differ less than two of this CLI's renders with independent seeds do."""
    import numpy as np
    from conftest import golden
    pt = os.path.join(REF_DIR, "pt")
    ours = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cuda-wavefront-pathtracer_b200", "pt")
    if not os.path.exists(pt):
        pytest.skip("oracle/_ref/pt not built")
    meshes, descs, first, mats, base, boxes = cwp.serving_scenes(n_scenes=1, seed=9, tris=(500, 4000), instances=(6, 16), blas_per_scene=(2, 3))
    mats = mats.copy()
    for b0 in base:
        mats[b0 + 1, 8:11] = (4.0, 3.0, 2.0)
    scene = write_reference_scene(tmp_path, meshes, descs, first, mats, base, frames=30)
    (_, req), = cwp.serving_requests(1, 100.0, boxes, seed=43, resolutions=[(96, 64)], spps=[256], max_depth=4, frames=30)
    c = req.cam
    c2w = [c.ax[0], c.ay[0], c.az[0], c.pos[0], c.ax[1], c.ay[1], c.az[1], c.pos[1], c.ax[2], c.ay[2], c.az[2], c.pos[2], 0, 0, 0, 1]
    with open(tmp_path / "camera.json", "w") as fp:
        fp.write('{"c2w_blender_zup": [' + ", ".join("%.9g" % x for x in c2w) + "]}\n")
    g = golden("env.npz")
    (tmp_path / "env.hdr").write_bytes(g["big_hdr"].tobytes())
    W = cwp.workloads
    with open(tmp_path / "lighting.json", "w") as fp:
        json.dump({"sun_dir_to_light_world_zup": list(W.SUN_TO), "sun_irradiance_W_m2": W.SUN_E, "sun_angle_rad": W.SUN_ANGLE_RAD,
                   "sky_radiance_rgb_linear": list(W.SKY), "env_map": str(tmp_path / "env.hdr"), "env_strength": 1.5, "env_rotation_deg": 30.0}, fp)
    args = ["--scene", scene, "--frame_start", "7", "--frames", "1", "--camera", str(tmp_path / "camera.json"), "--lighting", str(tmp_path / "lighting.json"),
            "--hfov", str(W.HFOV), "--width", "96", "--height", "64", "--spp", "256", "--batch", "64", "--bounces", "4", "--variant", "bvh2", "--warm", "0"]
    subprocess.run([pt] + args + ["--seed", "11", "--out", str(tmp_path / "ref")], check=True, capture_output=True, text=True, timeout=600)
    for seed, name in ((11, "ours"), (12, "other")):
        r = subprocess.run([ours] + args + ["--seed", str(seed), "--out", str(tmp_path / name)], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
    line = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")][-1]
    assert line["integrator"] == "full" and line["env"] == 1 and line["frame"] == 7 and line["rays_total"] > 0
    ref, a, b = (cwp.imageio.read_pfm(str(tmp_path / f"{n}.pfm")) for n in ("ref", "ours", "other"))
    db, floor = cwp.imageio.psnr(a, ref), cwp.imageio.psnr(a, b)
    print(json.dumps({"cli_psnr_vs_reference_db": db, "cli_psnr_independent_seeds_db": floor}))
    assert db >= floor, (db, floor)
