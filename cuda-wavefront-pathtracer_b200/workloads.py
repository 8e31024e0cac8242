"""Synthetic workloads of the diffuse benchmark path: seeded box-field scenes, the frame settings, and incoherent ray
batches. The reference's benchmark scene (116,855 triangles of Poly Haven models) is not redistributed, so a box field
of the same size stands in for it:

  boxes12k   1,024 boxes + ground = 12,290 triangles   (256x256, 16 spp, depth 4)
  boxes117k  9,750 boxes + ground = 117,002 triangles  (512x512 and 1280x720, 256 spp, depth 4; 16M-ray batches)

Boxes: centres uniform in x, z in [-20, 20], edges log-uniform in [0.2, 3] per axis, rotation about the vertical
uniform in [0, 2 pi), resting on a 40 x 40 ground, generated y-up and stored z-up. Lighting and camera (pinned here,
stated with every result): pinhole camera at (0, -34, 22) looking at the origin, 45 deg horizontal field of view;
sun towards (0.608749, -0.42625, 0.669131) at 3 W/m^2 with a 0.00918 rad disc, constant sky (0.30, 0.38, 0.50),
albedo 0.7, 1-pixel box filter, seed 1000, ray offset 1e-4 x scene extent.
"""
import json
import math

import numpy as np

SCENES = {"boxes12k": 1024, "boxes117k": 9750}
SCENE_SEED = 1
CAM_POS, CAM_TARGET, CAM_UP, HFOV = (0.0, -34.0, 22.0), (0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 45.0
SUN_TO = (0.608749, -0.42625, 0.669131)
SUN_E = 3.0
SUN_ANGLE_RAD = 0.00918
SKY = (0.30, 0.38, 0.50)
ALBEDO = 0.7
SEED = 1000
EPS_SCALE = 1e-4

__all__ = ["SCENES", "scene", "box_field_arrays", "frame_params", "scene_extent", "camera_rays", "incoherent_rays", "reference_inputs",
           "batch_scenes", "batch_rays", "serving_scenes", "serving_requests", "planar_uvs", "texture_images", "RESOLUTIONS", "SPPS", "HFOV", "SEED", "SUN_TO", "SUN_E", "SUN_ANGLE_RAD", "SKY", "ALBEDO"]


def box_field_arrays(n_boxes, seed=SCENE_SEED, half=20.0, edge_lo=0.2, edge_hi=3.0):
    """The box field of Mesh.box_field (cwp_mesh_box_field) in plain Python, without the CUDA library: (verts float32
    (nv, 3), faces int32 (nt, 3), face material int32 (nt,)). Same SplitMix64 stream, same double arithmetic through
    the C library's exp / log / cos / sin, same float rounding, so the arrays are bit-identical to the library's (a
    CPU test checks it). Used where the library must not be loaded: the reference arm of the benchmark."""
    M64 = (1 << 64) - 1
    state = [int(seed) & M64]

    def unit():
        state[0] = (state[0] + 0x9E3779B97F4A7C15) & M64
        z = state[0]
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return ((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0)
    half = float(np.float32(half))
    l_lo, l_hi = math.log(float(np.float32(edge_lo))), math.log(float(np.float32(edge_hi)))
    v = [(-half, 0.0, -half), (half, 0.0, -half), (half, 0.0, half), (-half, 0.0, half)]   # ground, y-up
    f = [(0, 2, 1), (0, 3, 2)]
    quads = ((0, 4, 6, 2), (1, 3, 7, 5), (0, 1, 5, 4), (2, 6, 7, 3), (0, 2, 3, 1), (4, 5, 7, 6))
    for _ in range(int(n_boxes)):
        cx = -half + 2.0 * half * unit(); cz = -half + 2.0 * half * unit()
        ex = math.exp(l_lo + (l_hi - l_lo) * unit()); ey = math.exp(l_lo + (l_hi - l_lo) * unit()); ez = math.exp(l_lo + (l_hi - l_lo) * unit())
        th = 2.0 * 3.14159265358979323846 * unit(); c, s = math.cos(th), math.sin(th)
        base = len(v)
        for k in range(8):
            lx = (0.5 if k & 1 else -0.5) * ex; ly = ey if k & 2 else 0.0; lz = (0.5 if k & 4 else -0.5) * ez
            v.append((cx + lx * c + lz * s, ly, cz - lx * s + lz * c))
        for q in quads:
            f.append((base + q[0], base + q[1], base + q[2])); f.append((base + q[0], base + q[2], base + q[3]))
    vd = np.array(v, np.float64)
    verts = np.stack([vd[:, 0], -vd[:, 2], vd[:, 1]], 1).astype(np.float32)   # y-up -> z-up, (x, y, z) -> (x, -z, y)
    faces = np.array(f, np.int32)
    return verts, faces, np.zeros(len(faces), np.int32)


def scene(name_or_boxes, variant=8, bins=32, leaf=4, collapse=0, threads=0, spatial=0.0):
    """(mesh, bvh) of a box-field scene; bvh.albedo is set to the benchmark albedo."""
    from . import Bvh, Mesh
    n = SCENES.get(name_or_boxes, name_or_boxes)
    mesh = Mesh.box_field(int(n), SCENE_SEED)
    bvh = Bvh(mesh, variant=variant, bins=bins, leaf=leaf, collapse=collapse, threads=threads, spatial=spatial)
    bvh.albedo = np.full((1, 3), ALBEDO, np.float32)
    return mesh, bvh


def scene_extent(mesh):
    v = mesh.arrays()[0]
    return float(np.max(v.max(0) - v.min(0)))


def frame_params(mesh, w, h, bounces=4, seed=SEED):
    """Params of the benchmark frame (the reference CLI's setupScene arithmetic for the same flags)."""
    from . import camera_look_at, params_defaults, params_finish
    p = params_defaults()
    p.cam = camera_look_at(CAM_POS, CAM_TARGET, CAM_UP, HFOV, w, h)
    p.sun_to[:] = SUN_TO
    p.sun_e[:] = (SUN_E,) * 3
    p.sky[:] = SKY
    p.max_b, p.seed, p.filter_bh, p.near_clip, p.has_n = bounces, seed, 0, 0.0, 0
    sun_deg = float(np.float32(SUN_ANGLE_RAD * 180.0 / math.pi))
    return params_finish(p, sun_deg, EPS_SCALE, scene_extent(mesh))


def camera_rays(p, n, seed=7):
    """n camera rays through seeded random pixels with box jitter: (o, d) float4 arrays (tmin 0, tmax 1e30)."""
    rng = np.random.default_rng(seed)
    c = p.cam
    px = rng.integers(0, c.w, n).astype(np.float32) + rng.random(n, np.float32)
    py = rng.integers(0, c.h, n).astype(np.float32) + rng.random(n, np.float32)
    dx = (px - np.float32(c.px)) / np.float32(c.fx)
    dy = -(py - np.float32(c.py)) / np.float32(c.fy)
    ax, ay, az = (np.array(list(v), np.float32) for v in (c.ax, c.ay, c.az))
    d = ax[None] * dx[:, None] + ay[None] * dy[:, None] - az[None]
    d /= np.sqrt((d * d).sum(1, dtype=np.float32))[:, None]
    o = np.zeros((n, 4), np.float32); o[:, :3] = np.array(list(c.pos), np.float32)
    dd = np.empty((n, 4), np.float32); dd[:, :3] = d; dd[:, 3] = 1e30
    return o, dd


def incoherent_rays(n, p, tris, trace_closest, seed=11):
    """Incoherent ray batch: origins on camera-visible surface points offset by eps along the geometric normal,
    directions cosine-weighted about the normal facing the camera. trace_closest(o, d) -> hits float4 is used to find
    the surface points (any exact implementation gives the same batch). Returns (o, d) float4, tmin 0, tmax 1e30."""
    out_o, out_d, have = [], [], 0
    rng = np.random.default_rng(seed)
    while have < n:
        m = int((n - have) * 1.4) + 1024
        o, d = camera_rays(p, m, seed=int(rng.integers(1 << 30)))
        hits = trace_closest(o, d)
        tri = hits[:, 3].view(np.int32)
        keep = tri >= 0
        o, d, hits, tri = o[keep], d[keep], hits[keep], tri[keep]
        t = hits[:, 0:1]
        pnt = o[:, :3] + d[:, :3] * t
        e1 = tris[3 * tri + 1, :3]; e2 = tris[3 * tri + 2, :3]
        ng = np.cross(e1, e2).astype(np.float32)
        ng /= np.maximum(np.sqrt((ng * ng).sum(1)), np.float32(1e-30))[:, None]
        flip = (ng * d[:, :3]).sum(1) > 0
        ng[flip] = -ng[flip]
        # cosine-weighted direction in the frame of ng (Duff et al. 2017)
        u0 = rng.random(len(ng), np.float32); u1 = rng.random(len(ng), np.float32)
        s = np.where(ng[:, 2] >= 0, np.float32(1), np.float32(-1))
        a = np.float32(-1) / (s + ng[:, 2]); b = ng[:, 0] * ng[:, 1] * a
        tx = np.stack([1 + s * ng[:, 0] * ng[:, 0] * a, s * b, -s * ng[:, 0]], 1)
        ty = np.stack([b, s + ng[:, 1] * ng[:, 1] * a, -ng[:, 1]], 1)
        r = np.sqrt(u0); ph = np.float32(2 * math.pi) * u1
        dirs = tx * (r * np.cos(ph))[:, None] + ty * (r * np.sin(ph))[:, None] + ng * np.sqrt(np.maximum(0, 1 - u0))[:, None]
        dirs /= np.sqrt((dirs * dirs).sum(1))[:, None]
        oo = np.zeros((len(ng), 4), np.float32); oo[:, :3] = pnt + ng * np.float32(p.eps)
        dd = np.empty((len(ng), 4), np.float32); dd[:, :3] = dirs; dd[:, 3] = 1e30
        out_o.append(oo); out_d.append(dd); have += len(oo)
    return np.concatenate(out_o)[:n].astype(np.float32), np.concatenate(out_d)[:n].astype(np.float32)


def reference_inputs(mesh, p, outdir, w, h, spp, batch, variant="bvh2"):
    """Writes the scene as binary PLY plus camera/lighting JSON for the reference's `pt`, and returns its arguments
    for the same frame (the reference computes fx from --hfov with the same formula)."""
    import os
    os.makedirs(outdir, exist_ok=True)
    ply, cam, light = (os.path.join(outdir, f) for f in ("scene.ply", "camera.json", "lighting.json"))
    mesh.write_ply(ply)
    c = p.cam
    c2w = [c.ax[0], c.ay[0], c.az[0], c.pos[0], c.ax[1], c.ay[1], c.az[1], c.pos[1], c.ax[2], c.ay[2], c.az[2], c.pos[2], 0, 0, 0, 1]
    with open(cam, "w") as f:
        f.write('{"c2w_blender_zup": [' + ", ".join("%.9g" % x for x in c2w) + "]}\n")
    with open(light, "w") as f:
        json.dump({"sun_dir_to_light_world_zup": list(SUN_TO), "sun_irradiance_W_m2": SUN_E, "sun_angle_rad": SUN_ANGLE_RAD,
                   "sky_radiance_rgb_linear": list(SKY)}, f)
    return ["--mesh", ply, "--camera", cam, "--lighting", light, "--albedo", str(ALBEDO), str(ALBEDO), str(ALBEDO),
            "--filter", "box", "--hfov", str(HFOV), "--width", str(w), "--height", str(h), "--spp", str(spp), "--bounces", str(p.max_b),
            "--variant", variant, "--tri", "woop", "--fuse", "1", "--batch", str(batch), "--seed", str(p.seed), "--leaf", "4"]


def _log_uniform_int(rng, lo, hi):
    return int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))


def batch_scenes(n_scenes=64, seed=5, tris=(1000, 500000), instances=(1, 4096), blas_per_scene=(1, 8)):
    """The batched-form workload: n_scenes two-level scenes, each a TLAS over a log-uniform number of instances of
    1-8 BLAS of its own; every BLAS is a box field of a log-uniform triangle count; every instance a random rigid
    transform (axis uniform on the sphere, angle uniform in [0, 2 pi), translation uniform in a cube that grows with
    the cube root of the instance count). Returns (meshes, xforms [n_inst, 12], mesh_of [n_inst], scene_first)."""
    from . import Mesh
    rng = np.random.default_rng(seed)
    meshes, xf, mesh_of, first = [], [], [], [0]
    for s in range(n_scenes):
        nb = int(rng.integers(blas_per_scene[0], blas_per_scene[1] + 1))
        ids = []
        for _ in range(nb):
            nt = _log_uniform_int(rng, *tris)
            ids.append(len(meshes))
            meshes.append(Mesh.box_field(max(1, (nt - 2) // 12), int(rng.integers(1 << 30))))
        ni = _log_uniform_int(rng, *instances)
        half = 20.0 * max(1.0, ni ** (1.0 / 3.0))
        for _ in range(ni):
            ax = rng.normal(size=3); ax /= np.linalg.norm(ax)
            ang = rng.uniform(0, 2 * math.pi); c, sn, k = math.cos(ang), math.sin(ang), 1 - math.cos(ang)
            x, y, z = ax
            R = np.array([[c + x * x * k, x * y * k - z * sn, x * z * k + y * sn],
                          [y * x * k + z * sn, c + y * y * k, y * z * k - x * sn],
                          [z * x * k - y * sn, z * y * k + x * sn, c + z * z * k]])
            t = rng.uniform(-half, half, 3)
            xf.append(np.concatenate([R, t[:, None]], 1).reshape(12))
            mesh_of.append(ids[int(rng.integers(len(ids)))])
        first.append(len(xf))
    return meshes, np.array(xf, np.float32).reshape(-1, 12), np.array(mesh_of, np.int32), np.array(first, np.int32)


def batch_rays(xforms, scene_first, rays_per_scene, seed=9, extent=40.0):
    """Rays of the batched workload, scene-major: origins uniform in each scene's instance-translation box grown by
    the mesh extent, directions uniform on the sphere, tmin 0, tmax 1e30. Returns (o, d float4, scene int32)."""
    rng = np.random.default_rng(seed)
    n_s = len(scene_first) - 1
    o = np.zeros((n_s * rays_per_scene, 4), np.float32); d = np.zeros_like(o); sc = np.repeat(np.arange(n_s, dtype=np.int32), rays_per_scene)
    for s in range(n_s):
        a, b = scene_first[s], scene_first[s + 1]
        sl = slice(s * rays_per_scene, (s + 1) * rays_per_scene)
        if b > a:
            t = xforms[a:b].reshape(-1, 3, 4)[:, :, 3]
            lo, hi = t.min(0) - extent, t.max(0) + extent
        else:
            lo, hi = np.full(3, -extent), np.full(3, extent)
        o[sl, :3] = rng.uniform(lo, hi, (rays_per_scene, 3))
        v = rng.normal(size=(rays_per_scene, 3)); v /= np.linalg.norm(v, axis=1, keepdims=True)
        d[sl, :3] = v; d[sl, 3] = 1e30
    return o, d, sc


RESOLUTIONS = [(256, 256), (512, 512), (1280, 720), (1920, 1080)]
SPPS = [1, 4, 16, 64, 256]


def serving_scenes(n_scenes=32, seed=7, tris=(1000, 500000), instances=(1, 4096), blas_per_scene=(1, 8), mats_per_mesh=8):
    """Resident scenes of the serving form: the batched form's generator (box-field BLAS of log-uniform size, a
    log-uniform number of instances per scene) with animated instances (per-frame translation and rotation) and
    OpenPBR materials per mesh: roughness uniform in [0.05, 1], metallic ~ Bernoulli(0.3), 10% glass at IOR 1.5.
    Returns (mesh arrays [(verts, faces, face_mat, None)], descs (InstanceDesc array), scene_first, materials [n, 16],
    mesh_mat_base, scene_boxes [n_scenes, 2, 3])."""
    from . import InstanceDesc, Mesh
    rng = np.random.default_rng(seed)
    meshes, descs, first, mats, base, boxes = [], [], [0], [], [], []
    for s in range(n_scenes):
        nb = int(rng.integers(blas_per_scene[0], blas_per_scene[1] + 1))
        ids = []
        for _ in range(nb):
            nt = _log_uniform_int(rng, *tris)
            m = Mesh.box_field(max(1, (nt - 2) // 12), int(rng.integers(1 << 30)))
            v, f, fm, _ = m.arrays()
            fm = np.zeros(len(f), np.int32); fm[2:] = (np.arange(len(f) - 2) // 12) % (mats_per_mesh - 1) + 1   # ground 0, boxes 1..
            ids.append(len(meshes)); meshes.append((v, f, fm, None)); base.append(len(mats))
            for k in range(mats_per_mesh):
                mt = np.zeros(16, np.float32)
                mt[0:3] = rng.uniform(0.2, 0.9, 3); mt[4:7] = 1.0; mt[7] = rng.uniform(0.05, 1.0); mt[11] = 1.5; mt[12] = 1.0
                if rng.random() < 0.1: mt[13] = 1.0                # glass
                elif rng.random() < 0.3: mt[3] = 1.0               # metal
                mats.append(mt)
        ni = _log_uniform_int(rng, *instances)
        half = 20.0 * max(1.0, ni ** (1.0 / 3.0))
        for _ in range(ni):
            d = InstanceDesc()
            d.mesh = ids[int(rng.integers(len(ids)))]
            d.translate[:] = tuple(rng.uniform(-half, half, 3)); d.translate_per_frame[:] = tuple(rng.normal(0, 0.2, 3))
            ax = rng.normal(size=3); ax /= np.linalg.norm(ax); d.axis[:] = tuple(ax)
            d.angle_deg = float(rng.uniform(0, 360)); d.angle_deg_per_frame = float(rng.uniform(-2, 2))
            d.scale[:] = (1.0, 1.0, 1.0); d.scale_per_frame[:] = (0.0, 0.0, 0.0)
            descs.append(d)
        first.append(len(descs))
        boxes.append([[-half - 30] * 3, [half + 30] * 3])
    arr = (InstanceDesc * len(descs))(*descs)
    return meshes, arr, np.array(first, np.int32), np.array(mats, np.float32), np.array(base, np.int32), np.array(boxes, np.float32)


def serving_requests(n, rate, scene_boxes, seed=11, resolutions=None, spps=None, max_depth=8, frames=30):
    """n requests of a Poisson stream at `rate` per second: arrival time, scene (uniform), animation frame (uniform in
    [0, frames)), resolution and spp uniform over the given sets, camera looking at the scene centre from a random
    direction above the horizon at the scene's extent. Returns a list of (arrival_s, Request)."""
    from . import camera_look_at, make_request
    rng = np.random.default_rng(seed)
    resolutions = resolutions or RESOLUTIONS; spps = spps or SPPS
    t, out = 0.0, []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        sc = int(rng.integers(len(scene_boxes))); lo, hi = scene_boxes[sc]
        c = (lo + hi) * 0.5; ext = float(np.max(hi - lo))
        th = rng.uniform(0, 2 * math.pi); el = rng.uniform(0.3, 1.2)
        pos = c + 0.7 * ext * np.array([math.cos(th) * math.cos(el), math.sin(th) * math.cos(el), math.sin(el)])
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        cam = camera_look_at(tuple(pos), tuple(c), (0, 0, 1), HFOV, w, h)
        out.append((t, make_request(sc, cam, int(spps[int(rng.integers(len(spps)))]), frame=int(rng.integers(frames)), max_depth=max_depth,
                                    seed=int(rng.integers(1 << 30)), eps=1e-4 * ext)))
    return out


def planar_uvs(meshes, scale=0.35):
    """Texture coordinates and tangents for box-field meshes: each triangle projected along its normal's dominant axis
    (u, v from the other two axes, scaled), the tangent along the u axis with the handedness that makes
    sign * (n x t) the v axis. Returns (uvs float32 [n, 8], tans float32 [n, 12]) over all meshes in mesh order."""
    uvs, tans = [], []
    for m in meshes:
        v, f = (m.arrays() if hasattr(m, "arrays") else m)[:2]
        p = v[f].astype(np.float64)
        n = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
        a = np.argmax(np.abs(n), axis=1); b = (a + 1) % 3; c = (a + 2) % 3
        idx = np.arange(len(f))
        uv = np.stack([p[idx[:, None], np.arange(3)[None, :], b[:, None]], p[idx[:, None], np.arange(3)[None, :], c[:, None]]], -1) * scale
        u = np.zeros((len(f), 8), np.float32)
        u[:, 0:2], u[:, 2:4], u[:, 4:6] = uv[:, 0], uv[:, 1], uv[:, 2]
        t = np.zeros((len(f), 3)); t[idx, b] = 1.0
        e_c = np.zeros((len(f), 3)); e_c[idx, c] = 1.0
        sg = np.where(np.einsum("ij,ij->i", np.cross(n, t), e_c) < 0, -1.0, 1.0)
        tg = np.zeros((len(f), 12), np.float32)
        for k in range(3):
            tg[:, 4 * k:4 * k + 3] = t; tg[:, 4 * k + 3] = sg
        uvs.append(u); tans.append(tg)
    return np.concatenate(uvs), np.concatenate(tans)


def texture_images(seed=1):
    """Procedural images: an sRGB colour checker (48x32), a linear roughness (G) / metalness (B) map (20x20), a
    tangent-space bump normal map (32x32), an sRGB emission spot map (16x16). List of (rgba uint8, srgb)."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:32, 0:48]
    chk = ((yy // 4 + xx // 6) % 2).astype(np.float64)
    col = np.stack([40 + 180 * chk, 200 - 120 * chk, 90 + 60 * rng.random((32, 48)), np.full((32, 48), 255)], -1)
    rm = np.stack([np.zeros((20, 20)), 40 + 200 * rng.random((20, 20)), 255.0 * (rng.random((20, 20)) < 0.3), np.full((20, 20), 255)], -1)
    y2, x2 = np.mgrid[0:32, 0:32] / 32.0
    nx, ny = 0.5 * np.sin(2 * np.pi * 3 * x2), 0.5 * np.cos(2 * np.pi * 2 * y2); nz = np.sqrt(np.maximum(0.0, 1 - nx ** 2 - ny ** 2))
    nrm = np.stack([(nx + 1) * 127.5, (ny + 1) * 127.5, (nz + 1) * 127.5, np.full((32, 32), 255)], -1)
    y3, x3 = np.mgrid[0:16, 0:16]
    em = np.where(((y3 - 8) ** 2 + (x3 - 8) ** 2) < 12, 255, 0)
    emi = np.stack([em, em * 0.8, em * 0.5, np.full((16, 16), 255)], -1)
    return [(np.clip(col, 0, 255).astype(np.uint8), True), (np.clip(rm, 0, 255).astype(np.uint8), False),
            (np.clip(nrm, 0, 255).astype(np.uint8), False), (np.clip(emi, 0, 255).astype(np.uint8), True)]
