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

__all__ = ["SCENES", "scene", "frame_params", "scene_extent", "camera_rays", "incoherent_rays", "reference_inputs",
           "HFOV", "SEED", "SUN_TO", "SUN_E", "SUN_ANGLE_RAD", "SKY", "ALBEDO"]


def scene(name_or_boxes, variant=8, bins=32, leaf=4, collapse=0, threads=0):
    """(mesh, bvh) of a box-field scene; bvh.albedo is set to the benchmark albedo."""
    from . import Bvh, Mesh
    n = SCENES.get(name_or_boxes, name_or_boxes)
    mesh = Mesh.box_field(int(n), SCENE_SEED)
    bvh = Bvh(mesh, variant=variant, bins=bins, leaf=leaf, collapse=collapse, threads=threads)
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
