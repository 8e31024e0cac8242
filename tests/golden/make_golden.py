"""Generates tests/golden/boxes64.npz from the reference's own code (oracle/_ref/libcwpref.so, compiled from the
reference sources by oracle/Makefile):

  inputs   the 64-box field (770 triangles, seed 1) and a 2,048-ray batch: 1,024 camera rays plus 1,024 incoherent
           rays from camera-visible surface points (cosine-weighted about the normal)
  outputs  the reference's BVH2, BVH4, greedy BVH8 and SAH-collapsed CWBVH node arrays, leaf orders, packed triangles
           and Woop rows (16 bins, leaf 4), and the reference traversal's closest hits and any-hit occluders for the
           batch over BVH2 and CWBVH with Woop and Moller-Trumbore triangles

and tests/golden/instances.npz:

  inputs   256 seeded object-to-world maps (rotation x scale x translation, some mirrored, some near-singular) and 64
           parametric instances (translate / axis / angle / scale with per-frame velocities) at frames 0, 1 and 7
  outputs  the reference's invertXform inverses and determinant signs and its instanceXform matrices; the reference
           traversal's closest hits and any-hit occluders over its BVH4 nodes of boxes64 (Woop and Moller-Trumbore)

and tests/golden/bsdf.npz:

  inputs   96 seeded materials (Lambertian, glossy-diffuse, rough and mirror conductors, rough and smooth glass, blends)
           and 2,048 (material, wo, wi, eta, glossy-diffuse random pair, sample triple) cases
  outputs  the reference's bsdfEval f and pdf and bsdfSample wi / weight / pdf / success (render/bsdf.h), with the
           glossy-diffuse energy compensation off and on

and tests/golden/env.npz:

  inputs   two Radiance RGBE files written here (a 40x20 map with run-length scanlines: a sky gradient, a bright sun
           disc, a dark band; a 6x4 map with flat scanlines), kept as bytes
  outputs  the reference's loadHDR radiance and buildEnvMap tables (texels x strength 1.5, marginal and conditional
           CDFs) for each file

and tests/golden/bsdf_bump.npz:

  inputs   the cases of bsdf.npz with an unperturbed normal per case (the bump-terminator term of the diffuse lobe)
  outputs  the reference's bsdfEval and bsdfSample with it, energy compensation off and on

The fixtures pin the oracle and the library where the reference sources are absent. Run from the repository root:
    python tests/golden/make_golden.py              (every fixture)
    python tests/golden/make_golden.py env          (env.npz only)
    python tests/golden/make_golden.py bsdf_bump    (bsdf_bump.npz only, from bsdf.npz's inputs)
"""
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT); sys.path.insert(0, os.path.join(ROOT, "tests"))


def main():
    from conftest import REF_DIR, Ref
    cwp = importlib.import_module("cuda-wavefront-pathtracer_b200")
    ref = Ref(os.path.join(REF_DIR, "libcwpref.so"))
    mesh = cwp.Mesh.box_field(64, 1)
    v, f, fm, _ = mesh.arrays()
    out = dict(verts=v, faces=f, face_mat=fm)
    for name, variant, collapse in (("bvh2", 2, 0), ("bvh4", 4, 0), ("bvh8g", 8, 1), ("cwbvh", 8, 0)):
        r = ref.build(v, f, fm, variant=variant, leaf=4, collapse=collapse)
        out[f"{name}_nodes"] = r["nodes"]; out[f"{name}_order"] = r["order"]
        if name in ("bvh2", "cwbvh"):
            out[f"{name}_tris"] = r["tris"]; out[f"{name}_woop"] = r["woop"]
    p = cwp.frame_params(mesh, 64, 64, bounces=4)
    o1, d1 = cwp.camera_rays(p, 1024, seed=3)
    o2, d2 = cwp.incoherent_rays(1024, p, out["bvh2_tris"], lambda o, d: ref.trace(2, 1, False, out["bvh2_nodes"], out["bvh2_woop"], o, d, threads=1), seed=5)
    o, d = np.concatenate([o1, o2]), np.concatenate([d1, d2])
    out["rays_o"], out["rays_d"] = o, d
    for name, variant in (("bvh2", 2), ("cwbvh", 8)):
        for tri, tv in ((1, out[f"{name}_woop"]), (0, out[f"{name}_tris"])):
            out[f"{name}_t{tri}_closest"] = ref.trace(variant, tri, False, out[f"{name}_nodes"], tv, o, d, threads=1)
            out[f"{name}_t{tri}_any"] = ref.trace(variant, tri, True, out[f"{name}_nodes"], tv, o, d, threads=1)
    np.savez_compressed(os.path.join(HERE, "boxes64.npz"), **out)
    print("wrote", os.path.join(HERE, "boxes64.npz"), sum(a.nbytes for a in out.values()), "bytes uncompressed")
    instances(ref, out)
    bsdf(ref)
    bsdf_bump(ref)
    envmaps(ref)


def instances(ref, box):
    import ctypes as C
    L = ref.L
    rng = np.random.default_rng(21)
    mats = []
    for k in range(256):
        ax = rng.normal(size=3); ax /= np.linalg.norm(ax); a = rng.uniform(0, 2 * np.pi)
        K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
        R = np.eye(3) + np.sin(a) * K + (1 - np.cos(a)) * K @ K
        S = np.diag(np.exp(rng.uniform(-2, 2, 3)) * (np.where(rng.random(3) < 0.1, -1.0, 1.0)))
        if k % 32 == 5: S[2, 2] = 1e-7   # near-singular
        mats.append(np.concatenate([R @ S, rng.uniform(-100, 100, (3, 1))], 1).reshape(12))
    mats = np.array(mats, np.float32)
    inv = np.zeros_like(mats); det = np.zeros(len(mats), np.float32)
    fp = C.POINTER(C.c_float)
    for i in range(len(mats)):
        L.ref_xform_invert(mats[i].ctypes.data_as(fp), inv[i].ctypes.data_as(fp), det[i:i + 1].ctypes.data_as(fp))
    n = 64
    desc = dict(translate=rng.uniform(-50, 50, (n, 3)), translate_vel=rng.uniform(-1, 1, (n, 3)), axis=rng.normal(size=(n, 3)),
                angle=rng.uniform(-180, 180, n), angle_vel=rng.uniform(-5, 5, n), scale=np.exp(rng.uniform(-1, 1, (n, 3))),
                scale_vel=rng.uniform(-0.01, 0.01, (n, 3)))
    desc = {k: np.ascontiguousarray(v, np.float32) for k, v in desc.items()}
    desc["axis"][0] = 0.0   # zero axis: +z
    frames = np.array([0, 1, 7], np.int32)
    anim = np.zeros((n, len(frames), 12), np.float32)
    for i in range(n):
        for j, f in enumerate(frames):
            L.ref_xform_animate(desc["translate"][i].ctypes.data_as(fp), desc["translate_vel"][i].ctypes.data_as(fp), desc["axis"][i].ctypes.data_as(fp),
                                C.c_float(desc["angle"][i]), C.c_float(desc["angle_vel"][i]), desc["scale"][i].ctypes.data_as(fp),
                                desc["scale_vel"][i].ctypes.data_as(fp), C.c_int(int(f)), anim[i, j].ctypes.data_as(fp))
    out = dict(mats=mats, inv=inv, det_sign=det, frames=frames, anim=anim, **{f"desc_{k}": v for k, v in desc.items()})
    # BVH4 traversal of boxes64 (tris for Moller-Trumbore, woop rows re-packed in the BVH4 leaf order)
    r = ref.build(box["verts"], box["faces"], box["face_mat"], variant=4, leaf=4, collapse=0)
    for tri, tv in ((1, r["woop"]), (0, r["tris"])):
        out[f"bvh4_t{tri}_closest"] = ref.trace(4, tri, False, r["nodes"], tv, box["rays_o"], box["rays_d"], threads=1)
        out[f"bvh4_t{tri}_any"] = ref.trace(4, tri, True, r["nodes"], tv, box["rays_o"], box["rays_d"], threads=1)
    out["bvh4_tris"], out["bvh4_woop"] = r["tris"], r["woop"]
    np.savez_compressed(os.path.join(HERE, "instances.npz"), **out)
    print("wrote", os.path.join(HERE, "instances.npz"), sum(a.nbytes for a in out.values()), "bytes uncompressed")


def materials(rng, n):
    """n materials as float32 [n, 16] in the cwp_material layout, spanning every base and blend"""
    m = np.zeros((n, 16), np.float32)
    for i in range(n):
        kind = i % 8
        base = rng.uniform(0.05, 0.95, 3); spec = rng.uniform(0.5, 1.0, 3)
        rough = rng.choice([0.0, 0.02, rng.uniform(0.05, 1.0)], p=[0.1, 0.1, 0.8])
        metallic, trans, ws = 0.0, 0.0, 1.0
        if kind == 0: ws, rough = 0.0, 1.0                       # Lambertian
        elif kind == 1: metallic = 1.0                           # conductor
        elif kind == 2: trans = 1.0                              # glass
        elif kind == 3: metallic = rng.uniform(0.2, 0.8)         # blend conductor / glossy-diffuse
        elif kind == 4: trans = rng.uniform(0.2, 0.8)            # blend glass / glossy-diffuse
        elif kind == 5: metallic, trans = 0.3, 0.5               # three bases
        m[i, 0:3] = base; m[i, 3] = metallic; m[i, 4:7] = spec; m[i, 7] = rough; m[i, 11] = 1.5; m[i, 12] = ws; m[i, 13] = trans
    return m


def bsdf(ref):
    import ctypes as C
    L = ref.L
    L.ref_bsdf_eval.restype = None; L.ref_bsdf_sample.restype = None
    rng = np.random.default_rng(33)
    mats = materials(rng, 96)
    n = 2048
    mat = rng.integers(0, len(mats), n).astype(np.int32)
    def hemi(k, up=True):
        v = rng.normal(size=(k, 3)); v /= np.linalg.norm(v, axis=1, keepdims=True)
        if up: v[:, 2] = np.abs(v[:, 2]) + 1e-3
        return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)
    wo = hemi(n); wi = hemi(n, up=False)
    wi[: n // 4] = (wo[: n // 4] * np.array([-1, -1, 1], np.float32))   # mirror directions
    eta = np.where(rng.random(n) < 0.5, 1.5, 1 / 1.5).astype(np.float32)
    ux = rng.random((n, 2)).astype(np.float32); uvw = rng.random((n, 3)).astype(np.float32)
    out = dict(mats=mats, mat=mat, wo=wo, wi=wi, eta=eta, ux=ux, uvw=uvw)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    for gd in (0, 1):
        f = np.zeros((n, 3), np.float32); pdf = np.zeros(n, np.float32)
        L.ref_bsdf_eval(p(mats), p(mat), p(wo), p(wi), p(eta), C.c_int(gd), p(ux), p(f), p(pdf), C.c_long(n))
        sw = np.zeros((n, 3), np.float32); sWt = np.zeros((n, 3), np.float32); spdf = np.zeros(n, np.float32); ok = np.zeros(n, np.int32)
        L.ref_bsdf_sample(p(mats), p(mat), p(wo), p(eta), C.c_int(gd), p(ux), p(uvw), p(sw), p(sWt), p(spdf), p(ok), C.c_long(n))
        out.update({f"f{gd}": f, f"pdf{gd}": pdf, f"s_wi{gd}": sw, f"s_w{gd}": sWt, f"s_pdf{gd}": spdf, f"s_ok{gd}": ok})
    np.savez_compressed(os.path.join(HERE, "bsdf.npz"), **out)
    print("wrote", os.path.join(HERE, "bsdf.npz"), sum(a.nbytes for a in out.values()), "bytes uncompressed")


def bsdf_bump(ref):
    """The bump-terminator term (render/bsdf.h:67-75): the inputs of bsdf.npz with an unperturbed normal nr per triple,
    tilted from the shading normal by up to ~70 degrees (nr.z > 0, the only case the integrator passes), and nr = +z
    exactly for the last quarter (the term is off there); the reference's bsdfEval / bsdfSample with it."""
    import ctypes as C
    L = ref.L
    g = np.load(os.path.join(HERE, "bsdf.npz"))
    mats, mat, wo, wi, eta, ux, uvw = (np.ascontiguousarray(g[k]) for k in ("mats", "mat", "wo", "wi", "eta", "ux", "uvw"))
    n = len(mat)
    rng = np.random.default_rng(35)
    nr = rng.normal(size=(n, 3)); nr[:, 2] = np.abs(nr[:, 2]) + 0.35
    nr /= np.linalg.norm(nr, axis=1, keepdims=True)
    nr[3 * n // 4:] = (0.0, 0.0, 1.0)
    nr = np.ascontiguousarray(nr, np.float32)
    out = dict(nr=nr)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    L.ref_bsdf_eval_nr.restype = None; L.ref_bsdf_sample_nr.restype = None
    for gd in (0, 1):
        f = np.zeros((n, 3), np.float32); pdf = np.zeros(n, np.float32)
        L.ref_bsdf_eval_nr(p(mats), p(mat), p(wo), p(wi), p(eta), C.c_int(gd), p(ux), p(nr), p(f), p(pdf), C.c_long(n))
        sw = np.zeros((n, 3), np.float32); sWt = np.zeros((n, 3), np.float32); spdf = np.zeros(n, np.float32); ok = np.zeros(n, np.int32)
        L.ref_bsdf_sample_nr(p(mats), p(mat), p(wo), p(eta), C.c_int(gd), p(ux), p(uvw), p(nr), p(sw), p(sWt), p(spdf), p(ok), C.c_long(n))
        out.update({f"f{gd}": f, f"pdf{gd}": pdf, f"s_wi{gd}": sw, f"s_w{gd}": sWt, f"s_pdf{gd}": spdf, f"s_ok{gd}": ok})
    np.savez_compressed(os.path.join(HERE, "bsdf_bump.npz"), **out)
    print("wrote", os.path.join(HERE, "bsdf_bump.npz"), sum(a.nbytes for a in out.values()), "bytes uncompressed")


def rgbe_bytes(rgb, rle):
    """Radiance RGBE file content for float rgb [h, w, 3] (new-style run-length scanlines when rle, else flat)"""
    h, w = rgb.shape[:2]
    out = bytearray(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {h} +X {w}\n".encode())
    px = np.zeros((h, w, 4), np.uint8)
    for y in range(h):
        for x in range(w):
            m = float(rgb[y, x].max())
            if m < 1e-32:
                continue
            mant, e = np.frexp(m)
            sc = mant * 256.0 / m
            px[y, x, :3] = np.clip((rgb[y, x] * sc).astype(np.int64), 0, 255); px[y, x, 3] = e + 128
    for y in range(h):
        if not rle:
            out += px[y].tobytes(); continue
        out += bytes([2, 2, w >> 8, w & 255])
        for c in range(4):
            v = px[y, :, c]; x = 0
            while x < w:
                r = 1
                while x + r < w and r < 127 and v[x + r] == v[x]:
                    r += 1
                if r >= 3:
                    out += bytes([128 + r, int(v[x])]); x += r; continue
                s0 = x
                while x < w and x - s0 < 128 and not (x + 2 < w and v[x] == v[x + 1] == v[x + 2]):
                    x += 1
                out += bytes([x - s0]) + v[s0:x].tobytes()
    return bytes(out)


def envmaps(ref):
    import ctypes as C
    import tempfile
    L = ref.L
    L.ref_env_build.restype = C.c_int
    L.ref_env_build.argtypes = [C.c_char_p, C.c_float] + [C.c_void_p] * 6
    h, w = 20, 40
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    big = np.stack([0.2 + 0.6 * (1 - yy / h), 0.3 + 0.5 * (1 - yy / h), 0.6 + 0.3 * (1 - yy / h)], -1)
    big[((yy - 5) ** 2 + (xx - 28) ** 2) < 4] = (40.0, 36.0, 30.0)   # sun disc
    big[14:16] = 0.0                                                  # dark band (zero-luminance rows)
    big[:, 3:9] = (0.5, 0.5, 0.5)                                     # a flat block (runs)
    small = np.random.default_rng(3).uniform(0, 4, (4, 6, 3)).astype(np.float32)
    out = {}
    for name, img, rle in (("big", big, True), ("small", small, False)):
        data = rgbe_bytes(img, rle)
        with tempfile.NamedTemporaryFile(suffix=".hdr", delete=False) as f:
            f.write(data); path = f.name
        ww, hh = C.c_int(), C.c_int()
        assert L.ref_env_build(path.encode(), 1.5, C.byref(ww), C.byref(hh), None, None, None, None) == 0
        W, H = ww.value, hh.value
        rgb = np.zeros((H, W, 3), np.float32); tex = np.zeros((H, W, 4), np.float32)
        marg = np.zeros(H + 1, np.float32); cond = np.zeros((H, W + 1), np.float32)
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        assert L.ref_env_build(path.encode(), 1.5, C.byref(ww), C.byref(hh), p(rgb), p(tex), p(marg), p(cond)) == 0
        os.unlink(path)
        out.update({f"{name}_hdr": np.frombuffer(data, np.uint8), f"{name}_rgb": rgb, f"{name}_tex": tex, f"{name}_marg": marg, f"{name}_cond": cond})
    np.savez_compressed(os.path.join(HERE, "env.npz"), **out)
    print("wrote", os.path.join(HERE, "env.npz"), sum(a.nbytes for a in out.values()), "bytes uncompressed")


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] in ("env", "bsdf_bump"):
        from conftest import REF_DIR, Ref
        (envmaps if sys.argv[1] == "env" else bsdf_bump)(Ref(os.path.join(REF_DIR, "libcwpref.so")))
    else:
        main()
