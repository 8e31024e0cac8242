"""Generates tests/golden/boxes64.npz from the reference's own code (oracle/_ref/libcwpref.so, compiled from the
reference sources by oracle/Makefile):

  inputs   the 64-box field (770 triangles, seed 1) and a 2,048-ray batch: 1,024 camera rays plus 1,024 incoherent
           rays from camera-visible surface points (cosine-weighted about the normal)
  outputs  the reference's BVH2, BVH4, greedy BVH8 and SAH-collapsed CWBVH node arrays, leaf orders, packed triangles
           and Woop rows (16 bins, leaf 4), and the reference traversal's closest hits and any-hit occluders for the
           batch over BVH2 and CWBVH with Woop and Moller-Trumbore triangles

The fixtures pin the oracle and the library where the reference sources are absent. Run from the repository root:
    python tests/golden/make_golden.py
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


if __name__ == "__main__":
    main()
