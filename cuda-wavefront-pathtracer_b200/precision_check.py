"""Comparison of float closest hits with the FP64 oracle traversal (cwp_trace_fp64): the precision form's lost-hit,
tie and t-error figures, and the checks that every disagreement is one the FP32 arithmetic allows. numpy only."""
import numpy as np


def classify_vs_fp64(h, t64, i64, ext, tol=1e-6, o=None, d=None, verts=None):
    """Float closest hits h (t, u, v, tri bits) against the FP64 oracle's (t64, i64), distances compared in units of
    max(t, ext) (FP32 t error scales with the scene, not with t). Returns a dict of counts:
      same   - the same triangle;   tie - another triangle within tol;
      lost   - the oracle hits and the float path misses, or reports a hit farther than tol beyond the oracle's (with
               o, d, verts given: unless the FP32 test itself places the oracle's triangle no closer, a t-order tie);
      extra  - the float path reports a hit closer than tol before the oracle's, or where the oracle misses (a ray
               within the conservative edge bound of a silhouette);
    and the masks "lost_mask", "extra_mask" plus "max_t_error" over same-triangle hits."""
    ih = h[:, 3].view(np.int32)
    t = h[:, 0].astype(np.float64)
    both = (i64 >= 0) & (ih >= 0)
    scale = np.maximum(np.where(i64 >= 0, t64, t), ext)
    dt = (t - t64) / scale
    same = both & (ih == i64)
    tie = both & (ih != i64) & (np.abs(dt) <= tol)
    lost = ((i64 >= 0) & (ih < 0)) | (both & (ih != i64) & (dt > tol))
    if verts is not None and lost.any():
        # a farther hit is a tie when the FP32 test accepts the oracle's triangle at a distance no smaller than the one
        # reported (FP32 rounding of t reorders the two; the oracle's triangle is found, not lost)
        k = np.where(lost & (ih >= 0))[0]
        acc, t32 = wt32(o[k], d[k], verts, i64[k])
        order = acc & (t32 >= h[k, 0])
        lost[k[order]] = False; tie[k[order]] = True
    extra = ((i64 < 0) & (ih >= 0)) | (both & (ih != i64) & (dt < -tol))
    return {"same": int(same.sum()), "tie": int(tie.sum()), "lost": int(lost.sum()), "extra": int(extra.sum()),
            "lost_mask": lost, "extra_mask": extra, "max_t_error": float(np.abs(dt[same]).max()) if same.any() else 0.0}


def wt32(o, d, verts, tri):
    """The precision form's FP32 triangle test (conservative watertight edges) for given (ray, triangle) pairs, in
    numpy float32 with the kernel's operation order: (accepted, t)."""
    f = np.float32
    o3 = o[:, :3].astype(f); d3 = d[:, :3].astype(f); r = np.arange(len(o3))
    ad = np.abs(d3)
    kz = np.where(ad[:, 0] >= ad[:, 1], np.where(ad[:, 0] >= ad[:, 2], 0, 2), np.where(ad[:, 1] >= ad[:, 2], 1, 2))
    kx = np.where(kz == 2, 0, kz + 1); ky = np.where(kx == 2, 0, kx + 1)
    neg = d3[r, kz] < 0
    kx, ky = np.where(neg, ky, kx), np.where(neg, kx, ky)
    dz = d3[r, kz]; sx = d3[r, kx] / dz; sy = d3[r, ky] / dz; sz = f(1) / dz
    P = [verts[3 * tri + k, :3].astype(f) - o3 for k in range(3)]
    Z, X, Y, S = [], [], [], []
    for Q in P:
        qz, qkx, qky = Q[r, kz], Q[r, kx], Q[r, ky]
        px, py = sx * qz, sy * qz
        Z.append(qz); X.append(qkx - px); Y.append(qky - py); S.append((np.abs(qkx) + np.abs(px), np.abs(qky) + np.abs(py)))
    (Ax, Bx, Cx), (Ay, By, Cy), (Az, Bz, Cz) = X, Y, Z
    (SAx, SAy), (SBx, SBy), (SCx, SCy) = S
    U = Cx * By - Cy * Bx; V = Ax * Cy - Ay * Cx; W = Bx * Ay - By * Ax
    k, a = f(1e-6), f(1e-30)
    eU = k * (SCx * SBy + SCy * SBx) + a; eV = k * (SAx * SCy + SAy * SCx) + a; eW = k * (SBx * SAy + SBy * SAx) + a
    rej = ((U < -eU) | (V < -eV) | (W < -eW)) & ((U > eU) | (V > eV) | (W > eW))
    det = U + V + W
    with np.errstate(divide="ignore", invalid="ignore"):
        T = U * (sz * Az) + V * (sz * Bz) + W * (sz * Cz)
        t = T / det
    return ~rej & (det != 0), t


def edge_excess(o, d, verts, tri):
    """For rays (o, d float4) and leaf-order triangles tri (exact corners verts, 3 float4 each): how far outside the
    triangle the ray passes in FP64, in units of the precision form's FP32 edge bound 1e-6 (Sx Sy' + Sy Sx'); <= 1
    means the conservative FP32 edge test may accept it, 0 means inside."""
    o = o[:, :3].astype(np.float64); d32 = d[:, :3]; dd = d32.astype(np.float64)
    ad = np.abs(d32)
    kz = np.where(ad[:, 0] >= ad[:, 1], np.where(ad[:, 0] >= ad[:, 2], 0, 2), np.where(ad[:, 1] >= ad[:, 2], 1, 2))
    kx = np.where(kz == 2, 0, kz + 1); ky = np.where(kx == 2, 0, kx + 1)
    neg = d32[np.arange(len(d32)), kz] < 0
    kx, ky = np.where(neg, ky, kx), np.where(neg, kx, ky)
    r = np.arange(len(o))
    sx = dd[r, kx] / dd[r, kz]; sy = dd[r, ky] / dd[r, kz]
    P = [verts[3 * tri + k, :3].astype(np.float64) - o for k in range(3)]
    sh, S = [], []
    for Q in P:
        qz = Q[r, kz]
        sh.append((Q[r, kx] - sx * qz, Q[r, ky] - sy * qz))
        S.append((np.abs(Q[r, kx]) + np.abs(sx * qz), np.abs(Q[r, ky]) + np.abs(sy * qz)))
    (Ax, Ay), (Bx, By), (Cx, Cy) = sh
    (SAx, SAy), (SBx, SBy), (SCx, SCy) = S
    E = np.stack([Cx * By - Cy * Bx, Ax * Cy - Ay * Cx, Bx * Ay - By * Ax], 1)
    e = 1e-6 * np.stack([SCx * SBy + SCy * SBx, SAx * SCy + SAy * SCx, SBx * SAy + SBy * SAx], 1) + 1e-30
    sgn = np.where(E.sum(1) >= 0, 1.0, -1.0)[:, None]
    return np.maximum(0.0, (-sgn * E / e).max(1))
