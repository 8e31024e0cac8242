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


def edge_margin(o, d, verts, tri):
    """For rays (o, d float4) and leaf-order triangles tri (exact corners verts, 3 float4 each): the signed distance
    of the ray from the triangle's edges in FP64, in units of the precision form's FP32 edge bound
    1e-6 (Sx Sy' + Sy Sx'): the largest of the three edge functions taken outward, so > 0 outside (by that much),
    <= 0 inside (|value| = the margin to the nearest edge)."""
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
    return (-sgn * E / e).max(1)


def edge_excess(o, d, verts, tri):
    """How far outside the triangle the ray passes in FP64, in the units of edge_margin; <= 1 means the conservative
    FP32 edge test may accept it, 0 means inside."""
    return np.maximum(0.0, edge_margin(o, d, verts, tri))


def fp64_hit(o, d, verts, tri):
    """FP64 test of given (ray, leaf-order triangle) pairs on the exact corners: (t of the triangle's plane, signed
    edge margin as edge_margin), nan / inf where tri < 0."""
    t = np.full(len(o), np.nan)
    m = np.full(len(o), np.inf)
    k = np.where(tri >= 0)[0]
    if not len(k):
        return t, m
    oo = o[k, :3].astype(np.float64); dd = d[k, :3].astype(np.float64); tt = tri[k]
    v = [verts[3 * tt + j, :3].astype(np.float64) for j in range(3)]
    n = np.cross(v[1] - v[0], v[2] - v[0])
    den = (n * dd).sum(1)
    with np.errstate(divide="ignore", invalid="ignore"):
        t[k] = np.where(den != 0, ((v[0] - oo) * n).sum(1) / den, np.nan)
    m[k] = edge_margin(o[k], d[k], verts, tt)
    return t, m


def explain_differences(o, d, verts, ours, other, any_hit=False, rel=1e-6, graze=16.0, ids=None):
    """Rays on which this library and another traversal of the same tree disagree, classified in FP64 on the exact
    corners. Closest hit: ours / other are float4 (t, u, v, leaf-order triangle bits) and a ray disagrees when the
    triangles differ; any hit: int32 triangle or -1, and a ray disagrees when one side finds an occluder and the
    other does not. Classes:
      tie         (closest) both hits within rel * t of each other;
      ours_exact  ours is the exact answer of the two: our triangle is hit in exact arithmetic (margin <= 0) and the
                  other reports none, a farther one, or one that exact arithmetic misses (margin > 0);
      graze       a triangle that one side reports and the other does not lies within `graze` edge-bound units of one
                  of its edges, inside or out (FP32 rounding decides such rays);
      unexplained anything else.
    ids (optional): the original mesh triangle of every leaf-order reference (tris[3k].w); with spatial splits one
    triangle has several references, and two references to the same triangle are the same hit ("same_triangle",
    counted, not classified).
    Returns (counts, rows), one row per disagreeing ray."""
    if any_hit:
        ia, ib = np.asarray(ours, np.int32), np.asarray(other, np.int32)
        diff = np.where((ia >= 0) != (ib >= 0))[0]
    else:
        ia, ib = ours[:, 3].view(np.int32), other[:, 3].view(np.int32)
        diff = np.where(ia != ib)[0]
    counts = {"rays": int(len(o)), "differ": 0, "same_triangle": 0, "tie": 0, "ours_exact": 0, "graze": 0, "unexplained": 0}
    if ids is not None and not any_hit and len(diff):
        ids = np.asarray(ids, np.int32)
        dup = (ia[diff] >= 0) & (ib[diff] >= 0) & (ids[np.maximum(ia[diff], 0)] == ids[np.maximum(ib[diff], 0)])
        counts["same_triangle"] = int(dup.sum())
        diff = diff[~dup]
    counts["differ"] = int(len(diff))
    rows = []
    if not len(diff):
        return counts, rows
    oo, dd = o[diff], d[diff]
    ta, ma = fp64_hit(oo, dd, verts, ia[diff])
    tb, mb = fp64_hit(oo, dd, verts, ib[diff])
    for j, i in enumerate(diff):
        a, b = int(ia[i]), int(ib[i])
        if not any_hit and a >= 0 and b >= 0 and abs(ours[i, 0] - other[i, 0]) <= rel * max(abs(ours[i, 0]), abs(other[i, 0])):
            c = "tie"
        elif a >= 0 and ma[j] <= 0 and (b < 0 or mb[j] > 0 or ta[j] < tb[j]):
            c = "ours_exact"
        elif any_hit and a < 0 and mb[j] > graze:
            c = "ours_exact"   # the other's occluder is missed by exact arithmetic
        elif (a >= 0 and abs(ma[j]) <= graze) or (b >= 0 and abs(mb[j]) <= graze):
            c = "graze"
        else:
            c = "unexplained"
        counts[c] += 1
        rows.append({"ray": int(i), "ours": a, "other": b, "t64_ours": float(ta[j]), "t64_other": float(tb[j]),
                     "margin_ours": float(ma[j]), "margin_other": float(mb[j]), "class": c,
                     **({} if any_hit else {"t_ours": float(ours[i, 0]), "t_other": float(other[i, 0]), "uv_ours": [float(ours[i, 1]), float(ours[i, 2])],
                                            "uv_other": [float(other[i, 1]), float(other[i, 2])]})})
    return counts, rows
