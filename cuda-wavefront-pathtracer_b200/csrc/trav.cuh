// trav.cuh - closest-hit and any-hit ray traversal of the BVH2 (64 B), BVH4 (128 B) and CWBVH (80 B) encodings on
// CUDA cores, with Moller-Trumbore (TRI = 0) or Woop unit-triangle (TRI = 1) leaf tests.
//
// Traversal order, tie rules and leaf handling are those of the reference's device traversal (accel/traverse.cuh):
// strict tmin < t < hitT (the first triangle found at a given t wins), nearer-child-first BVH2 descent, BVH4 children
// sorted by entry distance, CWBVH children visited in ray-octant order with the node's hit leaves tested in slot order
// before descending. So for the same ray the same triangle is reported, except at exact ties that rounding may break
// differently. (The CWBVH node visit runs its eight slab tests before its leaf tests, where the reference interleaves
// them; leaf order and descent order are unchanged, so only boxes that a closer hit would have culled a little earlier
// are visited and rejected one level lower.)
//
// Implementation for sm_100a: nodes and triangles are read with 16-byte read-only loads (ld.global.nc.v4), every
// slab/plane evaluation is one explicit FMA, the short stack lives in registers/local memory, and each traversal
// carries a visit budget and a stack bound: a ray that exceeds either stops and raises bit kTravOverflow in *err
// instead of running out of bounds or forever.
#pragma once
#include "vecmath.h"

namespace cwpb {

enum : int { kTravOverflow = 1, kTravBudget = 2 };
static constexpr int kStack2 = 64;          // BVH2 / BVH4 stack entries (the host rejects deeper trees)
static constexpr int kStack8 = 40;          // CWBVH stack entries of (child base, masks)
static constexpr int kVisitBudget = 1 << 22;

__device__ __forceinline__ float4 ld4(const float4* p) { return __ldg(p); }

// reciprocal direction with the reference's safe epsilon (traverse.cuh:48-50)
__device__ __forceinline__ float safe_rcp(float x) { const float eps = 1e-20f; return 1.f / (fabsf(x) > eps ? x : copysignf(eps, x)); }

// ---------------- leaf tests ----------------
template <bool ANY, int TRI>
__device__ __forceinline__ bool leaf_hit(const float4* __restrict__ tv, int first, int cnt, float3 o, float3 d, float tmin,
                                         float& hitT, int& hitTri, float& hu, float& hv) {
    for (int t = first; t < first + cnt; t++) {
        if (TRI == 0) {   // Moller-Trumbore on (v0, e1, e2)
            float4 a = ld4(tv + 3 * t), b = ld4(tv + 3 * t + 1), c = ld4(tv + 3 * t + 2);
            float3 v0 = xyz(a), e1 = xyz(b), e2 = xyz(c);
            float3 pv = f3(fmaf(d.y, e2.z, -d.z * e2.y), fmaf(d.z, e2.x, -d.x * e2.z), fmaf(d.x, e2.y, -d.y * e2.x));
            float det = fdot(e1, pv);
            if (fabsf(det) < 1e-12f) continue;
            float inv = 1.f / det; float3 tq = o - v0; float u = fdot(tq, pv) * inv;
            if (u < 0.f || u > 1.f) continue;
            float3 qv = f3(fmaf(tq.y, e1.z, -tq.z * e1.y), fmaf(tq.z, e1.x, -tq.x * e1.z), fmaf(tq.x, e1.y, -tq.y * e1.x));
            float v = fdot(d, qv) * inv;
            if (v < 0.f || u + v > 1.f) continue;
            float tt = fdot(e2, qv) * inv;
            if (tt > tmin && tt < hitT) { hitT = tt; hitTri = t; hu = u; hv = v; if (ANY) return true; }
        } else {          // Woop: plane row 2 first (distance), rows 0 and 1 only when the distance is in range
            float4 r2 = ld4(tv + 3 * t + 2);
            float Oz = frow(r2, o), Dz = fdot(d, xyz(r2));
            float tt = -Oz / Dz;
            if (tt > tmin && tt < hitT) {
                float4 r0 = ld4(tv + 3 * t);
                float u = fmaf(tt, fdot(d, xyz(r0)), frow(r0, o));
                if (u >= 0.f && u <= 1.f) {
                    float4 r1 = ld4(tv + 3 * t + 1);
                    float v = fmaf(tt, fdot(d, xyz(r1)), frow(r1, o));
                    if (v >= 0.f && u + v <= 1.f) { hitT = tt; hitTri = t; hu = u; hv = v; if (ANY) return true; }
                }
            }
        }
    }
    return false;
}

// ---------------- resumable traversal state ----------------
// TravState<V, ANY, TRI>: one ray's traversal, advanced one node visit at a time. begin() sets the ray up; step()
// visits the current node (its slab tests and hit leaves) and picks the next node, returning true when the ray is
// done (traversal exhausted, an any-hit found, or a bound exceeded). Running step() to completion is the plain
// while-while traversal; persistent kernels interleave the steps of many rays (render.cu, trace.cu). The traversal
// stack is the caller's array (TravState<V>::Stack), kept out of the struct so that its scalars stay in registers.
template <int V, bool ANY, int TRI> struct TravState;

// ---------------- BVH2 ----------------
template <bool ANY, int TRI>
struct TravState<2, ANY, TRI> {
    typedef int Stack[kStack2];
    float3 o, d; float idx, idy, idz, ox, oy, oz, tmin, hitT, hu, hv; int hitTri, node, sp, budget;

    __device__ __forceinline__ void begin(float3 o_, float3 d_, float tmin_, float tmax_, int root) {
        o = o_; d = d_; tmin = tmin_; hitT = tmax_; hu = hv = 0.f; hitTri = -1; node = root; sp = 0; budget = kVisitBudget;
        idx = safe_rcp(d.x); idy = safe_rcp(d.y); idz = safe_rcp(d.z);
        ox = -o.x * idx; oy = -o.y * idy; oz = -o.z * idz;
    }
    __device__ __forceinline__ bool step(const float4* __restrict__ nodes, const float4* __restrict__ tv, Stack& stack, int& err) {
        if (--budget < 0) { err |= kTravBudget; return true; }
        const float4* nb = nodes + 4 * (size_t)node;
        const float4 n0 = ld4(nb), n1 = ld4(nb + 1), nz = ld4(nb + 2), mt = ld4(nb + 3);
        int c0 = __float_as_int(mt.x), c1 = __float_as_int(mt.y); const int k0 = __float_as_int(mt.z), k1 = __float_as_int(mt.w);
        const float a0 = fmaf(n0.x, idx, ox), a1 = fmaf(n0.y, idx, ox), a2 = fmaf(n0.z, idy, oy), a3 = fmaf(n0.w, idy, oy), a4 = fmaf(nz.x, idz, oz), a5 = fmaf(nz.y, idz, oz);
        const float b0 = fmaf(n1.x, idx, ox), b1 = fmaf(n1.y, idx, ox), b2 = fmaf(n1.z, idy, oy), b3 = fmaf(n1.w, idy, oy), b4 = fmaf(nz.z, idz, oz), b5 = fmaf(nz.w, idz, oz);
        const float t0n = fmaxf(fmaxf(fminf(a0, a1), fminf(a2, a3)), fmaxf(fminf(a4, a5), tmin));
        const float t0f = fminf(fminf(fmaxf(a0, a1), fmaxf(a2, a3)), fminf(fmaxf(a4, a5), hitT));
        const float t1n = fmaxf(fmaxf(fminf(b0, b1), fminf(b2, b3)), fmaxf(fminf(b4, b5), tmin));
        const float t1f = fminf(fminf(fmaxf(b0, b1), fmaxf(b2, b3)), fminf(fmaxf(b4, b5), hitT));
        bool h0 = t0n <= t0f, h1 = t1n <= t1f;
        if (h0 && k0 > 0) { if (leaf_hit<ANY, TRI>(tv, c0, k0, o, d, tmin, hitT, hitTri, hu, hv) && ANY) return true; h0 = false; }
        if (h1 && k1 > 0) { if (leaf_hit<ANY, TRI>(tv, c1, k1, o, d, tmin, hitT, hitTri, hu, hv) && ANY) return true; h1 = false; }
        if (!h0 && !h1) { if (sp == 0) return true; node = stack[--sp]; }
        else if (h0 && h1) {
            if (t1n < t0n) { const int t = c0; c0 = c1; c1 = t; }
            if (sp == kStack2) { err |= kTravOverflow; return true; }
            stack[sp++] = c1; node = c0;
        } else node = h0 ? c0 : c1;
        return false;
    }
};

template <bool ANY, int TRI>
__device__ __forceinline__ bool trav_bvh2(const float4* __restrict__ nodes, const float4* __restrict__ tv, float3 o, float3 d, float tmin,
                                          float& hitT, int& hitTri, float& hu, float& hv, int root, int& err) {
    TravState<2, ANY, TRI> r; typename TravState<2, ANY, TRI>::Stack stack; r.begin(o, d, tmin, hitT, root);
    while (!r.step(nodes, tv, stack, err)) {}
    hitT = r.hitT; hitTri = r.hitTri; hu = r.hu; hv = r.hv;
    return hitTri >= 0;
}

// ---------------- BVH4 ----------------
template <bool ANY, int TRI>
__device__ __forceinline__ bool trav_bvh4(const float4* __restrict__ nodes, const float4* __restrict__ tv, float3 o, float3 d, float tmin,
                                          float& hitT, int& hitTri, float& hu, float& hv, int root, int& err) {
    int stack[kStack2]; int sp = 0, node = root, budget = kVisitBudget;
    const float idx = safe_rcp(d.x), idy = safe_rcp(d.y), idz = safe_rcp(d.z);
    const float ox = -o.x * idx, oy = -o.y * idy, oz = -o.z * idz;
    const float INF = 3.4e38f;
    while (true) {
        if (--budget < 0) { err |= kTravBudget; break; }
        const float4* nb = nodes + 8 * (size_t)node;
        const float4 lx = ld4(nb), hx = ld4(nb + 1), ly = ld4(nb + 2), hy = ld4(nb + 3), lz = ld4(nb + 4), hz = ld4(nb + 5), cf = ld4(nb + 6), kf = ld4(nb + 7);
        float ht[4]; int hc[4];
        const float LX[4] = { lx.x, lx.y, lx.z, lx.w }, HX[4] = { hx.x, hx.y, hx.z, hx.w }, LY[4] = { ly.x, ly.y, ly.z, ly.w };
        const float HY[4] = { hy.x, hy.y, hy.z, hy.w }, LZ[4] = { lz.x, lz.y, lz.z, lz.w }, HZ[4] = { hz.x, hz.y, hz.z, hz.w };
        const int CC[4] = { __float_as_int(cf.x), __float_as_int(cf.y), __float_as_int(cf.z), __float_as_int(cf.w) };
        const int KK[4] = { __float_as_int(kf.x), __float_as_int(kf.y), __float_as_int(kf.z), __float_as_int(kf.w) };
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float x0 = fmaf(LX[j], idx, ox), x1 = fmaf(HX[j], idx, ox), y0 = fmaf(LY[j], idy, oy), y1 = fmaf(HY[j], idy, oy), z0 = fmaf(LZ[j], idz, oz), z1 = fmaf(HZ[j], idz, oz);
            float tn = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
            float tf = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), hitT));
            ht[j] = INF; hc[j] = CC[j];
            if (tn <= tf) {
                if (KK[j] > 0) { if (leaf_hit<ANY, TRI>(tv, CC[j], KK[j], o, d, tmin, hitT, hitTri, hu, hv) && ANY) return true; }
                else ht[j] = tn;
            }
        }
        // sorting network on entry distance (traverse.cuh:99)
#define CWPB_CSWAP(a, b) { if (ht[b] < ht[a]) { float tf_ = ht[a]; ht[a] = ht[b]; ht[b] = tf_; int ti_ = hc[a]; hc[a] = hc[b]; hc[b] = ti_; } }
        CWPB_CSWAP(0, 1) CWPB_CSWAP(2, 3) CWPB_CSWAP(0, 2) CWPB_CSWAP(1, 3) CWPB_CSWAP(1, 2)
#undef CWPB_CSWAP
        if (ht[0] == INF) { if (sp == 0) break; node = stack[--sp]; continue; }
        if (sp + 3 > kStack2) { err |= kTravOverflow; break; }
        if (ht[3] < INF) stack[sp++] = hc[3];
        if (ht[2] < INF) stack[sp++] = hc[2];
        if (ht[1] < INF) stack[sp++] = hc[1];
        node = hc[0];
    }
    return hitTri >= 0;
}

// ---------------- CWBVH ----------------
__device__ __forceinline__ unsigned byte_of(unsigned w, int s) { return (w >> (8 * (s & 3))) & 255u; }
// Byte s of w as an exact float without an int->float conversion (those run on the quarter-rate XU pipe): the byte
// permute builds the bit pattern 0x4B0000bb, which is the float 2^23 + b, and the subtraction is exact.
__device__ __forceinline__ float qbyte(unsigned w, int s) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u | (unsigned)(s & 3))) - 8388608.0f;
}

template <bool ANY, int TRI>
struct TravState<8, ANY, TRI> {
    typedef uint2 Stack[kStack8];
    float3 o, d; float idx, idy, idz, tmin, hitT, hu, hv; int hitTri, node, sp, budget; unsigned oct, cb, im, hm;

    __device__ __forceinline__ void begin(float3 o_, float3 d_, float tmin_, float tmax_, int root) {
        o = o_; d = d_; tmin = tmin_; hitT = tmax_; hu = hv = 0.f; hitTri = -1; node = root; sp = 0; budget = kVisitBudget;
        idx = safe_rcp(d.x); idy = safe_rcp(d.y); idz = safe_rcp(d.z);
        oct = (d.x > 0.f ? 1u : 0u) | (d.y > 0.f ? 2u : 0u) | (d.z > 0.f ? 4u : 0u);
        cb = im = hm = 0;
    }
    __device__ __forceinline__ bool step(const float4* __restrict__ nodes, const float4* __restrict__ tv, Stack& stack, int& err) {
        if (--budget < 0) { err |= kTravBudget; return true; }
        const float4* nb = nodes + 5 * (size_t)node;
        const float4 f0 = ld4(nb), f1 = ld4(nb + 1), f2 = ld4(nb + 2), f3_ = ld4(nb + 3), f4_ = ld4(nb + 4);
        const unsigned ew = __float_as_uint(f0.w);
        const float sx = __uint_as_float((ew & 255u) << 23) * idx, sy = __uint_as_float(((ew >> 8) & 255u) << 23) * idy, sz = __uint_as_float(((ew >> 16) & 255u) << 23) * idz;
        const float ox = (f0.x - o.x) * idx, oy = (f0.y - o.y) * idy, oz = (f0.z - o.z) * idz;
        const unsigned imask = ew >> 24, m0 = __float_as_uint(f1.z), m1 = __float_as_uint(f1.w);
        const int childBase = __float_as_int(f1.x), triBase = __float_as_int(f1.y);
        // per axis, the plane a ray enters first: the low bound when the reciprocal is positive, else the high bound.
        // Selecting it replaces the min/max of each (low, high) pair and gives the same values: the fused affine map
        // q * s + o is monotonic in q for either sign of s.
        const bool fx = idx < 0.f, fy = idy < 0.f, fz = idz < 0.f;
        // quantised bounds: lo x (f2.x, f2.y), lo y (f2.z, f2.w), lo z (f3.x, f3.y), hi x (f3.z, f3.w), hi y (f4.x, f4.y), hi z (f4.z, f4.w)
        const unsigned nx0 = __float_as_uint(fx ? f3_.z : f2.x), nx1 = __float_as_uint(fx ? f3_.w : f2.y), px0 = __float_as_uint(fx ? f2.x : f3_.z), px1 = __float_as_uint(fx ? f2.y : f3_.w);
        const unsigned ny0 = __float_as_uint(fy ? f4_.x : f2.z), ny1 = __float_as_uint(fy ? f4_.y : f2.w), py0 = __float_as_uint(fy ? f2.z : f4_.x), py1 = __float_as_uint(fy ? f2.w : f4_.y);
        const unsigned nz0 = __float_as_uint(fz ? f4_.z : f3_.x), nz1 = __float_as_uint(fz ? f4_.w : f3_.y), pz0 = __float_as_uint(fz ? f3_.x : f4_.z), pz1 = __float_as_uint(fz ? f3_.y : f4_.w);
        // all eight slab tests first (predicated, no branches), then the hit leaves in slot order
        unsigned boxHit = 0;
#pragma unroll
        for (int s = 0; s < 8; s++) {
            const float xn = fmaf(qbyte(s < 4 ? nx0 : nx1, s), sx, ox), xf = fmaf(qbyte(s < 4 ? px0 : px1, s), sx, ox);
            const float yn = fmaf(qbyte(s < 4 ? ny0 : ny1, s), sy, oy), yf = fmaf(qbyte(s < 4 ? py0 : py1, s), sy, oy);
            const float zn = fmaf(qbyte(s < 4 ? nz0 : nz1, s), sz, oz), zf = fmaf(qbyte(s < 4 ? pz0 : pz1, s), sz, oz);
            // entry = max(xn, yn, zn, tmin), exit = min(xf, yf, zf, hitT) selected with 3-input integer min/max on the
            // float bits: for values >= +0 the integer order is the float order, entry >= tmin >= +0, and any negative
            // candidate for the exit makes the float comparison below fail whichever negative value is picked - so
            // the hit decision is the one the float min/max gives.
            const float tn = __int_as_float(__vimax3_s32(__float_as_int(xn), __float_as_int(yn), max(__float_as_int(zn), __float_as_int(tmin))));
            const float tf = __int_as_float(__vimin3_s32(__float_as_int(xf), __float_as_int(yf), min(__float_as_int(zf), __float_as_int(hitT))));
            boxHit |= (tn <= tf ? 1u : 0u) << s;
        }
        // leaf slots: meta bit 7 of each byte
        const unsigned leafMask = ((m0 >> 7) & 1u) | ((m0 >> 14) & 2u) | ((m0 >> 21) & 4u) | ((m0 >> 28) & 8u) |
                                  ((m1 >> 3) & 16u) | ((m1 >> 10) & 32u) | ((m1 >> 17) & 64u) | ((m1 >> 24) & 128u);
        unsigned leafHit = boxHit & leafMask;
        // internal children hit, re-indexed to octant order (slot s -> bit s ^ oct)
        unsigned hits = boxHit & imask;
        if (oct & 1u) hits = ((hits & 0x55u) << 1) | ((hits & 0xAAu) >> 1);
        if (oct & 2u) hits = ((hits & 0x33u) << 2) | ((hits & 0xCCu) >> 2);
        if (oct & 4u) hits = ((hits & 0x0Fu) << 4) | ((hits & 0xF0u) >> 4);
        while (leafHit) {
            const int s = __ffs(leafHit) - 1; leafHit &= leafHit - 1;
            const unsigned m = byte_of(s < 4 ? m0 : m1, s);
            if (leaf_hit<ANY, TRI>(tv, triBase + (int)(m & 31u), (int)((m >> 5) & 3u) + 1, o, d, tmin, hitT, hitTri, hu, hv) && ANY) return true;
        }
        if (hits) {
            if (hm) { if (sp == kStack8) { err |= kTravOverflow; return true; } stack[sp++] = make_uint2(cb, (im << 8) | hm); }
            cb = (unsigned)childBase; im = imask; hm = hits;
        }
        while (hm == 0) { if (sp == 0) return true; const uint2 e = stack[--sp]; cb = e.x; im = e.y >> 8; hm = e.y & 255u; }
        const unsigned k = __ffs(hm) - 1; hm &= hm - 1; const unsigned slot = k ^ oct;
        node = (int)cb + __popc(im & ((1u << slot) - 1u));
        return false;
    }
};

template <bool ANY, int TRI>
__device__ __forceinline__ bool trav_cwbvh(const float4* __restrict__ nodes, const float4* __restrict__ tv, float3 o, float3 d, float tmin,
                                           float& hitT, int& hitTri, float& hu, float& hv, int root, int& err) {
    TravState<8, ANY, TRI> r; typename TravState<8, ANY, TRI>::Stack stack; r.begin(o, d, tmin, hitT, root);
    while (!r.step(nodes, tv, stack, err)) {}
    hitT = r.hitT; hitTri = r.hitTri; hu = r.hu; hv = r.hv;
    return hitTri >= 0;
}

template <int V, bool ANY, int TRI>
__device__ __forceinline__ bool trace_ray(const float4* __restrict__ nodes, const float4* __restrict__ tv, float3 o, float3 d, float tmin,
                                          float& hitT, int& hitTri, float& hu, float& hv, int root, int& err) {
    if (V == 2) return trav_bvh2<ANY, TRI>(nodes, tv, o, d, tmin, hitT, hitTri, hu, hv, root, err);
    if (V == 4) return trav_bvh4<ANY, TRI>(nodes, tv, o, d, tmin, hitT, hitTri, hu, hv, root, err);
    return trav_cwbvh<ANY, TRI>(nodes, tv, o, d, tmin, hitT, hitTri, hu, hv, root, err);
}

}  // namespace cwpb
