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
#include <cuda_fp16.h>

namespace cwpb {

enum : int { kTravOverflow = 1, kTravBudget = 2 };
static constexpr int kStack2 = 64;          // BVH2 / BVH4 stack entries (the host rejects deeper trees)
static constexpr int kStack8 = 40;          // CWBVH stack entries of (child base, masks)
static constexpr int kVisitBudget = 1 << 22;

__device__ __forceinline__ float4 ld4(const float4* p) { return __ldg(p); }

// Where a traversal reads its nodes. A plain node pointer reads global memory through the read-only path;
// StagedNodes reads the first k nodes from a block's copy in shared memory and the rest from global memory. With a
// breadth-first node numbering the first k nodes are the tree's top levels, which every ray visits.
struct StagedNodes { const float4* __restrict__ g; const float4* s; int k; };
template <int W>
__device__ __forceinline__ void fetch_node(const float4* __restrict__ g, int node, float4 (&f)[W]) {
    const float4* p = g + (size_t)W * node;
#pragma unroll
    for (int i = 0; i < W; i++) f[i] = __ldg(p + i);
}
template <int W>
__device__ __forceinline__ void fetch_node(const StagedNodes& n, int node, float4 (&f)[W]) {
    if (node < n.k) {
        const float4* p = n.s + W * node;
#pragma unroll
        for (int i = 0; i < W; i++) f[i] = p[i];
    } else fetch_node<W>(n.g, node, f);
}

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
        } else {          // Woop: distance from row 2, then u and v from rows 0 and 1
            // all three rows are loaded at once: one memory latency per triangle instead of up to three dependent
            // ones (the traversal is bound by load latency, not by L1 bytes; measured 4% faster on frames)
            const float4 r2 = ld4(tv + 3 * t + 2), r0 = ld4(tv + 3 * t), r1 = ld4(tv + 3 * t + 1);
            float Oz = frow(r2, o), Dz = fdot(d, xyz(r2));
            float tt = -Oz / Dz;
            if (tt > tmin && tt < hitT) {
                float u = fmaf(tt, fdot(d, xyz(r0)), frow(r0, o));
                if (u >= 0.f && u <= 1.f) {
                    float v = fmaf(tt, fdot(d, xyz(r1)), frow(r1, o));
                    if (v >= 0.f && u + v <= 1.f) { hitT = tt; hitTri = t; hu = u; hv = v; if (ANY) return true; }
                }
            }
        }
    }
    return false;
}

// one triangle of the leaf-order arrays (the body of leaf_hit for one t)
template <bool ANY, int TRI>
__device__ __forceinline__ bool tri_hit(const float4* __restrict__ tv, int t, float3 o, float3 d, float tmin, float& hitT, int& hitTri, float& hu, float& hv) {
    return leaf_hit<ANY, TRI>(tv, t, 1, o, d, tmin, hitT, hitTri, hu, hv);
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
    template <class S>
    __device__ __forceinline__ bool step(const float4* __restrict__ nodes, const float4* __restrict__ tv, S& stack, int& err) {
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
struct TravState<4, ANY, TRI> {
    typedef int Stack[kStack2];
    float3 o, d; float idx, idy, idz, ox, oy, oz, tmin, hitT, hu, hv; int hitTri, node, sp, budget;

    __device__ __forceinline__ void begin(float3 o_, float3 d_, float tmin_, float tmax_, int root) {
        o = o_; d = d_; tmin = tmin_; hitT = tmax_; hu = hv = 0.f; hitTri = -1; node = root; sp = 0; budget = kVisitBudget;
        idx = safe_rcp(d.x); idy = safe_rcp(d.y); idz = safe_rcp(d.z);
        ox = -o.x * idx; oy = -o.y * idy; oz = -o.z * idz;
    }
    // one node: four slab tests, hit leaves tested in child order, hit inner children sorted by entry distance
    // (traverse.cuh:74-107), the nearest visited next and the others pushed
    template <class S>
    __device__ __forceinline__ bool step(const float4* __restrict__ nodes, const float4* __restrict__ tv, S& stack, int& err) {
        const float INF = 3.4e38f;
        if (--budget < 0) { err |= kTravBudget; return true; }
        const float4* nb = nodes + 8 * (size_t)node;
        const float4 lx = ld4(nb), hx = ld4(nb + 1), ly = ld4(nb + 2), hy = ld4(nb + 3), lz = ld4(nb + 4), hz = ld4(nb + 5), cf = ld4(nb + 6), kf = ld4(nb + 7);
        float ht[4]; int hc[4];
        const float LX[4] = { lx.x, lx.y, lx.z, lx.w }, HX[4] = { hx.x, hx.y, hx.z, hx.w }, LY[4] = { ly.x, ly.y, ly.z, ly.w };
        const float HY[4] = { hy.x, hy.y, hy.z, hy.w }, LZ[4] = { lz.x, lz.y, lz.z, lz.w }, HZ[4] = { hz.x, hz.y, hz.z, hz.w };
        const int CC[4] = { __float_as_int(cf.x), __float_as_int(cf.y), __float_as_int(cf.z), __float_as_int(cf.w) };
        const int KK[4] = { __float_as_int(kf.x), __float_as_int(kf.y), __float_as_int(kf.z), __float_as_int(kf.w) };
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float x0 = fmaf(LX[j], idx, ox), x1 = fmaf(HX[j], idx, ox), y0 = fmaf(LY[j], idy, oy), y1 = fmaf(HY[j], idy, oy), z0 = fmaf(LZ[j], idz, oz), z1 = fmaf(HZ[j], idz, oz);
            const float tn = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
            const float tf = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), hitT));
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
        if (ht[0] == INF) { if (sp == 0) return true; node = stack[--sp]; return false; }
        if (sp + 3 > kStack2) { err |= kTravOverflow; return true; }
        if (ht[3] < INF) stack[sp++] = hc[3];
        if (ht[2] < INF) stack[sp++] = hc[2];
        if (ht[1] < INF) stack[sp++] = hc[1];
        node = hc[0];
        return false;
    }
};

template <bool ANY, int TRI>
__device__ __forceinline__ bool trav_bvh4(const float4* __restrict__ nodes, const float4* __restrict__ tv, float3 o, float3 d, float tmin,
                                          float& hitT, int& hitTri, float& hu, float& hv, int root, int& err) {
    TravState<4, ANY, TRI> r; typename TravState<4, ANY, TRI>::Stack stack; r.begin(o, d, tmin, hitT, root);
    while (!r.step(nodes, tv, stack, err)) {}
    hitT = r.hitT; hitTri = r.hitTri; hu = r.hu; hv = r.hv;
    return hitTri >= 0;
}

// traversal stack kept in shared memory: entry i of this thread at base[i * stride] (stride = threads per block, so
// a warp's accesses to one entry hit consecutive words)
template <class T>
struct SharedStack {
    T* base; int stride;
    __device__ __forceinline__ T& operator[](int i) const { return base[(size_t)i * stride]; }
};


// ---------------- CWBVH ----------------
__device__ __forceinline__ __half2 h2_of_bits(unsigned u) { __half2 h; memcpy(&h, &u, 4); return h; }
__device__ __forceinline__ unsigned bits_of_h2(__half2 h) { unsigned u; memcpy(&u, &h, 4); return u; }
// CWBVH slots whose meta byte marks a leaf (bit 7 of each of the eight bytes in m0, m1), as an 8-bit mask: the four
// flag bits of a word, isolated at bits 0, 8, 16, 24, are gathered onto bits 28..31 by one multiply (no carries)
__device__ __forceinline__ unsigned leaf_slots(unsigned m0, unsigned m1) {
    return ((((m0 >> 7) & 0x01010101u) * 0x10204080u) >> 28) | (((((m1 >> 7) & 0x01010101u) * 0x10204080u) >> 24) & 0xF0u);
}
__device__ __forceinline__ unsigned byte_of(unsigned w, int s) { return (w >> (8 * (s & 3))) & 255u; }
// Byte s of w as an exact float without an int->float conversion (those run on the quarter-rate XU pipe): the byte
// permute builds the bit pattern 0x4B0000bb, which is the float 2^23 + b, and the subtraction is exact.
__device__ __forceinline__ float qbyte(unsigned w, int s) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u | (unsigned)(s & 3))) - 8388608.0f;
}

// FOCT >= 0: every ray of the launch has direction octant FOCT and no zero direction component (the caller checks
// per ray), so the near/far plane choice and the octant order are compile-time constants; -1: taken per ray
template <bool ANY, int TRI, int FOCT>
struct CwbvhTrav {
    typedef uint2 Stack[kStack8];
    float3 o, d; float idx, idy, idz, tmin, hitT, hu, hv; int hitTri, node, sp, budget; unsigned oct, cb, im, hm;

    __device__ __forceinline__ void begin(float3 o_, float3 d_, float tmin_, float tmax_, int root) {
        o = o_; d = d_; tmin = tmin_; hitT = tmax_; hu = hv = 0.f; hitTri = -1; node = root; sp = 0; budget = kVisitBudget;
        idx = safe_rcp(d.x); idy = safe_rcp(d.y); idz = safe_rcp(d.z);
        oct = (d.x > 0.f ? 1u : 0u) | (d.y > 0.f ? 2u : 0u) | (d.z > 0.f ? 4u : 0u);
        cb = im = hm = 0;
    }
    template <class N, class S>
    __device__ __forceinline__ bool step(const N& nodes, const float4* __restrict__ tv, S& stack, int& err) {
        if (--budget < 0) { err |= kTravBudget; return true; }
        float4 nf[5]; fetch_node<5>(nodes, node, nf);
        const float4 f0 = nf[0], f1 = nf[1], f2 = nf[2], f3_ = nf[3], f4_ = nf[4];
        const unsigned ew = __float_as_uint(f0.w);
        // 2^e / d per axis as the reference computes it, times 2^24 (exact whatever its range; the upload check on the
        // exponent bytes, at most 164, keeps it finite for |1/d| up to the 1e20 of the safe reciprocal)
        const float sx24 = (__uint_as_float((ew & 255u) << 23) * idx) * 16777216.f, sy24 = (__uint_as_float(((ew >> 8) & 255u) << 23) * idy) * 16777216.f,
                    sz24 = (__uint_as_float(((ew >> 16) & 255u) << 23) * idz) * 16777216.f;
        const float ox = (f0.x - o.x) * idx, oy = (f0.y - o.y) * idy, oz = (f0.z - o.z) * idz;
        const unsigned imask = ew >> 24, m0 = __float_as_uint(f1.z), m1 = __float_as_uint(f1.w);
        const int childBase = __float_as_int(f1.x), triBase = __float_as_int(f1.y);
        // per axis, the plane a ray enters first: the low bound when the reciprocal is positive, else the high bound.
        // Selecting it replaces the min/max of each (low, high) pair and gives the same values: the fused affine map
        // q * s + o is monotonic in q for either sign of s.
        const bool fx = FOCT >= 0 ? !(FOCT & 1) : idx < 0.f, fy = FOCT >= 0 ? !(FOCT & 2) : idy < 0.f, fz = FOCT >= 0 ? !(FOCT & 4) : idz < 0.f;
        const unsigned oc = FOCT >= 0 ? (unsigned)FOCT : oct;
        // quantised bounds: lo x (f2.x, f2.y), lo y (f2.z, f2.w), lo z (f3.x, f3.y), hi x (f3.z, f3.w), hi y (f4.x, f4.y), hi z (f4.z, f4.w)
        const unsigned nx0 = __float_as_uint(fx ? f3_.z : f2.x), nx1 = __float_as_uint(fx ? f3_.w : f2.y), px0 = __float_as_uint(fx ? f2.x : f3_.z), px1 = __float_as_uint(fx ? f2.y : f3_.w);
        const unsigned ny0 = __float_as_uint(fy ? f4_.x : f2.z), ny1 = __float_as_uint(fy ? f4_.y : f2.w), py0 = __float_as_uint(fy ? f2.z : f4_.x), py1 = __float_as_uint(fy ? f2.w : f4_.y);
        const unsigned nz0 = __float_as_uint(fz ? f4_.z : f3_.x), nz1 = __float_as_uint(fz ? f4_.w : f3_.y), pz0 = __float_as_uint(fz ? f3_.x : f4_.z), pz1 = __float_as_uint(fz ? f3_.y : f4_.w);
        // all eight slab tests first (predicated, no branches), then the hit leaves in slot order
        unsigned boxHit = 0;
        // The quantised planes q (bytes) enter the fused affine map as the f16 subnormals q 2^-24: one byte permute
        // places two bytes as two halves, and the f16 -> f32 conversions are exact; the per-axis scales carry the
        // factor 2^24 in their exponents (sx24 = 2^(e + 24) / d, exact), so fmaf(q 2^-24, sx24, ox) is bit for bit
        // fmaf(q, 2^e / d, ox) - the slab distances of the reference's decode - at one permute per two planes
        // instead of a permute and a subtraction per plane.
        float2 pbx, pby, pbz, pcx, pcy, pcz;
#pragma unroll
        for (int s = 0; s < 8; s++) {
            float2 bx, by, bz, cx, cy, cz;
            if ((s & 1) == 0) {
                const unsigned sel = (s & 2) ? 0x4342u : 0x4140u;
                bx = __half22float2(h2_of_bits(__byte_perm(s < 4 ? nx0 : nx1, 0u, sel))); cx = __half22float2(h2_of_bits(__byte_perm(s < 4 ? px0 : px1, 0u, sel)));
                by = __half22float2(h2_of_bits(__byte_perm(s < 4 ? ny0 : ny1, 0u, sel))); cy = __half22float2(h2_of_bits(__byte_perm(s < 4 ? py0 : py1, 0u, sel)));
                bz = __half22float2(h2_of_bits(__byte_perm(s < 4 ? nz0 : nz1, 0u, sel))); cz = __half22float2(h2_of_bits(__byte_perm(s < 4 ? pz0 : pz1, 0u, sel)));
                pbx = bx; pby = by; pbz = bz; pcx = cx; pcy = cy; pcz = cz;
            }
            const bool hi = s & 1;
            const float xn = fmaf(hi ? pbx.y : pbx.x, sx24, ox), xf = fmaf(hi ? pcx.y : pcx.x, sx24, ox);
            const float yn = fmaf(hi ? pby.y : pby.x, sy24, oy), yf = fmaf(hi ? pcy.y : pcy.x, sy24, oy);
            const float zn = fmaf(hi ? pbz.y : pbz.x, sz24, oz), zf = fmaf(hi ? pcz.y : pcz.x, sz24, oz);
            // entry = max(xn, yn, zn, tmin), exit = min(xf, yf, zf, hitT) selected with 3-input integer min/max on the
            // float bits: for values >= +0 the integer order is the float order, entry >= tmin >= +0, and any negative
            // candidate for the exit makes the float comparison below fail whichever negative value is picked - so
            // the hit decision is the one the float min/max gives.
            const float tn = __int_as_float(__vimax3_s32(__float_as_int(xn), __float_as_int(yn), max(__float_as_int(zn), __float_as_int(tmin))));
            const float tf = __int_as_float(__vimin3_s32(__float_as_int(xf), __float_as_int(yf), min(__float_as_int(zf), __float_as_int(hitT))));
            boxHit |= (tn <= tf ? 1u : 0u) << s;
        }
        unsigned leafHit = boxHit & leaf_slots(m0, m1);
        // internal children hit, re-indexed to octant order (slot s -> bit s ^ oct)
        unsigned hits = boxHit & imask;
        if (oc & 1u) hits = ((hits & 0x55u) << 1) | ((hits & 0xAAu) >> 1);
        if (oc & 2u) hits = ((hits & 0x33u) << 2) | ((hits & 0xCCu) >> 2);
        if (oc & 4u) hits = ((hits & 0x0Fu) << 4) | ((hits & 0xF0u) >> 4);
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
        const unsigned k = __ffs(hm) - 1; hm &= hm - 1; const unsigned slot = k ^ oc;
        node = (int)cb + __popc(im & ((1u << slot) - 1u));
        return false;
    }
};

template <bool ANY, int TRI> struct TravState<8, ANY, TRI> : CwbvhTrav<ANY, TRI, -1> {};

// direction octant of d (bit i set: component i positive), or -1 when a component is zero (its sign then decides the
// plane choice, not the octant bit)
__device__ __forceinline__ int octant_of(float3 d) {
    return d.x != 0.f && d.y != 0.f && d.z != 0.f ? (d.x > 0.f ? 1 : 0) | (d.y > 0.f ? 2 : 0) | (d.z > 0.f ? 4 : 0) : -1;
}

template <bool ANY, int TRI, int FOCT = -1, class N>
__device__ __forceinline__ bool trav_cwbvh(const N& nodes, const float4* __restrict__ tv, float3 o, float3 d, float tmin,
                                           float& hitT, int& hitTri, float& hu, float& hv, int root, int& err) {
    CwbvhTrav<ANY, TRI, FOCT> r; typename CwbvhTrav<ANY, TRI, FOCT>::Stack stack; r.begin(o, d, tmin, hitT, root);
    while (!r.step(nodes, tv, stack, err)) {}
    hitT = r.hitT; hitTri = r.hitTri; hu = r.hu; hv = r.hv;
    return hitTri >= 0;
}


// ---------------- precision form: FP16 conservative slabs + watertight FP32 triangles ----------------
// Box test: the CWBVH's 8-bit child planes q (0..255) sit at t = A + q B per axis, A = (node origin - ray origin) / d,
// B = 2^e / d. The test runs in f16x2, two children per instruction: a byte permute builds the halves 1024 + q, so
// t = A' + (1024 + q) B with A' = A - 1024 B. The per-node bases are rounded outward in f32 -> f16 (down for the planes
// a ray enters, up for those it leaves) after widening by m = (1.001 |A| + 1792 |B|) / 2048 + 1e-4. That bounds the
// rounding of B to f16 (<= 2^-11 |B| per unit of 1024 + q <= 1279: 0.625 |B|) plus the rounding of the f16 fused
// multiply-add to nearest (<= 2^-11 of a result within 0.625 |B| + m of A + q B, q <= 255: 2^-11 |A| + 0.125 |B| and a
// little), with 1e-4 for f16 subnormal spacing: the rounded near plane lies below, the far plane above, the exact ones.
// So every box the ray meets in exact arithmetic passes. (An earlier margin of (|A| + 2048 |B|) / 512 bounded the
// result by |A| + 2303 |B| and widened every box by four quantisation steps: 21% more node visits and 49% more
// triangle tests than the FP32 slabs on incoherent rays, against 7% and 27% now.)
// A node with an axis whose plane distances could leave the f16 range (a direction component near zero makes B large)
// runs its eight slab tests in FP32 instead, widened by 2^-20 (|A| + 256 |B|), which bounds the FP32 rounding of A, B
// and the fused decode (about 6 ulps); an axis with non-finite A or B is left unconstrained there.
// Triangle test: watertight ray/triangle intersection (Woop, Benthin & Wald, JCGT 2013): shear to the ray's dominant
// axis, edge functions from the exact shared corner positions (no fused operations, so a shared edge gives the same
// value with opposite sign in both triangles). An edge function counts as negative or positive only beyond its FP32
// rounding bound e = 1e-6 (Sx Sy' + Sy Sx') (Sx = |P_kx| + |sx P_kz| bounds a sheared coordinate, 1e-6 is about 17
// ulps against the 10 that the shear, the products and the difference can accumulate), so a ray that exact (or FP64)
// arithmetic puts inside a triangle is never rejected: no hit inside [tmin, tmax] can be lost. Rays within the bound
// of an edge may report the neighbouring triangle or a silhouette hit that exact arithmetic just misses.
struct WtRay { int kx, ky, kz; float sx, sy, sz; };
__device__ __forceinline__ float comp3(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
static constexpr float kEdgeRel = 1e-6f, kEdgeAbs = 1e-30f;

__device__ __forceinline__ WtRay wt_setup(float3 d) {
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    WtRay r; r.kz = ax >= ay ? (ax >= az ? 0 : 2) : (ay >= az ? 1 : 2);
    r.kx = r.kz == 2 ? 0 : r.kz + 1; r.ky = r.kx == 2 ? 0 : r.kx + 1;
    if (comp3(d, r.kz) < 0.f) { const int t = r.kx; r.kx = r.ky; r.ky = t; }   // keep the winding
    const float dz = comp3(d, r.kz);
    r.sx = comp3(d, r.kx) / dz; r.sy = comp3(d, r.ky) / dz; r.sz = 1.f / dz;
    return r;
}

// one watertight test of triangle t against the interval (tmin, tmax); true when it hits there, with its distance and
// barycentrics in tt, u, v
__device__ __forceinline__ bool wt_test(const float4* __restrict__ vt, int t, float3 o, const WtRay& r, float tmin, float tmax,
                                        float& tt, float& u, float& v) {
    {
        const float3 A = xyz(ld4(vt + 3 * t)) - o, B = xyz(ld4(vt + 3 * t + 1)) - o, C = xyz(ld4(vt + 3 * t + 2)) - o;
        const float Az = comp3(A, r.kz), Bz = comp3(B, r.kz), Cz = comp3(C, r.kz);
        const float Akx = comp3(A, r.kx), Aky = comp3(A, r.ky), Bkx = comp3(B, r.kx), Bky = comp3(B, r.ky), Ckx = comp3(C, r.kx), Cky = comp3(C, r.ky);
        const float pAx = r.sx * Az, pAy = r.sy * Az, pBx = r.sx * Bz, pBy = r.sy * Bz, pCx = r.sx * Cz, pCy = r.sy * Cz;
        const float Ax = Akx - pAx, Ay = Aky - pAy, Bx = Bkx - pBx, By = Bky - pBy, Cx = Ckx - pCx, Cy = Cky - pCy;
        const float U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
        const float SAx = fabsf(Akx) + fabsf(pAx), SAy = fabsf(Aky) + fabsf(pAy), SBx = fabsf(Bkx) + fabsf(pBx), SBy = fabsf(Bky) + fabsf(pBy);
        const float SCx = fabsf(Ckx) + fabsf(pCx), SCy = fabsf(Cky) + fabsf(pCy);
        const float eU = kEdgeRel * (SCx * SBy + SCy * SBx) + kEdgeAbs, eV = kEdgeRel * (SAx * SCy + SAy * SCx) + kEdgeAbs;
        const float eW = kEdgeRel * (SBx * SAy + SBy * SAx) + kEdgeAbs;
        if ((U < -eU || V < -eV || W < -eW) && (U > eU || V > eV || W > eW)) return false;
        const float det = U + V + W;
        if (det == 0.f) return false;
        const float T = U * (r.sz * Az) + V * (r.sz * Bz) + W * (r.sz * Cz);
        tt = T / det;
        if (!(tt > tmin && tt < tmax)) return false;
        u = V / det; v = W / det;
        return true;
    }
}
// one watertight test of triangle t; true when it became the closest hit
__device__ __forceinline__ bool wt_tri(const float4* __restrict__ vt, int t, float3 o, const WtRay& r, float tmin,
                                       float& hitT, int& hitTri, float& hu, float& hv) {
    float tt, u, v;
    if (!wt_test(vt, t, o, r, tmin, hitT, tt, u, v)) return false;
    hitT = tt; hitTri = t; hu = u; hv = v;
    return true;
}


// the margin that keeps the f16 planes outside the exact ones (see above)
__device__ __forceinline__ float h16_margin(float A, float B) { return (1.001f * fabsf(A) + 1792.f * fabsf(B)) * (1.f / 2048.f) + 1e-4f; }
// whether an axis's plane distances stay inside the f16 range (see above)
__device__ __forceinline__ bool h16_ok(float A, float B) {
    const float m = h16_margin(A, B), Ap = A - 1024.f * B;
    return fabsf(B) * 1279.f < 30000.f && fabsf(Ap) + m < 30000.f;
}
// outward-rounded f16 bases of one axis
__device__ __forceinline__ void h16_axis(float A, float B, __half2& lo2, __half2& hi2, __half2& b2) {
    const float m = h16_margin(A, B), Ap = A - 1024.f * B;
    const __half lo = __float2half_rd(Ap - m), hi = __float2half_ru(Ap + m);
    lo2 = __halves2half2(lo, lo); hi2 = __halves2half2(hi, hi); b2 = __float2half2_rn(B);   // (one conversion fills both halves)
}
// widened FP32 bases of one axis (nodes outside the f16 range)
__device__ __forceinline__ void f32_axis(float A, float B, float& lo, float& hi, float& b) {
    if (fabsf(A) < 1e30f && fabsf(B) < 1e30f) {
        const float m = (fabsf(A) + 256.f * fabsf(B)) * 9.5367431640625e-7f + 1e-30f;   // 2^-20
        lo = A - m; hi = A + m; b = B;
    } else { lo = -INFINITY; hi = INFINITY; b = 0.f; }
}

// A node visit and the triangle tests of its hit leaves are separate steps: step() visits a node only once the previous
// node's triangles are all tested, and runs one watertight test per call. Each ray still performs exactly the sequence
// of the fused traversal (visit, its leaves in slot order, the next visit), so hits are unchanged; but a lane with many
// hit triangles no longer holds the warp's other lanes for all of its (expensive) tests at once. Measured +10% on the
// 1M-ray precision batch; the same split of the FP32 traversal (TravState<8>, cheap Woop tests) measured 15-25%
// slower - its node visits, not its leaf tests, dominate (ncu: thread instructions +8%, active lanes 14.0 -> 13.1).
// The hit leaves' triangles are kept as a bit mask over the node's triangle range: both encoders here (host collapse,
// GPU emission) assign a node's leaf ranges in slot order, so ascending bits are slot order, and within a leaf its
// triangles in order. The closest-hit ray-batch kernel (trace.cu k_trace_prec_rf) calls visit() alone and tests the
// pending triangles (tb, tm) of all lanes together, with the same per-ray result.
template <bool ANY, int TRI>
struct TravState<16, ANY, TRI> {
    typedef uint2 Stack[kStack8];
    float3 o, d; float idx, idy, idz, tmin, hitT, hu, hv; int hitTri, node, sp, budget; unsigned oct, cb, im, hm, tb, tm, tint; WtRay wt;

    // the f16 interval [tmin rounded down, hitT rounded up], updated when hitT changes (not per node)
    __device__ __forceinline__ void set_tint() {
        tint = bits_of_h2(__halves2half2(__float2half_rd(tmin), __float2half_ru(hitT)));
    }
    __device__ __forceinline__ void begin(float3 o_, float3 d_, float tmin_, float tmax_, int root) {
        o = o_; d = d_; tmin = tmin_; hitT = tmax_; hu = hv = 0.f; hitTri = -1; node = root; sp = 0; budget = kVisitBudget;
        idx = safe_rcp(d.x); idy = safe_rcp(d.y); idz = safe_rcp(d.z);
        oct = (d.x > 0.f ? 1u : 0u) | (d.y > 0.f ? 2u : 0u) | (d.z > 0.f ? 4u : 0u);
        cb = im = hm = tb = tm = 0; wt = wt_setup(d); set_tint();
    }
    // A node visit: the node's hit leaves become the pending triangles (tm), and the next node is chosen. True when
    // the ray is finished (no node left and nothing pending, or an error).
    template <class N, class S>
    __device__ __forceinline__ bool visit(const N& nodes, S& stack, int& err) {
        {
            if (node < 0) return true;
            if (--budget < 0) { err |= kTravBudget; return true; }
            float4 nf[5]; fetch_node<5>(nodes, node, nf);
            const float4 f0 = nf[0], f1 = nf[1], f2 = nf[2], f3_ = nf[3], f4_ = nf[4];
            const unsigned ew = __float_as_uint(f0.w);
            const unsigned imask = ew >> 24, m0 = __float_as_uint(f1.z), m1 = __float_as_uint(f1.w);
            const int childBase = __float_as_int(f1.x);
            const float Ax = (f0.x - o.x) * idx, Bx = __uint_as_float((ew & 255u) << 23) * idx;
            const float Ay = (f0.y - o.y) * idy, By = __uint_as_float(((ew >> 8) & 255u) << 23) * idy;
            const float Az = (f0.z - o.z) * idz, Bz = __uint_as_float(((ew >> 16) & 255u) << 23) * idz;
            const bool fx = idx < 0.f, fy = idy < 0.f, fz = idz < 0.f;
            const unsigned nx0 = __float_as_uint(fx ? f3_.z : f2.x), nx1 = __float_as_uint(fx ? f3_.w : f2.y), px0 = __float_as_uint(fx ? f2.x : f3_.z), px1 = __float_as_uint(fx ? f2.y : f3_.w);
            const unsigned ny0 = __float_as_uint(fy ? f4_.x : f2.z), ny1 = __float_as_uint(fy ? f4_.y : f2.w), py0 = __float_as_uint(fy ? f2.z : f4_.x), py1 = __float_as_uint(fy ? f2.w : f4_.y);
            const unsigned nz0 = __float_as_uint(fz ? f4_.z : f3_.x), nz1 = __float_as_uint(fz ? f4_.w : f3_.y), pz0 = __float_as_uint(fz ? f3_.x : f4_.z), pz1 = __float_as_uint(fz ? f3_.y : f4_.w);
            unsigned boxHit = 0;
            if (h16_ok(Ax, Bx) && h16_ok(Ay, By) && h16_ok(Az, Bz)) {
                __half2 xlo, xhi, xb, ylo, yhi, yb, zlo, zhi, zb;
                h16_axis(Ax, Bx, xlo, xhi, xb); h16_axis(Ay, By, ylo, yhi, yb); h16_axis(Az, Bz, zlo, zhi, zb);
                const __half2 tmin2 = h2_of_bits(__byte_perm(tint, 0u, 0x1010u)), tmax2 = h2_of_bits(__byte_perm(tint, 0u, 0x3232u));
                unsigned hm2[4];   // per child pair: 0xffff in the low half for slot 2j, in the high half for slot 2j + 1
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const unsigned sel = (j & 1) ? 0x4342u : 0x4140u;   // bytes (2j, 2j+1) of the word, each under 0x64: halves 1024 + q
                    const __half2 xn = __hfma2(h2_of_bits(__byte_perm(j < 2 ? nx0 : nx1, 0x64646464u, sel)), xb, xlo);
                    const __half2 xf = __hfma2(h2_of_bits(__byte_perm(j < 2 ? px0 : px1, 0x64646464u, sel)), xb, xhi);
                    const __half2 yn = __hfma2(h2_of_bits(__byte_perm(j < 2 ? ny0 : ny1, 0x64646464u, sel)), yb, ylo);
                    const __half2 yf = __hfma2(h2_of_bits(__byte_perm(j < 2 ? py0 : py1, 0x64646464u, sel)), yb, yhi);
                    const __half2 zn = __hfma2(h2_of_bits(__byte_perm(j < 2 ? nz0 : nz1, 0x64646464u, sel)), zb, zlo);
                    const __half2 zf = __hfma2(h2_of_bits(__byte_perm(j < 2 ? pz0 : pz1, 0x64646464u, sel)), zb, zhi);
                    const __half2 tn = __hmax2(__hmax2(xn, yn), __hmax2(zn, tmin2));
                    const __half2 tf = __hmin2(__hmin2(xf, yf), __hmin2(zf, tmax2));
                    hm2[j] = __hle2_mask(tn, tf);
                }
                // one byte per slot (the low byte of each half), then the flags gathered onto bits 0..7 as in leaf_slots
                const unsigned w0 = __byte_perm(hm2[0], hm2[1], 0x6420u), w1 = __byte_perm(hm2[2], hm2[3], 0x6420u);
                boxHit = (((w0 & 0x01010101u) * 0x10204080u) >> 28) | ((((w1 & 0x01010101u) * 0x10204080u) >> 24) & 0xF0u);
            } else {
                float xlo, xhi, xb, ylo, yhi, yb, zlo, zhi, zb;
                f32_axis(Ax, Bx, xlo, xhi, xb); f32_axis(Ay, By, ylo, yhi, yb); f32_axis(Az, Bz, zlo, zhi, zb);
#pragma unroll
                for (int s = 0; s < 8; s++) {
                    const float xn = fmaf(qbyte(s < 4 ? nx0 : nx1, s), xb, xlo), xf = fmaf(qbyte(s < 4 ? px0 : px1, s), xb, xhi);
                    const float yn = fmaf(qbyte(s < 4 ? ny0 : ny1, s), yb, ylo), yf = fmaf(qbyte(s < 4 ? py0 : py1, s), yb, yhi);
                    const float zn = fmaf(qbyte(s < 4 ? nz0 : nz1, s), zb, zlo), zf = fmaf(qbyte(s < 4 ? pz0 : pz1, s), zb, zhi);
                    const float tn = fmaxf(fmaxf(xn, yn), fmaxf(zn, tmin)), tf = fminf(fminf(xf, yf), fminf(zf, hitT));
                    boxHit |= (tn <= tf ? 1u : 0u) << s;
                }
            }
            unsigned leafHit = boxHit & leaf_slots(m0, m1);
            tb = __float_as_uint(f1.y);
            while (leafHit) {
                const int s = __ffs(leafHit) - 1; leafHit &= leafHit - 1;
                const unsigned m = byte_of(s < 4 ? m0 : m1, s);
                tm |= ((2u << ((m >> 5) & 3u)) - 1u) << (m & 31u);
            }
            unsigned hits = boxHit & imask;
            if (oct & 1u) hits = ((hits & 0x55u) << 1) | ((hits & 0xAAu) >> 1);
            if (oct & 2u) hits = ((hits & 0x33u) << 2) | ((hits & 0xCCu) >> 2);
            if (oct & 4u) hits = ((hits & 0x0Fu) << 4) | ((hits & 0xF0u) >> 4);
            if (hits) {
                if (hm) { if (sp == kStack8) { err |= kTravOverflow; return true; } stack[sp++] = make_uint2(cb, (im << 8) | hm); }
                cb = (unsigned)childBase; im = imask; hm = hits;
            }
            while (hm == 0 && sp > 0) { const uint2 e = stack[--sp]; cb = e.x; im = e.y >> 8; hm = e.y & 255u; }
            if (hm) {
                const unsigned k = __ffs(hm) - 1; hm &= hm - 1; const unsigned slot = k ^ oct;
                node = (int)cb + __popc(im & ((1u << slot) - 1u));
            } else node = -1;
        }
        return tm == 0 && node < 0;
    }
    // One pending triangle test (tm != 0). True when the ray is finished.
    __device__ __forceinline__ bool tri(const float4* __restrict__ vt) {
        const int t = (int)tb + __ffs(tm) - 1; tm &= tm - 1;
        if (wt_tri(vt, t, o, wt, tmin, hitT, hitTri, hu, hv)) { if (ANY) return true; set_tint(); }
        return tm == 0 && node < 0;
    }
    // a visit when nothing is pending, then one pending triangle
    template <class N, class S>
    __device__ __forceinline__ bool step(const N& nodes, const float4* __restrict__ vt, S& stack, int& err) {
        if (tm == 0 && visit(nodes, stack, err)) return true;
        return tm ? tri(vt) : node < 0;
    }
};

// ---------------- FP64 reference traversal (the precision form's oracle) ----------------
// CWBVH nodes decoded exactly in double (origin + q 2^e), slab test in double widened by 1e-12 relative, watertight
// triangle test in double on the exact corners. Finds the closest hit in (tmin, tmax) to double accuracy.
__device__ __forceinline__ double dcomp(double3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

template <bool ANY>
__device__ __forceinline__ bool trav_fp64(const float4* __restrict__ nodes, const float4* __restrict__ vt, double3 o, double3 d, double tmin,
                                          double& hitT, int& hitTri, int& err) {
    uint2 stack[kStack8]; int sp = 0, budget = kVisitBudget, node = 0;
    const double ix = 1.0 / (fabs(d.x) > 1e-300 ? d.x : copysign(1e-300, d.x)), iy = 1.0 / (fabs(d.y) > 1e-300 ? d.y : copysign(1e-300, d.y)),
                 iz = 1.0 / (fabs(d.z) > 1e-300 ? d.z : copysign(1e-300, d.z));
    const double ad[3] = { fabs(d.x), fabs(d.y), fabs(d.z) };
    int kz = ad[0] >= ad[1] ? (ad[0] >= ad[2] ? 0 : 2) : (ad[1] >= ad[2] ? 1 : 2), kx = kz == 2 ? 0 : kz + 1, ky = kx == 2 ? 0 : kx + 1;
    if (dcomp(d, kz) < 0.0) { const int t = kx; kx = ky; ky = t; }
    const double sx = dcomp(d, kx) / dcomp(d, kz), sy = dcomp(d, ky) / dcomp(d, kz), sz = 1.0 / dcomp(d, kz);
    unsigned cb = 0, im = 0, hm = 0;
    while (true) {
        if (--budget < 0) { err |= kTravBudget; return hitTri >= 0; }
        const float4* nb = nodes + 5 * (size_t)node;
        const float4 f0 = ld4(nb), f1 = ld4(nb + 1);
        const unsigned ew = __float_as_uint(f0.w), imask = ew >> 24, m0 = __float_as_uint(f1.z), m1 = __float_as_uint(f1.w);
        const int childBase = __float_as_int(f1.x), triBase = __float_as_int(f1.y);
        const double ex = (double)__uint_as_float((ew & 255u) << 23), ey = (double)__uint_as_float(((ew >> 8) & 255u) << 23), ez = (double)__uint_as_float(((ew >> 16) & 255u) << 23);
        const unsigned* q = reinterpret_cast<const unsigned*>(nb + 2);
        unsigned boxHit = 0;
        for (int s = 0; s < 8; s++) {
            const int w = s < 4 ? 0 : 1;
            const double lx = (double)f0.x + byte_of(__ldg(q + 0 + w), s) * ex, ly = (double)f0.y + byte_of(__ldg(q + 2 + w), s) * ey, lz = (double)f0.z + byte_of(__ldg(q + 4 + w), s) * ez;
            const double hx = (double)f0.x + byte_of(__ldg(q + 6 + w), s) * ex, hy = (double)f0.y + byte_of(__ldg(q + 8 + w), s) * ey, hz = (double)f0.z + byte_of(__ldg(q + 10 + w), s) * ez;
            const double x0 = (lx - o.x) * ix, x1 = (hx - o.x) * ix, y0 = (ly - o.y) * iy, y1 = (hy - o.y) * iy, z0 = (lz - o.z) * iz, z1 = (hz - o.z) * iz;
            const double tn = fmax(fmax(fmin(x0, x1), fmin(y0, y1)), fmax(fmin(z0, z1), tmin));
            const double tf = fmin(fmin(fmax(x0, x1), fmax(y0, y1)), fmin(fmax(z0, z1), hitT));
            if (tn - 1e-12 * fabs(tn) <= tf + 1e-12 * fabs(tf)) boxHit |= 1u << s;
        }
        for (int s = 0; s < 8; s++) {
            if (!(boxHit & (1u << s))) continue;
            const unsigned m = byte_of(s < 4 ? m0 : m1, s);
            if (!(m & 0x80u)) continue;
            for (int t = triBase + (int)(m & 31u), e = t + (int)((m >> 5) & 3u) + 1; t < e; t++) {
                const float4 a = ld4(vt + 3 * t), b = ld4(vt + 3 * t + 1), c = ld4(vt + 3 * t + 2);
                const double3 A = make_double3(a.x - o.x, a.y - o.y, a.z - o.z), B = make_double3(b.x - o.x, b.y - o.y, b.z - o.z), C = make_double3(c.x - o.x, c.y - o.y, c.z - o.z);
                const double Az = dcomp(A, kz), Bz = dcomp(B, kz), Cz = dcomp(C, kz);
                const double Ax = dcomp(A, kx) - sx * Az, Ay = dcomp(A, ky) - sy * Az, Bx = dcomp(B, kx) - sx * Bz, By = dcomp(B, ky) - sy * Bz;
                const double Cx = dcomp(C, kx) - sx * Cz, Cy = dcomp(C, ky) - sy * Cz;
                const double U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
                if ((U < 0.0 || V < 0.0 || W < 0.0) && (U > 0.0 || V > 0.0 || W > 0.0)) continue;
                const double det = U + V + W;
                if (det == 0.0) continue;
                const double tt = (U * (sz * Az) + V * (sz * Bz) + W * (sz * Cz)) / det;
                if (tt > tmin && tt < hitT) { hitT = tt; hitTri = t; if (ANY) return true; }
            }
        }
        unsigned hits = boxHit & imask;
        const unsigned oct = (d.x > 0.0 ? 1u : 0u) | (d.y > 0.0 ? 2u : 0u) | (d.z > 0.0 ? 4u : 0u);
        unsigned ho = 0;
        for (int s = 0; s < 8; s++) if (hits & (1u << s)) ho |= 1u << (s ^ oct);
        if (ho) {
            if (hm) { if (sp == kStack8) { err |= kTravOverflow; return hitTri >= 0; } stack[sp++] = make_uint2(cb, (im << 8) | hm); }
            cb = (unsigned)childBase; im = imask; hm = ho;
        }
        while (hm == 0) { if (sp == 0) return hitTri >= 0; const uint2 e = stack[--sp]; cb = e.x; im = e.y >> 8; hm = e.y & 255u; }
        const unsigned k = __ffs(hm) - 1; hm &= hm - 1;
        node = (int)cb + __popc(im & ((1u << (k ^ oct)) - 1u));
    }
}

// nodes: a node pointer, or (CWBVH and the precision form) StagedNodes
template <int V, bool ANY, int TRI, class N>
__device__ __forceinline__ bool trace_ray(const N& nodes, const float4* __restrict__ tv, float3 o, float3 d, float tmin,
                                          float& hitT, int& hitTri, float& hu, float& hv, int root, int& err) {
    if constexpr (V == 2) return trav_bvh2<ANY, TRI>(nodes, tv, o, d, tmin, hitT, hitTri, hu, hv, root, err);
    else if constexpr (V == 4) return trav_bvh4<ANY, TRI>(nodes, tv, o, d, tmin, hitT, hitTri, hu, hv, root, err);
    else if constexpr (V == 16) {   // precision form: tv = exact corners
        TravState<16, ANY, TRI> r; typename TravState<16, ANY, TRI>::Stack stack; r.begin(o, d, tmin, hitT, root);
        while (!r.step(nodes, tv, stack, err)) {}
        hitT = r.hitT; hitTri = r.hitTri; hu = r.hu; hv = r.hv;
        return hitTri >= 0;
    } else return trav_cwbvh<ANY, TRI>(nodes, tv, o, d, tmin, hitT, hitTri, hu, hv, root, err);
}

}  // namespace cwpb
