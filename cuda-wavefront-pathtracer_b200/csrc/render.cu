// render.cu - wavefront path tracer for the diffuse (Lambert + sun + constant sky) path on sm_100a.
//
// Per pass of K samples per pixel, for depth = 0 .. bounces + 1:
//   k_trace_shade<depth 0>: camera ray generated in-kernel from the path index (no raygen pass, no state read),
//   k_trace_shade<depth > 0>: compacted path state read with coalesced 16-byte loads,
//   both: closest-hit traversal, then shading: miss -> sky; hit at depth <= bounces -> sun next-event estimation into
//   the shadow queue and a cosine continuation into the next depth's queue, both appended by one atomic per warp
//   (ballot + popc) so that every warp writes a contiguous run;
//   k_shadow: any-hit traversal of the shadow queue, unoccluded contributions added with one float4 atomic each.
// The semantics are those of the reference's legacy path (render/wavefront.cu:42-58 raygen, 94-136 shadeOne,
// 684-741 frame loop): same sample streams (pixel, sample, depth, dimension), same per-vertex decisions, so frames
// agree sample by sample with the reference's up to rounding.
// All traversal kernels are persistent (grid = resident blocks) with per-warp dynamic fetching of 32 paths, and read
// their queue lengths from device memory, so a whole frame is captured once as a CUDA graph and replayed.
#include "scene_dev.h"
#include "trav.cuh"
#include <algorithm>
#include <cstdio>
#include <mutex>
#include <cstring>
#include <string>
#include <vector>

namespace cwpb {

// path state (structure of arrays, one element per path in the queue):
//   s0 = (origin, path id bits), s1 = (direction, throughput.r), s2 = (throughput.g, throughput.b)
// shadow queue: h0 = (origin, pixel bits), h1 = (direction, contribution.r), h2 = (contribution.g, contribution.b)
struct Queues {
    float4* s0[2]; float4* s1[2]; float2* s2[2];
    float4* h0; float4* h1; float2* h2;
};

// per-depth counters, 4 ints each: [0] queue length, [1] shadow queue length, [2] trace fetch, [3] shadow fetch
struct KArgs {
    const float4* nodes; const float4* tv; const float4* tris; const float4* nrm; const float3* albedo;
    Queues q; float4* accum; int* cnt; int* err;
    int nk, N, sBase, depth;
    int staged;   // CWBVH nodes each block copies into shared memory (the first `staged`, i.e. the top levels)
};

// The node source of a traversal kernel: with STAGE, the block first copies the first a.staged nodes (the top levels
// of the breadth-first numbered CWBVH, which every ray visits) into its shared memory, and the traversal reads those
// from there and the rest from global memory.
template <bool STAGE>
__device__ __forceinline__ auto node_source(const KArgs& a) {
    if constexpr (STAGE) {
        extern __shared__ float4 sNodes[];
        for (int i = threadIdx.x; i < 5 * a.staged; i += blockDim.x) sNodes[i] = __ldg(a.nodes + i);
        __syncthreads();
        return StagedNodes{ a.nodes, sNodes, a.staged };
    } else return a.nodes;
}

__device__ __forceinline__ float rnd(const cwp_params& P, unsigned pix, unsigned smp, unsigned depth, unsigned dim) { return sample01(pix, smp, depth, dim, P.seed); }
__device__ __forceinline__ float3 v3(const float* a) { return f3(a[0], a[1], a[2]); }
__device__ __forceinline__ unsigned lanemask_lt() { unsigned m; asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m)); return m; }

// one atomic per warp: returns this lane's slot in a contiguous run reserved for the lanes with want set
__device__ __forceinline__ int warp_append(int* counter, bool want) {
    const unsigned m = __ballot_sync(0xffffffffu, want);
    if (!m) return -1;
    const int leader = __ffs(m) - 1, lane = threadIdx.x & 31;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    return want ? base + __popc(m & lanemask_lt()) : -1;
}

__device__ __forceinline__ void accum_add(float4* accum, int pix, float3 c) { atomicAdd(accum + pix, make_float4(c.x, c.y, c.z, 0.f)); }

// Pixel of path i: path i is sample sBase + i / N of pixel tile_pixel(i mod N). When the image is a whole number of
// 8 x 4 tiles, consecutive paths walk the pixels tile by tile, so a warp's 32 camera rays cover one 8 x 4 block
// (coherent traversal); otherwise row-major. Either way every (pixel, sample) pair is rendered exactly once.
__device__ __forceinline__ int tile_pixel(int j, int w, int h) {
    if ((w & 7) | (h & 3)) return j;
    const int t = j >> 5, r = j & 31, tilesX = w >> 3;
    return ((t / tilesX) * 4 + (r >> 3)) * w + (t % tilesX) * 8 + (r & 7);
}

// camera ray of path i (wavefront.cu:42-58): pixel tile_pixel(i mod N), sample sBase + i / N
__device__ __forceinline__ void camera_ray(const cwp_params& P, int i, int N, int sBase, float3& o, float3& d, int& pix, unsigned& smp) {
    const cwp_camera& C = P.cam;
    pix = tile_pixel(i % N, C.w, C.h); smp = (unsigned)(sBase + i / N);
    const int x = pix % C.w, y = pix / C.w;
    const float u0 = rnd(P, pix, smp, 0, 0), u1 = rnd(P, pix, smp, 0, 1);
    float jx, jy;
    if (P.filter_bh) { jx = table_lookup(P.ftab, CWP_FILTER_TABLE, u0); jy = table_lookup(P.ftab, CWP_FILTER_TABLE, u1); }
    else { jx = u0 - 0.5f; jy = u1 - 0.5f; }
    const float dx = (x + 0.5f + jx - C.px) / C.fx, dy = -(y + 0.5f + jy - C.py) / C.fy;
    const float3 ax = v3(C.ax), ay = v3(C.ay), az = v3(C.az), pos = v3(C.pos);
    d = normalize(ax * dx + ay * dy - az);
    o = pos;
    if (C.lens_r > 0.f) {
        float lx, ly; disk_map(rnd(P, pix, smp, 0, 2), rnd(P, pix, smp, 0, 3), lx, ly);
        const float3 pf = pos + (ax * dx + ay * dy - az) * C.focus_d;
        o = pos + ax * (lx * C.lens_r) + ay * (ly * C.lens_r);
        d = normalize(pf - o);
    }
}

static constexpr int kMaxStagedNodes = 512;    // 40 KB of shared memory per block at most
static constexpr int kDefaultStageLevels = -1;  // stage_levels = 0 means this

#ifndef CWPB_TRACE_MINB
#define CWPB_TRACE_MINB 8   // resident 128-thread blocks per SM the traversal kernels are compiled for
#endif

// Shading of path k after its closest-hit traversal (wavefront.cu:94-136): miss -> sky; hit at depth <= bounces ->
// sun next-event estimation (shadow queue) and cosine continuation (next depth's queue). Throughput and path id are
// read (or, for camera rays, recomputed) here, so that only the ray is live across the traversal. Every lane of the
// warp must call it (the appends are warp-wide); lanes with valid = false take part without a path.
template <bool PRIMARY>
__device__ __forceinline__ void shade_path(const KArgs& a, const cwp_params& P, bool valid, int k, float3 o, float3 d, float t, int tri, float hu, float hv) {
    int* const c = a.cnt + 4 * a.depth;
    const int rd = a.depth & 1, wr = rd ^ 1;
    const unsigned depthRng = (unsigned)a.depth + 1u;
    float3 T = f3(1.f, 1.f, 1.f); int id = k, pix = 0; unsigned smp = 0;
    if (valid) {
        if (!PRIMARY) {
            id = __float_as_int(__ldg(&a.q.s0[rd][k].w)); const float tr = __ldg(&a.q.s1[rd][k].w); const float2 s2 = __ldcs(a.q.s2[rd] + k);
            T = f3(tr, s2.x, s2.y);
        }
        pix = tile_pixel(id % a.N, P.cam.w, P.cam.h); smp = (unsigned)(a.sBase + id / a.N);
    }
    bool wantShadow = false, wantCont = false;
    float3 po = o, l = d, contrib = T, nd = d;
    if (valid) {
        if (tri < 0) accum_add(a.accum, pix, T * v3(P.sky));
        else if (a.depth <= P.max_b) {
            const float3 p = o + d * t;
            const float4 b = __ldg(a.tris + 3 * tri + 1), cc = __ldg(a.tris + 3 * tri + 2);
            float3 ng = normalize(cross(xyz(b), xyz(cc))), ns = ng;
            if (P.has_n && a.nrm) {
                const float3 n0 = xyz(__ldg(a.nrm + 3 * tri)), n1 = xyz(__ldg(a.nrm + 3 * tri + 1)), n2 = xyz(__ldg(a.nrm + 3 * tri + 2));
                const float3 nn = n0 * (1.f - hu - hv) + n1 * hu + n2 * hv; const float ln = length(nn);
                if (ln > 0.f) ns = nn * (1.f / ln);
                if (dot(ns, ng) < 0.f) ns = -ns;
            }
            if (dot(ng, d) > 0.f) { ng = -ng; ns = -ns; }
            const float3 alb = a.albedo[__float_as_int(b.w)];
            po = p + ng * P.eps;
            // sun next-event estimation: uniform direction in the sun's cone, Lambert BRDF alb / pi
            l = cone_dir(v3(P.sun_to), P.sun_cos, rnd(P, pix, smp, depthRng, 2), rnd(P, pix, smp, depthRng, 3));
            const float cl = dot(ns, l);
            if (cl > 0.f && dot(ng, l) > 0.f) { contrib = T * alb * v3(P.sun_e) * (cl * CWPB_INV_PI); wantShadow = true; }
            // continuation: cosine-weighted about the shading normal, throughput *= albedo
            nd = cosine_dir(ns, rnd(P, pix, smp, depthRng, 0), rnd(P, pix, smp, depthRng, 1));
            if (dot(nd, ng) > 0.f) { T = T * alb; wantCont = true; }
        }
    }
    const int sp = warp_append(c + 1, wantShadow);
    if (sp >= 0) {
        __stcs(a.q.h0 + sp, f4(po, __int_as_float(pix)));
        __stcs(a.q.h1 + sp, f4(l, contrib.x));
        __stcs(a.q.h2 + sp, make_float2(contrib.y, contrib.z));
    }
    const int cp = warp_append(c + 4, wantCont);
    if (cp >= 0) {
        __stcs(a.q.s0[wr] + cp, f4(po, __int_as_float(id)));
        __stcs(a.q.s1[wr] + cp, f4(nd, T.x));
        __stcs(a.q.s2[wr] + cp, make_float2(T.y, T.z));
    }
}

// the ray of path k at this depth: camera ray (depth 0) or the queued continuation
template <bool PRIMARY>
__device__ __forceinline__ void path_ray(const KArgs& a, const cwp_params& P, int k, float3& o, float3& d, float& tmin) {
    if (PRIMARY) { int pix; unsigned smp; camera_ray(P, k, a.N, a.sBase, o, d, pix, smp); tmin = P.near_clip; }
    else { const int rd = a.depth & 1; const float4 s0 = __ldcs(a.q.s0[rd] + k), s1 = __ldcs(a.q.s1[rd] + k); o = xyz(s0); d = xyz(s1); tmin = 0.f; }
}

// one warp fetch of 32 queue entries at a time, each ray traversed to completion, then the 32 shaded together
template <int V, int TRI, bool PRIMARY, bool STAGE = false>
__global__ void __launch_bounds__(128, CWPB_TRACE_MINB) k_trace_shade(const __grid_constant__ KArgs a, const __grid_constant__ cwp_params P) {
    const auto nodes = node_source<STAGE>(a);
    int* const c = a.cnt + 4 * a.depth;
    const int n = PRIMARY ? a.nk : c[0];
    const int lane = threadIdx.x & 31;
    int err = 0;
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(c + 2, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const int k = base + lane;
        const bool valid = k < n;
        float3 o = f3(0.f, 0.f, 0.f), d = f3(0.f, 0.f, 1.f); float tmin = 0.f;
        if (valid) path_ray<PRIMARY>(a, P, k, o, d, tmin);
        float t = 1e30f, hu = 0.f, hv = 0.f; int tri = -1;
        if (valid) trace_ray<V, false, TRI>(nodes, a.tv, o, d, tmin, t, tri, hu, hv, 0, err);
        shade_path<PRIMARY>(a, P, valid, k, o, d, t, tri, hu, hv);
    }
    if (err) atomicOr(a.err, err);
}

#ifndef CWPB_REFILL
#define CWPB_REFILL 24   // a warp refetches rays once this many of its lanes are idle (measured 12..32 on frame512:
                         // 12 74.6 ms, 16 72.7, 20 71.3, 24 70.8, 28 72.0, 32 76.6)
#endif

// Persistent traversal with dynamic refill (Aila & Laine 2009): every lane holds one ray's traversal state and
// advances it one node visit per step; once CWPB_REFILL lanes have finished, the warp shades those paths together,
// hands their lanes new queue entries with one atomic, and resumes. Lanes stay busy instead of waiting for the slowest
// ray of a 32-ray batch.
template <int V, int TRI, bool PRIMARY, bool STAGE = false>
__global__ void __launch_bounds__(128, CWPB_TRACE_MINB) k_trace_shade_rf(const __grid_constant__ KArgs a, const __grid_constant__ cwp_params P) {
    const auto nodes = node_source<STAGE>(a);
    int* const c = a.cnt + 4 * a.depth;
    const int n = PRIMARY ? a.nk : c[0];
    const int lane = threadIdx.x & 31;
    int err = 0;
    TravState<V, false, TRI> ray; typename TravState<V, false, TRI>::Stack stack;
    int k = -1; bool fin = false, drained = false;
    for (;;) {
        if (__any_sync(0xffffffffu, fin)) {
            shade_path<PRIMARY>(a, P, fin, k, ray.o, ray.d, ray.hitT, ray.hitTri, ray.hu, ray.hv);
            if (fin) { k = -1; fin = false; }
        }
        if (!drained) {
            const bool need = k < 0;
            const unsigned nm = __ballot_sync(0xffffffffu, need);
            if (nm) {
                const int leader = __ffs(nm) - 1;
                int base = 0;
                if (lane == leader) base = atomicAdd(c + 2, __popc(nm));
                base = __shfl_sync(0xffffffffu, base, leader);
                const int kk = base + __popc(nm & lanemask_lt());
                if (need && kk < n) { k = kk; float3 o, d; float tmin; path_ray<PRIMARY>(a, P, k, o, d, tmin); ray.begin(o, d, tmin, 1e30f, 0); }
                drained = __any_sync(0xffffffffu, need && kk >= n);   // the queue is empty from here on
            }
        }
        if (!__any_sync(0xffffffffu, k >= 0)) break;
        for (;;) {
            if (k >= 0 && !fin) fin = ray.step(nodes, a.tv, stack, err);
            const unsigned busy = __ballot_sync(0xffffffffu, k >= 0 && !fin);
            if (!busy || (!drained && 32 - __popc(busy) >= CWPB_REFILL)) break;
        }
    }
    if (err) atomicOr(a.err, err);
}

template <int V, int TRI, bool STAGE = false>
__global__ void __launch_bounds__(128, CWPB_TRACE_MINB) k_shadow_rf(const __grid_constant__ KArgs a) {
    const auto nodes = node_source<STAGE>(a);
    int* const c = a.cnt + 4 * a.depth;
    const int n = c[1];
    const int lane = threadIdx.x & 31;
    int err = 0;
    TravState<V, true, TRI> ray; typename TravState<V, true, TRI>::Stack stack;
    int k = -1; bool fin = false, drained = false;
    for (;;) {
        if (fin) {
            if (ray.hitTri < 0) { const float4 h0 = __ldg(a.q.h0 + k), h1 = __ldg(a.q.h1 + k); const float2 h2 = __ldcs(a.q.h2 + k); accum_add(a.accum, __float_as_int(h0.w), f3(h1.w, h2.x, h2.y)); }
            k = -1; fin = false;
        }
        if (!drained) {
            const bool need = k < 0;
            const unsigned nm = __ballot_sync(0xffffffffu, need);
            if (nm) {
                const int leader = __ffs(nm) - 1;
                int base = 0;
                if (lane == leader) base = atomicAdd(c + 3, __popc(nm));
                base = __shfl_sync(0xffffffffu, base, leader);
                const int kk = base + __popc(nm & lanemask_lt());
                if (need && kk < n) { k = kk; const float4 h0 = __ldg(a.q.h0 + k), h1 = __ldg(a.q.h1 + k); ray.begin(xyz(h0), xyz(h1), 0.f, 1e30f, 0); }
                drained = __any_sync(0xffffffffu, need && kk >= n);
            }
        }
        if (!__any_sync(0xffffffffu, k >= 0)) break;
        for (;;) {
            if (k >= 0 && !fin) fin = ray.step(nodes, a.tv, stack, err);
            const unsigned busy = __ballot_sync(0xffffffffu, k >= 0 && !fin);
            if (!busy || (!drained && 32 - __popc(busy) >= CWPB_REFILL)) break;
        }
    }
    if (err) atomicOr(a.err, err);
}

// FOCT >= 0 (CWBVH): the launch's shadow rays all point into octant FOCT (the sun's, when its cone stays inside one
// octant), so their traversal takes the plane choice and child order as constants; a ray outside it (or with a zero
// direction component) takes the per-ray form. Both visit the same nodes in the same order: the same result.
template <int V, int TRI, bool STAGE = false, int FOCT = -1>
__global__ void __launch_bounds__(128, CWPB_TRACE_MINB) k_shadow(const __grid_constant__ KArgs a) {
    const auto nodes = node_source<STAGE>(a);
    int* const c = a.cnt + 4 * a.depth;
    const int n = c[1];
    const int lane = threadIdx.x & 31;
    int err = 0;
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(c + 3, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const int k = base + lane;
        if (k < n) {
            const float4 h0 = __ldcs(a.q.h0 + k), h1 = __ldcs(a.q.h1 + k); const float2 h2 = __ldcs(a.q.h2 + k);
            float t = 1e30f, u, v; int tri = -1; bool hit;
            if constexpr (V == 8 && FOCT >= 0) {
                hit = octant_of(xyz(h1)) == FOCT ? trav_cwbvh<true, TRI, FOCT>(nodes, a.tv, xyz(h0), xyz(h1), 0.f, t, tri, u, v, 0, err)
                                                 : trav_cwbvh<true, TRI>(nodes, a.tv, xyz(h0), xyz(h1), 0.f, t, tri, u, v, 0, err);
            } else hit = trace_ray<V, true, TRI>(nodes, a.tv, xyz(h0), xyz(h1), 0.f, t, tri, u, v, 0, err);
            if (!hit) accum_add(a.accum, __float_as_int(h0.w), f3(h1.w, h2.x, h2.y));
        }
    }
    if (err) atomicOr(a.err, err);
}

// the octant every direction of the sun's cone lies in (all three components of the axis farther from zero than the
// cone's half-angle, with a factor 2 to spare), or -1
static int sun_octant(const cwp_params& P) {
    const float sx = P.sun_to[0], sy = P.sun_to[1], sz = P.sun_to[2];
    const float len = sqrtf(sx * sx + sy * sy + sz * sz);
    if (!(len > 0.f) || !(P.sun_cos > 0.f) || P.sun_cos > 1.f) return -1;
    const float half = acosf(P.sun_cos) * 2.f + 1e-6f;
    if (fabsf(sx) <= half * len || fabsf(sy) <= half * len || fabsf(sz) <= half * len) return -1;
    return (sx > 0.f ? 1 : 0) | (sy > 0.f ? 2 : 0) | (sz > 0.f ? 4 : 0);
}

// ---------------- continuation regrouping (cwp_render_options.sort) ----------------
// Before a bounce, the continuation rays are counting-sorted into bins of direction octant (and, for sort = 2, a 4 x 4 x
// 4 cell of the scene box around their origin), so the rays a warp fetches together descend the tree in the same order.
// Three light passes over the queue: histogram, exclusive scan of the bins, scatter of the 40-byte entries.
static constexpr int kSortBins = 512;
struct SortArgs { const float4* s0; const float4* s1; const float2* s2; float4* t0; float4* t1; float2* t2; const int* n; int* hist; int* cursor;
                  float3 lo, inv; int mode; };
__device__ __forceinline__ int sort_key(const SortArgs& a, float4 o, float4 d) {
    int k = (d.x < 0.f ? 1 : 0) | (d.y < 0.f ? 2 : 0) | (d.z < 0.f ? 4 : 0);
    if (a.mode == 2) {
        const int cx = min(max((int)((o.x - a.lo.x) * a.inv.x), 0), 3), cy = min(max((int)((o.y - a.lo.y) * a.inv.y), 0), 3), cz = min(max((int)((o.z - a.lo.z) * a.inv.z), 0), 3);
        k = (k << 6) | (cz << 4) | (cy << 2) | cx;
    }
    return k;
}
__global__ void __launch_bounds__(256) k_sort_hist(const SortArgs a) {
    __shared__ int h[kSortBins];
    for (int i = threadIdx.x; i < kSortBins; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const int n = *a.n;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) atomicAdd_block(&h[sort_key(a, __ldcs(a.s0 + k), __ldg(a.s1 + k))], 1);
    __syncthreads();
    for (int i = threadIdx.x; i < kSortBins; i += blockDim.x) if (h[i]) atomicAdd(&a.hist[i], h[i]);
}
__global__ void __launch_bounds__(kSortBins) k_sort_scan(const SortArgs a) {
    __shared__ int v[kSortBins];
    const int i = threadIdx.x, x = a.hist[i];
    v[i] = x; __syncthreads();
    for (int off = 1; off < kSortBins; off <<= 1) { const int y = i >= off ? v[i - off] : 0; __syncthreads(); v[i] += y; __syncthreads(); }
    a.cursor[i] = v[i] - x;
}
__global__ void __launch_bounds__(256) k_sort_scatter(const SortArgs a) {
    const int n = *a.n, lane = threadIdx.x & 31;
    for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < n; base += gridDim.x * blockDim.x) {
        const int k = base + lane; const bool ok = k < n;
        float4 o = make_float4(0.f, 0.f, 0.f, 0.f), d = o; float2 t = make_float2(0.f, 0.f);
        if (ok) { o = __ldcs(a.s0 + k); d = __ldcs(a.s1 + k); t = __ldcs(a.s2 + k); }
        const int key = ok ? sort_key(a, o, d) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        const int leader = __ffs(peers) - 1;
        int pos = 0;
        if (ok && lane == leader) pos = atomicAdd(&a.cursor[key], __popc(peers));
        pos = __shfl_sync(0xffffffffu, pos, leader) + __popc(peers & lanemask_lt());
        if (ok) { __stcs(a.t0 + pos, o); __stcs(a.t1 + pos, d); __stcs(a.t2 + pos, t); }
    }
}

// pass set-up: depth-0 queue length = nk; everything else zero
__global__ void k_pass_begin(int* cnt, int nInts, int nk, int* bins, int nBins) {
    for (int i = threadIdx.x; i < nInts; i += blockDim.x) cnt[i] = i == 0 ? nk : 0;
    for (int i = threadIdx.x; i < nBins; i += blockDim.x) bins[i] = 0;
}
// per-depth ray totals of a pass: tot[2 d] += queue length, tot[2 d + 1] += shadow queue length
__global__ void k_pass_end(const int* cnt, int depths, unsigned long long* tot) {
    for (int d = threadIdx.x; d < depths; d += blockDim.x) { tot[2 * d] += (unsigned)cnt[4 * d]; tot[2 * d + 1] += (unsigned)cnt[4 * d + 1]; }
}

}  // namespace cwpb

using namespace cwpb;

struct cwp_renderer {
    cwp_params P{}; cwp_render_options O{};
    DeviceScene scene;
    float4 *t0 = nullptr, *t1 = nullptr; float2* t2 = nullptr; int* sortBins = nullptr;   // regrouped continuation queue, bins per depth
    float3 boxLo{}, boxInv{};
    int N = 0, K = 1, depths = 0; long long nk = 0; bool ready = false;
    Queues q{};
    float4* accum = nullptr; int* cnt = nullptr; int* err = nullptr; unsigned long long* tot = nullptr;   // tot: 2 per depth
    std::vector<unsigned long long> htot;                 // last frame's per-depth totals
    std::vector<cudaEvent_t> ev; int evPasses = 0;        // profiling: 4 events per (pass, depth)
    std::vector<float> traceMs, shadowMs;                 // last frame's per-depth kernel times
    int* hcnt = nullptr;   // pinned copy of the counters (host loop)
    cudaStream_t st = nullptr; cudaEvent_t f0 = nullptr, f1 = nullptr;
    cudaGraphExec_t gexec = nullptr; int gSpp = -1, gBase = 0;
    int gridTrace = 0, gridTrace0 = 0, gridShadow = 0, nSM = 0; bool refill = false, refillShadow = false;
    int staged = 0;   // CWBVH nodes staged in each traversal block's shared memory (0 = none)
    std::vector<void*> allocs;
    double vramMB = 0; std::string gpuName;
};

namespace {

#ifdef CWPB_L1_CARVEOUT
template <class K> void prefer_l1(K* k) { cudaFuncSetAttribute((const void*)k, cudaFuncAttributePreferredSharedMemoryCarveout, CWPB_L1_CARVEOUT); }
#else
template <class K> void prefer_l1(K*) {}
#endif

template <int V, int TRI, bool STAGE = false> int occupancy_of(int& bt0, int& bt, int& bs, bool refill = false, size_t smem = 0) {
    if constexpr (!STAGE) {
        if constexpr (V != 4) { prefer_l1(k_trace_shade_rf<V, TRI, true>); prefer_l1(k_trace_shade_rf<V, TRI, false>); prefer_l1(k_shadow_rf<V, TRI>); }
        prefer_l1(k_trace_shade<V, TRI, true>); prefer_l1(k_trace_shade<V, TRI, false>); prefer_l1(k_shadow<V, TRI>);
    }
    if constexpr (V != 4) {
        if (refill) {
            CWPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt0, k_trace_shade_rf<V, TRI, true, STAGE>, 128, smem));
            CWPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt, k_trace_shade_rf<V, TRI, false, STAGE>, 128, smem));
            CWPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bs, k_shadow_rf<V, TRI, STAGE>, 128, smem));
            return CWP_OK;
        }
    }
    CWPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt0, k_trace_shade<V, TRI, true, STAGE>, 128, smem));
    CWPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt, k_trace_shade<V, TRI, false, STAGE>, 128, smem));
    CWPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bs, k_shadow<V, TRI, STAGE>, 128, smem));
    return CWP_OK;
}

// ev: 4 events (trace start/end, shadow start/end) or nullptr
template <int V, int TRI, bool STAGE = false> void launch_depth(cwp_renderer* r, KArgs a, int gt0, int gt, int gs, cudaEvent_t* ev) {
    // external records: inside a stream capture they become event-record nodes of the graph
    bool rf = false, rfShadow = false;
    const size_t sm = STAGE ? (size_t)80 * a.staged : 0;
    if constexpr (V != 4) { rf = r->refill; rfShadow = r->refillShadow; }
    if (ev) cudaEventRecordWithFlags(ev[0], r->st, cudaEventRecordExternal);
    if constexpr (V != 4) {
        if (rf) {
            if (a.depth == 0) k_trace_shade_rf<V, TRI, true, STAGE><<<gt0, 128, sm, r->st>>>(a, r->P);
            else k_trace_shade_rf<V, TRI, false, STAGE><<<gt, 128, sm, r->st>>>(a, r->P);
        }
    }
    if (!rf) {
        if (a.depth == 0) k_trace_shade<V, TRI, true, STAGE><<<gt0, 128, sm, r->st>>>(a, r->P);
        else k_trace_shade<V, TRI, false, STAGE><<<gt, 128, sm, r->st>>>(a, r->P);
    }
    if (r->O.sort && a.depth + 1 < r->depths) {   // regroup the continuations that the next bounce traces
        const int wr = (a.depth & 1) ^ 1;
        SortArgs sa{ r->q.s0[wr], r->q.s1[wr], r->q.s2[wr], r->t0, r->t1, r->t2, a.cnt + 4 * (a.depth + 1), r->sortBins + 2 * kSortBins * a.depth,
                     r->sortBins + 2 * kSortBins * a.depth + kSortBins, r->boxLo, r->boxInv, r->O.sort };
        k_sort_hist<<<r->nSM * 4, 256, 0, r->st>>>(sa);
        k_sort_scan<<<1, kSortBins, 0, r->st>>>(sa);
        k_sort_scatter<<<r->nSM * 8, 256, 0, r->st>>>(sa);
    }
    if (ev) { cudaEventRecordWithFlags(ev[1], r->st, cudaEventRecordExternal); cudaEventRecordWithFlags(ev[2], r->st, cudaEventRecordExternal); }
    if constexpr (V != 4) { if (rfShadow) k_shadow_rf<V, TRI, STAGE><<<gs, 128, sm, r->st>>>(a); }
    if (!rfShadow) {
        int foct = -1;
        if constexpr (V == 8 && !STAGE) foct = sun_octant(r->P);
        switch (foct) {
#define CWPB_SO(F) case F: if constexpr (V == 8 && !STAGE) k_shadow<8, TRI, false, F><<<gs, 128, sm, r->st>>>(a); break;
            CWPB_SO(0) CWPB_SO(1) CWPB_SO(2) CWPB_SO(3) CWPB_SO(4) CWPB_SO(5) CWPB_SO(6) CWPB_SO(7)
#undef CWPB_SO
            default: k_shadow<V, TRI, STAGE><<<gs, 128, sm, r->st>>>(a);
        }
    }
    if (ev) cudaEventRecordWithFlags(ev[3], r->st, cudaEventRecordExternal);
}

KArgs base_args(cwp_renderer* r) {
    KArgs a{};
    a.nodes = r->scene.nodes; a.tv = r->scene.leafData(); a.tris = r->scene.tris; a.nrm = r->scene.nrm; a.albedo = r->scene.albedo;
    a.q = r->q; a.accum = r->accum; a.cnt = r->cnt; a.err = r->err; a.nk = (int)r->nk; a.N = r->N; a.staged = r->staged;
    return a;
}

void dispatch_depth(cwp_renderer* r, KArgs a, int gt0, int gt, int gs, int pass) {
    const int V = r->scene.variant, T = r->scene.tri;
    if (r->O.sort && a.depth > 0) { const int rd = a.depth & 1; a.q.s0[rd] = r->t0; a.q.s1[rd] = r->t1; a.q.s2[rd] = r->t2; }
    cudaEvent_t* ev = r->O.profile ? &r->ev[((size_t)pass * r->depths + a.depth) * 4] : nullptr;
    if (V == 2) { if (T) launch_depth<2, 1>(r, a, gt0, gt, gs, ev); else launch_depth<2, 0>(r, a, gt0, gt, gs, ev); }
    else if (V == 4) { if (T) launch_depth<4, 1>(r, a, gt0, gt, gs, ev); else launch_depth<4, 0>(r, a, gt0, gt, gs, ev); }
    else if (r->staged) { if (T) launch_depth<8, 1, true>(r, a, gt0, gt, gs, ev); else launch_depth<8, 0, true>(r, a, gt0, gt, gs, ev); }
    else { if (T) launch_depth<8, 1>(r, a, gt0, gt, gs, ev); else launch_depth<8, 0>(r, a, gt0, gt, gs, ev); }
}

// profiling events for `passes` passes (created on first need, kept)
int ensure_events(cwp_renderer* r, int passes) {
    const size_t need = (size_t)passes * r->depths * 4;
    while (r->ev.size() < need) { cudaEvent_t e; CWPB_CUDA(cudaEventCreate(&e)); r->ev.push_back(e); }
    r->evPasses = passes;
    return CWP_OK;
}

// all passes of a frame with device-side queue lengths and persistent grids (the captured sequence)
int enqueue_passes(cwp_renderer* r, int spp, int sBase) {
    const int nInts = 4 * (r->depths + 1);
    for (int s = sBase, pass = 0; s < sBase + spp; s += r->K, pass++) {
        k_pass_begin<<<1, 128, 0, r->st>>>(r->cnt, nInts, (int)r->nk, r->sortBins, r->sortBins ? 2 * kSortBins * r->depths : 0);
        KArgs a = base_args(r); a.sBase = s;
        for (int d = 0; d < r->depths; d++) { a.depth = d; dispatch_depth(r, a, r->gridTrace0, r->gridTrace, r->gridShadow, pass); }
        k_pass_end<<<1, 32, 0, r->st>>>(r->cnt, r->depths, r->tot);
    }
    CWPB_CUDA(cudaGetLastError());
    return CWP_OK;
}

void release(cwp_renderer* r) {
    if (r->st) cudaStreamSynchronize(r->st);
    for (cudaEvent_t e : r->ev) cudaEventDestroy(e);
    r->ev.clear(); r->evPasses = 0;
    if (r->gexec) cudaGraphExecDestroy(r->gexec);
    r->gexec = nullptr; r->gSpp = -1;
    for (void* p : r->allocs) cudaFree(p);
    r->allocs.clear();
    r->t0 = r->t1 = nullptr; r->t2 = nullptr; r->sortBins = nullptr;
    if (r->hcnt) cudaFreeHost(r->hcnt);
    r->hcnt = nullptr;
    free_scene(r->scene);
    r->ready = false;
}

}  // namespace

extern "C" int cwp_renderer_create(cwp_renderer** out) {
    CWPB_CHECK(out, CWP_ERR_INVALID, "out is NULL");
    *out = new cwp_renderer();
    return CWP_OK;
}

extern "C" void cwp_renderer_destroy(cwp_renderer* r) {
    if (!r) return;
    cudaSetDevice(r->O.device);
    release(r);
    if (r->st) cudaStreamDestroy(r->st);
    if (r->f0) cudaEventDestroy(r->f0);
    if (r->f1) cudaEventDestroy(r->f1);
    delete r;
}

extern "C" int cwp_renderer_init(cwp_renderer* r, const cwp_params* p, const cwp_scene_buffers* s, const cwp_render_options* o) {
    CWPB_CHECK(r && p && s && o, CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(p->cam.w > 0 && p->cam.h > 0, CWP_ERR_INVALID, "image size %dx%d", p->cam.w, p->cam.h);
    CWPB_CHECK(o->batch >= 1, CWP_ERR_INVALID, "batch must be >= 1");
    CWPB_CHECK(o->bounces >= 0 && o->bounces <= 1000, CWP_ERR_INVALID, "bounces out of range");
    CWPB_CHECK(p->max_b <= o->bounces, CWP_ERR_INVALID, "params max_b %d exceeds the initialised bounce limit %d", p->max_b, o->bounces);
    const long long nk = (long long)p->cam.w * p->cam.h * o->batch;
    CWPB_CHECK(nk < (1ll << 31), CWP_ERR_INVALID, "w*h*batch = %lld paths in flight exceeds 2^31", nk);
    CWPB_CUDA(cudaSetDevice(o->device));
    release(r);
    size_t free0 = 0, total = 0;
    CWPB_CUDA(cudaMemGetInfo(&free0, &total));
    if (int rc = upload_scene(s, o->tri, o->device, r->scene)) return rc;
    CWPB_CHECK(r->scene.variant == o->variant, CWP_ERR_INVALID, "options.variant %d does not match the node stride (layout %d)", o->variant, r->scene.variant);
    r->P = *p; r->O = *o;
    r->N = p->cam.w * p->cam.h; r->K = o->batch; r->nk = nk; r->depths = o->bounces + 2;
    if (!r->st) { CWPB_CUDA(cudaStreamCreateWithFlags(&r->st, cudaStreamNonBlocking)); CWPB_CUDA(cudaEventCreate(&r->f0)); CWPB_CUDA(cudaEventCreate(&r->f1)); }
    auto alloc = [&](void** dst, size_t bytes) -> int {
        cudaError_t e = cudaMalloc(dst, bytes);
        if (e != cudaSuccess) { release(r); return set_error(CWP_ERR_NOMEM, "cannot allocate %.1f MB of path state: %s", bytes / 1e6, cudaGetErrorString(e)); }
        r->allocs.push_back(*dst); return CWP_OK;
    };
    const size_t NK = (size_t)nk;
    int rc = 0;
    for (int b = 0; b < 2 && !rc; b++) {
        rc = alloc((void**)&r->q.s0[b], NK * 16); if (!rc) rc = alloc((void**)&r->q.s1[b], NK * 16); if (!rc) rc = alloc((void**)&r->q.s2[b], NK * 8);
    }
    CWPB_CHECK(o->sort >= 0 && o->sort <= 2, CWP_ERR_INVALID, "sort %d is not 0, 1 or 2", o->sort);
    if (o->sort) {
        rc = alloc((void**)&r->t0, NK * 16); if (!rc) rc = alloc((void**)&r->t1, NK * 16); if (!rc) rc = alloc((void**)&r->t2, NK * 8);
        if (!rc) rc = alloc((void**)&r->sortBins, (size_t)2 * kSortBins * r->depths * sizeof(int));
        // scene box from the triangles (v0, v0 + e1, v0 + e2) for the origin cells
        float lo[3] = { 3e38f, 3e38f, 3e38f }, hi[3] = { -3e38f, -3e38f, -3e38f };
        for (int64_t t = 0; t < s->n_tris && !rc; t++)
            for (int c = 0; c < 3; c++) {
                const float* v = s->tris + 12 * t;
                for (int ax = 0; ax < 3; ax++) { const float x = v[ax] + (c ? s->tris[12 * t + 4 * c + ax] : 0.f); lo[ax] = std::min(lo[ax], x); hi[ax] = std::max(hi[ax], x); }
            }
        r->boxLo = f3(lo[0], lo[1], lo[2]);
        r->boxInv = f3(4.f / std::max(hi[0] - lo[0], 1e-30f), 4.f / std::max(hi[1] - lo[1], 1e-30f), 4.f / std::max(hi[2] - lo[2], 1e-30f));
    }
    if (!rc) rc = alloc((void**)&r->q.h0, NK * 16);
    if (!rc) rc = alloc((void**)&r->q.h1, NK * 16);
    if (!rc) rc = alloc((void**)&r->q.h2, NK * 8);
    if (!rc) rc = alloc((void**)&r->accum, (size_t)r->N * 16);
    if (!rc) rc = alloc((void**)&r->cnt, (size_t)4 * (r->depths + 1) * sizeof(int));
    if (!rc) rc = alloc((void**)&r->err, sizeof(int));
    if (!rc) rc = alloc((void**)&r->tot, 2 * (size_t)r->depths * sizeof(unsigned long long));
    if (rc) return rc;
    CWPB_CUDA(cudaMallocHost(&r->hcnt, (size_t)4 * (r->depths + 1) * sizeof(int)));
    CWPB_CUDA(cudaMemset(r->err, 0, sizeof(int)));
    CWPB_CUDA(cudaMemset(r->accum, 0, (size_t)r->N * 16));
    size_t free1 = 0; CWPB_CUDA(cudaMemGetInfo(&free1, &total));
    r->vramMB = (double)(free0 - free1) / 1048576.0;
    cudaDeviceProp prop; CWPB_CUDA(cudaGetDeviceProperties(&prop, o->device));
    r->gpuName = prop.name; r->nSM = prop.multiProcessorCount;
    int bt0 = 0, bt = 0, bs = 0;
    const int V = r->scene.variant, T = r->scene.tri;
    CWPB_CHECK(o->traversal >= 0 && o->traversal <= 2, CWP_ERR_INVALID, "traversal %d is not 0, 1 or 2", o->traversal);
    CWPB_CHECK(!(o->traversal == 1 && V == 4), CWP_ERR_INVALID, "refill traversal is available for BVH2 and CWBVH, not BVH4");
    // auto (measured on B200, 117k-triangle box field): refill pays for CWBVH closest-hit traversal; the shadow pass
    // (coherent rays towards the sun) and BVH2 (bound by dependent node-fetch latency) run faster per 32-ray batch
    r->refill = o->traversal == 1 || (o->traversal == 0 && V == 8);
    r->refillShadow = o->traversal == 1;
    // CWBVH top levels staged in shared memory: stage_levels 0 = the default, < 0 none, 1..3 levels 0..L (at most
    // kMaxStagedNodes nodes)
    CWPB_CHECK(o->stage_levels <= 3, CWP_ERR_INVALID, "stage_levels %d is above 3", o->stage_levels);
    r->staged = 0;
    if (V == 8) {
        const int L = o->stage_levels == 0 ? kDefaultStageLevels : o->stage_levels;
        if (L > 0) r->staged = std::min(r->scene.levelEnd[L], kMaxStagedNodes);
    }
    const size_t sm = (size_t)80 * r->staged;
    int b0 = 0, b1 = 0;
    if (V == 2) rc = T ? occupancy_of<2, 1>(bt0, bt, b0, r->refill) : occupancy_of<2, 0>(bt0, bt, b0, r->refill);
    else if (V == 4) rc = T ? occupancy_of<4, 1>(bt0, bt, b0) : occupancy_of<4, 0>(bt0, bt, b0);
    else if (r->staged) rc = T ? occupancy_of<8, 1, true>(bt0, bt, b0, r->refill, sm) : occupancy_of<8, 0, true>(bt0, bt, b0, r->refill, sm);
    else rc = T ? occupancy_of<8, 1>(bt0, bt, b0, r->refill) : occupancy_of<8, 0>(bt0, bt, b0, r->refill);
    if (rc) return rc;
    int d0 = 0, d1 = 0;   // shadow grid from the shadow kernel actually used
    if (V == 2) rc = T ? occupancy_of<2, 1>(d0, d1, bs, r->refillShadow) : occupancy_of<2, 0>(d0, d1, bs, r->refillShadow);
    else if (V == 4) rc = T ? occupancy_of<4, 1>(d0, d1, bs) : occupancy_of<4, 0>(d0, d1, bs);
    else if (r->staged) rc = T ? occupancy_of<8, 1, true>(d0, d1, bs, r->refillShadow, sm) : occupancy_of<8, 0, true>(d0, d1, bs, r->refillShadow, sm);
    else rc = T ? occupancy_of<8, 1>(d0, d1, bs, r->refillShadow) : occupancy_of<8, 0>(d0, d1, bs, r->refillShadow);
    (void)b1;
    if (rc) return rc;
    r->gridTrace0 = bt0 * r->nSM; r->gridTrace = bt * r->nSM; r->gridShadow = bs * r->nSM;
    r->ready = true;
    return CWP_OK;
}

extern "C" int cwp_renderer_render(cwp_renderer* r, int32_t spp, cwp_frame_stats* st, int32_t sBase, int32_t clear) {
    CWPB_CHECK(r && st, CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(r->ready, CWP_ERR_STATE, "render before a successful init");
    CWPB_CHECK(spp > 0 && spp % r->K == 0, CWP_ERR_INVALID, "spp %d must be a positive multiple of batch %d", spp, r->K);
    CWPB_CHECK(sBase >= 0, CWP_ERR_INVALID, "negative sample base");
    CWPB_CUDA(cudaSetDevice(r->O.device));
    *st = cwp_frame_stats{};
    if (clear) CWPB_CUDA(cudaMemsetAsync(r->accum, 0, (size_t)r->N * 16, r->st));
    CWPB_CUDA(cudaMemsetAsync(r->tot, 0, 2 * (size_t)r->depths * sizeof(unsigned long long), r->st));
    const int passes = spp / r->K;
    if (r->O.profile && r->evPasses < passes) {
        if (r->gexec) { CWPB_CUDA(cudaGraphExecDestroy(r->gexec)); r->gexec = nullptr; r->gSpp = -1; }   // events are captured nodes
        if (int rc = ensure_events(r, passes)) return rc;
    }
    CWPB_CUDA(cudaEventRecord(r->f0, r->st));
    if (r->O.graph) {
        if (!r->gexec || r->gSpp != spp || r->gBase != sBase) {   // the sample range is part of the captured launches
            if (r->gexec) { CWPB_CUDA(cudaGraphExecDestroy(r->gexec)); r->gexec = nullptr; }
            cudaGraph_t g;
            CWPB_CUDA(cudaStreamBeginCapture(r->st, cudaStreamCaptureModeThreadLocal));
            int rc = enqueue_passes(r, spp, sBase);
            cudaError_t e = cudaStreamEndCapture(r->st, &g);
            if (rc) { if (e == cudaSuccess) cudaGraphDestroy(g); return rc; }
            CWPB_CUDA(e);
            e = cudaGraphInstantiate(&r->gexec, g, 0);
            cudaGraphDestroy(g);
            CWPB_CUDA(e);
            r->gSpp = spp; r->gBase = sBase;
        }
        CWPB_CUDA(cudaGraphLaunch(r->gexec, r->st));
    } else {
        // host loop: exact grids from the queue lengths read back after each depth (one sync per bounce)
        const int nInts = 4 * (r->depths + 1);
        for (int s = sBase, pass = 0; s < sBase + spp; s += r->K, pass++) {
            k_pass_begin<<<1, 128, 0, r->st>>>(r->cnt, nInts, (int)r->nk, r->sortBins, r->sortBins ? 2 * kSortBins * r->depths : 0);
            KArgs a = base_args(r); a.sBase = s;
            int n = (int)r->nk;
            if (r->O.profile) for (int d = 0; d < r->depths; d++) for (int j = 0; j < 4; j++) CWPB_CUDA(cudaEventRecord(r->ev[((size_t)pass * r->depths + d) * 4 + j], r->st));
            for (int d = 0; d < r->depths && n > 0; d++) {
                a.depth = d;
                const int need = (n + 127) / 128;
                const int gt = need < r->gridTrace ? need : r->gridTrace, gt0 = need < r->gridTrace0 ? need : r->gridTrace0;
                dispatch_depth(r, a, gt0, gt, r->gridShadow, pass);
                CWPB_CUDA(cudaMemcpyAsync(r->hcnt, r->cnt, (size_t)nInts * sizeof(int), cudaMemcpyDeviceToHost, r->st));
                CWPB_CUDA(cudaStreamSynchronize(r->st));
                n = r->hcnt[4 * (d + 1)];
            }
            k_pass_end<<<1, 32, 0, r->st>>>(r->cnt, r->depths, r->tot);
        }
        CWPB_CUDA(cudaGetLastError());
    }
    CWPB_CUDA(cudaEventRecord(r->f1, r->st));
    CWPB_CUDA(cudaEventSynchronize(r->f1));
    float ms = 0.f; CWPB_CUDA(cudaEventElapsedTime(&ms, r->f0, r->f1));
    int herr = 0;
    r->htot.assign(2 * (size_t)r->depths, 0);
    CWPB_CUDA(cudaMemcpy(r->htot.data(), r->tot, r->htot.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    CWPB_CUDA(cudaMemcpy(&herr, r->err, sizeof(int), cudaMemcpyDeviceToHost));
    double rays = 0, shadow = 0;
    for (int d = 0; d < r->depths; d++) { rays += (double)r->htot[2 * d]; shadow += (double)r->htot[2 * d + 1]; }
    st->frame_ms = ms; st->trace_ms = ms; st->rays = rays; st->shadow_rays = shadow;
    r->traceMs.assign(r->depths, 0.f); r->shadowMs.assign(r->depths, 0.f);
    if (r->O.profile) {
        for (int pass = 0; pass < passes; pass++)
            for (int d = 0; d < r->depths; d++) {
                cudaEvent_t* e = &r->ev[((size_t)pass * r->depths + d) * 4]; float a = 0.f, b = 0.f;
                CWPB_CUDA(cudaEventElapsedTime(&a, e[0], e[1])); CWPB_CUDA(cudaEventElapsedTime(&b, e[2], e[3]));
                r->traceMs[d] += a; r->shadowMs[d] += b;
            }
        double t = 0; for (int d = 0; d < r->depths; d++) t += r->traceMs[d] + r->shadowMs[d];
        st->trace_ms = t;
    }
    if (herr) { cudaMemset(r->err, 0, sizeof(int)); return set_error(CWP_ERR_TRAVERSAL, "traversal stopped early on some rays (status 0x%x)", herr); }
    return CWP_OK;
}

extern "C" int cwp_renderer_read_accum(const cwp_renderer* r, float* dst) {
    CWPB_CHECK(r && dst, CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(r->ready, CWP_ERR_STATE, "read before a successful init");
    CWPB_CUDA(cudaSetDevice(r->O.device));
    CWPB_CUDA(cudaStreamSynchronize(r->st));
    CWPB_CUDA(cudaMemcpy(dst, r->accum, (size_t)r->N * 16, cudaMemcpyDeviceToHost));
    return CWP_OK;
}

extern "C" const void* cwp_renderer_accum_device(const cwp_renderer* r) { return r ? r->accum : nullptr; }

extern "C" int cwp_renderer_set_params(cwp_renderer* r, const cwp_params* p) {
    CWPB_CHECK(r && p, CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(r->ready, CWP_ERR_STATE, "set_params before a successful init");
    CWPB_CHECK(p->cam.w == r->P.cam.w && p->cam.h == r->P.cam.h, CWP_ERR_INVALID, "image size cannot change after init");
    CWPB_CHECK(p->max_b <= r->O.bounces, CWP_ERR_INVALID, "max_b %d exceeds the initialised bounce limit %d", p->max_b, r->O.bounces);
    CWPB_CUDA(cudaSetDevice(r->O.device));
    CWPB_CUDA(cudaStreamSynchronize(r->st));
    r->P = *p;
    if (r->gexec) { CWPB_CUDA(cudaGraphExecDestroy(r->gexec)); r->gexec = nullptr; r->gSpp = -1; }   // parameters are baked into the graph
    return CWP_OK;
}

extern "C" int cwp_renderer_set_materials(cwp_renderer* r, const float* albedo, int32_t n) {
    CWPB_CHECK(r && albedo, CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(r->ready, CWP_ERR_STATE, "set_materials before a successful init");
    CWPB_CHECK(n == r->scene.nAlbedo, CWP_ERR_INVALID, "material count %d differs from the initialised %d", n, r->scene.nAlbedo);
    CWPB_CUDA(cudaSetDevice(r->O.device));
    CWPB_CUDA(cudaStreamSynchronize(r->st));
    std::vector<float3> a(n);
    for (int i = 0; i < n; i++) a[i] = make_float3(albedo[3 * i], albedo[3 * i + 1], albedo[3 * i + 2]);
    CWPB_CUDA(cudaMemcpy(r->scene.albedo, a.data(), n * sizeof(float3), cudaMemcpyHostToDevice));
    return CWP_OK;
}

extern "C" int cwp_renderer_depth_stats(const cwp_renderer* r, int64_t* closest, int64_t* shadow, float* trace_ms, float* shadow_ms, int32_t n) {
    CWPB_CHECK(r, CWP_ERR_INVALID, "NULL renderer");
    CWPB_CHECK(n >= 0, CWP_ERR_INVALID, "negative depth count");
    for (int d = 0; d < n; d++) {
        const bool have = d < r->depths && r->htot.size() == 2 * (size_t)r->depths;
        if (closest) closest[d] = have ? (int64_t)r->htot[2 * d] : 0;
        if (shadow) shadow[d] = have ? (int64_t)r->htot[2 * d + 1] : 0;
        if (trace_ms) trace_ms[d] = d < (int)r->traceMs.size() ? r->traceMs[d] : 0.f;
        if (shadow_ms) shadow_ms[d] = d < (int)r->shadowMs.size() ? r->shadowMs[d] : 0.f;
    }
    return CWP_OK;
}

extern "C" int cwp_renderer_info_of(const cwp_renderer* r, cwp_renderer_info* out) {
    CWPB_CHECK(r && out, CWP_ERR_INVALID, "NULL argument");
    memset(out, 0, sizeof *out);
    out->vram_mb = r->vramMB; out->tlas_ms = 0; out->pt_blocks = r->gridTrace; out->n_sm = r->nSM;
    snprintf(out->gpu_name, sizeof out->gpu_name, "%s", r->gpuName.c_str());
    return CWP_OK;
}

// ---------------------------------------------------------------------------------------------------------------
// Rendering without any allocation. Some callers cannot call cudaMalloc: a plugin inside a host application that owns
// the GPU's memory budget, a serving loop that must not stall on cudaMalloc / cudaFree (both can synchronise the
// device), or code that must not fail on an allocation in the middle of a frame. cwp_render_noalloc gives them the
// frame of cwp_renderer_render with every scratch buffer (path state, shadow queue, counters) in the fixed array
// below, which every GPU that loads this library holds until the process exits. The caller passes the scene and the
// accumulation buffer as device pointers.
namespace cwpb {

static constexpr long long kNoAllocMaxPaths = 262144;     // w * h * batch of one pass
static constexpr int kNoAllocMaxBounces = 62;
static constexpr size_t kNoAllocStateBytes = (size_t)kNoAllocMaxPaths * (2 * (16 + 16 + 8) + (16 + 16 + 8));
static constexpr size_t kNoAllocCountBytes = 256 * ((4 * (kNoAllocMaxBounces + 3) * sizeof(int) + 255) / 256);
static constexpr size_t kNoAllocTotBytes = 256 * ((2 * (kNoAllocMaxBounces + 2) * sizeof(unsigned long long) + 255) / 256);
static constexpr size_t kNoAllocBytes = kNoAllocStateBytes + kNoAllocCountBytes + kNoAllocTotBytes + 256;

// the scratch: 31.5 MB of path state and queues, then the counters, per-depth ray totals and the status word
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

struct NoAllocDevice { unsigned char* base = nullptr; int gridTrace0 = 0, gridTrace = 0, gridShadow = 0; };

// device address of the scratch on the current device, looked up once per device (host code cannot use the symbol
// itself: on the host it names a stand-in, not device memory). The table is guarded by a mutex, so host threads that
// make their first calls at the same time each see a complete entry.
static int noalloc_setup(int dev, NoAllocDevice& out) {
    static std::mutex mu;
    static NoAllocDevice table[64];
    static bool ready[64] = { false };
    CWPB_CHECK(dev >= 0 && dev < 64, CWP_ERR_INVALID, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(mu);
    if (!ready[dev]) {
        void* p = nullptr;
        CWPB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        NoAllocDevice d; d.base = (unsigned char*)p;
        int nSM = 0; CWPB_CUDA(cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, dev));
        int bt0 = 0, bt = 0, bs = 0;
        // occupancy of the Woop / CWBVH kernels bounds every variant's grid (all share the launch bounds)
        if (int rc = occupancy_of<8, 1>(bt0, bt, bs)) return rc;
        d.gridTrace0 = bt0 * nSM; d.gridTrace = bt * nSM; d.gridShadow = bs * nSM;
        table[dev] = d; ready[dev] = true;
    }
    out = table[dev];
    return CWP_OK;
}

// a caller's buffer must be device (or managed) memory that the current device can address
static int noalloc_check_ptr(const void* ptr, int dev, const char* what) {
    if (!ptr) return CWP_OK;
    cudaPointerAttributes at{};
    CWPB_CUDA(cudaPointerGetAttributes(&at, ptr));
    CWPB_CHECK(at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged, CWP_ERR_INVALID, "%s is not device memory", what);
    CWPB_CHECK(at.type == cudaMemoryTypeManaged || at.device == dev, CWP_ERR_INVALID, "%s lives on device %d, not on the current device %d", what, at.device, dev);
    return CWP_OK;
}

}  // namespace cwpb

extern "C" int cwp_render_noalloc(const cwp_params* p, const cwp_device_scene* s, const cwp_render_options* o, int32_t spp, int32_t s_base,
                                  int32_t clear, float* d_accum, int64_t* h_rays, void* stream) {
    CWPB_CHECK(p && s && o && d_accum, CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(s->nodes && s->tris && s->albedo && (o->tri == 0 || s->woop), CWP_ERR_INVALID, "scene buffers missing");
    CWPB_CHECK(o->variant == 2 || o->variant == 4 || o->variant == 8, CWP_ERR_INVALID, "variant %d is not 2, 4 or 8", o->variant);
    CWPB_CHECK(o->tri == 0 || o->tri == 1, CWP_ERR_INVALID, "tri must be 0 or 1");
    CWPB_CHECK(p->cam.w > 0 && p->cam.h > 0 && o->batch >= 1, CWP_ERR_INVALID, "bad image size or batch");
    const long long nk = (long long)p->cam.w * p->cam.h * o->batch;
    CWPB_CHECK(nk <= kNoAllocMaxPaths, CWP_ERR_INVALID, "w*h*batch = %lld paths exceeds the no-allocation limit of %lld per pass (use a smaller batch, or cwp_renderer_*)", nk, kNoAllocMaxPaths);
    CWPB_CHECK(o->bounces >= 0 && o->bounces <= kNoAllocMaxBounces, CWP_ERR_INVALID, "bounces %d outside [0, %d] of the no-allocation path", o->bounces, kNoAllocMaxBounces);
    CWPB_CHECK(p->max_b <= o->bounces, CWP_ERR_INVALID, "params max_b %d exceeds bounces %d", p->max_b, o->bounces);
    CWPB_CHECK(spp > 0 && spp % o->batch == 0 && s_base >= 0, CWP_ERR_INVALID, "spp %d must be a positive multiple of batch %d", spp, o->batch);
    CWPB_CHECK(o->traversal == 0 || o->traversal == 2, CWP_ERR_INVALID, "traversal %d: the no-allocation path runs one 32-ray fetch per warp (0 or 2)", o->traversal);
    CWPB_CHECK(o->sort == 0, CWP_ERR_INVALID, "sort %d: the no-allocation path has no regrouping buffers (sort must be 0)", o->sort);
    int dev = 0; CWPB_CUDA(cudaGetDevice(&dev));
    CWPB_CHECK(o->device == dev, CWP_ERR_INVALID, "options.device %d is not the current device %d (make it current before the call)", o->device, dev);
    {
        const void* ptrs[6] = { s->nodes, s->tris, s->woop, s->nrm, s->albedo, d_accum };
        const char* names[6] = { "scene nodes", "scene tris", "scene woop", "scene nrm", "scene albedo", "accumulation buffer" };
        for (int k = 0; k < 6; k++) if (int rc = noalloc_check_ptr(ptrs[k], dev, names[k])) return rc;
    }
    NoAllocDevice na; if (int rc = noalloc_setup(dev, na)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t NK = (size_t)kNoAllocMaxPaths;
    unsigned char* b = na.base;
    Queues q{};
    for (int k = 0; k < 2; k++) { q.s0[k] = (float4*)b; b += NK * 16; q.s1[k] = (float4*)b; b += NK * 16; q.s2[k] = (float2*)b; b += NK * 8; }
    q.h0 = (float4*)b; b += NK * 16; q.h1 = (float4*)b; b += NK * 16; q.h2 = (float2*)b; b += NK * 8;
    int* cnt = (int*)b; b += kNoAllocCountBytes;
    unsigned long long* tot = (unsigned long long*)b; b += kNoAllocTotBytes;
    int* err = (int*)b;
    const int depths = o->bounces + 2, N = p->cam.w * p->cam.h;
    // the scratch keeps the previous call's contents: totals and status start at zero, counters are reset per pass
    CWPB_CUDA(cudaMemsetAsync(tot, 0, 2 * (size_t)depths * sizeof(unsigned long long), st));
    CWPB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    if (clear) CWPB_CUDA(cudaMemsetAsync(d_accum, 0, (size_t)N * 16, st));
    KArgs a{};
    a.nodes = (const float4*)s->nodes; a.tv = (const float4*)(o->tri ? s->woop : s->tris); a.tris = (const float4*)s->tris;
    a.nrm = (const float4*)s->nrm; a.albedo = (const float3*)s->albedo;
    a.q = q; a.accum = (float4*)d_accum; a.cnt = cnt; a.err = err; a.nk = (int)nk; a.N = N;
    for (int sb = s_base; sb < s_base + spp; sb += o->batch) {
        k_pass_begin<<<1, 128, 0, st>>>(cnt, 4 * (depths + 1), (int)nk, nullptr, 0);
        a.sBase = sb;
        for (int d = 0; d < depths; d++) {
            a.depth = d;
#define CWPB_NA(VV, TT) do { if (d == 0) k_trace_shade<VV, TT, true><<<na.gridTrace0, 128, 0, st>>>(a, *p); \
                             else k_trace_shade<VV, TT, false><<<na.gridTrace, 128, 0, st>>>(a, *p); \
                             k_shadow<VV, TT><<<na.gridShadow, 128, 0, st>>>(a); } while (0)
            if (o->variant == 2) { if (o->tri) CWPB_NA(2, 1); else CWPB_NA(2, 0); }
            else if (o->variant == 4) { if (o->tri) CWPB_NA(4, 1); else CWPB_NA(4, 0); }
            else { if (o->tri) CWPB_NA(8, 1); else CWPB_NA(8, 0); }
#undef CWPB_NA
        }
        k_pass_end<<<1, 32, 0, st>>>(cnt, depths, tot);
    }
    CWPB_CUDA(cudaGetLastError());
    if (h_rays) {   // optional: wait for the frame and report (closest, shadow) ray totals and the traversal status
        unsigned long long ht[2 * (kNoAllocMaxBounces + 2)]; int herr = 0;
        CWPB_CUDA(cudaMemcpyAsync(ht, tot, 2 * (size_t)depths * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        CWPB_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        CWPB_CUDA(cudaStreamSynchronize(st));
        h_rays[0] = h_rays[1] = 0;
        for (int d = 0; d < depths; d++) { h_rays[0] += (int64_t)ht[2 * d]; h_rays[1] += (int64_t)ht[2 * d + 1]; }
        CWPB_CHECK(herr == 0, CWP_ERR_TRAVERSAL, "traversal stopped early on some rays (status 0x%x)", herr);
    }
    return CWP_OK;
}
