// trace.cu - device scene upload/validation and the standalone closest-hit / any-hit ray-batch kernels.
#include "scene_dev.h"
#include "trav.cuh"
#include <algorithm>
#include <cstring>
#include <vector>

namespace cwpb {

// ---------------- validation + upload ----------------
int validate_nodes(const float* nodes, int64_t nF4, int stride, int64_t nTris, int* variantOut) {
    CWPB_CHECK(nodes && nF4 > 0, CWP_ERR_INVALID, "empty node array");
    CWPB_CHECK(stride == 4 || stride == 5 || stride == 8, CWP_ERR_INVALID, "node stride %d is not 4 (BVH2), 8 (BVH4) or 5 (CWBVH)", stride);
    CWPB_CHECK(nF4 % stride == 0, CWP_ERR_INVALID, "node array of %lld float4 is not a multiple of the stride %d", (long long)nF4, stride);
    const int64_t nNodes = nF4 / stride;
    const int32_t* w = reinterpret_cast<const int32_t*>(nodes);
    auto leafOk = [&](int64_t first, int64_t cnt) { return first >= 0 && cnt > 0 && first + cnt <= nTris; };
    if (stride == 4 || stride == 8) {
        const int width = stride == 4 ? 2 : 4;
        for (int64_t n = 0; n < nNodes; n++) {
            const int32_t* m = w + n * stride * 4 + (stride == 4 ? 12 : 24);
            for (int j = 0; j < width; j++) {
                int32_t c = m[j], k = m[j + (stride == 4 ? 2 : 4)];
                bool ok = k > 0 ? leafOk(c, k) : (k == 0 && (c == -1 || (c >= 0 && c < nNodes)));
                CWPB_CHECK(ok, CWP_ERR_INVALID, "node %lld child %d: reference (%d, %d) out of range (%lld nodes, %lld triangles)", (long long)n, j, c, k, (long long)nNodes, (long long)nTris);
            }
        }
        *variantOut = stride == 4 ? 2 : 4;
    } else {
        for (int64_t n = 0; n < nNodes; n++) {
            const int32_t* q = w + n * 20;
            uint32_t ew = (uint32_t)q[3], imask = ew >> 24; int32_t childBase = q[4], triBase = q[5];
            // the traversal scales 2^e / d by 2^24: biased exponents up to 164 (quantisation steps up to 2^37, child boxes
            // up to about 3.5e13 across) keep that finite for |1/d| <= 1e20
            CWPB_CHECK((ew & 255u) <= 164u && ((ew >> 8) & 255u) <= 164u && ((ew >> 16) & 255u) <= 164u, CWP_ERR_INVALID,
                       "CWBVH node %lld: quantisation exponent above 164 (child boxes beyond 3.5e13)", (long long)n);
            int nInt = __builtin_popcount(imask);
            CWPB_CHECK(nInt == 0 || (childBase >= 0 && (int64_t)childBase + nInt <= nNodes), CWP_ERR_INVALID, "CWBVH node %lld: children [%d, +%d) out of range", (long long)n, childBase, nInt);
            for (int s = 0; s < 8; s++) {
                uint32_t m = ((uint32_t)q[6 + s / 4] >> (8 * (s & 3))) & 255u;
                if (m & 0x80u) {
                    int64_t first = (int64_t)triBase + (m & 31u), cnt = ((m >> 5) & 3u) + 1;
                    CWPB_CHECK(leafOk(first, cnt), CWP_ERR_INVALID, "CWBVH node %lld slot %d: leaf [%lld, +%lld) out of range", (long long)n, s, (long long)first, (long long)cnt);
                    // the traversal keeps a node's hit triangles as a 32-bit mask over offsets from triBase
                    CWPB_CHECK((m & 31u) + cnt <= 32, CWP_ERR_INVALID, "CWBVH node %lld slot %d: leaf offset %u + %lld triangles exceeds 32", (long long)n, s, m & 31u, (long long)cnt);
                } else if (m) {
                    CWPB_CHECK(imask & (1u << s), CWP_ERR_INVALID, "CWBVH node %lld slot %d: internal child without imask bit", (long long)n, s);
                }
            }
        }
        *variantOut = 8;
    }
    return CWP_OK;
}

bool cwbvh_breadth_first(const float* in, int64_t nNodes, std::vector<float>& out, int levelEnd[4]) {
    out.assign((size_t)nNodes * 20, 0.f);
    std::vector<int32_t> order; order.reserve((size_t)nNodes);   // old index of each new index
    std::vector<int> level; level.reserve((size_t)nNodes);
    std::vector<char> seen((size_t)nNodes, 0);
    order.push_back(0); level.push_back(0); seen[0] = 1;
    for (size_t q = 0; q < order.size(); q++) {
        const int32_t* w = reinterpret_cast<const int32_t*>(in) + (int64_t)order[q] * 20;
        const int nInt = __builtin_popcount((uint32_t)w[3] >> 24);
        const int32_t newBase = (int32_t)order.size();
        for (int c = 0; c < nInt; c++) {
            const int32_t old = w[4] + c;   // in range: validate_nodes checked every child group
            if (seen[old]) return false;    // a node with two parents: not a tree
            seen[old] = 1; order.push_back(old); level.push_back(level[q] + 1);
        }
        int32_t* o = reinterpret_cast<int32_t*>(out.data()) + (int64_t)q * 20;
        memcpy(o, w, 80);
        if (nInt) o[4] = newBase;
    }
    if ((int64_t)order.size() != nNodes) return false;   // unreachable nodes
    for (int L = 0; L < 4; L++) { int64_t k = 0; while (k < (int64_t)level.size() && level[k] <= L) k++; levelEnd[L] = (int)k; }
    return true;
}

void free_scene(DeviceScene& s) {
    if (s.arena) { cudaSetDevice(s.device); cudaFree(s.arena); }
    s = DeviceScene();
}

int upload_scene(const cwp_scene_buffers* s, int tri, int device, DeviceScene& out) {
    CWPB_CHECK(s, CWP_ERR_INVALID, "scene buffers are NULL");
    CWPB_CHECK(tri == 0 || tri == 1, CWP_ERR_INVALID, "tri must be 0 (Moller-Trumbore) or 1 (Woop)");
    CWPB_CHECK(s->tris && s->n_tris > 0, CWP_ERR_INVALID, "scene has no triangles");
    CWPB_CHECK(tri == 0 || s->woop, CWP_ERR_INVALID, "Woop triangle test requested without Woop rows");
    int variant = 2;
    if (int rc = validate_nodes(s->nodes, s->n_node_float4, s->node_stride, s->n_tris, &variant)) return rc;
    free_scene(out);
    out.device = device; out.variant = variant; out.tri = tri;
    out.nNodes = s->n_node_float4 / s->node_stride; out.nTris = s->n_tris;
    CWPB_CUDA(cudaSetDevice(device));
    std::vector<float3> alb;
    for (int i = 0; i < s->n_albedo; i++) alb.push_back(make_float3(s->albedo[3 * i], s->albedo[3 * i + 1], s->albedo[3 * i + 2]));
    if (alb.empty()) alb.push_back(make_float3(0.8f, 0.8f, 0.8f));
    out.nAlbedo = (int)alb.size();
    // one allocation, the traversal's data first (nodes, leaf rows, triangles, exact corners), so that a single L2
    // access-policy window can cover what every ray reads
    struct Part { void** dst; const void* src; size_t bytes; };
    const size_t tb = (size_t)s->n_tris * 48;
    std::vector<float> bfs;
    const float* nodeSrc = s->nodes;
    if (variant == 8) {
        CWPB_CHECK(cwbvh_breadth_first(s->nodes, out.nNodes, bfs, out.levelEnd), CWP_ERR_INVALID,
                   "CWBVH of %lld nodes is not a tree rooted at node 0 (a node unreachable or with two parents)", (long long)out.nNodes);
        nodeSrc = bfs.data();
    }
    const Part parts[] = { { (void**)&out.nodes, nodeSrc, (size_t)s->n_node_float4 * 16 }, { (void**)&out.woop, s->woop, s->woop ? tb : 0 },
                           { (void**)&out.tris, s->tris, tb }, { (void**)&out.verts, s->verts, s->verts ? tb : 0 },
                           { (void**)&out.nrm, s->nrm, s->nrm ? tb : 0 }, { (void**)&out.albedo, alb.data(), alb.size() * sizeof(float3) } };
    size_t total = 0, hot = 0;
    for (int i = 0; i < 6; i++) { total += (parts[i].bytes + 255) & ~(size_t)255; if (i == 3) hot = total; }
    cudaError_t e = cudaMalloc(&out.arena, total);
    if (e == cudaSuccess) {
        out.bytes = total; out.hotBytes = hot;
        size_t off = 0;
        for (int i = 0; i < 6 && e == cudaSuccess; i++) {
            if (!parts[i].bytes) { *parts[i].dst = nullptr; continue; }
            *parts[i].dst = static_cast<char*>(out.arena) + off;
            e = cudaMemcpy(*parts[i].dst, parts[i].src, parts[i].bytes, cudaMemcpyHostToDevice);
            off += (parts[i].bytes + 255) & ~(size_t)255;
        }
    }
    if (e != cudaSuccess) { free_scene(out); return set_error(e == cudaErrorMemoryAllocation ? CWP_ERR_NOMEM : CWP_ERR_CUDA, "scene upload: %s", cudaGetErrorString(e)); }
    // every material id referenced by a triangle must have an albedo entry
    const int32_t* tw = reinterpret_cast<const int32_t*>(s->tris);
    for (int64_t t = 0; t < s->n_tris; t++) {
        int32_t mat = tw[t * 12 + 7];
        if (mat < 0 || mat >= out.nAlbedo) { free_scene(out); return set_error(CWP_ERR_INVALID, "triangle %lld: material %d has no albedo entry", (long long)t, mat); }
    }
    return CWP_OK;
}

// ---------------- ray-batch kernels ----------------
static constexpr int kBatchBlock = 128;

template <int V, int TRI>
__global__ void __launch_bounds__(kBatchBlock) k_trace_closest(const float4* __restrict__ nodes, const float4* __restrict__ tv, const float4* __restrict__ ro,
                                                               const float4* __restrict__ rd, float4* __restrict__ hits, long long n, int* err) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 O = __ldcs(ro + i), D = __ldcs(rd + i);
    float t = D.w, u = 0.f, v = 0.f; int tri = -1, e = 0;
    trace_ray<V, false, TRI>(nodes, tv, xyz(O), xyz(D), O.w, t, tri, u, v, 0, e);
    __stcs(hits + i, make_float4(t, u, v, __int_as_float(tri)));
    if (e) atomicOr(err, e);
}

template <int V, int TRI>
__global__ void __launch_bounds__(kBatchBlock) k_trace_any(const float4* __restrict__ nodes, const float4* __restrict__ tv, const float4* __restrict__ ro,
                                                           const float4* __restrict__ rd, int* __restrict__ occ, long long n, int* err) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 O = __ldcs(ro + i), D = __ldcs(rd + i);
    float t = D.w, u = 0.f, v = 0.f; int tri = -1, e = 0;
    trace_ray<V, true, TRI>(nodes, tv, xyz(O), xyz(D), O.w, t, tri, u, v, 0, e);
    __stcs(occ + i, tri);
    if (e) atomicOr(err, e);
}

// Persistent variant with dynamic refill: each lane advances its ray one node visit per step and the warp refetches
// rays (one atomic on *fetch) once kRefillBatch lanes are idle. *fetch must be zero at launch.
#ifndef CWPB_BATCH_REFILL
#define CWPB_BATCH_REFILL 12
#endif
static constexpr int kRefillBatch = CWPB_BATCH_REFILL;
__device__ __forceinline__ unsigned lane_lt() { unsigned m; asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m)); return m; }

template <int V, int TRI, bool ANY>
__global__ void __launch_bounds__(kBatchBlock, 8) k_trace_rf(const float4* __restrict__ nodes, const float4* __restrict__ tv, const float4* __restrict__ ro,
                                                             const float4* __restrict__ rd, float4* __restrict__ hits, int* __restrict__ occ, long long n, int* fetch, int* err) {
    const int lane = threadIdx.x & 31;
    int e = 0;
    TravState<V, ANY, TRI> ray; typename TravState<V, ANY, TRI>::Stack stack;
    long long k = -1; bool fin = false, drained = false;
    for (;;) {
        if (fin) {
            if (ANY) __stcs(occ + k, ray.hitTri);
            else __stcs(hits + k, make_float4(ray.hitT, ray.hu, ray.hv, __int_as_float(ray.hitTri)));
            k = -1; fin = false;
        }
        if (!drained) {
            const bool need = k < 0;
            const unsigned nm = __ballot_sync(0xffffffffu, need);
            if (nm) {
                const int leader = __ffs(nm) - 1;
                long long base = 0;
                if (lane == leader) base = atomicAdd((unsigned long long*)fetch, (unsigned long long)__popc(nm));
                base = __shfl_sync(0xffffffffu, base, leader);
                const long long kk = base + __popc(nm & lane_lt());
                if (need && kk < n) { k = kk; const float4 O = __ldcs(ro + k), D = __ldcs(rd + k); ray.begin(xyz(O), xyz(D), O.w, D.w, 0); }
                drained = __any_sync(0xffffffffu, need && kk >= n);
            }
        }
        if (!__any_sync(0xffffffffu, k >= 0)) break;
        for (;;) {
            if (k >= 0 && !fin) fin = ray.step(nodes, tv, stack, e);
            const unsigned busy = __ballot_sync(0xffffffffu, k >= 0 && !fin);
            if (!busy || (!drained && 32 - __popc(busy) >= kRefillBatch)) break;
        }
    }
    if (e) atomicOr(err, e);
}

// Precision form, closest hits: persistent with refill, with the watertight triangle tests shared out over the warp.
// Each iteration every active lane visits one node (TravState<16>::visit: f16 slab tests; the hit leaves' triangles
// become its pending mask). Then the warp tests all lanes' pending triangles together, 32 per round: slot i of the
// warp's concatenated list goes to lane i mod 32, which takes the owning ray's data by shuffles. A lane whose test hits
// in the owner's interval proposes (t, slot) to the owner by a 64-bit atomic minimum in shared memory, and the owner
// takes the smallest t, the earliest slot among equal ones. That is the hit the owner's own tests in slot order keep
// (a later triangle replaces the hit only when strictly closer), so every ray gets the result of the sequential
// traversal (TravState<16>::step) bit for bit. Rounds of one owner follow one another, each against the interval the
// previous round left. The watertight test costs several slab tests, and one lane's run of tests no longer holds the
// warp's other lanes: 8% less time than one test per lane and step on the 1M-ray batch. Any-hit rays keep that form
// (k_trace_rf<16, 1, true>): they stop at their first hit, and sharing their tests measured 6% slower.
// The warp refills once 8 lanes are idle (12: +1.5%, 16: +5% time).
static constexpr int kRefillPrec = 8;
__device__ __forceinline__ unsigned long long wt_key(float t, int slot) {
    const unsigned u = __float_as_uint(t);
    return ((unsigned long long)((u & 0x80000000u) ? ~u : (u | 0x80000000u)) << 32) | (unsigned)slot;   // float order, then slot
}

__global__ void __launch_bounds__(kBatchBlock, 8) k_trace_prec_rf(const float4* __restrict__ nodes, const float4* __restrict__ vt, const float4* __restrict__ ro,
                                                                  const float4* __restrict__ rd, float4* __restrict__ hits, long long n, int* fetch, int* err) {
    __shared__ unsigned long long best[kBatchBlock];   // per lane: the smallest (t, slot) its pending triangles gave this round
    const int lane = threadIdx.x & 31;
    unsigned long long* myBest = best + threadIdx.x;
    int e = 0;
    TravState<16, false, 1> ray; TravState<16, false, 1>::Stack stack;
    ray.tm = ray.tb = 0u; ray.node = -1;   // (a lane without a ray owns no slot; its fields are shuffled but not used)
    long long k = -1; bool fin = false, drained = false;
    for (;;) {
        if (fin) { __stcs(hits + k, make_float4(ray.hitT, ray.hu, ray.hv, __int_as_float(ray.hitTri))); k = -1; fin = false; }
        if (!drained) {
            const bool need = k < 0;
            const unsigned nm = __ballot_sync(0xffffffffu, need);
            if (nm) {
                const int leader = __ffs(nm) - 1;
                long long base = 0;
                if (lane == leader) base = atomicAdd((unsigned long long*)fetch, (unsigned long long)__popc(nm));
                base = __shfl_sync(0xffffffffu, base, leader);
                const long long kk = base + __popc(nm & lane_lt());
                if (need && kk < n) { k = kk; const float4 O = __ldcs(ro + k), D = __ldcs(rd + k); ray.begin(xyz(O), xyz(D), O.w, D.w, 0); }
                drained = __any_sync(0xffffffffu, need && kk >= n);
            }
        }
        if (!__any_sync(0xffffffffu, k >= 0)) break;
        for (;;) {
            // one node visit per active ray (true: the ray stopped on a bound; its pending triangles are dropped)
            if (k >= 0 && !fin && ray.visit(nodes, stack, e)) fin = true;
            const unsigned pend = (k >= 0 && !fin) ? ray.tm : 0u;
            ray.tm = 0;
            // the warp's pending triangles, concatenated in lane order: this lane's are slots [incl - cnt, incl)
            const int cnt = __popc(pend);
            int incl = cnt;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) { const int v = __shfl_up_sync(0xffffffffu, incl, off); if (lane >= off) incl += v; }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            for (int base = 0; base < total; base += 32) {
                *myBest = ~0ull;
                __syncwarp();
                const int slot = base + lane;
                int owner = 0;   // the first lane whose inclusive count exceeds slot
#pragma unroll
                for (int step = 16; step; step >>= 1) if (__shfl_sync(0xffffffffu, incl, owner + step - 1) <= slot) owner += step;
                const unsigned om = __shfl_sync(0xffffffffu, pend, owner);
                const int oFirst = __shfl_sync(0xffffffffu, incl - cnt, owner);
                const int oTb = __shfl_sync(0xffffffffu, (int)ray.tb, owner);
                const float3 o = make_float3(__shfl_sync(0xffffffffu, ray.o.x, owner), __shfl_sync(0xffffffffu, ray.o.y, owner), __shfl_sync(0xffffffffu, ray.o.z, owner));
                WtRay w;
                const int kk = __shfl_sync(0xffffffffu, ray.wt.kx | (ray.wt.ky << 2) | (ray.wt.kz << 4), owner);
                w.kx = kk & 3; w.ky = (kk >> 2) & 3; w.kz = kk >> 4;
                w.sx = __shfl_sync(0xffffffffu, ray.wt.sx, owner); w.sy = __shfl_sync(0xffffffffu, ray.wt.sy, owner); w.sz = __shfl_sync(0xffffffffu, ray.wt.sz, owner);
                const float tmin = __shfl_sync(0xffffffffu, ray.tmin, owner), tmax = __shfl_sync(0xffffffffu, ray.hitT, owner);
                // the owner's (slot - oFirst)-th pending triangle in bit order (lanes past the list compute an unused index)
                const int t = oTb + (int)__fns(om, 0, slot - oFirst + 1);
                float tt = 0.f, u = 0.f, v = 0.f;
                if (slot < total && wt_test(vt, t, o, w, tmin, tmax, tt, u, v)) atomicMin(best + (threadIdx.x - lane) + owner, wt_key(tt, slot));
                __syncwarp();
                const unsigned long long b = *myBest;
                const int src = b == ~0ull ? lane : (int)(b & 31u);   // the lane that tested this ray's winning slot
                const float wT = __shfl_sync(0xffffffffu, tt, src), wU = __shfl_sync(0xffffffffu, u, src), wV = __shfl_sync(0xffffffffu, v, src);
                const int wTri = __shfl_sync(0xffffffffu, t, src);
                if (b != ~0ull) { ray.hitT = wT; ray.hitTri = wTri; ray.hu = wU; ray.hv = wV; ray.set_tint(); }
                __syncwarp();
            }
            if (k >= 0 && !fin && ray.node < 0) fin = true;
            const unsigned busy = __ballot_sync(0xffffffffu, k >= 0 && !fin);
            if (!busy || (!drained && 32 - __popc(busy) >= kRefillPrec)) break;
        }
    }
    if (e) atomicOr(err, e);
}

template <bool ANY>
static int launch_batch(const DeviceScene& s, const float4* o, const float4* d, void* out, long long n, int* err, cudaStream_t st, int* fetch, int refillGrid) {
    if (n <= 0) return CWP_OK;
    const float4* tv0 = s.leafData();
    if (fetch && s.variant != 4) {   // persistent refill kernels (BVH2, CWBVH, precision form)
        CWPB_CUDA(cudaMemsetAsync(fetch, 0, sizeof(unsigned long long), st));
#define CWPB_R(VV, TT) k_trace_rf<VV, TT, ANY><<<refillGrid, kBatchBlock, 0, st>>>(s.nodes, tv0, o, d, (float4*)out, (int*)out, n, fetch, err)
        if (s.precise) {   // closest hits share their triangle tests over the warp; any-hit rays keep their own
            if (ANY) CWPB_R(16, 1);
            else k_trace_prec_rf<<<refillGrid, kBatchBlock, 0, st>>>(s.nodes, tv0, o, d, (float4*)out, n, fetch, err);
        }
        else if (s.variant == 2) { if (s.tri) CWPB_R(2, 1); else CWPB_R(2, 0); }
        else { if (s.tri) CWPB_R(8, 1); else CWPB_R(8, 0); }
#undef CWPB_R
        CWPB_CUDA(cudaGetLastError());
        return CWP_OK;
    }
    const unsigned grid = (unsigned)((n + kBatchBlock - 1) / kBatchBlock);
    const float4* tv = s.leafData();
#define CWPB_L(VV, TT) do { if (ANY) k_trace_any<VV, TT><<<grid, kBatchBlock, 0, st>>>(s.nodes, tv, o, d, (int*)out, n, err); \
                            else k_trace_closest<VV, TT><<<grid, kBatchBlock, 0, st>>>(s.nodes, tv, o, d, (float4*)out, n, err); } while (0)
    if (s.precise) CWPB_L(16, 1);
    else if (s.variant == 2) { if (s.tri) CWPB_L(2, 1); else CWPB_L(2, 0); }
    else if (s.variant == 4) { if (s.tri) CWPB_L(4, 1); else CWPB_L(4, 0); }
    else { if (s.tri) CWPB_L(8, 1); else CWPB_L(8, 0); }
#undef CWPB_L
    CWPB_CUDA(cudaGetLastError());
    return CWP_OK;
}

// FP64 reference traversal of a ray batch (the precision form's oracle): t in double, leaf-order triangle or -1
template <bool ANY>
__global__ void __launch_bounds__(kBatchBlock) k_trace_fp64(const float4* __restrict__ nodes, const float4* __restrict__ verts, const float4* __restrict__ ro,
                                                            const float4* __restrict__ rd, double* __restrict__ tOut, int* __restrict__ triOut, long long n, int* err) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 O = ro[i], D = rd[i];
    double t = D.w; int tri = -1, e = 0;
    trav_fp64<ANY>(nodes, verts, make_double3(O.x, O.y, O.z), make_double3(D.x, D.y, D.z), (double)O.w, t, tri, e);
    tOut[i] = t; triOut[i] = tri;
    if (e) atomicOr(err, e);
}

}  // namespace cwpb

using namespace cwpb;

struct cwp_accel {
    DeviceScene scene;
    int* err = nullptr;                 // device traversal status bits
    int* fetch = nullptr;               // refill kernels' ray cursor (8 bytes)
    int refillGrid = 0;                 // resident blocks of the refill kernels
    bool refill = true;                 // use them (cwp_accel_set_traversal; set at creation by the automatic rule)
    cudaStream_t st = nullptr, st2 = nullptr;   // streams of the host-buffer entry points (chunks alternate)
    int* fetch2 = nullptr;              // their refill cursors, one 8-byte counter per stream
    cudaEvent_t e0 = nullptr, e1 = nullptr, ej = nullptr;
    float4 *bo = nullptr, *bd = nullptr; void* bh = nullptr; size_t cap = 0;   // staging for host-buffer calls
};

extern "C" int cwp_accel_create(const cwp_scene_buffers* s, int32_t tri, int32_t device, cwp_accel** out) {
    CWPB_CHECK(out, CWP_ERR_INVALID, "out is NULL");
    *out = nullptr;
    cwp_accel* a = new cwp_accel();
    int rc = upload_scene(s, tri, device, a->scene);
    if (rc) { delete a; return rc; }
    cudaError_t e = cudaMalloc(&a->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(a->err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&a->fetch, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&a->fetch2, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess && a->scene.variant != 4) {
        int nSM = 0, b = 0;
        e = cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, device);
        const bool t = a->scene.tri == 1;
        if (e == cudaSuccess) e = a->scene.variant == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, t ? k_trace_rf<2, 1, false> : k_trace_rf<2, 0, false>, kBatchBlock, 0)
                                                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, t ? k_trace_rf<8, 1, false> : k_trace_rf<8, 0, false>, kBatchBlock, 0);
        a->refillGrid = b * nSM;
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&a->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&a->st2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&a->e0);
    if (e == cudaSuccess) e = cudaEventCreate(&a->e1);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&a->ej, cudaEventDisableTiming);
    if (e != cudaSuccess) { cwp_accel_destroy(a); return set_error(CWP_ERR_CUDA, "accel setup: %s", cudaGetErrorString(e)); }
    a->refill = a->scene.variant == 8;
    *out = a;
    return CWP_OK;
}

extern "C" void cwp_accel_destroy(cwp_accel* a) {
    if (!a) return;
    cudaSetDevice(a->scene.device);
    if (a->st) cudaStreamSynchronize(a->st);
    if (a->st2) cudaStreamSynchronize(a->st2);
    cudaFree(a->err); cudaFree(a->fetch); cudaFree(a->fetch2); cudaFree(a->bo); cudaFree(a->bd); cudaFree(a->bh);
    if (a->st) cudaStreamDestroy(a->st);
    if (a->st2) cudaStreamDestroy(a->st2);
    if (a->e0) cudaEventDestroy(a->e0);
    if (a->e1) cudaEventDestroy(a->e1);
    if (a->ej) cudaEventDestroy(a->ej);
    free_scene(a->scene);
    delete a;
}

extern "C" int cwp_trace_closest(cwp_accel* a, const float* o, const float* d, float* hits, int64_t n, void* stream) {
    CWPB_CHECK(a, CWP_ERR_INVALID, "accel is NULL");
    CWPB_CHECK(n >= 0, CWP_ERR_INVALID, "negative ray count");
    CWPB_CHECK(n == 0 || (o && d && hits), CWP_ERR_INVALID, "NULL ray or hit buffer");
    CWPB_CUDA(cudaSetDevice(a->scene.device));
    return launch_batch<false>(a->scene, (const float4*)o, (const float4*)d, hits, n, a->err, (cudaStream_t)stream, a->refill ? a->fetch : nullptr, a->refillGrid);
}

extern "C" int cwp_trace_any(cwp_accel* a, const float* o, const float* d, int32_t* occ, int64_t n, void* stream) {
    CWPB_CHECK(a, CWP_ERR_INVALID, "accel is NULL");
    CWPB_CHECK(n >= 0, CWP_ERR_INVALID, "negative ray count");
    CWPB_CHECK(n == 0 || (o && d && occ), CWP_ERR_INVALID, "NULL ray or result buffer");
    CWPB_CUDA(cudaSetDevice(a->scene.device));
    return launch_batch<true>(a->scene, (const float4*)o, (const float4*)d, occ, n, a->err, (cudaStream_t)stream, a->refill ? a->fetch : nullptr, a->refillGrid);
}

// Host-buffer calls pipeline the copies with the traversal: the batch is cut into up to 8 chunks of at least 256k rays
// that alternate over two streams, so one chunk's rays travel in while the one before it is traced and the results
// of the one before that travel out (separate copy engines per direction).
static constexpr int64_t kHostChunkMin = 1 << 18;
template <bool ANY>
static int host_call(cwp_accel* a, const float* o, const float* d, void* res, int64_t n, float* ms) {
    CWPB_CHECK(a, CWP_ERR_INVALID, "accel is NULL");
    CWPB_CHECK(n >= 0, CWP_ERR_INVALID, "negative ray count");
    CWPB_CHECK(n == 0 || (o && d && res), CWP_ERR_INVALID, "NULL host buffer");
    if (ms) *ms = 0.f;
    if (n == 0) return CWP_OK;
    CWPB_CUDA(cudaSetDevice(a->scene.device));
    const size_t resBytes = ANY ? 4 : 16;
    if ((size_t)n > a->cap) {
        cudaFree(a->bo); cudaFree(a->bd); cudaFree(a->bh); a->bo = a->bd = nullptr; a->bh = nullptr; a->cap = 0;
        CWPB_CUDA(cudaMalloc(&a->bo, (size_t)n * 16)); CWPB_CUDA(cudaMalloc(&a->bd, (size_t)n * 16)); CWPB_CUDA(cudaMalloc(&a->bh, (size_t)n * 16));
        a->cap = (size_t)n;
    }
    const int nc = (int)std::max<int64_t>(1, std::min<int64_t>(8, n / kHostChunkMin));
    const cudaStream_t ss[2] = { a->st, a->st2 };
    CWPB_CUDA(cudaEventRecord(a->e0, a->st));
    CWPB_CUDA(cudaStreamWaitEvent(a->st2, a->e0, 0));
    for (int c = 0; c < nc; c++) {
        const int64_t b0 = n * c / nc, m = n * (c + 1) / nc - b0;
        const cudaStream_t s = ss[c & 1];
        char* out = (char*)a->bh + (size_t)b0 * resBytes;
        CWPB_CUDA(cudaMemcpyAsync(a->bo + b0, o + 4 * b0, (size_t)m * 16, cudaMemcpyHostToDevice, s));
        CWPB_CUDA(cudaMemcpyAsync(a->bd + b0, d + 4 * b0, (size_t)m * 16, cudaMemcpyHostToDevice, s));
        if (int rc = launch_batch<ANY>(a->scene, a->bo + b0, a->bd + b0, out, m, a->err, s, a->refill ? a->fetch2 + 2 * (c & 1) : nullptr, a->refillGrid)) return rc;
        CWPB_CUDA(cudaMemcpyAsync((char*)res + (size_t)b0 * resBytes, out, (size_t)m * resBytes, cudaMemcpyDeviceToHost, s));
    }
    CWPB_CUDA(cudaEventRecord(a->ej, a->st2));
    CWPB_CUDA(cudaStreamWaitEvent(a->st, a->ej, 0));
    CWPB_CUDA(cudaEventRecord(a->e1, a->st));
    CWPB_CUDA(cudaEventSynchronize(a->e1));
    if (ms) CWPB_CUDA(cudaEventElapsedTime(ms, a->e0, a->e1));
    return CWP_OK;
}

extern "C" int cwp_trace_closest_host(cwp_accel* a, const float* o, const float* d, float* hits, int64_t n, float* ms) { return host_call<false>(a, o, d, hits, n, ms); }
extern "C" int cwp_trace_any_host(cwp_accel* a, const float* o, const float* d, int32_t* occ, int64_t n, float* ms) { return host_call<true>(a, o, d, occ, n, ms); }

extern "C" int cwp_accel_set_traversal(cwp_accel* a, int32_t mode) {
    CWPB_CHECK(a, CWP_ERR_INVALID, "accel is NULL");
    CWPB_CHECK(mode >= 0 && mode <= 2, CWP_ERR_INVALID, "traversal %d is not 0, 1 or 2", mode);
    CWPB_CHECK(!(mode == 1 && a->scene.variant == 4), CWP_ERR_INVALID, "refill traversal is available for BVH2 and CWBVH, not BVH4");
    // auto: refill for CWBVH (measured faster on incoherent batches), one ray per thread for BVH2 and BVH4
    a->refill = mode == 1 || (mode == 0 && a->scene.variant == 8);
    return CWP_OK;
}

extern "C" int cwp_accel_set_precision(cwp_accel* a, int32_t mode) {
    CWPB_CHECK(a, CWP_ERR_INVALID, "accel is NULL");
    CWPB_CHECK(mode == 0 || mode == 1, CWP_ERR_INVALID, "precision mode %d is not 0 (plain) or 1 (precision form)", mode);
    CWPB_CHECK(mode == 0 || (a->scene.variant == 8 && a->scene.verts), CWP_ERR_INVALID, "the precision form needs a CWBVH and the exact corner buffer (cwp_scene_buffers.verts)");
    int nSM = 0, b = 0;
    CWPB_CUDA(cudaSetDevice(a->scene.device));
    CWPB_CUDA(cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, a->scene.device));
    if (mode == 1) {   // closest hits: the shared-test kernel; any-hit: k_trace_rf<16, 1, true>; one grid fits both
        int b2 = 0;
        CWPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_trace_prec_rf, kBatchBlock, 0));
        CWPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, k_trace_rf<16, 1, true>, kBatchBlock, 0));
        b = std::min(b, b2);
    } else CWPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, a->scene.tri == 1 ? k_trace_rf<8, 1, false> : k_trace_rf<8, 0, false>, kBatchBlock, 0));
    a->scene.precise = mode == 1;
    a->refillGrid = b * nSM;
    return CWP_OK;
}

extern "C" int cwp_trace_fp64(cwp_accel* a, int32_t any_hit, const float* d_o, const float* d_d, double* d_t, int32_t* d_tri, int64_t n, void* stream) {
    CWPB_CHECK(a, CWP_ERR_INVALID, "accel is NULL");
    CWPB_CHECK(n >= 0, CWP_ERR_INVALID, "negative ray count");
    CWPB_CHECK(a->scene.variant == 8 && a->scene.verts, CWP_ERR_INVALID, "the FP64 traversal needs a CWBVH and the exact corner buffer");
    if (n == 0) return CWP_OK;
    CWPB_CHECK(d_o && d_d && d_t && d_tri, CWP_ERR_INVALID, "NULL buffer");
    CWPB_CUDA(cudaSetDevice(a->scene.device));
    const unsigned grid = (unsigned)((n + kBatchBlock - 1) / kBatchBlock);
    if (any_hit) k_trace_fp64<true><<<grid, kBatchBlock, 0, (cudaStream_t)stream>>>(a->scene.nodes, a->scene.verts, (const float4*)d_o, (const float4*)d_d, d_t, d_tri, n, a->err);
    else k_trace_fp64<false><<<grid, kBatchBlock, 0, (cudaStream_t)stream>>>(a->scene.nodes, a->scene.verts, (const float4*)d_o, (const float4*)d_d, d_t, d_tri, n, a->err);
    CWPB_CUDA(cudaGetLastError());
    return CWP_OK;
}

extern "C" int cwp_accel_status(cwp_accel* a) {
    CWPB_CHECK(a, CWP_ERR_INVALID, "accel is NULL");
    CWPB_CUDA(cudaSetDevice(a->scene.device));
    CWPB_CUDA(cudaDeviceSynchronize());
    int h = 0;
    CWPB_CUDA(cudaMemcpy(&h, a->err, sizeof(int), cudaMemcpyDeviceToHost));
    CWPB_CUDA(cudaMemset(a->err, 0, sizeof(int)));
    CWPB_CHECK(h == 0, CWP_ERR_TRAVERSAL, "traversal stopped early on some rays (status bits 0x%x: 1 = stack bound, 2 = visit budget)", h);
    return CWP_OK;
}
