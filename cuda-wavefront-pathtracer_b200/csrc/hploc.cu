// hploc.cu - segmented H-PLOC: many BVH2s built on the device in one pass (see hploc.h).
#include "hploc.h"
#include "vecmath.h"
#include <cub/device/device_radix_sort.cuh>
#include <vector>

namespace cwpb {

static constexpr int kPlocT = 16;          // clusters kept per LBVH subtree: half a warp, so both children fit one warp
static constexpr int kPlocR = 8;           // PLOC nearest-neighbour search radius (positions)
static constexpr int kClimbBlock = 128;
static constexpr unsigned kFull = 0xffffffffu;

// float <-> unsigned map that preserves order, for atomicMin / atomicMax on float bounds
__device__ __forceinline__ unsigned ord_of(float f) { const unsigned u = __float_as_uint(f); return (u >> 31) ? ~u : (u | 0x80000000u); }
__device__ __forceinline__ float float_of(unsigned o) { return __uint_as_float((o >> 31) ? (o & 0x7fffffffu) : ~o); }
__device__ __forceinline__ unsigned lanes_below() { unsigned m; asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m)); return m; }

// segment of primitive i: the largest s with segFirst[s] <= i
__device__ __forceinline__ int seg_of(const int* __restrict__ segFirst, int nSeg, int i) {
    int lo = 0, hi = nSeg - 1;
    while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (__ldg(segFirst + mid) <= i) lo = mid; else hi = mid - 1; }
    return lo;
}

__global__ void k_seg_init(unsigned* cbox, int* counters, const int* __restrict__ segFirst, int nSeg) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nSeg) return;
    for (int a = 0; a < 3; a++) { cbox[6 * s + a] = 0xffffffffu; cbox[6 * s + 3 + a] = 0u; }
    const int f = segFirst[s], m = segFirst[s + 1] - f;
    counters[s] = 2 * f - s + m;   // internal nodes follow the segment's m leaves
}

// per-segment centroid bounds; a warp whose primitives all lie in one segment reduces before its atomics
__global__ void k_seg_bounds(const float4* __restrict__ lo, const float4* __restrict__ hi, int n, const int* __restrict__ segFirst, int nSeg, unsigned* cbox) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = i < n;
    const int s = ok ? seg_of(segFirst, nSeg, i) : -1;
    float3 c = f3(0.f, 0.f, 0.f);
    if (ok) { const float4 a = lo[i], b = hi[i]; c = f3((a.x + b.x) * 0.5f, (a.y + b.y) * 0.5f, (a.z + b.z) * 0.5f); }
    const int s0 = __shfl_sync(kFull, s, 0);
    if (__all_sync(kFull, !ok || s == s0)) {
        float mn[3] = { ok ? c.x : 3.4e38f, ok ? c.y : 3.4e38f, ok ? c.z : 3.4e38f }, mx[3] = { ok ? c.x : -3.4e38f, ok ? c.y : -3.4e38f, ok ? c.z : -3.4e38f };
#pragma unroll
        for (int a = 0; a < 3; a++)
            for (int k = 16; k > 0; k >>= 1) { mn[a] = fminf(mn[a], __shfl_xor_sync(kFull, mn[a], k)); mx[a] = fmaxf(mx[a], __shfl_xor_sync(kFull, mx[a], k)); }
        if ((threadIdx.x & 31) == 0 && s0 >= 0)
            for (int a = 0; a < 3; a++) { atomicMin(&cbox[6 * s0 + a], ord_of(mn[a])); atomicMax(&cbox[6 * s0 + 3 + a], ord_of(mx[a])); }
    } else if (ok) {
        const float cc[3] = { c.x, c.y, c.z };
        for (int a = 0; a < 3; a++) { atomicMin(&cbox[6 * s + a], ord_of(cc[a])); atomicMax(&cbox[6 * s + 3 + a], ord_of(cc[a])); }
    }
}

// bit b of v -> bit 3 b
__device__ __forceinline__ unsigned long long spread3(unsigned v) {
    unsigned long long r = 0;
#pragma unroll
    for (int b = 0; b < 18; b++) r |= (unsigned long long)((v >> b) & 1u) << (3 * b);
    return r;
}

__global__ void k_seg_keys(const float4* __restrict__ lo, const float4* __restrict__ hi, int n, const int* __restrict__ segFirst, int nSeg,
                           const unsigned* __restrict__ cbox, unsigned long long* keys, int* vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = seg_of(segFirst, nSeg, i);
    const float4 a = lo[i], b = hi[i];
    const float c[3] = { (a.x + b.x) * 0.5f, (a.y + b.y) * 0.5f, (a.z + b.z) * 0.5f };
    unsigned q[3];
    for (int k = 0; k < 3; k++) {
        const float l = float_of(cbox[6 * s + k]), h = float_of(cbox[6 * s + 3 + k]), e = h - l;
        const float u = e > 0.f ? (c[k] - l) / e : 0.f;
        q[k] = (unsigned)fminf(fmaxf(u * 262144.f, 0.f), 262143.f);
    }
    keys[i] = ((unsigned long long)s << kMortonBits) | (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
    vals[i] = i;
}

__global__ void k_seg_leaves(const float4* __restrict__ lo, const float4* __restrict__ hi, const unsigned long long* __restrict__ keys,
                             const int* __restrict__ vals, int n, const int* __restrict__ segFirst, float4* nodes, int* count, int* C, int* bounds) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = vals[i], s = (int)(keys[i] >> kMortonBits), f = segFirst[s];
    const int node = 2 * f - s + (i - f);
    const float4 a = lo[p], b = hi[p];
    nodes[2 * node] = make_float4(a.x, a.y, a.z, __int_as_float(p));
    nodes[2 * node + 1] = make_float4(b.x, b.y, b.z, __int_as_float(-1));
    count[node] = 1;
    C[i] = node; bounds[i] = -1;
}

struct PlocScratch { int id[32]; int cnt[32]; float box[32 * 6]; };

__device__ __forceinline__ float half_area(float3 l, float3 h) { const float3 e = h - l; return e.x * e.y + e.y * e.z + e.z * e.x; }
__device__ __forceinline__ float3 shfl3(float3 v, int src) { return f3(__shfl_sync(kFull, v.x, src), __shfl_sync(kFull, v.y, src), __shfl_sync(kFull, v.z, src)); }
__device__ __forceinline__ float3 shfl3_down(float3 v, int d) { return f3(__shfl_down_sync(kFull, v.x, d), __shfl_down_sync(kFull, v.y, d), __shfl_down_sync(kFull, v.z, d)); }

// The warp merges the clusters of LBVH range [L, R] (children [L, split] and [split + 1, R], clusters at the start of
// each child's range, unused slots -1) by PLOC until kPlocT clusters remain (1 for a segment root), allocating new
// nodes from *counter, and writes the survivors to the start of [L, R]. All 32 lanes take part.
__device__ void ploc_merge(int lane, int L, int R, int split, bool root, float4* nodes, int* count, int* C, int* counter, PlocScratch& ws) {
    const unsigned below = lanes_below();
    const int nL = min(split - L + 1, kPlocT), nR = min(R - split, kPlocT);
    const int slot = lane < nL ? L + lane : (lane < nL + nR ? split + 1 + (lane - nL) : -1);
    int id = slot >= 0 ? __ldcg(C + slot) : -1;
    const unsigned have = __ballot_sync(kFull, id >= 0);
    int num = __popc(have);
    if (id >= 0) ws.id[__popc(have & below)] = id;
    __syncwarp();
    id = lane < num ? ws.id[lane] : -1;
    __syncwarp();
    float3 lo = f3(0.f, 0.f, 0.f), hi = lo; int cnt = 0;
    if (id >= 0) {
        const float4 a = __ldcg(nodes + 2 * id), b = __ldcg(nodes + 2 * id + 1);
        lo = f3(a.x, a.y, a.z); hi = f3(b.x, b.y, b.z); cnt = __ldcg(count + id);
    }
    const int target = root ? 1 : kPlocT;
    while (num > target) {
        // nearest neighbour: pairs ordered by (merged area, lower lane, upper lane), so the best pair of the whole
        // list is mutual and every round merges at least one pair
        unsigned long long best = ~0ull;
#pragma unroll
        for (int r = 1; r <= kPlocR; r++) {
            const float3 olo = shfl3_down(lo, r), ohi = shfl3_down(hi, r);
            unsigned long long key = ~0ull;
            if (lane + r < num) key = ((unsigned long long)__float_as_uint(half_area(vmin(lo, olo), vmax(hi, ohi))) << 32) | ((unsigned)lane << 8) | (unsigned)(lane + r);
            best = key < best ? key : best;
            const unsigned long long up = __shfl_up_sync(kFull, key, r);
            if (lane >= r && up < best) best = up;
        }
        const int pa = (int)((best >> 8) & 0xffu), pb = (int)(best & 0xffu);
        const int nn = lane < num ? (pa == lane ? pb : pa) : lane;
        const int back = __shfl_sync(kFull, nn, nn & 31);
        const bool mutual = lane < num && nn != lane && back == lane;
        const bool lead = mutual && lane < nn;
        const float3 plo = shfl3(lo, nn & 31), phi = shfl3(hi, nn & 31);
        const int pid = __shfl_sync(kFull, id, nn & 31), pcnt = __shfl_sync(kFull, cnt, nn & 31);
        const unsigned leads = __ballot_sync(kFull, lead);
        int base = 0;
        if (lane == 0) base = atomicAdd(counter, __popc(leads));
        base = __shfl_sync(kFull, base, 0);
        if (lead) {
            const int nid = base + __popc(leads & below);
            lo = vmin(lo, plo); hi = vmax(hi, phi); cnt += pcnt;
            nodes[2 * nid] = make_float4(lo.x, lo.y, lo.z, __int_as_float(id));
            nodes[2 * nid + 1] = make_float4(hi.x, hi.y, hi.z, __int_as_float(pid));
            count[nid] = cnt;
            id = nid;
        }
        const bool keep = lane < num && !(mutual && !lead);
        const unsigned km = __ballot_sync(kFull, keep);
        if (keep) {
            const int k = __popc(km & below);
            ws.id[k] = id; ws.cnt[k] = cnt;
            ws.box[6 * k] = lo.x; ws.box[6 * k + 1] = lo.y; ws.box[6 * k + 2] = lo.z; ws.box[6 * k + 3] = hi.x; ws.box[6 * k + 4] = hi.y; ws.box[6 * k + 5] = hi.z;
        }
        __syncwarp();
        num = __popc(km);
        if (lane < num) {
            id = ws.id[lane]; cnt = ws.cnt[lane];
            lo = f3(ws.box[6 * lane], ws.box[6 * lane + 1], ws.box[6 * lane + 2]); hi = f3(ws.box[6 * lane + 3], ws.box[6 * lane + 4], ws.box[6 * lane + 5]);
        } else id = -1;
        __syncwarp();
    }
    if (slot >= 0) C[slot] = -1;
    __syncwarp();
    if (lane < num) C[L + lane] = id;
    __syncwarp();
}

// delta(R) < delta(L - 1), delta(i) = key[i] ^ key[i + 1] with position as the tie-break for equal keys
__device__ __forceinline__ bool parent_right(const unsigned long long* __restrict__ keys, int L, int R) {
    const unsigned long long a = keys[R] ^ keys[R + 1], b = keys[L - 1] ^ keys[L];
    if (a != b) return a < b;
    return (unsigned)(R ^ (R + 1)) < (unsigned)((L - 1) ^ L);
}

__global__ void __launch_bounds__(kClimbBlock) k_seg_hploc(float4* nodes, int* count, const unsigned long long* __restrict__ keys, int* C, int* bounds,
                                                           const int* __restrict__ segFirst, int* counters, int n) {
    __shared__ PlocScratch scratch[kClimbBlock / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool active = i < n;
    int s = 0, s0 = 0, s1 = 0;
    if (active) { s = (int)(keys[i] >> kMortonBits); s0 = segFirst[s]; s1 = segFirst[s + 1] - 1; if (s0 == s1) active = false; }
    int L = i, R = i;
    while (__any_sync(kFull, active)) {
        __syncwarp();
        __threadfence();   // this warp's node and cluster writes are visible before a parent is handed over
        int split = 0; bool merge = false;
        if (active) {
            const bool right = L == s0 || (R != s1 && parent_right(keys, L, R));
            int other;
            if (right) { split = R; other = atomicExch(&bounds[R], L); if (other >= 0) R = other; }
            else { split = L - 1; other = atomicExch(&bounds[L - 1], R); if (other >= 0) L = other; }
            if (other < 0) active = false;   // first child to arrive: the sibling's thread continues
            else { __threadfence(); merge = (R - L + 1 > kPlocT) || (L == s0 && R == s1); }
        }
        unsigned todo = __ballot_sync(kFull, merge);
        while (todo) {
            const int src = __ffs(todo) - 1; todo &= todo - 1;
            const int l = __shfl_sync(kFull, L, src), r = __shfl_sync(kFull, R, src), sp = __shfl_sync(kFull, split, src);
            const int sg = __shfl_sync(kFull, s, src), a0 = __shfl_sync(kFull, s0, src), a1 = __shfl_sync(kFull, s1, src);
            ploc_merge(lane, l, r, sp, l == a0 && r == a1, nodes, count, C, counters + sg, scratch[w]);
        }
        if (active && L == s0 && R == s1) active = false;
    }
}

int SegBuilder::reserve(int64_t n, int nSeg) {
    if (n <= capPrims && nSeg <= capSegs) return CWP_OK;
    release();
    CWPB_CHECK(n < (1ll << 30), CWP_ERR_INVALID, "%lld primitives in one build (limit 2^30)", (long long)n);
    CWPB_CUDA(cudaSetDevice(device));
    const int64_t cap = n > capPrims ? n : capPrims; const int cs = nSeg > capSegs ? nSeg : capSegs;
    CWPB_CUDA(cudaMalloc(&nodes, (size_t)2 * 2 * cap * sizeof(float4)));
    CWPB_CUDA(cudaMalloc(&count, (size_t)2 * cap * sizeof(int)));
    CWPB_CUDA(cudaMalloc(&keys, (size_t)cap * 8)); CWPB_CUDA(cudaMalloc(&keysSorted, (size_t)cap * 8));
    CWPB_CUDA(cudaMalloc(&vals, (size_t)cap * 4)); CWPB_CUDA(cudaMalloc(&valsSorted, (size_t)cap * 4));
    CWPB_CUDA(cudaMalloc(&clusters, (size_t)cap * 4)); CWPB_CUDA(cudaMalloc(&bounds, (size_t)cap * 4));
    CWPB_CUDA(cudaMalloc(&segFirst, (size_t)(cs + 1) * 4)); CWPB_CUDA(cudaMalloc(&counters, (size_t)cs * 4));
    CWPB_CUDA(cudaMalloc(&cbox, (size_t)cs * 6 * 4));
    tmpBytes = 0;
    CWPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmpBytes, keys, keysSorted, vals, valsSorted, (int)cap, 0, 64));
    CWPB_CUDA(cudaMalloc(&tmp, tmpBytes > 0 ? tmpBytes : 16));
    capPrims = cap; capSegs = cs;
    return CWP_OK;
}

void SegBuilder::release() {
    if (!capPrims && !capSegs) return;
    cudaSetDevice(device);
    cudaFree(nodes); cudaFree(count); cudaFree(keys); cudaFree(keysSorted); cudaFree(vals); cudaFree(valsSorted);
    cudaFree(clusters); cudaFree(bounds); cudaFree(segFirst); cudaFree(counters); cudaFree(cbox); cudaFree(tmp);
    nodes = nullptr; count = nullptr; keys = keysSorted = nullptr; vals = valsSorted = nullptr; clusters = bounds = nullptr;
    segFirst = counters = nullptr; cbox = nullptr; tmp = nullptr; tmpBytes = 0; capPrims = 0; capSegs = 0;
}

int SegBuilder::build(const float4* lo, const float4* hi, int64_t n64, const int* segFirstHost, int nSeg, cudaStream_t st) {
    CWPB_CHECK(nSeg >= 1 && nSeg <= (1 << kSegBits), CWP_ERR_INVALID, "%d segments in one build (1..%d)", nSeg, 1 << kSegBits);
    CWPB_CHECK(segFirstHost[0] == 0 && segFirstHost[nSeg] == n64, CWP_ERR_INVALID, "segment offsets do not cover the primitives");
    for (int s = 0; s < nSeg; s++) CWPB_CHECK(segFirstHost[s + 1] > segFirstHost[s], CWP_ERR_INVALID, "segment %d is empty", s);
    if (int rc = reserve(n64, nSeg)) return rc;
    const int n = (int)n64;
    CWPB_CUDA(cudaMemcpyAsync(segFirst, segFirstHost, (size_t)(nSeg + 1) * 4, cudaMemcpyHostToDevice, st));
    const int g = (n + 255) / 256;
    k_seg_init<<<(nSeg + 127) / 128, 128, 0, st>>>(cbox, counters, segFirst, nSeg);
    k_seg_bounds<<<g, 256, 0, st>>>(lo, hi, n, segFirst, nSeg, cbox);
    k_seg_keys<<<g, 256, 0, st>>>(lo, hi, n, segFirst, nSeg, cbox, keys, vals);
    int segBits = 0; while ((1 << segBits) < nSeg) segBits++;
    size_t tb = tmpBytes;
    CWPB_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keysSorted, vals, valsSorted, n, 0, kMortonBits + segBits, st));
    k_seg_leaves<<<g, 256, 0, st>>>(lo, hi, keysSorted, valsSorted, n, segFirst, nodes, count, clusters, bounds);
    k_seg_hploc<<<(n + kClimbBlock - 1) / kClimbBlock, kClimbBlock, 0, st>>>(nodes, count, keysSorted, clusters, bounds, segFirst, counters, n);
    CWPB_CUDA(cudaGetLastError());
    return CWP_OK;
}

// ---------------- one mesh, for the host layouts ----------------
int hploc_build_mesh(const float* v, const int* f, int64_t nt, int device, std::vector<float4>& nodesOut, double& gpuMs) {
    CWPB_CHECK(nt > 0 && nt < (1ll << 30), CWP_ERR_INVALID, "%lld triangles", (long long)nt);
    CWPB_CUDA(cudaSetDevice(device));
    std::vector<float4> lo((size_t)nt), hi((size_t)nt);
    for (int64_t t = 0; t < nt; t++) {
        float3 a = f3(3e38f, 3e38f, 3e38f), b = f3(-3e38f, -3e38f, -3e38f);
        for (int k = 0; k < 3; k++) { const float* p = v + 3 * (int64_t)f[3 * t + k]; const float3 q = f3(p[0], p[1], p[2]); a = vmin(a, q); b = vmax(b, q); }
        lo[(size_t)t] = make_float4(a.x, a.y, a.z, 0.f); hi[(size_t)t] = make_float4(b.x, b.y, b.z, 0.f);
    }
    float4 *dLo = nullptr, *dHi = nullptr; cudaStream_t st = nullptr; cudaEvent_t e0 = nullptr, e1 = nullptr;
    SegBuilder B; B.device = device;
    const int seg[2] = { 0, (int)nt };
    int rc = CWP_OK;
    auto ck = [&](cudaError_t e) { if (e != cudaSuccess && rc == CWP_OK) rc = set_error(CWP_ERR_CUDA, "H-PLOC build: %s", cudaGetErrorString(e)); return rc == CWP_OK; };
    if (ck(cudaMalloc(&dLo, (size_t)nt * 16)) && ck(cudaMalloc(&dHi, (size_t)nt * 16)) && ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) &&
        ck(cudaEventCreate(&e0)) && ck(cudaEventCreate(&e1)) &&
        ck(cudaMemcpyAsync(dLo, lo.data(), (size_t)nt * 16, cudaMemcpyHostToDevice, st)) && ck(cudaMemcpyAsync(dHi, hi.data(), (size_t)nt * 16, cudaMemcpyHostToDevice, st))) {
        // a first build loads the kernels and allocates; the second is timed
        rc = B.build(dLo, dHi, nt, seg, 1, st);
        if (rc == CWP_OK && ck(cudaEventRecord(e0, st))) rc = B.build(dLo, dHi, nt, seg, 1, st);
        if (rc == CWP_OK && ck(cudaEventRecord(e1, st)) && ck(cudaEventSynchronize(e1))) {
            float ms = 0.f; ck(cudaEventElapsedTime(&ms, e0, e1)); gpuMs = ms;
            nodesOut.resize((size_t)2 * (2 * nt - 1));
            ck(cudaMemcpy(nodesOut.data(), B.nodes, nodesOut.size() * 16, cudaMemcpyDeviceToHost));
        }
    }
    B.release(); cudaFree(dLo); cudaFree(dHi);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    return rc;
}

}  // namespace cwpb
