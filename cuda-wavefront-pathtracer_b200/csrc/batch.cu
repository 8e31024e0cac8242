// batch.cu - the batched form: every BLAS built on the device at once, every scene's TLAS rebuilt per frame at once,
// and one persistent two-level traversal launch over a ray queue whose rays carry their scene id. The launch shape
// (block size, BLAS width, fetch granularity, stack placement) is a runtime tuning that cwp_batch_autotune measures.
#include "cwp_b200.h"
#include "batch_internal.h"
#include "host_bvh.h"
#include "hploc.h"
#include "runtime.h"
#include "trav.cuh"
#include "wide_emit.h"
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <thread>
#include <type_traits>
#include <vector>

using namespace cwpb;

namespace cwpb {

static constexpr int kTlasStack = 64;

static constexpr int kBatchMaxBlock = 512;

struct BatchArgs {
    const float4* nodes; const float4* tris;        // BLAS layout of the chosen width (absolute indices, MT records)
    const float4* tlas; const int* sceneRoot; const float4* inst;   // TLAS nodes, root per scene, instances (7 float4)
    int tlasW;                                                        // TLAS node width: 2 (4 float4 per node) or 4 (8 float4)
    const int* meshRoot;                                              // BLAS root of each mesh in the traced layout
    int nScenes;
    const float4* ro; const float4* rd; const int* sceneOf;
    float4* hits; int* hitInst; long long n; const int* nDev;   // nDev: ray count on the device (overrides n), or null
    unsigned long long* cursor; int fetch; int* err;
};

// One ray through a two-level scene, one node visit per step: TLAS (BVH2 over instances, nearer child first) or the
// current instance's BLAS (TravState<V>, object-space ray o' = inv o, d' = inv d, so t is shared). TLAS leaves are
// pushed like inner nodes (as ~instance) and entered when they come up.
template <int V, bool ANY>
struct TwoLevel {
    float3 o, d; float tmin, idx, idy, idz, ox, oy, oz;
    float hitT, hu, hv; int hitTri, hitInst;
    int next, tsp, inst, budget;
    TravState<V, ANY, 0> blas;

    __device__ __forceinline__ bool begin(float3 o_, float3 d_, float tmin_, float tmax_, int troot) {
        o = o_; d = d_; tmin = tmin_; hitT = tmax_; hu = hv = 0.f; hitTri = -1; hitInst = -1;
        idx = safe_rcp(d.x); idy = safe_rcp(d.y); idz = safe_rcp(d.z);
        ox = -o.x * idx; oy = -o.y * idy; oz = -o.z * idz;
        next = troot; tsp = 0; inst = -1; budget = kVisitBudget;
        return troot < 0;   // an empty scene: nothing to traverse
    }
    // enter instance k: ray into object space, BLAS traversal from the instance's root
    __device__ __forceinline__ void enter(const float4* __restrict__ instances, const int* __restrict__ meshRoot, int k) {
        const float4* I = instances + 7 * (size_t)k;
        const float4 r0 = ld4(I), r1 = ld4(I + 1), r2 = ld4(I + 2);
        const int root = __ldg(meshRoot + __float_as_int(ld4(I + 6).y));
        const float3 lo_ = f3(r0.x * o.x + r0.y * o.y + r0.z * o.z + r0.w, r1.x * o.x + r1.y * o.y + r1.z * o.z + r1.w, r2.x * o.x + r2.y * o.y + r2.z * o.z + r2.w);
        const float3 ld_ = f3(r0.x * d.x + r0.y * d.y + r0.z * d.z, r1.x * d.x + r1.y * d.y + r1.z * d.z, r2.x * d.x + r2.y * d.y + r2.z * d.z);
        blas.begin(lo_, ld_, tmin, hitT, root);
        inst = k;
    }
    // one BLAS node visit of the current instance (inst >= 0); on leaving the instance, its hit is merged and the next
    // TLAS entry taken. True when the ray is finished.
    template <class TS, class BS>
    __device__ __forceinline__ bool step_blas(const BatchArgs& a, TS& tstack, BS& bstack, int& err) {
        if (!blas.step(a.nodes, a.tris, bstack, err)) return false;
        if (blas.hitTri >= 0 && blas.hitT < hitT) { hitT = blas.hitT; hitTri = blas.hitTri; hu = blas.hu; hv = blas.hv; hitInst = inst; }
        inst = -1;
        if (ANY && hitTri >= 0) return true;
        if (tsp == 0) return true;
        next = tstack[--tsp];
        if (next < 0) { enter(a.inst, a.meshRoot, ~next); return false; }
        return false;
    }
    template <class TS, class BS>
    __device__ __forceinline__ bool step(const BatchArgs& a, TS& tstack, BS& bstack, int& err) {
        return inst >= 0 ? step_blas(a, tstack, bstack, err) : step_tlas(a, tstack, err);
    }
    // one TLAS node visit (inst < 0): nearer children first, an instance entered when it comes up. True when the ray
    // is finished.
    template <class TS>
    __device__ __forceinline__ bool step_tlas(const BatchArgs& a, TS& tstack, int& err) {
        if (--budget < 0) { err |= kTravBudget; return true; }
        if (a.tlasW == 4) {   // four children, hit ones sorted by entry distance, nearest taken, others pushed far to near
            const float INF = 3.4e38f;
            const float4* nb = a.tlas + 8 * (size_t)next;
            const float4 lx = ld4(nb), hx = ld4(nb + 1), ly = ld4(nb + 2), hy = ld4(nb + 3), lz = ld4(nb + 4), hz = ld4(nb + 5), cf = ld4(nb + 6), kf = ld4(nb + 7);
            const float LX[4] = { lx.x, lx.y, lx.z, lx.w }, HX[4] = { hx.x, hx.y, hx.z, hx.w }, LY[4] = { ly.x, ly.y, ly.z, ly.w };
            const float HY[4] = { hy.x, hy.y, hy.z, hy.w }, LZ[4] = { lz.x, lz.y, lz.z, lz.w }, HZ[4] = { hz.x, hz.y, hz.z, hz.w };
            const int CC[4] = { __float_as_int(cf.x), __float_as_int(cf.y), __float_as_int(cf.z), __float_as_int(cf.w) };
            const int KK[4] = { __float_as_int(kf.x), __float_as_int(kf.y), __float_as_int(kf.z), __float_as_int(kf.w) };
            float ht[4]; int he[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float x0 = fmaf(LX[j], idx, ox), x1 = fmaf(HX[j], idx, ox), y0 = fmaf(LY[j], idy, oy), y1 = fmaf(HY[j], idy, oy), z0 = fmaf(LZ[j], idz, oz), z1 = fmaf(HZ[j], idz, oz);
                const float tn = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
                const float tf = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), hitT));
                ht[j] = CC[j] >= 0 && tn <= tf ? tn : INF;
                he[j] = KK[j] > 0 ? ~CC[j] : CC[j];
            }
#define CWPB_CSWAP(p, q) { if (ht[q] < ht[p]) { const float tf_ = ht[p]; ht[p] = ht[q]; ht[q] = tf_; const int ti_ = he[p]; he[p] = he[q]; he[q] = ti_; } }
            CWPB_CSWAP(0, 1) CWPB_CSWAP(2, 3) CWPB_CSWAP(0, 2) CWPB_CSWAP(1, 3) CWPB_CSWAP(1, 2)
#undef CWPB_CSWAP
            int go;
            if (ht[0] == INF) { if (tsp == 0) return true; go = tstack[--tsp]; }
            else {
                if (tsp + 3 > kTlasStack) { err |= kTravOverflow; return true; }
                if (ht[3] < INF) tstack[tsp++] = he[3];
                if (ht[2] < INF) tstack[tsp++] = he[2];
                if (ht[1] < INF) tstack[tsp++] = he[1];
                go = he[0];
            }
            if (go < 0) enter(a.inst, a.meshRoot, ~go); else next = go;
            return false;
        }
        const float4* nb = a.tlas + 4 * (size_t)next;
        const float4 n0 = ld4(nb), n1 = ld4(nb + 1), nz = ld4(nb + 2), mt = ld4(nb + 3);
        const int c0 = __float_as_int(mt.x), c1 = __float_as_int(mt.y), k0 = __float_as_int(mt.z), k1 = __float_as_int(mt.w);
        const float a0 = fmaf(n0.x, idx, ox), a1 = fmaf(n0.y, idx, ox), a2 = fmaf(n0.z, idy, oy), a3 = fmaf(n0.w, idy, oy), a4 = fmaf(nz.x, idz, oz), a5 = fmaf(nz.y, idz, oz);
        const float b0 = fmaf(n1.x, idx, ox), b1 = fmaf(n1.y, idx, ox), b2 = fmaf(n1.z, idy, oy), b3 = fmaf(n1.w, idy, oy), b4 = fmaf(nz.z, idz, oz), b5 = fmaf(nz.w, idz, oz);
        const float t0n = fmaxf(fmaxf(fminf(a0, a1), fminf(a2, a3)), fmaxf(fminf(a4, a5), tmin));
        const float t0f = fminf(fminf(fmaxf(a0, a1), fmaxf(a2, a3)), fminf(fmaxf(a4, a5), hitT));
        const float t1n = fmaxf(fmaxf(fminf(b0, b1), fminf(b2, b3)), fmaxf(fminf(b4, b5), tmin));
        const float t1f = fminf(fminf(fmaxf(b0, b1), fmaxf(b2, b3)), fminf(fmaxf(b4, b5), hitT));
        const bool h0 = c0 >= 0 && t0n <= t0f, h1 = c1 >= 0 && t1n <= t1f;
        int e0 = k0 > 0 ? ~c0 : c0, e1 = k1 > 0 ? ~c1 : c1;   // entries: node >= 0, instance as ~id
        int go;
        if (h0 && h1) {
            if (t1n < t0n) { const int t = e0; e0 = e1; e1 = t; }
            if (tsp == kTlasStack) { err |= kTravOverflow; return true; }
            tstack[tsp++] = e1; go = e0;
        } else if (h0 || h1) go = h0 ? e0 : e1;
        else { if (tsp == 0) return true; go = tstack[--tsp]; }
        if (go < 0) enter(a.inst, a.meshRoot, ~go); else next = go;
        return false;
    }
};

__device__ __forceinline__ unsigned lane_mask_lt() { unsigned m; asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m)); return m; }

// Persistent launch: each lane advances its ray one node visit at a time; a warp refetches rays (one atomic on the
// queue cursor) once a.fetch of its lanes are idle. SMEM: the BLAS stack in shared memory, entry-major.
template <int V, bool ANY, bool SMEM>
// 64 registers (two 512-thread blocks per SM) with 132 bytes of spills: measured faster than 80 registers without
// spills (1.83 vs 1.80 Grays/s on 64 scenes) or 128 registers (1.41); resident warps matter more than the spills
__global__ void __launch_bounds__(kBatchMaxBlock, 2) k_batch_trace(const BatchArgs a) {
    typedef typename TravState<V, ANY, 0>::Stack LocalStack;
    typedef typename std::conditional<V == 8, uint2, int>::type Entry;
    extern __shared__ unsigned char smem[];
    const int lane = threadIdx.x & 31;
    int e = 0;
    TwoLevel<V, ANY> ray;
    int tstack[kTlasStack];
    const long long nRays = a.nDev ? (long long)*a.nDev : a.n;
    LocalStack lstack;
    SharedStack<Entry> sstack{ reinterpret_cast<Entry*>(smem) + threadIdx.x, (int)blockDim.x };
    long long k = -1; bool fin = false, drained = false;
    for (;;) {
        if (fin) {
            if (!ANY) a.hits[k] = make_float4(ray.hitT, ray.hu, ray.hv, __int_as_float(ray.hitTri));
            else if (a.hits) a.hits[k] = make_float4(ray.hitT, ray.hu, ray.hv, __int_as_float(ray.hitTri));
            a.hitInst[k] = ray.hitInst;
            k = -1; fin = false;
        }
        if (!drained) {
            const bool need = k < 0;
            const unsigned nm = __ballot_sync(0xffffffffu, need);
            if (nm) {
                const int leader = __ffs(nm) - 1;
                long long base = 0;
                if (lane == leader) base = (long long)atomicAdd(a.cursor, (unsigned long long)__popc(nm));
                base = __shfl_sync(0xffffffffu, base, leader);
                const long long kk = base + __popc(nm & lane_mask_lt());
                if (need && kk < nRays) {
                    k = kk;
                    const float4 O = __ldcs(a.ro + k), D = __ldcs(a.rd + k);
                    const int sc = __ldcs(a.sceneOf + k);
                    const int root = sc >= 0 && sc < a.nScenes ? __ldg(a.sceneRoot + sc) : -1;
                    fin = ray.begin(xyz(O), xyz(D), O.w, D.w, root);
                }
                drained = __any_sync(0xffffffffu, need && kk >= nRays);
            }
        }
        if (!__any_sync(0xffffffffu, k >= 0)) break;
        for (;;) {
            // one level per iteration, so the warp runs one code path: the lanes in a BLAS step when they are at least
            // twice as many as those in the TLAS, else the TLAS lanes (measured: both levels every iteration 1.64
            // Grays/s on 64 scenes; 1:1 1.80; 2:1 1.82; 3:1 1.80; TLAS first 1.41)
            bool act = k >= 0 && !fin;
            {
                const unsigned inB = __ballot_sync(0xffffffffu, act && ray.inst >= 0), inT = __ballot_sync(0xffffffffu, act && ray.inst < 0);
                const bool doB = __popc(inB) >= 2 * __popc(inT);
                act = act && ((ray.inst >= 0) == doB);
            }
            if (act) fin = ray.inst >= 0 ? (SMEM ? ray.step_blas(a, tstack, sstack, e) : ray.step_blas(a, tstack, lstack, e)) : ray.step_tlas(a, tstack, e);
            const unsigned busy = __ballot_sync(0xffffffffu, k >= 0 && !fin);
            if (!busy || (!drained && 32 - __popc(busy) >= a.fetch)) break;
        }
    }
    if (e) atomicOr(a.err, e);
}

template <int V> constexpr size_t stack_entry_bytes() { return V == 8 ? sizeof(uint2) : sizeof(int); }
template <int V> constexpr int stack_entries() { return V == 8 ? kStack8 : kStack2; }

typedef void (*BatchKernel)(const BatchArgs);
static BatchKernel pick_kernel(int width, bool any, bool smem) {
#define CWPB_K(VV) (any ? (smem ? k_batch_trace<VV, true, true> : k_batch_trace<VV, true, false>) : (smem ? k_batch_trace<VV, false, true> : k_batch_trace<VV, false, false>))
    return width == 2 ? CWPB_K(2) : width == 4 ? CWPB_K(4) : CWPB_K(8);
#undef CWPB_K
}
static size_t smem_bytes(int width, int block) {
    return (size_t)block * (width == 8 ? stack_entries<8>() * stack_entry_bytes<8>() : width == 4 ? stack_entries<4>() * stack_entry_bytes<4>() : stack_entries<2>() * stack_entry_bytes<2>());
}

}  // namespace cwpb

struct cwp_batch {
    int device = 0, leaf = 4, widths = 0;
    int nMesh = 0; int64_t nTris = 0;
    std::vector<int> meshFirst;          // nMesh + 1 triangle offsets
    float4* triV = nullptr;              // input triangles, 3 float4 each
    float4* nrm = nullptr;               // corner normals, 3 float4 per triangle in mesh order (zero for meshes without), or null
    float4 *primLo = nullptr, *primHi = nullptr, *meshBox = nullptr;
    int* meshFirstDev = nullptr;
    int* meshRoot[3] = { nullptr, nullptr, nullptr }; std::vector<int> meshRootHost[3];   // per layout width
    int builder = 0;
    SegBuilder blasB, tlasB;
    WideLayout lay[3];                   // width 2, 4, 8
    // scenes
    int nScenes = 0; int64_t nInst = 0;
    std::vector<int> sceneFirst;         // nScenes + 1
    cwp_instance* inst = nullptr; int64_t capInst = 0;
    float4 *instLo = nullptr, *instHi = nullptr, *tlas = nullptr, *tlas4 = nullptr;   // TLAS in BVH2 and width-4 form
    int tlasWidth = 4;                   // the form the traversal reads
    int *sceneRoot = nullptr, *segFirstTlas = nullptr; int capScenes = 0;
    // incremental form: fixed regions of `fixedCap` instances per scene, updates built over a compact copy
    int fixedCap = 0;
    cwp_instance* uInst = nullptr; float4 *uLo = nullptr, *uHi = nullptr; int64_t capU = 0;
    int* dstFirstTlas = nullptr; int capDst = 0;
    // launch
    cwp_batch_tuning tuning{};
    int* err = nullptr; unsigned long long* cursor = nullptr;
    cudaStream_t st = nullptr; cudaEvent_t e0 = nullptr, e1 = nullptr;
    double blasMs = 0, tlasMs = 0; int nSm = 0;
    int64_t refs[3] = { 0, 0, 0 };   // triangle records per layout (host build with spatial splits: more than nTris)
};

static int lay_index(int w) { return w == 2 ? 0 : w == 4 ? 1 : w == 8 ? 2 : -1; }

static void batch_free(cwp_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    for (auto& l : b->lay) free_wide(l);
    b->blasB.release(); b->tlasB.release();
    cudaFree(b->triV); cudaFree(b->nrm); cudaFree(b->primLo); cudaFree(b->primHi); cudaFree(b->meshBox); cudaFree(b->meshFirstDev);
    cudaFree(b->inst); cudaFree(b->instLo); cudaFree(b->instHi); cudaFree(b->tlas); cudaFree(b->tlas4); cudaFree(b->sceneRoot); cudaFree(b->segFirstTlas);
    cudaFree(b->uInst); cudaFree(b->uLo); cudaFree(b->uHi); cudaFree(b->dstFirstTlas);
    cudaFree(b->err); cudaFree(b->cursor);
    for (int i = 0; i < 3; i++) cudaFree(b->meshRoot[i]);
    if (b->st) cudaStreamDestroy(b->st);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    delete b;
}

extern "C" void cwp_batch_destroy(cwp_batch* b) { batch_free(b); }

// append a BVH4 array with indices relative to its own nodes and triangles
static int append_bvh4(std::vector<float4>& all, const std::vector<float4>& blas, int triBase) {
    const int base = (int)(all.size() / 8);
    for (size_t i = 0; i < blas.size(); i += 8) {
        float4 c = blas[i + 6]; const float4 k = blas[i + 7];
        int* cc = reinterpret_cast<int*>(&c); const int* kk = reinterpret_cast<const int*>(&k);
        for (int j = 0; j < 4; j++) { if (kk[j] > 0) cc[j] += triBase; else if (cc[j] >= 0) cc[j] += base; }
        for (int j = 0; j < 6; j++) all.push_back(blas[i + j]);
        all.push_back(c); all.push_back(k);
    }
    return base;
}

// Every BLAS built on the host cores (meshes in parallel, one thread each): binned SAH with 32 bins, spatial splits
// when spatial > 0, BVH2 / BVH4 layouts from leaf-`leaf` trees and the SAH-collapsed CWBVH from a leaf-1 tree,
// concatenated with absolute indices; per-layout mesh roots; Moller-Trumbore records in each layout's leaf order.
static int host_build(cwp_batch* b, const cwp_mesh_view* meshes, int n, float spatial) {
    CWPB_CHECK(spatial >= 0.f && spatial < 1.f, CWP_ERR_INVALID, "spatial %g out of [0, 1)", spatial);
    struct Out { std::vector<float4> nodes[3], tris[3]; Box3 box; };
    std::vector<Out> out(n);
    auto build_one = [&](int m) {
        const cwp_mesh_view& v = meshes[m];
        Mesh M; M.v.assign(v.verts, v.verts + 3 * v.n_verts); M.f.assign(v.faces, v.faces + 3 * v.n_tris);
        if (v.face_mat) M.fm.assign(v.face_mat, v.face_mat + v.n_tris); else M.fm.assign(v.n_tris, 0);
        for (size_t i = 0; i < M.nv(); i++) out[m].box.grow(M.vert((int)i));
        SahOptions so; so.bins = 32; so.threads = 1;
        std::vector<float4> nrm;
        if (b->widths & ((1 << 2) | (1 << 4))) {
            so.leafMax = b->leaf; BinaryBvh B;
            if (spatial > 0.f) build_sbvh(M, so, spatial, 0.3f, B); else build_sah(M, so, B);
            if (b->widths & (1 << 2)) { BinaryBvh B2 = B; layout_bvh2(B2, out[m].nodes[0]); pack_tris(M, B2.prim, out[m].tris[0], nrm); }
            if (b->widths & (1 << 4)) { BinaryBvh B4 = B; layout_bvh4(B4, out[m].nodes[1]); pack_tris(M, B4.prim, out[m].tris[1], nrm); }
        }
        if (b->widths & (1 << 8)) {
            so.leafMax = 1; BinaryBvh B;
            if (spatial > 0.f) build_sbvh(M, so, spatial, 0.3f, B); else build_sah(M, so, B);
            WideBvh W; collapse_cwbvh(B, W);
            out[m].nodes[2].swap(W.nodes); pack_tris(M, W.order, out[m].tris[2], nrm);
        }
    };
    const auto t0 = std::chrono::steady_clock::now();
    const int threads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<int> next{ 0 };
    std::vector<std::thread> ts;
    for (int t = 0; t < std::min(threads, n); t++) ts.emplace_back([&] { for (int m; (m = next++) < n;) build_one(m); });
    for (auto& t : ts) t.join();
    std::vector<float4> box(2 * (size_t)n);
    for (int m = 0; m < n; m++) { box[2 * m] = make_float4(out[m].box.lo.x, out[m].box.lo.y, out[m].box.lo.z, 0.f); box[2 * m + 1] = make_float4(out[m].box.hi.x, out[m].box.hi.y, out[m].box.hi.z, 0.f); }
    CWPB_CUDA(cudaMemcpy(b->meshBox, box.data(), box.size() * sizeof(float4), cudaMemcpyHostToDevice));
    for (int w : { 2, 4, 8 }) {
        if (!(b->widths & (1 << w))) continue;
        const int li = lay_index(w);
        std::vector<float4> nodes, tris; b->meshRootHost[li].resize(n);
        for (int m = 0; m < n; m++) {
            const int triBase = (int)(tris.size() / 3);
            b->meshRootHost[li][m] = w == 2 ? append_bvh2(nodes, out[m].nodes[li], triBase) : w == 4 ? append_bvh4(nodes, out[m].nodes[li], triBase)
                                                                                          : append_bvh8(nodes, out[m].nodes[li], triBase);
            tris.insert(tris.end(), out[m].tris[li].begin(), out[m].tris[li].end());
            std::vector<float4>().swap(out[m].nodes[li]); std::vector<float4>().swap(out[m].tris[li]);
        }
        WideLayout& L = b->lay[li];
        L.width = w; L.nNodes = (int64_t)nodes.size() / L.stride(); L.capNodes = L.nNodes;
        CWPB_CUDA(cudaMalloc(&L.nodes, nodes.size() * sizeof(float4)));
        CWPB_CUDA(cudaMalloc(&L.tris, tris.size() * sizeof(float4)));
        CWPB_CUDA(cudaMemcpy(L.nodes, nodes.data(), nodes.size() * sizeof(float4), cudaMemcpyHostToDevice));
        CWPB_CUDA(cudaMemcpy(L.tris, tris.data(), tris.size() * sizeof(float4), cudaMemcpyHostToDevice));
        b->refs[li] = (int64_t)tris.size() / 3;
    }
    b->blasMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return CWP_OK;
}

static int batch_create(const cwp_mesh_view* meshes, int32_t n, const cwp_batch_options* opt, cwp_batch* b) {
    b->device = opt ? opt->device : 0;
    b->leaf = opt && opt->leaf > 0 ? opt->leaf : 4;
    b->widths = opt && opt->widths ? opt->widths : ((1 << 2) | (1 << 4) | (1 << 8));
    CWPB_CHECK(b->leaf <= 8, CWP_ERR_INVALID, "leaf size %d above 8", b->leaf);
    CWPB_CHECK((b->widths & ~((1 << 2) | (1 << 4) | (1 << 8))) == 0, CWP_ERR_INVALID, "layout mask 0x%x has bits other than 1<<2, 1<<4, 1<<8", b->widths);
    CWPB_CUDA(cudaSetDevice(b->device));
    CWPB_CUDA(cudaDeviceGetAttribute(&b->nSm, cudaDevAttrMultiProcessorCount, b->device));
    b->nMesh = n;
    b->meshFirst.assign(n + 1, 0);
    for (int m = 0; m < n; m++) {
        const cwp_mesh_view& v = meshes[m];
        CWPB_CHECK(v.verts && v.faces && v.n_tris > 0 && v.n_verts > 0, CWP_ERR_INVALID, "mesh %d is empty or has NULL arrays", m);
        b->meshFirst[m + 1] = b->meshFirst[m] + (int)v.n_tris;
        CWPB_CHECK((int64_t)b->meshFirst[m + 1] < (1ll << 30), CWP_ERR_INVALID, "more than 2^30 triangles in one batch");
    }
    b->nTris = b->meshFirst[n];
    // triangle soup, 3 float4 per triangle: (v0, local id), (v1, material), (v2, 0); vertex indices and coordinates checked
    std::vector<float4> soup((size_t)3 * b->nTris);
    for (int m = 0; m < n; m++) {
        const cwp_mesh_view& v = meshes[m];
        for (int64_t t = 0; t < v.n_tris; t++) {
            float4* o = &soup[(size_t)3 * (b->meshFirst[m] + t)];
            for (int k = 0; k < 3; k++) {
                const int vi = v.faces[3 * t + k];
                CWPB_CHECK(vi >= 0 && vi < v.n_verts, CWP_ERR_INVALID, "mesh %d triangle %lld: vertex index %d out of range", m, (long long)t, vi);
                const float* p = v.verts + 3 * (size_t)vi;
                CWPB_CHECK(std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]), CWP_ERR_INVALID, "mesh %d: non-finite vertex %d", m, vi);
                o[k] = make_float4(p[0], p[1], p[2], 0.f);
            }
            int id = (int)t, mat = v.face_mat ? v.face_mat[t] : 0;
            memcpy(&o[0].w, &id, 4); memcpy(&o[1].w, &mat, 4);
        }
    }
    // corner normals of the meshes that have them (shading normals of the serving integrator)
    std::vector<float4> nr;
    for (int m = 0; m < n; m++) {
        const cwp_mesh_view& v = meshes[m];
        if (!v.normals) continue;
        if (nr.empty()) nr.assign((size_t)3 * b->nTris, make_float4(0.f, 0.f, 0.f, 0.f));
        for (int64_t t = 0; t < v.n_tris; t++)
            for (int k = 0; k < 3; k++) {
                const float* q = v.normals + 3 * (size_t)v.faces[3 * t + k];
                CWPB_CHECK(std::isfinite(q[0]) && std::isfinite(q[1]) && std::isfinite(q[2]), CWP_ERR_INVALID, "mesh %d: non-finite normal", m);
                nr[(size_t)3 * (b->meshFirst[m] + t) + k] = make_float4(q[0], q[1], q[2], 0.f);
            }
    }
    CWPB_CUDA(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
    CWPB_CUDA(cudaEventCreate(&b->e0)); CWPB_CUDA(cudaEventCreate(&b->e1));
    if (!nr.empty()) {
        CWPB_CUDA(cudaMalloc(&b->nrm, nr.size() * sizeof(float4)));
        CWPB_CUDA(cudaMemcpy(b->nrm, nr.data(), nr.size() * sizeof(float4), cudaMemcpyHostToDevice));
    }
    CWPB_CUDA(cudaMalloc(&b->err, sizeof(int))); CWPB_CUDA(cudaMemset(b->err, 0, sizeof(int)));
    CWPB_CUDA(cudaMalloc(&b->cursor, sizeof(unsigned long long)));
    CWPB_CUDA(cudaMalloc(&b->triV, soup.size() * sizeof(float4)));
    CWPB_CUDA(cudaMalloc(&b->primLo, (size_t)b->nTris * sizeof(float4))); CWPB_CUDA(cudaMalloc(&b->primHi, (size_t)b->nTris * sizeof(float4)));
    CWPB_CUDA(cudaMalloc(&b->meshBox, (size_t)2 * n * sizeof(float4)));
    CWPB_CUDA(cudaMalloc(&b->meshFirstDev, (size_t)(n + 1) * sizeof(int)));
    CWPB_CUDA(cudaMemcpyAsync(b->triV, soup.data(), soup.size() * sizeof(float4), cudaMemcpyHostToDevice, b->st));
    CWPB_CUDA(cudaMemcpyAsync(b->meshFirstDev, b->meshFirst.data(), (size_t)(n + 1) * sizeof(int), cudaMemcpyHostToDevice, b->st));
    b->blasB.device = b->device; b->tlasB.device = b->device;
    b->builder = opt ? opt->builder : 0;
    CWPB_CHECK(b->builder == 0 || b->builder == 1, CWP_ERR_INVALID, "builder %d is not 0 (GPU) or 1 (host)", b->builder);
    b->tlasWidth = opt && opt->tlas_width ? opt->tlas_width : 4;
    CWPB_CHECK(b->tlasWidth == 2 || b->tlasWidth == 4, CWP_ERR_INVALID, "TLAS width %d is not 2 or 4", b->tlasWidth);
    if (b->builder == 1) {
        if (int rc = host_build(b, meshes, n, opt ? opt->spatial : 0.f)) return rc;
    } else {
        if (int rc = b->blasB.reserve(b->nTris, n)) return rc;
        CWPB_CUDA(cudaStreamSynchronize(b->st));
        // the timed build: boxes, keys, sort, one H-PLOC launch, root boxes, layouts
        CWPB_CUDA(cudaEventRecord(b->e0, b->st));
        triangle_boxes(b->triV, b->nTris, b->primLo, b->primHi, b->st);
        if (int rc = b->blasB.build(b->primLo, b->primHi, b->nTris, b->meshFirst.data(), n, b->st)) return rc;
        root_boxes(b->blasB, b->meshFirstDev, n, b->meshBox, b->st);
        for (int w : { 2, 4, 8 }) {
            if (!(b->widths & (1 << w))) continue;
            if (int rc = emit_wide(b->blasB, b->meshFirst.data(), n, b->triV, w, w == 8 ? std::min(b->leaf, 3) : b->leaf, b->lay[lay_index(w)], b->st)) return rc;
            b->meshRootHost[lay_index(w)].resize(n);
            for (int m = 0; m < n; m++) b->meshRootHost[lay_index(w)][m] = m;   // mesh m's root is node m
        }
        CWPB_CUDA(cudaEventRecord(b->e1, b->st));
        CWPB_CUDA(cudaEventSynchronize(b->e1));
        float ms = 0; CWPB_CUDA(cudaEventElapsedTime(&ms, b->e0, b->e1)); b->blasMs = ms;
        CWPB_CUDA(cudaGetLastError());
    }
    for (int i = 0; i < 3; i++) {
        if (b->meshRootHost[i].empty()) continue;
        CWPB_CUDA(cudaMalloc(&b->meshRoot[i], (size_t)n * sizeof(int)));
        CWPB_CUDA(cudaMemcpy(b->meshRoot[i], b->meshRootHost[i].data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice));
    }
    for (int i = 0; i < 3; i++) {
        if (!b->lay[i].nodes) continue;
        if (!b->refs[i]) b->refs[i] = b->nTris;
        if (int rc = check_wide(b->lay[i], b->refs[i], b->err, b->st)) return rc;
    }
    b->tuning.block = 128; b->tuning.width = (b->widths & (1 << 8)) ? 8 : (b->widths & (1 << 4)) ? 4 : 2; b->tuning.fetch = 12; b->tuning.smem_stack = 0; b->tuning.ms = 0;
    return CWP_OK;
}

extern "C" int cwp_batch_create(const cwp_mesh_view* meshes, int32_t n, const cwp_batch_options* opt, cwp_batch** out) {
    CWPB_CHECK(out, CWP_ERR_INVALID, "out is NULL");
    *out = nullptr;
    CWPB_CHECK(meshes && n >= 1 && n <= (1 << kSegBits), CWP_ERR_INVALID, "%d meshes (1..%d)", n, 1 << kSegBits);
    cwp_batch* b = new cwp_batch();
    if (int rc = batch_create(meshes, n, opt, b)) { batch_free(b); return rc; }
    *out = b;
    return CWP_OK;
}

static int check_instances(const cwp_batch* b, const cwp_instance* h, int64_t n, int64_t at) {
    for (int64_t i = 0; i < n; i++) {
        CWPB_CHECK(h[i].mesh >= 0 && h[i].mesh < b->nMesh, CWP_ERR_INVALID, "instance %lld: mesh %d out of range", (long long)(at + i), h[i].mesh);
        for (int k = 0; k < 12; k++) CWPB_CHECK(std::isfinite(h[i].inv[k]) && std::isfinite(h[i].fwd[k]), CWP_ERR_INVALID, "instance %lld: non-finite transform", (long long)(at + i));
    }
    return CWP_OK;
}

extern "C" int cwp_batch_set_scenes(cwp_batch* b, const cwp_instance* inst, int64_t n, const int32_t* first, int32_t nScenes) {
    CWPB_CHECK(b, CWP_ERR_INVALID, "batch is NULL");
    CWPB_CHECK(first && nScenes >= 1, CWP_ERR_INVALID, "no scenes");
    CWPB_CHECK(first[0] == 0 && first[nScenes] == n, CWP_ERR_INVALID, "scene offsets do not cover the %lld instances", (long long)n);
    CWPB_CHECK(n >= 0 && n < (1ll << 30), CWP_ERR_INVALID, "%lld instances", (long long)n);
    CWPB_CHECK(n == 0 || inst, CWP_ERR_INVALID, "instances are NULL");
    for (int s = 0; s < nScenes; s++) CWPB_CHECK(first[s + 1] >= first[s], CWP_ERR_INVALID, "scene offsets decrease at scene %d", s);
    if (int rc = check_instances(b, inst, n, 0)) return rc;
    // segments: the non-empty scenes (their instance ranges are contiguous and cover the array)
    std::vector<int> seg; seg.push_back(0);
    std::vector<int> rootHost(nScenes, -1);
    for (int s = 0; s < nScenes; s++) {
        const int m = first[s + 1] - first[s];
        if (m == 0) continue;
        rootHost[s] = m == 1 ? first[s] : first[s] + m - 2;
        seg.push_back(first[s + 1]);
    }
    const int nSeg = (int)seg.size() - 1;
    CWPB_CHECK(nSeg <= (1 << kSegBits), CWP_ERR_INVALID, "%d non-empty scenes (limit %d)", nSeg, 1 << kSegBits);
    CWPB_CUDA(cudaSetDevice(b->device));
    if (n > b->capInst) {
        cudaFree(b->inst); cudaFree(b->instLo); cudaFree(b->instHi); cudaFree(b->tlas); cudaFree(b->tlas4);
        b->inst = nullptr; b->instLo = b->instHi = b->tlas = b->tlas4 = nullptr; b->capInst = 0;
        CWPB_CUDA(cudaMalloc(&b->inst, (size_t)n * sizeof(cwp_instance)));
        CWPB_CUDA(cudaMalloc(&b->instLo, (size_t)n * sizeof(float4))); CWPB_CUDA(cudaMalloc(&b->instHi, (size_t)n * sizeof(float4)));
        CWPB_CUDA(cudaMalloc(&b->tlas, (size_t)4 * n * sizeof(float4)));
        CWPB_CUDA(cudaMalloc(&b->tlas4, (size_t)8 * n * sizeof(float4)));
        b->capInst = n;
    }
    if (nScenes + 1 > b->capScenes) {
        cudaFree(b->sceneRoot); cudaFree(b->segFirstTlas); b->sceneRoot = b->segFirstTlas = nullptr;
        CWPB_CUDA(cudaMalloc(&b->sceneRoot, (size_t)(nScenes + 1) * sizeof(int)));
        CWPB_CUDA(cudaMalloc(&b->segFirstTlas, (size_t)(nScenes + 1) * sizeof(int)));
        b->capScenes = nScenes + 1;
    }
    CWPB_CUDA(cudaEventRecord(b->e0, b->st));
    if (n > 0) CWPB_CUDA(cudaMemcpyAsync(b->inst, inst, (size_t)n * sizeof(cwp_instance), cudaMemcpyHostToDevice, b->st));
    CWPB_CUDA(cudaMemcpyAsync(b->sceneRoot, rootHost.data(), (size_t)nScenes * sizeof(int), cudaMemcpyHostToDevice, b->st));
    CWPB_CUDA(cudaMemcpyAsync(b->segFirstTlas, seg.data(), seg.size() * sizeof(int), cudaMemcpyHostToDevice, b->st));
    if (n > 0) {
        instance_boxes(b->inst, (int)n, b->meshBox, b->instLo, b->instHi, b->st);
        if (int rc = b->tlasB.build(b->instLo, b->instHi, n, seg.data(), nSeg, b->st)) return rc;
        emit_tlas(b->tlasB, (int)n, b->segFirstTlas, nSeg, b->tlas, b->st, nullptr, b->tlas4);
    }
    CWPB_CUDA(cudaEventRecord(b->e1, b->st));
    CWPB_CUDA(cudaEventSynchronize(b->e1));
    float ms = 0; CWPB_CUDA(cudaEventElapsedTime(&ms, b->e0, b->e1)); b->tlasMs = ms;
    CWPB_CUDA(cudaGetLastError());
    b->nScenes = 0;   // not traceable until the new TLAS passes its check
    if (int rc = check_tlas(b->tlas, (int)n, b->segFirstTlas, nSeg, b->err, b->st, nullptr, b->tlas4)) return rc;
    b->nScenes = nScenes; b->nInst = n; b->sceneFirst.assign(first, first + nScenes + 1); b->fixedCap = 0;
    return CWP_OK;
}

extern "C" int cwp_batch_reserve_scenes(cwp_batch* b, int32_t nScenes, int32_t cap) {
    CWPB_CHECK(b, CWP_ERR_INVALID, "batch is NULL");
    CWPB_CHECK(nScenes >= 1 && cap >= 1 && (int64_t)nScenes * cap < (1ll << 30), CWP_ERR_INVALID, "%d scenes of %d instances", nScenes, cap);
    CWPB_CHECK(nScenes <= (1 << kSegBits), CWP_ERR_INVALID, "%d scenes (limit %d)", nScenes, 1 << kSegBits);
    CWPB_CUDA(cudaSetDevice(b->device));
    const int64_t n = (int64_t)nScenes * cap;
    b->nScenes = 0;   // not traceable while the arrays change
    if (n > b->capInst) {
        cudaFree(b->inst); cudaFree(b->instLo); cudaFree(b->instHi); cudaFree(b->tlas); cudaFree(b->tlas4);
        b->inst = nullptr; b->instLo = b->instHi = b->tlas = b->tlas4 = nullptr; b->capInst = 0;
        CWPB_CUDA(cudaMalloc(&b->inst, (size_t)n * sizeof(cwp_instance)));
        CWPB_CUDA(cudaMalloc(&b->instLo, (size_t)n * sizeof(float4))); CWPB_CUDA(cudaMalloc(&b->instHi, (size_t)n * sizeof(float4)));
        CWPB_CUDA(cudaMalloc(&b->tlas, (size_t)4 * n * sizeof(float4)));
        CWPB_CUDA(cudaMalloc(&b->tlas4, (size_t)8 * n * sizeof(float4)));
        b->capInst = n;
    }
    if (n > b->capU) {
        cudaFree(b->uInst); cudaFree(b->uLo); cudaFree(b->uHi); b->uInst = nullptr; b->uLo = b->uHi = nullptr; b->capU = 0;
        CWPB_CUDA(cudaMalloc(&b->uInst, (size_t)n * sizeof(cwp_instance)));
        CWPB_CUDA(cudaMalloc(&b->uLo, (size_t)n * sizeof(float4))); CWPB_CUDA(cudaMalloc(&b->uHi, (size_t)n * sizeof(float4)));
        b->capU = n;
    }
    if (nScenes + 1 > b->capScenes) {
        cudaFree(b->sceneRoot); cudaFree(b->segFirstTlas); b->sceneRoot = b->segFirstTlas = nullptr;
        CWPB_CUDA(cudaMalloc(&b->sceneRoot, (size_t)(nScenes + 1) * sizeof(int)));
        CWPB_CUDA(cudaMalloc(&b->segFirstTlas, (size_t)(nScenes + 1) * sizeof(int)));
        b->capScenes = nScenes + 1;
    }
    if (nScenes > b->capDst) {
        cudaFree(b->dstFirstTlas); b->dstFirstTlas = nullptr;
        CWPB_CUDA(cudaMalloc(&b->dstFirstTlas, (size_t)nScenes * sizeof(int)));
        b->capDst = nScenes;
    }
    // every scene empty: root -1 (its rays miss); zeroed instances and nodes keep the downloads well-formed
    CWPB_CUDA(cudaMemsetAsync(b->sceneRoot, 0xff, (size_t)nScenes * sizeof(int), b->st));
    CWPB_CUDA(cudaMemsetAsync(b->inst, 0, (size_t)n * sizeof(cwp_instance), b->st));
    CWPB_CUDA(cudaMemsetAsync(b->tlas, 0, (size_t)4 * n * sizeof(float4), b->st));
    CWPB_CUDA(cudaMemsetAsync(b->tlas4, 0, (size_t)8 * n * sizeof(float4), b->st));
    CWPB_CUDA(cudaStreamSynchronize(b->st));
    b->fixedCap = cap; b->nInst = n; b->nScenes = nScenes;
    b->sceneFirst.resize(nScenes + 1);
    for (int s = 0; s <= nScenes; s++) b->sceneFirst[s] = s * cap;
    return CWP_OK;
}

extern "C" int cwp_batch_update_scenes(cwp_batch* b, const int32_t* scenes, int32_t nUpd, const cwp_instance* inst, const int32_t* counts) {
    CWPB_CHECK(b, CWP_ERR_INVALID, "batch is NULL");
    CWPB_CHECK(b->fixedCap > 0 && b->nScenes > 0, CWP_ERR_STATE, "no reserved scenes (cwp_batch_reserve_scenes)");
    CWPB_CHECK(nUpd >= 0 && (nUpd == 0 || (scenes && counts)), CWP_ERR_INVALID, "NULL scene list");
    if (nUpd == 0) return CWP_OK;
    const int cap = b->fixedCap;
    std::vector<char> seen(b->nScenes, 0);
    int64_t total = 0;
    for (int i = 0; i < nUpd; i++) {
        CWPB_CHECK(scenes[i] >= 0 && scenes[i] < b->nScenes, CWP_ERR_INVALID, "scene %d out of range", scenes[i]);
        CWPB_CHECK(!seen[scenes[i]], CWP_ERR_INVALID, "scene %d listed twice", scenes[i]);
        CWPB_CHECK(counts[i] >= 0 && counts[i] <= cap, CWP_ERR_INVALID, "scene %d: %d instances (room for %d)", scenes[i], counts[i], cap);
        seen[scenes[i]] = 1; total += counts[i];
    }
    CWPB_CHECK(total == 0 || inst, CWP_ERR_INVALID, "instances are NULL");
    if (int rc = check_instances(b, inst, total, 0)) return rc;
    CWPB_CUDA(cudaSetDevice(b->device));
    // segments over the compact copy (non-empty scenes), their regions, and the roots they will get
    std::vector<int> seg{ 0 }, dst, rootOf(nUpd, -1);
    for (int i = 0; i < nUpd; i++) {
        if (counts[i] == 0) continue;
        const int r0 = scenes[i] * cap, m = counts[i];
        dst.push_back(r0); seg.push_back(seg.back() + m);
        rootOf[i] = m == 1 ? r0 : r0 + m - 2;
    }
    const int nSeg = (int)dst.size();
    CWPB_CUDA(cudaEventRecord(b->e0, b->st));
    const int minus1 = -1;
    for (int i = 0; i < nUpd; i++)   // the updated scenes are untraceable until their TLAS passes its check
        CWPB_CUDA(cudaMemcpyAsync(b->sceneRoot + scenes[i], &minus1, sizeof(int), cudaMemcpyHostToDevice, b->st));
    if (total > 0) {
        CWPB_CUDA(cudaMemcpyAsync(b->uInst, inst, (size_t)total * sizeof(cwp_instance), cudaMemcpyHostToDevice, b->st));
        for (int k = 0, at = 0; k < nSeg; k++) {   // the scene's region holds its instances (the traversal reads them there)
            const int m = seg[k + 1] - seg[k];
            CWPB_CUDA(cudaMemcpyAsync(b->inst + dst[k], b->uInst + at, (size_t)m * sizeof(cwp_instance), cudaMemcpyDeviceToDevice, b->st));
            at += m;
        }
        CWPB_CUDA(cudaMemcpyAsync(b->dstFirstTlas, dst.data(), (size_t)nSeg * sizeof(int), cudaMemcpyHostToDevice, b->st));
        CWPB_CUDA(cudaMemcpyAsync(b->segFirstTlas, seg.data(), (size_t)(nSeg + 1) * sizeof(int), cudaMemcpyHostToDevice, b->st));
        instance_boxes(b->uInst, (int)total, b->meshBox, b->uLo, b->uHi, b->st);
        if (int rc = b->tlasB.build(b->uLo, b->uHi, total, seg.data(), nSeg, b->st)) return rc;
        emit_tlas(b->tlasB, (int)total, b->segFirstTlas, nSeg, b->tlas, b->st, b->dstFirstTlas, b->tlas4);
        CWPB_CUDA(cudaGetLastError());
        if (int rc = check_tlas(b->tlas, (int)total, b->segFirstTlas, nSeg, b->err, b->st, b->dstFirstTlas, b->tlas4)) return rc;
    }
    for (int i = 0; i < nUpd; i++)
        if (rootOf[i] >= 0) CWPB_CUDA(cudaMemcpyAsync(b->sceneRoot + scenes[i], &rootOf[i], sizeof(int), cudaMemcpyHostToDevice, b->st));
    CWPB_CUDA(cudaEventRecord(b->e1, b->st));
    CWPB_CUDA(cudaEventSynchronize(b->e1));
    float ms = 0; CWPB_CUDA(cudaEventElapsedTime(&ms, b->e0, b->e1)); b->tlasMs = ms;
    return CWP_OK;
}

static int launch(cwp_batch* b, const cwp_batch_tuning& t, bool any, const float* o, const float* d, const int* sc, float* hits, int* hinst, int64_t n, cudaStream_t st,
                  const int* nDev = nullptr) {
    const WideLayout& L = b->lay[lay_index(t.width)];
    CWPB_CHECK(L.nodes, CWP_ERR_STATE, "layout width %d was not emitted (cwp_batch_options.widths)", t.width);
    BatchArgs a;
    a.nodes = L.nodes; a.tris = L.tris; a.tlas = b->tlasWidth == 4 ? b->tlas4 : b->tlas; a.tlasW = b->tlasWidth;
    a.sceneRoot = b->sceneRoot; a.inst = reinterpret_cast<const float4*>(b->inst);
    a.meshRoot = b->meshRoot[lay_index(t.width)];
    a.nScenes = b->nScenes; a.ro = (const float4*)o; a.rd = (const float4*)d; a.sceneOf = sc; a.hits = (float4*)hits; a.hitInst = hinst;
    a.n = n; a.nDev = nDev; a.cursor = b->cursor; a.fetch = t.fetch; a.err = b->err;
    BatchKernel k = pick_kernel(t.width, any, t.smem_stack != 0);
    const size_t sm = t.smem_stack ? smem_bytes(t.width, t.block) : 0;
    if (sm > 48 * 1024) CWPB_CUDA(cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per = 0;
    CWPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, t.block, sm));
    CWPB_CHECK(per > 0, CWP_ERR_INVALID, "tuning (block %d, width %d, shared stack %d) does not fit an SM", t.block, t.width, t.smem_stack);
    CWPB_CUDA(cudaMemsetAsync(b->cursor, 0, sizeof(unsigned long long), st));
    k<<<per * b->nSm, t.block, sm, st>>>(a);
    CWPB_CUDA(cudaGetLastError());
    return CWP_OK;
}

static int check_tuning(const cwp_batch* b, const cwp_batch_tuning* t) {
    CWPB_CHECK(t, CWP_ERR_INVALID, "tuning is NULL");
    CWPB_CHECK(t->block >= 32 && t->block <= kBatchMaxBlock && t->block % 32 == 0, CWP_ERR_INVALID, "block %d is not a multiple of 32 in 32..%d", t->block, kBatchMaxBlock);
    CWPB_CHECK(lay_index(t->width) >= 0, CWP_ERR_INVALID, "width %d is not 2, 4 or 8", t->width);
    CWPB_CHECK(b->lay[lay_index(t->width)].nodes, CWP_ERR_STATE, "layout width %d was not emitted", t->width);
    CWPB_CHECK(t->fetch >= 1 && t->fetch <= 32, CWP_ERR_INVALID, "fetch %d is not in 1..32", t->fetch);
    CWPB_CHECK(t->smem_stack == 0 || t->smem_stack == 1, CWP_ERR_INVALID, "smem_stack %d is not 0 or 1", t->smem_stack);
    return CWP_OK;
}

extern "C" int cwp_batch_trace(cwp_batch* b, int32_t any, const float* o, const float* d, const int32_t* sc, float* hits, int32_t* hinst, int64_t n, void* stream) {
    CWPB_CHECK(b, CWP_ERR_INVALID, "batch is NULL");
    CWPB_CHECK(b->nScenes > 0, CWP_ERR_STATE, "no scenes (cwp_batch_set_scenes)");
    CWPB_CHECK(n >= 0, CWP_ERR_INVALID, "negative ray count");
    if (n == 0) return CWP_OK;
    CWPB_CHECK(o && d && sc && hinst && (any || hits), CWP_ERR_INVALID, "NULL buffer");
    CWPB_CUDA(cudaSetDevice(b->device));
    return launch(b, b->tuning, any != 0, o, d, sc, hits, hinst, n, (cudaStream_t)stream);
}

extern "C" int cwp_batch_set_tuning(cwp_batch* b, const cwp_batch_tuning* t) {
    CWPB_CHECK(b, CWP_ERR_INVALID, "batch is NULL");
    if (int rc = check_tuning(b, t)) return rc;
    b->tuning = *t;
    return CWP_OK;
}
extern "C" int cwp_batch_get_tuning(const cwp_batch* b, cwp_batch_tuning* t) {
    CWPB_CHECK(b && t, CWP_ERR_INVALID, "NULL argument");
    *t = b->tuning;
    return CWP_OK;
}

extern "C" int cwp_batch_autotune(cwp_batch* b, const float* o, const float* d, const int32_t* sc, float* hits, int32_t* hinst, int64_t n, cwp_batch_tuning* best) {
    CWPB_CHECK(b, CWP_ERR_INVALID, "batch is NULL");
    CWPB_CHECK(b->nScenes > 0, CWP_ERR_STATE, "no scenes (cwp_batch_set_scenes)");
    CWPB_CHECK(n > 0 && o && d && sc && hits && hinst, CWP_ERR_INVALID, "empty sample or NULL buffer");
    CWPB_CUDA(cudaSetDevice(b->device));
    cwp_batch_tuning win{}; win.ms = 3e38f;
    for (int width : { 2, 4, 8 }) {
        if (!b->lay[lay_index(width)].nodes) continue;
        for (int block : { 64, 128, 256, 512 })
            for (int smem : { 0, 1 })
                for (int fetch : { 1, 2, 4, 8, 16, 32 }) {
                    cwp_batch_tuning t{}; t.block = block; t.width = width; t.fetch = fetch; t.smem_stack = smem;
                    int per = 0; const size_t sm = smem ? smem_bytes(width, block) : 0;
                    BatchKernel k = pick_kernel(width, false, smem != 0);
                    if (sm > 48 * 1024) CWPB_CUDA(cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                    if (sm > 227 * 1024 || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, block, sm) != cudaSuccess || per == 0) { cudaGetLastError(); continue; }
                    float bestMs = 3e38f;
                    for (int rep = 0; rep < 3; rep++) {   // first run warms up; the faster of the next two counts
                        CWPB_CUDA(cudaEventRecord(b->e0, b->st));
                        if (int rc = launch(b, t, false, o, d, sc, hits, hinst, n, b->st)) return rc;
                        if (int rc = launch(b, t, true, o, d, sc, nullptr, hinst, n, b->st)) return rc;
                        CWPB_CUDA(cudaEventRecord(b->e1, b->st));
                        CWPB_CUDA(cudaEventSynchronize(b->e1));
                        float ms = 0; CWPB_CUDA(cudaEventElapsedTime(&ms, b->e0, b->e1));
                        if (rep > 0) bestMs = std::min(bestMs, ms);
                    }
                    if (bestMs < win.ms) { win = t; win.ms = bestMs; }
                }
    }
    CWPB_CHECK(win.block > 0, CWP_ERR_STATE, "no tuning fits the device");
    b->tuning = win;
    if (best) *best = win;
    return cwp_batch_status(b);
}

extern "C" int cwp_batch_set_tlas_width(cwp_batch* b, int32_t width) {
    CWPB_CHECK(b, CWP_ERR_INVALID, "batch is NULL");
    CWPB_CHECK(width == 2 || width == 4, CWP_ERR_INVALID, "TLAS width %d is not 2 or 4", width);
    b->tlasWidth = width;   // both forms are always built: the next traces read the chosen one
    return CWP_OK;
}

extern "C" int cwp_batch_status(cwp_batch* b) {
    CWPB_CHECK(b, CWP_ERR_INVALID, "batch is NULL");
    CWPB_CUDA(cudaSetDevice(b->device));
    CWPB_CUDA(cudaDeviceSynchronize());
    int h = 0;
    CWPB_CUDA(cudaMemcpy(&h, b->err, sizeof(int), cudaMemcpyDeviceToHost));
    CWPB_CUDA(cudaMemset(b->err, 0, sizeof(int)));
    CWPB_CHECK(h == 0, CWP_ERR_TRAVERSAL, "traversal stopped early on some rays (status bits 0x%x: 1 = stack bound, 2 = visit budget)", h);
    return CWP_OK;
}

extern "C" int cwp_batch_info_of(const cwp_batch* b, cwp_batch_info* out) {
    CWPB_CHECK(b && out, CWP_ERR_INVALID, "NULL argument");
    memset(out, 0, sizeof(*out));
    out->n_blas = b->nMesh; out->n_scenes = b->nScenes; out->n_tris = b->nTris; out->n_instances = b->nInst;
    for (int i = 0; i < 3; i++) out->node_bytes[i] = b->lay[i].nNodes * b->lay[i].stride() * 16;
    out->blas_build_ms = b->blasMs; out->tlas_build_ms = b->tlasMs; out->blas_hploc_launches = 1;
    return CWP_OK;
}

extern "C" int cwp_batch_download(const cwp_batch* b, int32_t width, float* nodes, int64_t* nNodeF4, float* tris, int64_t* nTriF4) {
    CWPB_CHECK(b, CWP_ERR_INVALID, "batch is NULL");
    CWPB_CHECK(lay_index(width) >= 0, CWP_ERR_INVALID, "width %d is not 2, 4 or 8", width);
    const WideLayout& L = b->lay[lay_index(width)];
    CWPB_CHECK(L.nodes, CWP_ERR_STATE, "layout width %d was not emitted", width);
    CWPB_CUDA(cudaSetDevice(b->device));
    if (nNodeF4) *nNodeF4 = L.nNodes * L.stride();
    const int64_t nr = b->refs[lay_index(width)] ? b->refs[lay_index(width)] : b->nTris;
    if (nTriF4) *nTriF4 = 3 * nr;
    if (nodes) CWPB_CUDA(cudaMemcpy(nodes, L.nodes, (size_t)L.nNodes * L.stride() * sizeof(float4), cudaMemcpyDeviceToHost));
    if (tris) CWPB_CUDA(cudaMemcpy(tris, L.tris, (size_t)3 * nr * sizeof(float4), cudaMemcpyDeviceToHost));
    return CWP_OK;
}

extern "C" int cwp_batch_blas_root(const cwp_batch* b, int32_t width, int32_t mesh, int32_t* root) {
    CWPB_CHECK(b && root, CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(lay_index(width) >= 0 && b->lay[lay_index(width)].nodes, CWP_ERR_STATE, "layout width %d was not emitted", width);
    CWPB_CHECK(mesh >= 0 && mesh < b->nMesh, CWP_ERR_INVALID, "mesh %d out of range", mesh);
    *root = b->meshRootHost[lay_index(width)][mesh];
    return CWP_OK;
}

extern "C" int cwp_batch_download_tlas(const cwp_batch* b, float* nodes, int64_t* nNodeF4, int32_t* roots, cwp_instance* inst) {
    CWPB_CHECK(b, CWP_ERR_INVALID, "batch is NULL");
    CWPB_CHECK(b->nScenes > 0, CWP_ERR_STATE, "no scenes");
    CWPB_CUDA(cudaSetDevice(b->device));
    const int64_t stride = b->tlasWidth == 4 ? 8 : 4;   // the form the traversal reads
    if (nNodeF4) *nNodeF4 = stride * b->nInst;
    if (nodes && b->nInst) CWPB_CUDA(cudaMemcpy(nodes, b->tlasWidth == 4 ? b->tlas4 : b->tlas, (size_t)stride * b->nInst * sizeof(float4), cudaMemcpyDeviceToHost));
    if (roots) CWPB_CUDA(cudaMemcpy(roots, b->sceneRoot, (size_t)b->nScenes * sizeof(int), cudaMemcpyDeviceToHost));
    if (inst && b->nInst) {
        CWPB_CUDA(cudaMemcpy(inst, b->inst, (size_t)b->nInst * sizeof(cwp_instance), cudaMemcpyDeviceToHost));
        const std::vector<int>& R = b->meshRootHost[lay_index(b->tuning.width)];
        for (int64_t i = 0; i < b->nInst; i++) inst[i].root = R[inst[i].mesh];   // roots of the layout the tuning traces
    }
    return CWP_OK;
}

namespace cwpb {
int batch_trace_dev(cwp_batch* b, bool any, const float4* o, const float4* d, const int* sc, float4* hits, int* inst, int64_t n, cudaStream_t st, const int* nDev) {
    CWPB_CHECK(b->nScenes > 0, CWP_ERR_STATE, "no scenes");
    if (n <= 0 && !nDev) return CWP_OK;
    return launch(b, b->tuning, any, (const float*)o, (const float*)d, sc, (float*)hits, inst, n, st, nDev);
}
const float4* batch_tris(const cwp_batch* b) { return b->lay[lay_index(b->tuning.width)].tris; }
const cwp_instance* batch_instances(const cwp_batch* b) { return b->inst; }
int batch_mesh_count(const cwp_batch* b) { return b->nMesh; }
const int* batch_mesh_first(const cwp_batch* b) { return b->meshFirstDev; }
int64_t batch_tri_count(const cwp_batch* b) { return b->nTris; }
const float4* batch_tri_soup(const cwp_batch* b) { return b->triV; }
const float4* batch_normals(const cwp_batch* b) { return b->nrm; }
const int* batch_mesh_first_host(const cwp_batch* b) { return b->meshFirst.data(); }
int batch_device(const cwp_batch* b) { return b->device; }
}  // namespace cwpb
