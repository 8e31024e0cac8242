// wide_emit.cu - encodings of segmented H-PLOC trees (see wide_emit.h).
#include "wide_emit.h"
#include "vecmath.h"
#include <cub/device/device_scan.cuh>
#include <vector>

namespace cwpb {

static const float kEmpty = 3e37f;   // bounds of an empty child slot (never hit before tmax)

__device__ __forceinline__ float3 node_lo(const float4* bn, int i) { const float4 a = __ldg(bn + 2 * i); return f3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 node_hi(const float4* bn, int i) { const float4 a = __ldg(bn + 2 * i + 1); return f3(a.x, a.y, a.z); }
__device__ __forceinline__ int node_left(const float4* bn, int i) { return __float_as_int(__ldg(bn + 2 * i).w); }
__device__ __forceinline__ int node_right(const float4* bn, int i) { return __float_as_int(__ldg(bn + 2 * i + 1).w); }
__device__ __forceinline__ float half_area3(float3 l, float3 h) { const float3 e = h - l; return e.x * e.y + e.y * e.z + e.z * e.x; }

__global__ void k_tri_boxes(const float4* __restrict__ triV, int64_t n, float4* lo, float4* hi) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = triV[3 * i], b = triV[3 * i + 1], c = triV[3 * i + 2];
    lo[i] = make_float4(fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)), fminf(a.z, fminf(b.z, c.z)), 0.f);
    hi[i] = make_float4(fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)), fmaxf(a.z, fmaxf(b.z, c.z)), 0.f);
}
void triangle_boxes(const float4* triV, int64_t n, float4* lo, float4* hi, cudaStream_t st) {
    if (n > 0) k_tri_boxes<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(triV, n, lo, hi);
}

__device__ __forceinline__ int seg_root(const int* segFirst, int s) {
    const int f = segFirst[s], m = segFirst[s + 1] - f;
    return 2 * f - s + (m > 1 ? 2 * m - 2 : 0);
}

__global__ void k_root_boxes(const float4* __restrict__ bn, const int* __restrict__ segFirst, int nSeg, float4* box) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nSeg) return;
    const int r = seg_root(segFirst, s);
    box[2 * s] = bn[2 * r]; box[2 * s + 1] = bn[2 * r + 1];
}
void root_boxes(const SegBuilder& B, const int* segFirstDev, int nSeg, float4* meshBox, cudaStream_t st) {
    k_root_boxes<<<(nSeg + 127) / 128, 128, 0, st>>>(B.nodes, segFirstDev, nSeg, meshBox);
}

// ---------------- level-by-level emission ----------------
// plan: the children of each item's wide node (binary node ids, in child order for widths 2 / 4 and in slot order
// for width 8, -1 = empty) and the packed counts (inner children << 32 | leaf triangles) that the scan turns into
// child and triangle offsets.
__global__ void k_wide_plan(int W, int leafMax, const int* __restrict__ items, int nItems, int rootLevel, const float4* __restrict__ bn,
                            const int* __restrict__ bcnt, int nBin, int* plan, unsigned long long* sums, int* err) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nItems) return;
    const int b = items[j];
    int ch[8]; int nc = 0;
    // a binary node id outside the node array means a broken build: flag it and emit nothing under this node
    auto bad = [&](int x) { if (x < 0 || x >= nBin) { atomicOr(err, 1); return true; } return false; };
    if (bad(b)) { for (int k = 0; k < 8; k++) plan[8 * j + k] = -1; sums[j] = 0; return; }
    if (rootLevel && bcnt[b] <= leafMax) { ch[0] = b; nc = 1; }   // the whole mesh is one leaf under the root
    else {
        ch[0] = node_left(bn, b); ch[1] = node_right(bn, b); nc = 2;
        if (bad(ch[0]) || bad(ch[1])) { for (int k = 0; k < 8; k++) plan[8 * j + k] = -1; sums[j] = 0; return; }
        while (nc < W) {   // open the largest-area child that is too big to be a leaf
            int best = -1; float bestA = -1.f;
            for (int k = 0; k < nc; k++)
                if (bcnt[ch[k]] > leafMax) { const float a = half_area3(node_lo(bn, ch[k]), node_hi(bn, ch[k])); if (a > bestA) { bestA = a; best = k; } }
            if (best < 0) break;
            const int o = ch[best], l = node_left(bn, o), r = node_right(bn, o);
            if (bad(l) || bad(r)) break;
            ch[best] = l; ch[nc++] = r;
        }
    }
    int out[8];
    for (int k = 0; k < 8; k++) out[k] = k < nc ? ch[k] : -1;
    if (W == 8) {
        // slots: repeatedly the (child, free slot) pair of lowest cost, slot s costing -dot(child centre - node centre,
        // octant direction of s) with bit set = negative axis, so the ray-octant traversal order visits near children first
        const float3 nl = node_lo(bn, b), nh = node_hi(bn, b), pc = (nl + nh) * 0.5f;
        float cost[8][8]; bool used[8] = { false, false, false, false, false, false, false, false };
        for (int k = 0; k < 8; k++) out[k] = -1;
        for (int c = 0; c < nc; c++) {
            const float3 cc = (node_lo(bn, ch[c]) + node_hi(bn, ch[c])) * 0.5f - pc;
            for (int s = 0; s < 8; s++) cost[c][s] = -(cc.x * (s & 1 ? -1.f : 1.f) + cc.y * (s & 2 ? -1.f : 1.f) + cc.z * (s & 4 ? -1.f : 1.f));
        }
        for (int it = 0; it < nc; it++) {
            float bc = 3e38f; int bi = -1, bs = -1;
            for (int c = 0; c < nc; c++) if (!used[c]) for (int s = 0; s < 8; s++) if (out[s] < 0 && cost[c][s] < bc) { bc = cost[c][s]; bi = c; bs = s; }
            if (bi < 0) for (int c = 0; c < nc && bi < 0; c++) if (!used[c]) for (int s = 0; s < 8; s++) if (out[s] < 0) { bi = c; bs = s; break; }
            used[bi] = true; out[bs] = ch[bi];
        }
    }
    unsigned nInner = 0, nTri = 0;
    for (int k = 0; k < 8; k++) {
        const int c = out[k];
        if (c < 0) continue;
        if (bcnt[c] > leafMax) nInner++; else nTri += (unsigned)max(bcnt[c], 0);
    }
    for (int k = 0; k < 8; k++) plan[8 * j + k] = out[k];
    sums[j] = ((unsigned long long)nInner << 32) | nTri;
}

// smallest exponent e with lo + 255 * 2^e >= hi (-100 for a flat axis)
__device__ __forceinline__ int quant_exp(float lo, float hi) {
    const float ext = hi - lo;
    if (!(ext > 0.f)) return -100;
    int e; const float f = frexpf(ext / 255.f, &e);   // ext / 255 = f 2^e, f in [0.5, 1)
    if (f == 0.5f) e -= 1;                               // an exact power of two
    if (e < -100) e = -100;
    while (lo + 255.f * ldexpf(1.f, e) < hi) e++;
    return e;
}
// conservative 8-bit plane: the difference is rounded outward before floor / ceil
__device__ __forceinline__ unsigned quant_plane(float v, float origin, float scaleInv, bool up) {
    const float f = (up ? __fsub_ru(v, origin) : __fsub_rd(v, origin)) * scaleInv;
    const float q = up ? ceilf(f) : floorf(f);
    return (unsigned)fminf(fmaxf(q, 0.f), 255.f);
}

__global__ void k_wide_emit(int W, int leafMax, const int* __restrict__ items, int nItems, int64_t levelStart, int64_t nextStart, int rootLevel,
                            const int* __restrict__ plan, const unsigned long long* __restrict__ prefix, int64_t triCursor,
                            const float4* __restrict__ bn, const int* __restrict__ bcnt, int nBin, const float4* __restrict__ triV, int nPrim,
                            float4* wnodes, float4* wtris, int* nextItems, int* err) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nItems) return;
    const int b = items[j];
    if (b < 0 || b >= nBin) { atomicOr(err, 1); return; }   // flagged by the plan pass; the build is rejected
    const unsigned long long p = prefix[j];
    const int innerOff = (int)(p >> 32);
    const int64_t childBase = nextStart + innerOff, triBase = triCursor + (int64_t)(p & 0xffffffffull);
    int cref[8], ccnt[8]; float3 clo[8], chi[8];
    int ord = 0, off = 0;
    for (int k = 0; k < 8; k++) {
        const int c = plan[8 * j + k];
        cref[k] = -1; ccnt[k] = 0;
        clo[k] = f3(kEmpty, kEmpty, kEmpty); chi[k] = clo[k];
        if (c < 0 || (W == 2 && k >= 2) || (W == 4 && k >= 4)) continue;
        clo[k] = node_lo(bn, c); chi[k] = node_hi(bn, c);
        if (bcnt[c] > leafMax) {   // inner child: next level, numbered in this order
            nextItems[innerOff + ord] = c;
            cref[k] = (int)(childBase + ord); ccnt[k] = 0; ord++;
        } else {                   // leaf: the subtree's triangles, left to right
            int stack[8], sp = 0, n = 0; stack[sp++] = c;
            const int want = bcnt[c];
            while (sp > 0) {
                const int x = stack[--sp];
                if (x < 0 || x >= nBin) { atomicOr(err, 1); continue; }
                if (node_right(bn, x) < 0) {
                    const int prim = node_left(bn, x);
                    if (prim < 0 || prim >= nPrim || n >= want) { atomicOr(err, 1); continue; }
                    const float4 v0 = triV[3 * (size_t)prim], v1 = triV[3 * (size_t)prim + 1], v2 = triV[3 * (size_t)prim + 2];
                    float4* o = wtris + 3 * (size_t)(triBase + off + n);
                    o[0] = v0;
                    o[1] = make_float4(v1.x - v0.x, v1.y - v0.y, v1.z - v0.z, v1.w);
                    o[2] = make_float4(v2.x - v0.x, v2.y - v0.y, v2.z - v0.z, 0.f);
                    n++;
                } else if (sp + 2 <= 8) { stack[sp++] = node_right(bn, x); stack[sp++] = node_left(bn, x); }
            }
            cref[k] = W == 8 ? off : (int)(triBase + off); ccnt[k] = n; off += n;
        }
    }
    const int64_t w = levelStart + j;
    if (W == 2) {
        float4* o = wnodes + 4 * (size_t)w;
        o[0] = make_float4(clo[0].x, chi[0].x, clo[0].y, chi[0].y);
        o[1] = make_float4(clo[1].x, chi[1].x, clo[1].y, chi[1].y);
        o[2] = make_float4(clo[0].z, chi[0].z, clo[1].z, chi[1].z);
        o[3] = make_float4(__int_as_float(cref[0]), __int_as_float(cref[1]), __int_as_float(ccnt[0]), __int_as_float(ccnt[1]));
    } else if (W == 4) {
        float4* o = wnodes + 8 * (size_t)w;
        o[0] = make_float4(clo[0].x, clo[1].x, clo[2].x, clo[3].x); o[1] = make_float4(chi[0].x, chi[1].x, chi[2].x, chi[3].x);
        o[2] = make_float4(clo[0].y, clo[1].y, clo[2].y, clo[3].y); o[3] = make_float4(chi[0].y, chi[1].y, chi[2].y, chi[3].y);
        o[4] = make_float4(clo[0].z, clo[1].z, clo[2].z, clo[3].z); o[5] = make_float4(chi[0].z, chi[1].z, chi[2].z, chi[3].z);
        o[6] = make_float4(__int_as_float(cref[0]), __int_as_float(cref[1]), __int_as_float(cref[2]), __int_as_float(cref[3]));
        o[7] = make_float4(__int_as_float(ccnt[0]), __int_as_float(ccnt[1]), __int_as_float(ccnt[2]), __int_as_float(ccnt[3]));
    } else {
        const float3 nl = node_lo(bn, b), nh = node_hi(bn, b);
        const int ex = quant_exp(nl.x, nh.x), ey = quant_exp(nl.y, nh.y), ez = quant_exp(nl.z, nh.z);
        const float ix = ldexpf(1.f, -ex), iy = ldexpf(1.f, -ey), iz = ldexpf(1.f, -ez);
        unsigned q[6][2] = { { 0u, 0u }, { 0u, 0u }, { 0u, 0u }, { 0u, 0u }, { 0u, 0u }, { 0u, 0u } }, meta[2] = { 0u, 0u }, imask = 0;
        for (int s = 0; s < 8; s++) {
            const int c = plan[8 * j + s];
            if (c < 0) continue;
            const int wd = s >> 2, sh = 8 * (s & 3);
            unsigned m;
            if (ccnt[s] > 0) m = 0x80u | ((unsigned)(ccnt[s] - 1) << 5) | (unsigned)cref[s];
            else { m = 0x40u; imask |= 1u << s; }
            meta[wd] |= m << sh;
            q[0][wd] |= quant_plane(clo[s].x, nl.x, ix, false) << sh; q[3][wd] |= quant_plane(chi[s].x, nl.x, ix, true) << sh;
            q[1][wd] |= quant_plane(clo[s].y, nl.y, iy, false) << sh; q[4][wd] |= quant_plane(chi[s].y, nl.y, iy, true) << sh;
            q[2][wd] |= quant_plane(clo[s].z, nl.z, iz, false) << sh; q[5][wd] |= quant_plane(chi[s].z, nl.z, iz, true) << sh;
        }
        const unsigned ew = (unsigned)(ex + 127) | ((unsigned)(ey + 127) << 8) | ((unsigned)(ez + 127) << 16) | (imask << 24);
        float4* o = wnodes + 5 * (size_t)w;
        o[0] = make_float4(nl.x, nl.y, nl.z, __uint_as_float(ew));
        o[1] = make_float4(__int_as_float((int)childBase), __int_as_float((int)triBase), __uint_as_float(meta[0]), __uint_as_float(meta[1]));
        o[2] = make_float4(__uint_as_float(q[0][0]), __uint_as_float(q[0][1]), __uint_as_float(q[1][0]), __uint_as_float(q[1][1]));
        o[3] = make_float4(__uint_as_float(q[2][0]), __uint_as_float(q[2][1]), __uint_as_float(q[3][0]), __uint_as_float(q[3][1]));
        o[4] = make_float4(__uint_as_float(q[4][0]), __uint_as_float(q[4][1]), __uint_as_float(q[5][0]), __uint_as_float(q[5][1]));
    }
    (void)rootLevel;
}

void free_wide(WideLayout& w) {
    cudaFree(w.nodes); cudaFree(w.tris);
    w.nodes = nullptr; w.tris = nullptr; w.nNodes = w.capNodes = 0;
}

int emit_wide(const SegBuilder& B, const int* segFirstHost, int nSeg, const float4* triV, int width, int leafMax, WideLayout& out, cudaStream_t st) {
    CWPB_CHECK(width == 2 || width == 4 || width == 8, CWP_ERR_INVALID, "layout width %d is not 2, 4 or 8", width);
    CWPB_CHECK(leafMax >= 1 && leafMax <= (width == 8 ? 3 : 8), CWP_ERR_INVALID, "leaf size %d out of range for width %d", leafMax, width);
    const int64_t n = segFirstHost[nSeg];
    free_wide(out);
    out.width = width;
    // wide nodes: at most the binary nodes above leaf size (<= 2 n / (leafMax + 1)) plus one root per mesh
    out.capNodes = 2 * n / (leafMax + 1) + nSeg + 64;
    CWPB_CUDA(cudaMalloc(&out.nodes, (size_t)out.capNodes * out.stride() * sizeof(float4)));
    CWPB_CUDA(cudaMalloc(&out.tris, (size_t)3 * n * sizeof(float4)));
    int *items = nullptr, *next = nullptr, *plan = nullptr, *err = nullptr; unsigned long long *sums = nullptr, *prefix = nullptr; void* tmp = nullptr; size_t tmpBytes = 0;
    unsigned long long* hostTot = nullptr;
    const int64_t capItems = out.capNodes;
    const int nBin = (int)(2 * n - nSeg);
    auto cleanup = [&]() { cudaFree(items); cudaFree(next); cudaFree(plan); cudaFree(err); cudaFree(sums); cudaFree(prefix); cudaFree(tmp); cudaFreeHost(hostTot); };
    cudaError_t e = cudaMalloc(&items, (size_t)capItems * 4);
    if (e == cudaSuccess) e = cudaMalloc(&err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMalloc(&next, (size_t)capItems * 4);
    if (e == cudaSuccess) e = cudaMalloc(&plan, (size_t)capItems * 8 * 4);
    if (e == cudaSuccess) e = cudaMalloc(&sums, (size_t)capItems * 8);
    if (e == cudaSuccess) e = cudaMalloc(&prefix, (size_t)capItems * 8);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tmpBytes, sums, prefix, (int)capItems);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tmpBytes > 0 ? tmpBytes : 16);
    if (e == cudaSuccess) e = cudaMallocHost(&hostTot, 2 * sizeof(unsigned long long));
    if (e != cudaSuccess) { cleanup(); return set_error(CWP_ERR_NOMEM, "layout scratch: %s", cudaGetErrorString(e)); }
    std::vector<int> roots(nSeg);
    for (int s = 0; s < nSeg; s++) { const int f = segFirstHost[s], m = segFirstHost[s + 1] - f; roots[s] = 2 * f - s + (m > 1 ? 2 * m - 2 : 0); }
    e = cudaMemcpyAsync(items, roots.data(), (size_t)nSeg * 4, cudaMemcpyHostToDevice, st);
    int64_t nItems = nSeg, levelStart = 0, cursor = nSeg, triCursor = 0; int rootLevel = 1;
    while (e == cudaSuccess && nItems > 0) {
        const unsigned g = (unsigned)((nItems + 127) / 128);
        k_wide_plan<<<g, 128, 0, st>>>(width, leafMax, items, (int)nItems, rootLevel, B.nodes, B.count, nBin, plan, sums, err);
        size_t tb = tmpBytes;
        e = cub::DeviceScan::ExclusiveSum(tmp, tb, sums, prefix, (int)nItems, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hostTot, prefix + nItems - 1, 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hostTot + 1, sums + nItems - 1, 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) break;
        const unsigned long long tot = hostTot[0] + hostTot[1];
        const int64_t nNext = (int64_t)(tot >> 32), nTri = (int64_t)(tot & 0xffffffffull);
        if (cursor + nNext > out.capNodes || triCursor + nTri > n) { cleanup(); return set_error(CWP_ERR_INVALID, "layout emission overflow (level of %lld nodes)", (long long)nItems); }
        k_wide_emit<<<g, 128, 0, st>>>(width, leafMax, items, (int)nItems, levelStart, cursor, rootLevel, plan, prefix, triCursor, B.nodes, B.count, nBin,
                                       triV, (int)n, out.nodes, out.tris, next, err);
        e = cudaGetLastError();
        levelStart = cursor; cursor += nNext; triCursor += nTri; nItems = nNext; rootLevel = 0;
        int* t = items; items = next; next = t;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost);
    cleanup();
    if (e != cudaSuccess) return set_error(CWP_ERR_CUDA, "layout emission: %s", cudaGetErrorString(e));
    CWPB_CHECK(herr == 0, CWP_ERR_INVALID, "layout emission found a broken binary tree (node or primitive reference out of range)");
    CWPB_CHECK(triCursor == n, CWP_ERR_INVALID, "layout emission placed %lld of %lld triangles", (long long)triCursor, (long long)n);
    out.nNodes = cursor;
    return CWP_OK;
}

// ---------------- TLAS ----------------
// One thread per binary inner node of a scene (or its single leaf): writes that node's TLAS entry in BVH2 form (two
// children) and, when tlas4 is given, in width-4 form (its grandchildren: a child that is an instance stays one child,
// an inner child contributes its two children). Every binary inner node gets an entry of each form, so both are
// written in one pass with no numbering step; traversal of the width-4 form starts at the same root and only reaches
// every other level. dstFirst (may be NULL = segFirst): where segment s's nodes and instances live in the TLAS /
// instance arrays, when the build ran over a compact copy of some scenes' instances (incremental updates of fixed
// per-scene regions).
__global__ void k_tlas(const float4* __restrict__ bn, int nInst, const int* __restrict__ segFirst, int nSeg, float4* tlas, float4* tlas4,
                       const int* __restrict__ dstFirst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nInst) return;
    int lo = 0, hi = nSeg - 1;
    while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (segFirst[mid] <= i) lo = mid; else hi = mid - 1; }
    const int s = lo, f = segFirst[s], m = segFirst[s + 1] - f, base = 2 * f - s, j = i - f, d0 = dstFirst ? dstFirst[s] : f;
    const int end = base + 2 * m - 1;   // the scene's binary nodes: leaves [base, base + m), inner [base + m, end)
    auto inside = [&](int c) { return c >= base && c < end; };
    int ch[2]; int outNode;
    if (m == 1) { if (j != 0) return; ch[0] = base; ch[1] = -1; outNode = d0; }
    else { if (j >= m - 1) return; const int b = base + m + j; ch[0] = node_left(bn, b); ch[1] = node_right(bn, b); outNode = d0 + j; }
    for (int q = 0; q < 2; q++) if (!inside(ch[q])) ch[q] = -1;   // outside the scene's region
    // a child entry: box, reference (instance or output node), count (1 instance, 0 inner)
    auto entry = [&](int c, float3& l, float3& h, int& ref, int& cnt) {
        if (c < 0) { l = h = f3(kEmpty, kEmpty, kEmpty); ref = -1; cnt = 0; return; }
        l = node_lo(bn, c); h = node_hi(bn, c);
        if (c < base + m) { ref = d0 + (node_left(bn, c) - f); cnt = 1; }   // a leaf: the instance
        else { ref = d0 + (c - base - m); cnt = 0; }
    };
    float3 l[2], h[2]; int c[2], k[2];
    for (int q = 0; q < 2; q++) entry(ch[q], l[q], h[q], c[q], k[q]);
    if (tlas) {
        float4* o = tlas + 4 * (size_t)outNode;
        o[0] = make_float4(l[0].x, h[0].x, l[0].y, h[0].y);
        o[1] = make_float4(l[1].x, h[1].x, l[1].y, h[1].y);
        o[2] = make_float4(l[0].z, h[0].z, l[1].z, h[1].z);
        o[3] = make_float4(__int_as_float(c[0]), __int_as_float(c[1]), __int_as_float(k[0]), __int_as_float(k[1]));
    }
    if (tlas4) {
        int g[4] = { -1, -1, -1, -1 }, ng = 0;
        for (int q = 0; q < 2; q++) {
            if (ch[q] < 0) continue;
            if (ch[q] < base + m) g[ng++] = ch[q];
            else for (int r = 0; r < 2; r++) { const int x = r ? node_right(bn, ch[q]) : node_left(bn, ch[q]); if (inside(x)) g[ng++] = x; }
        }
        float3 gl[4], gh[4]; int gc[4], gk[4];
        for (int q = 0; q < 4; q++) entry(g[q], gl[q], gh[q], gc[q], gk[q]);
        float4* o = tlas4 + 8 * (size_t)outNode;
        o[0] = make_float4(gl[0].x, gl[1].x, gl[2].x, gl[3].x); o[1] = make_float4(gh[0].x, gh[1].x, gh[2].x, gh[3].x);
        o[2] = make_float4(gl[0].y, gl[1].y, gl[2].y, gl[3].y); o[3] = make_float4(gh[0].y, gh[1].y, gh[2].y, gh[3].y);
        o[4] = make_float4(gl[0].z, gl[1].z, gl[2].z, gl[3].z); o[5] = make_float4(gh[0].z, gh[1].z, gh[2].z, gh[3].z);
        o[6] = make_float4(__int_as_float(gc[0]), __int_as_float(gc[1]), __int_as_float(gc[2]), __int_as_float(gc[3]));
        o[7] = make_float4(__int_as_float(gk[0]), __int_as_float(gk[1]), __int_as_float(gk[2]), __int_as_float(gk[3]));
    }
}
void emit_tlas(const SegBuilder& B, int nInst, const int* segFirstDev, int nSeg, float4* tlas, cudaStream_t st, const int* dstFirstDev, float4* tlas4) {
    if (nInst > 0) k_tlas<<<(nInst + 127) / 128, 128, 0, st>>>(B.nodes, nInst, segFirstDev, nSeg, tlas, tlas4, dstFirstDev);
}

__global__ void k_inst_boxes(const cwp_instance* __restrict__ inst, int n, const float4* __restrict__ meshBox, float4* lo, float4* hi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const cwp_instance& I = inst[i];
    const float4 bl = meshBox[2 * I.mesh], bh = meshBox[2 * I.mesh + 1];
    float3 mn = f3(3.4e38f, 3.4e38f, 3.4e38f), mx = f3(-3.4e38f, -3.4e38f, -3.4e38f);
    for (int c = 0; c < 8; c++) {
        const float x = c & 1 ? bh.x : bl.x, y = c & 2 ? bh.y : bl.y, z = c & 4 ? bh.z : bl.z;
        const float3 w = f3(I.fwd[0] * x + I.fwd[1] * y + I.fwd[2] * z + I.fwd[3], I.fwd[4] * x + I.fwd[5] * y + I.fwd[6] * z + I.fwd[7],
                            I.fwd[8] * x + I.fwd[9] * y + I.fwd[10] * z + I.fwd[11]);
        mn = vmin(mn, w); mx = vmax(mx, w);
    }
    // the corners are rounded images of the exact ones: widen by a few ulps so the box stays conservative
    const float3 e = (vmax(f3(fabsf(mn.x), fabsf(mn.y), fabsf(mn.z)), f3(fabsf(mx.x), fabsf(mx.y), fabsf(mx.z)))) * 4.8e-7f;
    lo[i] = make_float4(mn.x - e.x, mn.y - e.y, mn.z - e.z, 0.f); hi[i] = make_float4(mx.x + e.x, mx.y + e.y, mx.z + e.z, 0.f);
}
void instance_boxes(const cwp_instance* inst, int nInst, const float4* meshBox, float4* lo, float4* hi, cudaStream_t st) {
    if (nInst > 0) k_inst_boxes<<<(nInst + 127) / 128, 128, 0, st>>>(inst, nInst, meshBox, lo, hi);
}

}  // namespace cwpb

namespace cwpb {
// Every child and leaf reference of a wide layout lies inside the arrays, and inner children come after their parent
// (so traversal terminates): the check that stands between the builder and the traversal kernels.
__global__ void k_check_wide(int W, const float4* __restrict__ nodes, int64_t nNodes, int64_t nTris, int* bad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nNodes) return;
    bool ok = true;
    if (W == 2) {
        const float4 m = nodes[4 * i + 3];
        const int c[2] = { __float_as_int(m.x), __float_as_int(m.y) }, k[2] = { __float_as_int(m.z), __float_as_int(m.w) };
        for (int q = 0; q < 2; q++) {
            if (k[q] > 0) ok &= c[q] >= 0 && (int64_t)c[q] + k[q] <= nTris;
            else if (k[q] == 0) ok &= c[q] == -1 || (c[q] > i && c[q] < nNodes);
            else ok = false;
        }
    } else if (W == 4) {
        const float4 cf = nodes[8 * i + 6], kf = nodes[8 * i + 7];
        const int c[4] = { __float_as_int(cf.x), __float_as_int(cf.y), __float_as_int(cf.z), __float_as_int(cf.w) };
        const int k[4] = { __float_as_int(kf.x), __float_as_int(kf.y), __float_as_int(kf.z), __float_as_int(kf.w) };
        for (int q = 0; q < 4; q++) {
            if (k[q] > 0) ok &= c[q] >= 0 && (int64_t)c[q] + k[q] <= nTris;
            else if (k[q] == 0) ok &= c[q] == -1 || (c[q] > i && c[q] < nNodes);
            else ok = false;
        }
    } else {
        const float4 f0 = nodes[5 * i], f1 = nodes[5 * i + 1];
        const unsigned imask = __float_as_uint(f0.w) >> 24, m0 = __float_as_uint(f1.z), m1 = __float_as_uint(f1.w);
        const int childBase = __float_as_int(f1.x), triBase = __float_as_int(f1.y);
        if (imask) ok &= childBase > i && (int64_t)childBase + __popc(imask) <= nNodes;
        for (int s = 0; s < 8; s++) {
            const unsigned m = ((s < 4 ? m0 : m1) >> (8 * (s & 3))) & 255u;
            if (m & 0x80u) ok &= triBase >= 0 && (int64_t)triBase + (m & 31u) + ((m >> 5) & 3u) + 1 <= nTris;
        }
    }
    if (!ok) atomicOr(bad, 1);
}
__global__ void k_check_tlas(const float4* __restrict__ tlas, int nInst, const int* __restrict__ segFirst, int nSeg, int* bad, const int* __restrict__ dstFirst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nInst) return;
    int lo = 0, hi = nSeg - 1;
    while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (segFirst[mid] <= i) lo = mid; else hi = mid - 1; }
    const int m = segFirst[lo + 1] - segFirst[lo], j = i - segFirst[lo], f = dstFirst ? dstFirst[lo] : segFirst[lo];
    if (j >= (m == 1 ? 1 : m - 1)) return;   // unused slot of the scene's region
    const int node = f + j;
    const float4 mt = tlas[4 * (size_t)node + 3];
    const int c[2] = { __float_as_int(mt.x), __float_as_int(mt.y) }, k[2] = { __float_as_int(mt.z), __float_as_int(mt.w) };
    bool ok = true;
    for (int q = 0; q < 2; q++) {
        if (c[q] == -1) continue;
        if (k[q] > 0) ok &= k[q] == 1 && c[q] >= f && c[q] < f + m;           // an instance of this scene
        else ok &= k[q] == 0 && c[q] >= f && c[q] < node;                     // an inner node of this scene, built before its parent
    }
    if (!ok) atomicOr(bad, 1);
}
int check_wide(const WideLayout& w, int64_t nTris, int* dBad, cudaStream_t st) {
    CWPB_CUDA(cudaMemsetAsync(dBad, 0, sizeof(int), st));
    if (w.nNodes > 0) k_check_wide<<<(unsigned)((w.nNodes + 255) / 256), 256, 0, st>>>(w.width, w.nodes, w.nNodes, nTris, dBad);
    int h = 0;
    CWPB_CUDA(cudaMemcpyAsync(&h, dBad, sizeof(int), cudaMemcpyDeviceToHost, st));
    CWPB_CUDA(cudaStreamSynchronize(st));
    CWPB_CHECK(h == 0, CWP_ERR_INVALID, "width-%d layout has an out-of-range child or triangle reference", w.width);
    return CWP_OK;
}
// the width-4 entries: every instance reference inside the scene's instances, every inner reference an entry written
// before its parent (grandchildren of the H-PLOC tree have lower indices), empty slots marked -1
__global__ void k_check_tlas4(const float4* __restrict__ tlas4, int nInst, const int* __restrict__ segFirst, int nSeg, int* bad, const int* __restrict__ dstFirst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nInst) return;
    int lo = 0, hi = nSeg - 1;
    while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (segFirst[mid] <= i) lo = mid; else hi = mid - 1; }
    const int m = segFirst[lo + 1] - segFirst[lo], j = i - segFirst[lo], f = dstFirst ? dstFirst[lo] : segFirst[lo];
    if (j >= (m == 1 ? 1 : m - 1)) return;
    const int node = f + j;
    const float4 cf = tlas4[8 * (size_t)node + 6], kf = tlas4[8 * (size_t)node + 7];
    const int c[4] = { __float_as_int(cf.x), __float_as_int(cf.y), __float_as_int(cf.z), __float_as_int(cf.w) };
    const int k[4] = { __float_as_int(kf.x), __float_as_int(kf.y), __float_as_int(kf.z), __float_as_int(kf.w) };
    bool ok = true;
    for (int q = 0; q < 4; q++) {
        if (c[q] == -1) { ok &= k[q] == 0; continue; }
        if (k[q] > 0) ok &= k[q] == 1 && c[q] >= f && c[q] < f + m;
        else ok &= k[q] == 0 && c[q] >= f && c[q] < node;
    }
    if (!ok) atomicOr(bad, 1);
}
int check_tlas(const float4* tlas, int nInst, const int* segFirstDev, int nSeg, int* dBad, cudaStream_t st, const int* dstFirstDev, const float4* tlas4) {
    CWPB_CUDA(cudaMemsetAsync(dBad, 0, sizeof(int), st));
    if (nInst > 0) k_check_tlas<<<(nInst + 127) / 128, 128, 0, st>>>(tlas, nInst, segFirstDev, nSeg, dBad, dstFirstDev);
    if (nInst > 0 && tlas4) k_check_tlas4<<<(nInst + 127) / 128, 128, 0, st>>>(tlas4, nInst, segFirstDev, nSeg, dBad, dstFirstDev);
    int h = 0;
    CWPB_CUDA(cudaMemcpyAsync(&h, dBad, sizeof(int), cudaMemcpyDeviceToHost, st));
    CWPB_CUDA(cudaStreamSynchronize(st));
    CWPB_CHECK(h == 0, CWP_ERR_INVALID, "TLAS has an out-of-range child or instance reference");
    return CWP_OK;
}
}  // namespace cwpb
