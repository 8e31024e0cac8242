/* oracle.c - TEST INFRASTRUCTURE ONLY: a scalar CPU restatement of the reference path tracer's algorithms for the
 * diffuse benchmark path (YJLi-new/cuda-wavefront-pathtracer). It is the checker the parity tests compare the CUDA
 * library against; nothing in the product links or calls it.
 *
 * Parity pin: tests/test_oracle_pin.py checks every function here against the reference's own code compiled from
 * its sources (oracle/_ref, recipe oracle/Makefile) and against the committed fixtures in tests/golden/ that the
 * reference produced (tests/golden/make_golden.py).
 *
 * Arithmetic: compiled with -ffp-contract=off; fused multiply-adds only where written as fmaf(), at the same places
 * as the CUDA kernels (so traversal results agree bit for bit with them). Where the reference's host build rounds
 * differently (it has no fused operations), only exact ties can resolve differently.
 *
 * Contents (reference file:line each follows):
 *   sample hash and warps ........ core/rng.h:6-12, core/sampling.h:13-52
 *   binned-SAH BVH2 build ........ accel/bvh_builder.cpp:5-68 (bin count as a parameter; the reference fixes 16)
 *   BVH2 layout .................. accel/bvh_layouts.cpp:6-30
 *   CWBVH SAH collapse ........... accel/bvh_tools.cpp:46-168
 *   triangle / Woop packing ...... accel/tri_pack.cpp:6-38
 *   traversal (BVH2, CWBVH) ...... accel/traverse.cuh:10-70, 112-152 (a CWBVH node's slab tests all run before its
 *                                  leaf tests, in slot order; descent order as the reference)
 *   camera ray + legacy shading .. render/wavefront.cu:42-58, 94-136, frame loop 684-741
 *   FP64 watertight reference .... not in the reference (precision-form oracle; Woop, Benthin & Wald, JCGT 2013)
 *   precision form ............... not in the reference (f16x2 conservative slabs + watertight FP32 triangles, the
 *                                  CUDA precision form restated with exact f16 emulation)
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { float x, y, z; } V3;
typedef struct { float x, y, z, w; } V4;

static V3 v3(float x, float y, float z) { V3 r = { x, y, z }; return r; }
static V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static V3 neg(V3 a) { return v3(-a.x, -a.y, -a.z); }
static V3 mulv(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static V3 muls(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
static float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static V3 cross3(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static V3 normz(V3 a) { float l = sqrtf(dot3(a, a)); return l > 0.f ? muls(a, 1.0f / l) : a; }
static V3 xyz4(V4 a) { return v3(a.x, a.y, a.z); }
static float fdot(V3 a, V3 b) { return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)); }
static float frow(V4 r, V3 a) { return fmaf(a.z, r.z, fmaf(a.y, r.y, fmaf(a.x, r.x, r.w))); }
static int fi(float f) { int i; memcpy(&i, &f, 4); return i; }
static unsigned fu(float f) { unsigned u; memcpy(&u, &f, 4); return u; }
static float iff(int i) { float f; memcpy(&f, &i, 4); return f; }
static float uf(unsigned u) { float f; memcpy(&f, &u, 4); return f; }

/* ------------------------------------------------------------------ sample hash + warps (core/rng.h, sampling.h) */
static unsigned hash32(unsigned x) { x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16; return x; }
float orc_rng(unsigned pix, unsigned smp, unsigned depth, unsigned dim, unsigned seed) {
    unsigned h = hash32(pix * 0x9E3779B1U ^ hash32(smp * 0x85EBCA77U ^ hash32((depth * 8u + dim) * 0xC2B2AE3DU ^ seed)));
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}
static void onb(V3 n, V3* t, V3* b) {
    float s = n.z >= 0.f ? 1.f : -1.f; float a = -1.f / (s + n.z); float c = n.x * n.y * a;
    *t = v3(1.f + s * n.x * n.x * a, s * c, -s * n.x); *b = v3(c, s + n.y * n.y * a, -n.y);
}
static V3 cos_hemi(V3 n, float u0, float u1) {
    float r = sqrtf(u0), ph = 6.2831853f * u1; V3 t, b; onb(n, &t, &b);
    return normz(add(add(muls(t, r * cosf(ph)), muls(b, r * sinf(ph))), muls(n, sqrtf(fmaxf(0.f, 1.f - u0)))));
}
static V3 cone_dir(V3 axis, float cosMax, float u0, float u1) {
    float cz = 1.f - u0 * (1.f - cosMax); float sz = sqrtf(fmaxf(0.f, 1.f - cz * cz)); float ph = 6.2831853f * u1;
    V3 t, b; onb(axis, &t, &b);
    return normz(add(add(muls(axis, cz), muls(t, sz * cosf(ph))), muls(b, sz * sinf(ph))));
}
static float table_lookup(const float* tab, int n, float u) {
    float f = u * n; int k = (int)f; k = k < n - 1 ? k : n - 1; float t = f - k; return tab[k] * (1.f - t) + tab[k + 1] * t;
}

/* ------------------------------------------------------------------ binned-SAH BVH2 (bvh_builder.cpp:5-68) */
typedef struct { V3 lo, hi; } Box;
static Box box_empty(void) { Box b; b.lo = v3(FLT_MAX, FLT_MAX, FLT_MAX); b.hi = v3(-FLT_MAX, -FLT_MAX, -FLT_MAX); return b; }
static void grow_p(Box* b, V3 p) { b->lo = v3(fminf(b->lo.x, p.x), fminf(b->lo.y, p.y), fminf(b->lo.z, p.z)); b->hi = v3(fmaxf(b->hi.x, p.x), fmaxf(b->hi.y, p.y), fmaxf(b->hi.z, p.z)); }
static void grow_b(Box* b, const Box* c) {
    b->lo = v3(fminf(b->lo.x, c->lo.x), fminf(b->lo.y, c->lo.y), fminf(b->lo.z, c->lo.z));
    b->hi = v3(fmaxf(b->hi.x, c->hi.x), fmaxf(b->hi.y, c->hi.y), fmaxf(b->hi.z, c->hi.z));
}
static float box_area(const Box* b) { if (b->hi.x < b->lo.x) return 0.f; V3 d = sub(b->hi, b->lo); return 2.f * (d.x * d.y + d.y * d.z + d.z * d.x); }
static float comp(V3 v, int a) { return a == 0 ? v.x : a == 1 ? v.y : v.z; }

typedef struct { Box box; int left, right, first, count; } Node;
typedef struct {
    const float* v; const int* f; int nb, leafMax;
    Box* tb; V3* cent; int* idx;
    Node* nodes; int nNodes, cap; int maxDepth;
} Build;

static int push_node(Build* B) {
    if (B->nNodes == B->cap) { B->cap = B->cap ? 2 * B->cap : 1024; B->nodes = (Node*)realloc(B->nodes, sizeof(Node) * B->cap); }
    Node* n = &B->nodes[B->nNodes]; n->box = box_empty(); n->left = n->right = -1; n->first = n->count = 0;
    return B->nNodes++;
}
static int bin_of(float c, float lo, float scale, int nb) { int b = (int)((c - lo) * scale); return b < 0 ? 0 : b > nb - 1 ? nb - 1 : b; }

/* in-place two-sided partition: scan from the left for an element failing the predicate and from the right for one
 * satisfying it, swap, repeat (the classic bidirectional partition, same permutation as the C++ library's) */
static int partition(Build* B, int begin, int end, int axis, float lo, float scale, int bestBin) {
    int first = begin, last = end;
    for (;;) {
        for (;;) { if (first == last) return first; if (bin_of(comp(B->cent[B->idx[first]], axis), lo, scale, B->nb) <= bestBin) first++; else break; }
        last--;
        for (;;) { if (first == last) return first; if (!(bin_of(comp(B->cent[B->idx[last]], axis), lo, scale, B->nb) <= bestBin)) last--; else break; }
        { int t = B->idx[first]; B->idx[first] = B->idx[last]; B->idx[last] = t; }
        first++;
    }
}

static int rec(Build* B, int begin, int end, int depth) {
    int id = push_node(B), n = end - begin, i, axis, b;
    if (depth > B->maxDepth) B->maxDepth = depth;
    Box box = box_empty(), cb = box_empty();
    for (i = begin; i < end; i++) { grow_b(&box, &B->tb[B->idx[i]]); grow_p(&cb, B->cent[B->idx[i]]); }
    B->nodes[id].box = box;
    if (n <= B->leafMax || depth >= 62) { B->nodes[id].first = begin; B->nodes[id].count = n; return id; }
    const int NB = B->nb;
    float bestCost = FLT_MAX; int bestAxis = -1, bestBin = -1;
    V3 ext = sub(cb.hi, cb.lo);
    Box* bb = (Box*)malloc(sizeof(Box) * NB); int* bc = (int*)malloc(sizeof(int) * NB);
    float* rA = (float*)malloc(sizeof(float) * NB); int* rC = (int*)malloc(sizeof(int) * NB);
    for (axis = 0; axis < 3; axis++) {
        float lo = comp(cb.lo, axis), e = comp(ext, axis);
        if (e <= 1e-12f) continue;
        float scale = NB / e;
        for (b = 0; b < NB; b++) { bb[b] = box_empty(); bc[b] = 0; }
        for (i = begin; i < end; i++) { int k = bin_of(comp(B->cent[B->idx[i]], axis), lo, scale, NB); grow_b(&bb[k], &B->tb[B->idx[i]]); bc[k]++; }
        Box acc = box_empty(); int cnt = 0;
        for (b = NB - 1; b > 0; b--) { grow_b(&acc, &bb[b]); cnt += bc[b]; rA[b] = box_area(&acc); rC[b] = cnt; }
        Box lacc = box_empty(); int lcnt = 0;
        for (b = 0; b < NB - 1; b++) {
            grow_b(&lacc, &bb[b]); lcnt += bc[b];
            if (lcnt == 0 || rC[b + 1] == 0) continue;
            float cost = box_area(&lacc) * lcnt + rA[b + 1] * rC[b + 1];
            if (cost < bestCost) { bestCost = cost; bestAxis = axis; bestBin = b; }
        }
    }
    free(bb); free(bc); free(rA); free(rC);
    int mid;
    if (bestAxis < 0) mid = (begin + end) / 2;
    else {
        float lo = comp(cb.lo, bestAxis), e = comp(ext, bestAxis), scale = NB / e;
        mid = partition(B, begin, end, bestAxis, lo, scale, bestBin);
        if (mid == begin || mid == end) mid = (begin + end) / 2;
    }
    int l = rec(B, begin, mid, depth + 1), r = rec(B, mid, end, depth + 1);
    B->nodes[id].left = l; B->nodes[id].right = r;
    return id;
}

static V3 vert(const float* v, int i) { return v3(v[3 * i], v[3 * i + 1], v[3 * i + 2]); }

static void sah_build(Build* B, const float* v, const int* f, int nt, int nb, int leafMax) {
    memset(B, 0, sizeof *B);
    B->v = v; B->f = f; B->nb = nb; B->leafMax = leafMax;
    B->tb = (Box*)malloc(sizeof(Box) * (nt > 0 ? nt : 1)); B->cent = (V3*)malloc(sizeof(V3) * (nt > 0 ? nt : 1)); B->idx = (int*)malloc(sizeof(int) * (nt > 0 ? nt : 1));
    for (int i = 0; i < nt; i++) {
        Box b = box_empty(); grow_p(&b, vert(v, f[3 * i])); grow_p(&b, vert(v, f[3 * i + 1])); grow_p(&b, vert(v, f[3 * i + 2]));
        B->tb[i] = b; B->cent[i] = muls(add(b.lo, b.hi), 0.5f); B->idx[i] = i;
    }
    rec(B, 0, nt, 0);
}
static void build_free(Build* B) { free(B->tb); free(B->cent); free(B->idx); free(B->nodes); }

/* ------------------------------------------------------------------ BVH2 layout (bvh_layouts.cpp:6-30) */
typedef struct { V4* a; int n, cap; } V4Vec;
static void v4_resize(V4Vec* s, int n) { if (n > s->cap) { while (s->cap < n) s->cap = s->cap ? 2 * s->cap : 1024; s->a = (V4*)realloc(s->a, sizeof(V4) * s->cap); } s->n = n; }
static V4 mk4(float x, float y, float z, float w) { V4 r = { x, y, z, w }; return r; }
static const float kEmpty = 3e37f;

static int emit2(const Build* B, int bn, V4Vec* out) {
    const Node* nd = &B->nodes[bn];
    int id = out->n / 4; v4_resize(out, out->n + 4);
    int ch[2] = { nd->left, nd->right }, c[2], k[2]; Box bx[2];
    for (int j = 0; j < 2; j++) {
        if (ch[j] < 0) { c[j] = -1; k[j] = 0; bx[j].lo = bx[j].hi = v3(kEmpty, kEmpty, kEmpty); continue; }
        const Node* cn = &B->nodes[ch[j]]; bx[j] = cn->box;
        if (cn->count > 0) { c[j] = cn->first; k[j] = cn->count; } else { k[j] = 0; c[j] = emit2(B, ch[j], out); }
    }
    V4* n = &out->a[id * 4];
    n[0] = mk4(bx[0].lo.x, bx[0].hi.x, bx[0].lo.y, bx[0].hi.y);
    n[1] = mk4(bx[1].lo.x, bx[1].hi.x, bx[1].lo.y, bx[1].hi.y);
    n[2] = mk4(bx[0].lo.z, bx[0].hi.z, bx[1].lo.z, bx[1].hi.z);
    n[3] = mk4(iff(c[0]), iff(c[1]), iff(k[0]), iff(k[1]));
    return id;
}
static void wrap_root(Build* B) { int r = push_node(B); B->nodes[r].box = B->nodes[0].box; B->nodes[r].left = 0; B->nodes[r].right = -1; }

/* ------------------------------------------------------------------ CWBVH collapse (bvh_tools.cpp:46-168) */
enum { LEAF = 0, NODEC = 1, PREV = 2, DIST = 10 };
typedef struct { Box* box; int *L, *R, *first, *cnt, *p; float* C; unsigned char *D, *K8; int n, cap; const int* prim; } CW;
static void cw_push(CW* w) {
    if (w->n == w->cap) {
        w->cap = w->cap ? 2 * w->cap : 1024;
        w->box = (Box*)realloc(w->box, sizeof(Box) * w->cap); w->L = (int*)realloc(w->L, 4 * w->cap); w->R = (int*)realloc(w->R, 4 * w->cap);
        w->first = (int*)realloc(w->first, 4 * w->cap); w->cnt = (int*)realloc(w->cnt, 4 * w->cap);
    }
    w->n++;
}
static int cw_isleaf(const CW* w, int n) { return w->L[n] < 0 || w->D[(size_t)n * 8 + 1] == LEAF; }
typedef struct { int* a; int n, cap; } IVec;
static void ipush(IVec* s, int x) { if (s->n == s->cap) { s->cap = s->cap ? 2 * s->cap : 64; s->a = (int*)realloc(s->a, 4 * s->cap); } s->a[s->n++] = x; }
static void cw_roots(const CW* w, int n, int i, IVec* out) {
    for (;;) {
        if (i == 1) { ipush(out, n); return; }
        unsigned char d = w->D[(size_t)n * 8 + i];
        if (d == PREV) { i--; continue; }
        int k = d - DIST; cw_roots(w, w->L[n], k, out); cw_roots(w, w->R[n], i - k, out); return;
    }
}
static void cw_prims(const CW* w, int n, IVec* out) {
    IVec st = { 0 }; ipush(&st, n);
    while (st.n) { int h = st.a[--st.n]; if (w->L[h] < 0) { for (int t = 0; t < w->cnt[h]; t++) ipush(out, w->prim[w->first[h] + t]); } else { ipush(&st, w->R[h]); ipush(&st, w->L[h]); } }
    free(st.a);
}
static int expo8(float ext, float lo, float hi) {
    if (!(ext > 0.f)) return -100;
    int e = (int)ceilf(log2f(ext / 255.f)); if (e < -100) e = -100;
    while (lo + 255.f * ldexpf(1.f, e) < hi) e++;
    return e;
}
static int qz(float v, float o, float sc, int up) { float f = (v - o) / sc; int i = up ? (int)ceilf(f) : (int)floorf(f); return i < 0 ? 0 : i > 255 ? 255 : i; }
static unsigned pack4(const int* q, int b) { return (unsigned)q[b] | ((unsigned)q[b + 1] << 8) | ((unsigned)q[b + 2] << 16) | ((unsigned)q[b + 3] << 24); }

static double cw_build(const Build* B, V4Vec* nodes, IVec* order) {
    const int pMax = 3; const float cNode = 1.f, cPrim = 0.3f, INF = 3e38f;
    CW w; memset(&w, 0, sizeof w); w.prim = B->idx;
    for (int i = 0; i < B->nNodes; i++) {
        cw_push(&w); const Node* b = &B->nodes[i]; int lf = b->count > 0;
        w.box[i] = b->box; w.L[i] = lf ? -1 : b->left; w.R[i] = lf ? -1 : b->right; w.first[i] = b->first; w.cnt[i] = lf ? b->count : 0;
    }
    for (int i = 0; i < w.n; i++) {
        if (w.L[i] >= 0 || w.cnt[i] <= pMax) continue;
        int h = w.cnt[i] / 2, a = w.n; Box bx = w.box[i];
        cw_push(&w); cw_push(&w);
        w.box[a] = bx; w.box[a + 1] = bx; w.L[a] = w.L[a + 1] = w.R[a] = w.R[a + 1] = -1;
        w.first[a] = w.first[i]; w.cnt[a] = h; w.first[a + 1] = w.first[i] + h; w.cnt[a + 1] = w.cnt[i] - h;
        w.L[i] = a; w.R[i] = a + 1; w.cnt[i] = 0;
    }
    const int N = w.n;
    w.C = (float*)calloc((size_t)N * 8, 4); w.D = (unsigned char*)calloc((size_t)N * 8, 1); w.K8 = (unsigned char*)malloc(N); w.p = (int*)calloc(N, 4);
    memset(w.K8, 1, N);
    for (int n = N - 1; n >= 0; n--) {
        float A = box_area(&w.box[n]); float* c = &w.C[(size_t)n * 8]; unsigned char* d = &w.D[(size_t)n * 8];
        if (w.L[n] < 0) { w.p[n] = w.cnt[n]; float cl = A * w.p[n] * cPrim; for (int i = 1; i < 8; i++) { c[i] = cl; d[i] = i == 1 ? LEAF : PREV; } continue; }
        int l = w.L[n], r = w.R[n]; w.p[n] = w.p[l] + w.p[r];
        const float* cl = &w.C[(size_t)l * 8]; const float* cr = &w.C[(size_t)r * 8];
        float dist[9]; int dk[9];
        for (int j = 2; j <= 8; j++) { dist[j] = INF; dk[j] = 1; for (int k = 1; k < j; k++) { float x = cl[k] + cr[j - k]; if (x < dist[j]) { dist[j] = x; dk[j] = k; } } }
        float cLeaf = w.p[n] <= pMax ? A * w.p[n] * cPrim : INF, cInt = dist[8] + A * cNode;
        if (cLeaf <= cInt) { c[1] = cLeaf; d[1] = LEAF; } else { c[1] = cInt; d[1] = NODEC; }
        w.K8[n] = (unsigned char)dk[8];
        for (int i = 2; i < 8; i++) { if (dist[i] < c[i - 1]) { c[i] = dist[i]; d[i] = (unsigned char)(DIST + dk[i]); } else { c[i] = c[i - 1]; d[i] = PREV; } }
    }
    const float Ar = box_area(&w.box[0]); const int rootLeaf = cw_isleaf(&w, 0); double sah;
    if (rootLeaf) sah = Ar > 0 ? (Ar * w.p[0] * cPrim + Ar * cNode) / Ar : 0;
    else { float d8 = INF; for (int k = 1; k < 8; k++) { float x = w.C[(size_t)w.L[0] * 8 + k] + w.C[(size_t)w.R[0] * 8 + 8 - k]; d8 = x < d8 ? x : d8; } sah = Ar > 0 ? (d8 + Ar * cNode) / Ar : 0; }
    /* emission: LIFO job stack, children of a node contiguous */
    typedef struct { int bn, out, asLeaf; } Job;
    Job* jobs = (Job*)malloc(sizeof(Job) * (N + 8)); int nj = 0;
    nodes->n = 0; v4_resize(nodes, 5); order->n = 0;
    jobs[nj].bn = 0; jobs[nj].out = 0; jobs[nj].asLeaf = rootLeaf; nj++;
    IVec ch = { 0 }, pr = { 0 };
    while (nj) {
        Job jb = jobs[--nj]; int n = jb.bn;
        ch.n = 0;
        if (jb.asLeaf) ipush(&ch, n); else { cw_roots(&w, w.L[n], w.K8[n], &ch); cw_roots(&w, w.R[n], 8 - w.K8[n], &ch); }
        Box box = w.box[n]; V3 pc = muls(add(box.lo, box.hi), 0.5f);
        int slot[8], used[8] = { 0 }; float cost[8][8];
        for (int s = 0; s < 8; s++) slot[s] = -1;
        for (int c = 0; c < ch.n; c++) {
            V3 cc = sub(muls(add(w.box[ch.a[c]].lo, w.box[ch.a[c]].hi), 0.5f), pc);
            for (int s = 0; s < 8; s++) cost[c][s] = -(cc.x * (s & 1 ? -1.f : 1.f) + cc.y * (s & 2 ? -1.f : 1.f) + cc.z * (s & 4 ? -1.f : 1.f));
        }
        for (int it = 0; it < ch.n; it++) {
            float bc = INF; int bi = -1, bs = -1;
            for (int c = 0; c < ch.n; c++) if (!used[c]) for (int s = 0; s < 8; s++) if (slot[s] < 0 && cost[c][s] < bc) { bc = cost[c][s]; bi = c; bs = s; }
            if (bi < 0) for (int c = 0; c < ch.n && bi < 0; c++) if (!used[c]) for (int s = 0; s < 8; s++) if (slot[s] < 0) { bi = c; bs = s; break; }
            used[bi] = 1; slot[bs] = ch.a[bi];
        }
        V3 ext = sub(box.hi, box.lo);
        int ex = expo8(ext.x, box.lo.x, box.hi.x), ey = expo8(ext.y, box.lo.y, box.hi.y), ez = expo8(ext.z, box.lo.z, box.hi.z);
        float sx = ldexpf(1.f, ex), sy = ldexpf(1.f, ey), sz = ldexpf(1.f, ez);
        int q[6][8], meta[8], isLeafC[8]; int triBase = order->n, nInt = 0; unsigned imask = 0;
        for (int s = 0; s < 8; s++) {
            for (int a = 0; a < 6; a++) q[a][s] = 0;
            meta[s] = 0; isLeafC[s] = 0;
            int cn = slot[s]; if (cn < 0) continue;
            Box cb = w.box[cn];
            q[0][s] = qz(cb.lo.x, box.lo.x, sx, 0); q[3][s] = qz(cb.hi.x, box.lo.x, sx, 1);
            q[1][s] = qz(cb.lo.y, box.lo.y, sy, 0); q[4][s] = qz(cb.hi.y, box.lo.y, sy, 1);
            q[2][s] = qz(cb.lo.z, box.lo.z, sz, 0); q[5][s] = qz(cb.hi.z, box.lo.z, sz, 1);
            if (jb.asLeaf || cw_isleaf(&w, cn)) {
                pr.n = 0; cw_prims(&w, cn, &pr);
                int off = order->n - triBase;
                for (int t = 0; t < pr.n; t++) ipush(order, pr.a[t]);
                meta[s] = 0x80 | ((pr.n - 1) << 5) | off; isLeafC[s] = 1;
            } else { meta[s] = 0x40; imask |= 1u << s; nInt++; }
        }
        int childBase = nodes->n / 5;
        v4_resize(nodes, nodes->n + 5 * nInt);
        V4* o = &nodes->a[jb.out * 5];
        unsigned ew = (unsigned)(ex + 127) | ((unsigned)(ey + 127) << 8) | ((unsigned)(ez + 127) << 16) | (imask << 24);
        o[0] = mk4(box.lo.x, box.lo.y, box.lo.z, uf(ew));
        o[1] = mk4(iff(childBase), iff(triBase), uf(pack4(meta, 0)), uf(pack4(meta, 4)));
        unsigned u[12]; for (int a = 0; a < 6; a++) { u[2 * a] = pack4(q[a], 0); u[2 * a + 1] = pack4(q[a], 4); }
        for (int j = 0; j < 3; j++) o[2 + j] = mk4(uf(u[4 * j]), uf(u[4 * j + 1]), uf(u[4 * j + 2]), uf(u[4 * j + 3]));
        int ord = 0;
        for (int s = 0; s < 8; s++) if (slot[s] >= 0 && !isLeafC[s]) { jobs[nj].bn = slot[s]; jobs[nj].out = childBase + ord; jobs[nj].asLeaf = 0; nj++; ord++; }
    }
    free(jobs); free(ch.a); free(pr.a);
    free(w.box); free(w.L); free(w.R); free(w.first); free(w.cnt); free(w.p); free(w.C); free(w.D); free(w.K8);
    return sah;
}

/* ------------------------------------------------------------------ public build entry point
 * variant 2: BVH2 from leaves <= leafMax; variant 8: CWBVH by the SAH collapse from single-triangle leaves.
 * nodes_out capacity: variant 2 -> 4 (nt + 1) float4, variant 8 -> 5 (2 nt) float4. order_out: nt ints.
 * Returns the node count in float4 units (or -1), fills *max_depth. */
long orc_build(const float* v, const int* f, int nt, int bins, int leafMax, int variant, float* nodes_out, long cap_f4, int* order_out, int* max_depth, double* sah) {
    Build B; V4Vec nodes = { 0 }; IVec order = { 0 }; long n = -1;
    if (nt <= 0 || bins < 2) return -1;
    sah_build(&B, v, f, nt, bins, variant == 8 ? 1 : leafMax);
    *max_depth = B.maxDepth;
    if (variant == 2) {
        if (B.nodes[0].count > 0) { wrap_root(&B); emit2(&B, B.nNodes - 1, &nodes); } else emit2(&B, 0, &nodes);
        for (int i = 0; i < nt; i++) order_out[i] = B.idx[i];
        *sah = 0;
    } else {
        *sah = cw_build(&B, &nodes, &order);
        for (int i = 0; i < order.n && i < nt; i++) order_out[i] = order.a[i];
    }
    if (nodes.n <= cap_f4) { memcpy(nodes_out, nodes.a, sizeof(V4) * nodes.n); n = nodes.n; }
    free(nodes.a); free(order.a); build_free(&B);
    return n;
}

/* triangles in leaf order (tri_pack.cpp:6-16) and Woop rows (tri_pack.cpp:18-38) */
void orc_pack(const float* v, const int* f, const int* fm, const int* order, int n, float* tris, float* woop) {
    for (int k = 0; k < n; k++) {
        int t = order[k]; V3 v0 = vert(v, f[3 * t]), e1 = sub(vert(v, f[3 * t + 1]), v0), e2 = sub(vert(v, f[3 * t + 2]), v0), nn = cross3(e1, e2);
        int mat = fm ? fm[t] : 0;
        float* o = tris + 12 * (size_t)k;
        o[0] = v0.x; o[1] = v0.y; o[2] = v0.z; o[3] = iff(t); o[4] = e1.x; o[5] = e1.y; o[6] = e1.z; o[7] = iff(mat); o[8] = e2.x; o[9] = e2.y; o[10] = e2.z; o[11] = 0.f;
        double a[3][3] = { { e1.x, e2.x, nn.x }, { e1.y, e2.y, nn.y }, { e1.z, e2.z, nn.z } };
        double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) + a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
        double m[3][3] = { { 0 } };
        if (!(fabs(det) < 1e-300)) {
            double id = 1.0 / det;
            m[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) * id; m[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) * id; m[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) * id;
            m[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) * id; m[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * id; m[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) * id;
            m[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) * id; m[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) * id; m[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * id;
        }
        float* w = woop + 12 * (size_t)k;
        for (int r = 0; r < 3; r++) {
            double tt = -(m[r][0] * v0.x + m[r][1] * v0.y + m[r][2] * v0.z);
            w[4 * r] = (float)m[r][0]; w[4 * r + 1] = (float)m[r][1]; w[4 * r + 2] = (float)m[r][2]; w[4 * r + 3] = (float)tt;
        }
    }
}

/* ------------------------------------------------------------------ traversal (traverse.cuh) */
static int leaf_hit(const V4* tv, int first, int cnt, V3 o, V3 d, float tmin, int any, int tri, float* hitT, int* hitTri, float* hu, float* hv) {
    for (int t = first; t < first + cnt; t++) {
        if (tri == 0) {
            V3 v0 = xyz4(tv[3 * t]), e1 = xyz4(tv[3 * t + 1]), e2 = xyz4(tv[3 * t + 2]);
            V3 pv = v3(fmaf(d.y, e2.z, -d.z * e2.y), fmaf(d.z, e2.x, -d.x * e2.z), fmaf(d.x, e2.y, -d.y * e2.x));
            float det = fdot(e1, pv);
            if (fabsf(det) < 1e-12f) continue;
            float inv = 1.f / det; V3 tq = sub(o, v0); float u = fdot(tq, pv) * inv;
            if (u < 0.f || u > 1.f) continue;
            V3 qv = v3(fmaf(tq.y, e1.z, -tq.z * e1.y), fmaf(tq.z, e1.x, -tq.x * e1.z), fmaf(tq.x, e1.y, -tq.y * e1.x));
            float vv = fdot(d, qv) * inv;
            if (vv < 0.f || u + vv > 1.f) continue;
            float tt = fdot(e2, qv) * inv;
            if (tt > tmin && tt < *hitT) { *hitT = tt; *hitTri = t; *hu = u; *hv = vv; if (any) return 1; }
        } else {
            V4 r2 = tv[3 * t + 2];
            float Oz = frow(r2, o), Dz = fdot(d, xyz4(r2)), tt = -Oz / Dz;
            if (tt > tmin && tt < *hitT) {
                V4 r0 = tv[3 * t];
                float u = fmaf(tt, fdot(d, xyz4(r0)), frow(r0, o));
                if (u >= 0.f && u <= 1.f) {
                    V4 r1 = tv[3 * t + 1];
                    float vv = fmaf(tt, fdot(d, xyz4(r1)), frow(r1, o));
                    if (vv >= 0.f && u + vv <= 1.f) { *hitT = tt; *hitTri = t; *hu = u; *hv = vv; if (any) return 1; }
                }
            }
        }
    }
    return 0;
}
static float safe_rcp(float x) { return 1.f / (fabsf(x) > 1e-20f ? x : copysignf(1e-20f, x)); }

/* visit counters (for the algorithmic-bytes figures) */
typedef struct { long long nodes, tris; } Stats;
static int leaf_hit_s(const V4* tv, int first, int cnt, V3 o, V3 d, float tmin, int any, int tri, float* T, int* I, float* U, float* W, Stats* st) {
    if (st) { /* count tests the same way the loop runs them */
        int before = *I; float bt = *T; (void)before; (void)bt;
        int r = 0;
        for (int t = first; t < first + cnt; t++) { st->tris++; if (leaf_hit(tv, t, 1, o, d, tmin, any, tri, T, I, U, W)) { r = 1; if (any) break; } }
        return r;
    }
    return leaf_hit(tv, first, cnt, o, d, tmin, any, tri, T, I, U, W);
}

static int trav2r(const V4* nodes, const V4* tv, V3 o, V3 d, float tmin, int any, int tri, float* hitT, int* hitTri, float* hu, float* hv, Stats* st, int root) {
    int stack[64], sp = 0, node = root;
    const float idx = safe_rcp(d.x), idy = safe_rcp(d.y), idz = safe_rcp(d.z), ox = -o.x * idx, oy = -o.y * idy, oz = -o.z * idz;
    for (;;) {
        if (st) st->nodes++;
        const V4 n0 = nodes[4 * node], n1 = nodes[4 * node + 1], nz = nodes[4 * node + 2], mt = nodes[4 * node + 3];
        int c0 = fi(mt.x), c1 = fi(mt.y), k0 = fi(mt.z), k1 = fi(mt.w);
        float a0 = fmaf(n0.x, idx, ox), a1 = fmaf(n0.y, idx, ox), a2 = fmaf(n0.z, idy, oy), a3 = fmaf(n0.w, idy, oy), a4 = fmaf(nz.x, idz, oz), a5 = fmaf(nz.y, idz, oz);
        float b0 = fmaf(n1.x, idx, ox), b1 = fmaf(n1.y, idx, ox), b2 = fmaf(n1.z, idy, oy), b3 = fmaf(n1.w, idy, oy), b4 = fmaf(nz.z, idz, oz), b5 = fmaf(nz.w, idz, oz);
        float t0n = fmaxf(fmaxf(fminf(a0, a1), fminf(a2, a3)), fmaxf(fminf(a4, a5), tmin));
        float t0f = fminf(fminf(fmaxf(a0, a1), fmaxf(a2, a3)), fminf(fmaxf(a4, a5), *hitT));
        float t1n = fmaxf(fmaxf(fminf(b0, b1), fminf(b2, b3)), fmaxf(fminf(b4, b5), tmin));
        float t1f = fminf(fminf(fmaxf(b0, b1), fmaxf(b2, b3)), fminf(fmaxf(b4, b5), *hitT));
        int h0 = t0n <= t0f, h1 = t1n <= t1f;
        if (h0 && k0 > 0) { if (leaf_hit_s(tv, c0, k0, o, d, tmin, any, tri, hitT, hitTri, hu, hv, st) && any) return 1; h0 = 0; }
        if (h1 && k1 > 0) { if (leaf_hit_s(tv, c1, k1, o, d, tmin, any, tri, hitT, hitTri, hu, hv, st) && any) return 1; h1 = 0; }
        if (!h0 && !h1) { if (sp == 0) break; node = stack[--sp]; }
        else if (h0 && h1) { if (t1n < t0n) { int t = c0; c0 = c1; c1 = t; } if (sp == 64) return -1; stack[sp++] = c1; node = c0; }
        else node = h0 ? c0 : c1;
    }
    return *hitTri >= 0;
}

static unsigned byte_of(unsigned w, int s) { return (w >> (8 * (s & 3))) & 255u; }
static int trav8r(const V4* nodes, const V4* tv, V3 o, V3 d, float tmin, int any, int tri, float* hitT, int* hitTri, float* hu, float* hv, Stats* st, int root) {
    unsigned stk[40][2]; int sp = 0, node = root;
    const float idx = safe_rcp(d.x), idy = safe_rcp(d.y), idz = safe_rcp(d.z);
    const unsigned oct = (d.x > 0.f ? 1u : 0u) | (d.y > 0.f ? 2u : 0u) | (d.z > 0.f ? 4u : 0u);
    unsigned cb = 0, im = 0, hm = 0;
    for (;;) {
        if (st) st->nodes++;
        const V4* nb = nodes + 5 * node;
        V4 f0 = nb[0], f1 = nb[1], f2 = nb[2], f3 = nb[3], f4 = nb[4];
        unsigned ew = fu(f0.w);
        float sx = uf((ew & 255u) << 23) * idx, sy = uf(((ew >> 8) & 255u) << 23) * idy, sz = uf(((ew >> 16) & 255u) << 23) * idz;
        float ox = (f0.x - o.x) * idx, oy = (f0.y - o.y) * idy, oz = (f0.z - o.z) * idz;
        unsigned imask = ew >> 24, m0 = fu(f1.z), m1 = fu(f1.w); int childBase = fi(f1.x), triBase = fi(f1.y);
        unsigned q[12] = { fu(f2.x), fu(f2.y), fu(f2.z), fu(f2.w), fu(f3.x), fu(f3.y), fu(f3.z), fu(f3.w), fu(f4.x), fu(f4.y), fu(f4.z), fu(f4.w) };
        /* the eight slab tests first, then the hit leaves in slot order, then descent (the library's node visit) */
        unsigned hits = 0, leafHit = 0;
        for (int s = 0; s < 8; s++) {
            unsigned m = byte_of(s < 4 ? m0 : m1, s); int hi = s < 4 ? 0 : 1;
            if (m == 0) continue;
            float x0 = fmaf((float)byte_of(q[0 + hi], s), sx, ox), x1 = fmaf((float)byte_of(q[6 + hi], s), sx, ox);
            float y0 = fmaf((float)byte_of(q[2 + hi], s), sy, oy), y1 = fmaf((float)byte_of(q[8 + hi], s), sy, oy);
            float z0 = fmaf((float)byte_of(q[4 + hi], s), sz, oz), z1 = fmaf((float)byte_of(q[10 + hi], s), sz, oz);
            float tn = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
            float tf = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), *hitT));
            if (tn <= tf) { if (m & 0x80u) leafHit |= 1u << s; else hits |= 1u << (s ^ oct); }
        }
        for (int s = 0; s < 8; s++) if (leafHit & (1u << s)) {
            unsigned m = byte_of(s < 4 ? m0 : m1, s);
            if (leaf_hit_s(tv, triBase + (int)(m & 31u), (int)((m >> 5) & 3u) + 1, o, d, tmin, any, tri, hitT, hitTri, hu, hv, st) && any) return 1;
        }
        if (hits) { if (hm) { if (sp == 40) return -1; stk[sp][0] = cb; stk[sp][1] = (im << 8) | hm; sp++; } cb = (unsigned)childBase; im = imask; hm = hits; }
        while (hm == 0) { if (sp == 0) return *hitTri >= 0; sp--; cb = stk[sp][0]; im = stk[sp][1] >> 8; hm = stk[sp][1] & 255u; }
        unsigned k = (unsigned)__builtin_ctz(hm); hm &= hm - 1; unsigned slot = k ^ oct;
        node = (int)cb + __builtin_popcount(im & ((1u << slot) - 1u));
    }
}

static int trav2(const V4* nodes, const V4* tv, V3 o, V3 d, float tmin, int any, int tri, float* hitT, int* hitTri, float* hu, float* hv, Stats* st) {
    return trav2r(nodes, tv, o, d, tmin, any, tri, hitT, hitTri, hu, hv, st, 0);
}
static int trav8(const V4* nodes, const V4* tv, V3 o, V3 d, float tmin, int any, int tri, float* hitT, int* hitTri, float* hu, float* hv, Stats* st) {
    return trav8r(nodes, tv, o, d, tmin, any, tri, hitT, hitTri, hu, hv, st, 0);
}
/* BVH4 (traverse.cuh:74-107): four slab tests, hit leaves tested in child order, inner children sorted by entry
 * distance with the five-exchange network, nearest visited next, the others pushed farthest first */
static int trav4r(const V4* nodes, const V4* tv, V3 o, V3 d, float tmin, int any, int tri, float* hitT, int* hitTri, float* hu, float* hv, Stats* st, int root) {
    int stack[64], sp = 0, node = root;
    const float idx = safe_rcp(d.x), idy = safe_rcp(d.y), idz = safe_rcp(d.z), ox = -o.x * idx, oy = -o.y * idy, oz = -o.z * idz;
    const float INF = 3.4e38f;
    for (;;) {
        if (st) st->nodes++;
        const V4* nb = nodes + 8 * node;
        const float LX[4] = { nb[0].x, nb[0].y, nb[0].z, nb[0].w }, HX[4] = { nb[1].x, nb[1].y, nb[1].z, nb[1].w };
        const float LY[4] = { nb[2].x, nb[2].y, nb[2].z, nb[2].w }, HY[4] = { nb[3].x, nb[3].y, nb[3].z, nb[3].w };
        const float LZ[4] = { nb[4].x, nb[4].y, nb[4].z, nb[4].w }, HZ[4] = { nb[5].x, nb[5].y, nb[5].z, nb[5].w };
        const int CC[4] = { fi(nb[6].x), fi(nb[6].y), fi(nb[6].z), fi(nb[6].w) }, KK[4] = { fi(nb[7].x), fi(nb[7].y), fi(nb[7].z), fi(nb[7].w) };
        float ht[4]; int hc[4];
        for (int j = 0; j < 4; j++) {
            float x0 = fmaf(LX[j], idx, ox), x1 = fmaf(HX[j], idx, ox), y0 = fmaf(LY[j], idy, oy), y1 = fmaf(HY[j], idy, oy), z0 = fmaf(LZ[j], idz, oz), z1 = fmaf(HZ[j], idz, oz);
            float tn = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
            float tf = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), *hitT));
            ht[j] = INF; hc[j] = CC[j];
            if (tn <= tf) {
                if (KK[j] > 0) { if (leaf_hit_s(tv, CC[j], KK[j], o, d, tmin, any, tri, hitT, hitTri, hu, hv, st) && any) return 1; }
                else ht[j] = tn;
            }
        }
        static const int net[5][2] = { { 0, 1 }, { 2, 3 }, { 0, 2 }, { 1, 3 }, { 1, 2 } };
        for (int q = 0; q < 5; q++) {
            const int a = net[q][0], b = net[q][1];
            if (ht[b] < ht[a]) { float t = ht[a]; ht[a] = ht[b]; ht[b] = t; int c = hc[a]; hc[a] = hc[b]; hc[b] = c; }
        }
        if (ht[0] == INF) { if (sp == 0) break; node = stack[--sp]; continue; }
        if (sp + 3 > 64) return -1;
        if (ht[3] < INF) stack[sp++] = hc[3];
        if (ht[2] < INF) stack[sp++] = hc[2];
        if (ht[1] < INF) stack[sp++] = hc[1];
        node = hc[0];
    }
    return *hitTri >= 0;
}

/* ray batch: o/d float4 (tmin / tmax in w). Closest: hits float4 (t, u, v, tri bits). Any: occ = first occluder or -1.
 * stats (may be NULL): [0] node visits, [1] triangle tests summed over the batch. Returns the number of rays that hit
 * a stack bound. */
long orc_trace(int variant, int tri, int any, const float* nodes, const float* tv, const float* ro, const float* rd, long n, float* hits, int* occ, long long* stats) {
    long bad = 0; Stats st = { 0, 0 };
    for (long i = 0; i < n; i++) {
        V3 o = v3(ro[4 * i], ro[4 * i + 1], ro[4 * i + 2]), d = v3(rd[4 * i], rd[4 * i + 1], rd[4 * i + 2]);
        float tmin = ro[4 * i + 3], t = rd[4 * i + 3], u = 0.f, vv = 0.f; int h = -1, r;
        if (variant == 2) r = trav2((const V4*)nodes, (const V4*)tv, o, d, tmin, any, tri, &t, &h, &u, &vv, stats ? &st : NULL);
        else if (variant == 4) r = trav4r((const V4*)nodes, (const V4*)tv, o, d, tmin, any, tri, &t, &h, &u, &vv, stats ? &st : NULL, 0);
        else r = trav8((const V4*)nodes, (const V4*)tv, o, d, tmin, any, tri, &t, &h, &u, &vv, stats ? &st : NULL);
        if (r < 0) bad++;
        if (any) occ[i] = h;
        else { hits[4 * i] = t; hits[4 * i + 1] = u; hits[4 * i + 2] = vv; hits[4 * i + 3] = iff(h); }
    }
    if (stats) { stats[0] = st.nodes; stats[1] = st.tris; }
    return bad;
}

/* ------------------------------------------------------------------ legacy diffuse frame (wavefront.cu:42-136) */
typedef struct {
    float pos[3], ax[3], ay[3], az[3]; float fx, fy, px, py; int w, h; float lens_r, focus_d;
    float sun_to[3], sun_e[3], sky[3]; float sun_cos; int max_b; unsigned seed; float eps, near_clip; int has_n, filter_bh; float ftab[65];
} OrcParams;   /* same layout as cwp_params of the library's C ABI */

static V3 a3(const float* a) { return v3(a[0], a[1], a[2]); }

/* Traversal work of orc_render, for the on-chip roofline: [0] node visits and [1] triangle tests of closest-hit rays,
 * [2] and [3] of shadow rays. orc_render_stats(1, NULL) zeroes and enables the counters; (0, out) reads and disables. */
static long long g_render_stats[4]; static int g_render_stats_on;
void orc_render_stats(int on, long long* out) { if (out) memcpy(out, g_render_stats, sizeof g_render_stats); memset(g_render_stats, 0, sizeof g_render_stats); g_render_stats_on = on; }

/* Renders samples [s_base, s_base + spp) of pixels [pix0, pix1) with `bounces` as the frame's depth limit
 * (depths 0 .. bounces + 1 are traced) and adds radiance sums to accum (float4 per pixel). Each path is traced
 * to completion before the next; the per-vertex decisions and sample dimensions are those of the wavefront loop.
 * ray_counts (may be NULL): [0] closest rays, [1] shadow rays. */
void orc_render(const OrcParams* P, int variant, int tri, const float* nodes, const float* tv, const float* tris, const float* albedo,
                int bounces, int spp, int s_base, int pix0, int pix1, float* accum, long long* ray_counts) {
    const int N = P->w * P->h, depths = bounces + 2;
    long long nc = 0, ns = 0;
    for (int pix = pix0; pix < pix1; pix++) {
        const int x = pix % P->w, y = pix / P->w;
        for (int smp = s_base; smp < s_base + spp; smp++) {
            float u0 = orc_rng(pix, smp, 0, 0, P->seed), u1 = orc_rng(pix, smp, 0, 1, P->seed), jx, jy;
            if (P->filter_bh) { jx = table_lookup(P->ftab, 64, u0); jy = table_lookup(P->ftab, 64, u1); } else { jx = u0 - 0.5f; jy = u1 - 0.5f; }
            float dx = (x + 0.5f + jx - P->px) / P->fx, dy = -(y + 0.5f + jy - P->py) / P->fy;
            V3 d = normz(sub(add(muls(a3(P->ax), dx), muls(a3(P->ay), dy)), a3(P->az))), o = a3(P->pos), T = v3(1.f, 1.f, 1.f);
            float tmin = P->near_clip;
            for (int depth = 0; depth < depths; depth++) {
                nc++;
                float t = 1e30f, u = 0.f, vv = 0.f; int h = -1; Stats cs = {0, 0};
                if (variant == 2) trav2((const V4*)nodes, (const V4*)tv, o, d, tmin, 0, tri, &t, &h, &u, &vv, g_render_stats_on ? &cs : NULL);
                else trav8((const V4*)nodes, (const V4*)tv, o, d, tmin, 0, tri, &t, &h, &u, &vv, g_render_stats_on ? &cs : NULL);
                g_render_stats[0] += cs.nodes; g_render_stats[1] += cs.tris;
                if (h < 0) { V3 c = mulv(T, a3(P->sky)); accum[4 * pix] += c.x; accum[4 * pix + 1] += c.y; accum[4 * pix + 2] += c.z; break; }
                if (depth > P->max_b) break;
                V3 p = add(o, muls(d, t));
                const float* tb = tris + 12 * (size_t)h;
                V3 e1 = v3(tb[4], tb[5], tb[6]), e2 = v3(tb[8], tb[9], tb[10]);
                V3 ng = normz(cross3(e1, e2)), nsh = ng;
                if (dot3(ng, d) > 0.f) { ng = neg(ng); nsh = neg(nsh); }
                int mat = fi(tb[7]); V3 alb = a3(albedo + 3 * mat);
                V3 po = add(p, muls(ng, P->eps));
                const unsigned dr = (unsigned)depth + 1u;
                V3 l = cone_dir(a3(P->sun_to), P->sun_cos, orc_rng(pix, smp, dr, 2, P->seed), orc_rng(pix, smp, dr, 3, P->seed));
                float cl = dot3(nsh, l);
                if (cl > 0.f && dot3(ng, l) > 0.f) {
                    V3 contrib = muls(mulv(mulv(T, alb), a3(P->sun_e)), cl * 0.31830989f);
                    ns++;
                    float st = 1e30f, su, sv; int sh = -1, occ; Stats ss = {0, 0};
                    if (variant == 2) occ = trav2((const V4*)nodes, (const V4*)tv, po, l, 0.f, 1, tri, &st, &sh, &su, &sv, g_render_stats_on ? &ss : NULL);
                    else occ = trav8((const V4*)nodes, (const V4*)tv, po, l, 0.f, 1, tri, &st, &sh, &su, &sv, g_render_stats_on ? &ss : NULL);
                    g_render_stats[2] += ss.nodes; g_render_stats[3] += ss.tris;
                    if (occ == 0) { accum[4 * pix] += contrib.x; accum[4 * pix + 1] += contrib.y; accum[4 * pix + 2] += contrib.z; }
                }
                V3 nd = cos_hemi(nsh, orc_rng(pix, smp, dr, 0, P->seed), orc_rng(pix, smp, dr, 1, P->seed));
                if (dot3(nd, ng) <= 0.f) break;
                T = mulv(T, alb); o = po; d = nd; tmin = 0.f;
            }
        }
    }
    (void)N;
    if (ray_counts) { ray_counts[0] += nc; ray_counts[1] += ns; }
}

/* ------------------------------------------------------------------ FP64 watertight reference (precision form)
 * Not in the reference. Restates the watertight ray/triangle test (Woop, Benthin & Wald, JCGT 2013) in double over the
 * exact corners (verts: 3 float4 per leaf-order triangle), driven either by the CWBVH (nodes != NULL: child boxes
 * decoded exactly in double, slab test widened by 1e-12 relative) or by brute force over all n_tris triangles
 * (nodes == NULL). t_out = closest t in (tmin, tmax) (tmax on a miss), tri_out = leaf-order triangle or -1. */
static double dcomp3(const double* v, int k) { return v[k]; }
static int wt64(const float* vt, int t, const double* o, int kx, int ky, int kz, double sx, double sy, double sz, double tmin, double* hitT) {
    const float* a = vt + 12 * (size_t)t; const float* b = a + 4; const float* c = a + 8;
    double A[3] = { a[0] - o[0], a[1] - o[1], a[2] - o[2] }, B[3] = { b[0] - o[0], b[1] - o[1], b[2] - o[2] }, C[3] = { c[0] - o[0], c[1] - o[1], c[2] - o[2] };
    double Az = dcomp3(A, kz), Bz = dcomp3(B, kz), Cz = dcomp3(C, kz);
    double Ax = A[kx] - sx * Az, Ay = A[ky] - sy * Az, Bx = B[kx] - sx * Bz, By = B[ky] - sy * Bz, Cx = C[kx] - sx * Cz, Cy = C[ky] - sy * Cz;
    double U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
    if ((U < 0.0 || V < 0.0 || W < 0.0) && (U > 0.0 || V > 0.0 || W > 0.0)) return 0;
    double det = U + V + W;
    if (det == 0.0) return 0;
    double tt = (U * (sz * Az) + V * (sz * Bz) + W * (sz * Cz)) / det;
    if (tt > tmin && tt < *hitT) { *hitT = tt; return 1; }
    return 0;
}
long orc_trace_fp64(const float* nodes, const float* vt, int n_tris, const float* ro, const float* rd, long n, int any, double* t_out, int* tri_out) {
    for (long i = 0; i < n; i++) {
        const double o[3] = { ro[4 * i], ro[4 * i + 1], ro[4 * i + 2] }, d[3] = { rd[4 * i], rd[4 * i + 1], rd[4 * i + 2] };
        const double tmin = ro[4 * i + 3]; double hitT = rd[4 * i + 3]; int hit = -1;
        const double ad[3] = { fabs(d[0]), fabs(d[1]), fabs(d[2]) };
        int kz = ad[0] >= ad[1] ? (ad[0] >= ad[2] ? 0 : 2) : (ad[1] >= ad[2] ? 1 : 2), kx = kz == 2 ? 0 : kz + 1, ky = kx == 2 ? 0 : kx + 1;
        if (d[kz] < 0.0) { int t = kx; kx = ky; ky = t; }
        const double sx = d[kx] / d[kz], sy = d[ky] / d[kz], sz = 1.0 / d[kz];
        if (!nodes) {
            for (int t = 0; t < n_tris; t++) if (wt64(vt, t, o, kx, ky, kz, sx, sy, sz, tmin, &hitT)) { hit = t; if (any) break; }
        } else {
            const double inv[3] = { 1.0 / (fabs(d[0]) > 1e-300 ? d[0] : copysign(1e-300, d[0])), 1.0 / (fabs(d[1]) > 1e-300 ? d[1] : copysign(1e-300, d[1])),
                                    1.0 / (fabs(d[2]) > 1e-300 ? d[2] : copysign(1e-300, d[2])) };
            const unsigned oct = (d[0] > 0.0 ? 1u : 0u) | (d[1] > 0.0 ? 2u : 0u) | (d[2] > 0.0 ? 4u : 0u);
            unsigned stk[40][2]; int sp = 0, node = 0, done = 0; unsigned cb = 0, im = 0, hm = 0;
            while (!done) {
                const V4* nb = (const V4*)nodes + 5 * node;
                unsigned ew = fu(nb[0].w), imask = ew >> 24, m0 = fu(nb[1].z), m1 = fu(nb[1].w);
                int childBase = fi(nb[1].x), triBase = fi(nb[1].y);
                double e[3] = { uf((ew & 255u) << 23), uf(((ew >> 8) & 255u) << 23), uf(((ew >> 16) & 255u) << 23) };
                double org[3] = { nb[0].x, nb[0].y, nb[0].z };
                const unsigned* q = (const unsigned*)(nb + 2);
                unsigned boxHit = 0;
                for (int s = 0; s < 8; s++) {
                    int w = s < 4 ? 0 : 1; double lo[3], hi[3], tn = tmin, tf = hitT;
                    for (int ax = 0; ax < 3; ax++) {
                        lo[ax] = org[ax] + byte_of(q[2 * ax + w], s) * e[ax]; hi[ax] = org[ax] + byte_of(q[6 + 2 * ax + w], s) * e[ax];
                    }
                    double x0 = (lo[0] - o[0]) * inv[0], x1 = (hi[0] - o[0]) * inv[0], y0 = (lo[1] - o[1]) * inv[1], y1 = (hi[1] - o[1]) * inv[1], z0 = (lo[2] - o[2]) * inv[2], z1 = (hi[2] - o[2]) * inv[2];
                    tn = fmax(fmax(fmin(x0, x1), fmin(y0, y1)), fmax(fmin(z0, z1), tmin));
                    tf = fmin(fmin(fmax(x0, x1), fmax(y0, y1)), fmin(fmax(z0, z1), hitT));
                    if (tn - 1e-12 * fabs(tn) <= tf + 1e-12 * fabs(tf)) boxHit |= 1u << s;
                }
                for (int s = 0; s < 8 && !done; s++) {
                    if (!(boxHit & (1u << s))) continue;
                    unsigned m = byte_of(s < 4 ? m0 : m1, s);
                    if (!(m & 0x80u)) continue;
                    for (int t = triBase + (int)(m & 31u), e2 = t + (int)((m >> 5) & 3u) + 1; t < e2; t++)
                        if (wt64(vt, t, o, kx, ky, kz, sx, sy, sz, tmin, &hitT)) { hit = t; if (any) { done = 1; break; } }
                }
                if (done) break;
                unsigned hits = boxHit & imask, ho = 0;
                for (int s = 0; s < 8; s++) if (hits & (1u << s)) ho |= 1u << (s ^ oct);
                if (ho) { if (hm) { if (sp == 40) return -1; stk[sp][0] = cb; stk[sp][1] = (im << 8) | hm; sp++; } cb = (unsigned)childBase; im = imask; hm = ho; }
                while (hm == 0) { if (sp == 0) { done = 1; break; } sp--; cb = stk[sp][0]; im = stk[sp][1] >> 8; hm = stk[sp][1] & 255u; }
                if (done) break;
                unsigned k = (unsigned)__builtin_ctz(hm); hm &= hm - 1;
                node = (int)cb + __builtin_popcount(im & ((1u << (k ^ oct)) - 1u));
            }
        }
        t_out[i] = hitT; tri_out[i] = hit;
    }
    return 0;
}

/* ------------------------------------------------------------------ precision form, restated bit for bit
 * Not in the reference. The CUDA precision form (f16x2 conservative slab tests over the CWBVH, watertight FP32
 * triangle test on the exact corners) with every f16 operation emulated exactly: a product of two halves is exact in
 * double and the sum with a third is exact or far from a rounding midpoint, so rounding the double result once to the
 * nearest half gives the hardware's fused multiply-add; conversions round down / up / to nearest as the kernel asks.
 * Closest: hits float4 (t, u, v, tri bits); any: occ = first occluder or -1. stats as orc_trace. */
static double hround(double x, int mode) { /* mode 0 nearest-even, -1 toward -inf, +1 toward +inf */
    if (x != x || isinf(x) || x == 0.0) return x;
    const int neg = x < 0.0; const double a = fabs(x);
    int e; frexp(a, &e); int ex = e - 1; if (ex < -14) ex = -14;
    const double qn = ldexp(1.0, ex - 10), k = a / qn, kf = floor(k), r = k - kf;
    int up;
    if (mode == 0) up = r > 0.5 || (r == 0.5 && fmod(kf, 2.0) == 1.0);
    else up = r > 0.0 && ((mode > 0) != neg);
    double m = (kf + up) * qn;
    if (m > 65504.0) m = (mode == 0 || up) ? INFINITY : 65504.0;
    return neg ? -m : m;
}
static double hfma(double a, double b, double c) { return hround(a * b + c, 0); }
double orc_half_round(double x, int mode) { return hround(x, mode); }
static float h16_margin(float A, float B) { return (1.001f * fabsf(A) + 1792.f * fabsf(B)) * (1.f / 2048.f) + 1e-4f; }
static int h16_ok(float A, float B) {
    const float m = h16_margin(A, B), Ap = A - 1024.f * B;
    return fabsf(B) * 1279.f < 30000.f && fabsf(Ap) + m < 30000.f;
}
static void h16_axis(float A, float B, double* lo, double* hi, double* b) {
    const float m = h16_margin(A, B), Ap = A - 1024.f * B;
    *lo = hround(Ap - m, -1); *hi = hround(Ap + m, 1); *b = hround(B, 0);
}
static void f32_axis(float A, float B, float* lo, float* hi, float* b) {
    if (fabsf(A) < 1e30f && fabsf(B) < 1e30f) { const float m = (fabsf(A) + 256.f * fabsf(B)) * 9.5367431640625e-7f + 1e-30f; *lo = A - m; *hi = A + m; *b = B; }
    else { *lo = -INFINITY; *hi = INFINITY; *b = 0.f; }
}
typedef struct { int kx, ky, kz; float sx, sy, sz; } WtRay;
static WtRay wt_setup(V3 d) {
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    WtRay r; r.kz = ax >= ay ? (ax >= az ? 0 : 2) : (ay >= az ? 1 : 2);
    r.kx = r.kz == 2 ? 0 : r.kz + 1; r.ky = r.kx == 2 ? 0 : r.kx + 1;
    if (comp(d, r.kz) < 0.f) { int t = r.kx; r.kx = r.ky; r.ky = t; }
    const float dz = comp(d, r.kz);
    r.sx = comp(d, r.kx) / dz; r.sy = comp(d, r.ky) / dz; r.sz = 1.f / dz;
    return r;
}
static int wt_leaf(const V4* vt, int first, int cnt, V3 o, const WtRay* r, float tmin, int any, float* hitT, int* hitTri, float* hu, float* hv, Stats* st) {
    for (int t = first; t < first + cnt; t++) {
        if (st) st->tris++;
        const V3 A = sub(xyz4(vt[3 * t]), o), B = sub(xyz4(vt[3 * t + 1]), o), C = sub(xyz4(vt[3 * t + 2]), o);
        const float Az = comp(A, r->kz), Bz = comp(B, r->kz), Cz = comp(C, r->kz);
        const float Akx = comp(A, r->kx), Aky = comp(A, r->ky), Bkx = comp(B, r->kx), Bky = comp(B, r->ky), Ckx = comp(C, r->kx), Cky = comp(C, r->ky);
        const float pAx = r->sx * Az, pAy = r->sy * Az, pBx = r->sx * Bz, pBy = r->sy * Bz, pCx = r->sx * Cz, pCy = r->sy * Cz;
        const float Ax = Akx - pAx, Ay = Aky - pAy, Bx = Bkx - pBx, By = Bky - pBy, Cx = Ckx - pCx, Cy = Cky - pCy;
        const float U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
        const float SAx = fabsf(Akx) + fabsf(pAx), SAy = fabsf(Aky) + fabsf(pAy), SBx = fabsf(Bkx) + fabsf(pBx), SBy = fabsf(Bky) + fabsf(pBy);
        const float SCx = fabsf(Ckx) + fabsf(pCx), SCy = fabsf(Cky) + fabsf(pCy);
        const float eU = 1e-6f * (SCx * SBy + SCy * SBx) + 1e-30f, eV = 1e-6f * (SAx * SCy + SAy * SCx) + 1e-30f, eW = 1e-6f * (SBx * SAy + SBy * SAx) + 1e-30f;
        if ((U < -eU || V < -eV || W < -eW) && (U > eU || V > eV || W > eW)) continue;
        const float det = U + V + W;
        if (det == 0.f) continue;
        const float T = U * (r->sz * Az) + V * (r->sz * Bz) + W * (r->sz * Cz);
        const float tt = T / det;
        if (!(tt > tmin && tt < *hitT)) continue;
        *hitT = tt; *hitTri = t; *hu = V / det; *hv = W / det;
        if (any) return 1;
    }
    return 0;
}
static int trav_prec(const V4* nodes, const V4* vt, V3 o, V3 d, float tmin, int any, float* hitT, int* hitTri, float* hu, float* hv, Stats* st) {
    unsigned stk[40][2]; int sp = 0, node = 0;
    const float idx = safe_rcp(d.x), idy = safe_rcp(d.y), idz = safe_rcp(d.z);
    const unsigned oct = (d.x > 0.f ? 1u : 0u) | (d.y > 0.f ? 2u : 0u) | (d.z > 0.f ? 4u : 0u);
    const WtRay wt = wt_setup(d);
    unsigned cb = 0, im = 0, hm = 0;
    for (;;) {
        if (st) st->nodes++;
        const V4* nb = nodes + 5 * node;
        const V4 f0 = nb[0], f1 = nb[1];
        const unsigned ew = fu(f0.w), imask = ew >> 24, m0 = fu(f1.z), m1 = fu(f1.w);
        const int childBase = fi(f1.x), triBase = fi(f1.y);
        const unsigned* q = (const unsigned*)(nb + 2);   /* lo.x[2], lo.y[2], lo.z[2], hi.x[2], hi.y[2], hi.z[2] */
        const float A[3] = { (f0.x - o.x) * idx, (f0.y - o.y) * idy, (f0.z - o.z) * idz };
        const float Bq[3] = { uf((ew & 255u) << 23) * idx, uf(((ew >> 8) & 255u) << 23) * idy, uf(((ew >> 16) & 255u) << 23) * idz };
        const int flip[3] = { idx < 0.f, idy < 0.f, idz < 0.f };
        unsigned boxHit = 0;
        if (h16_ok(A[0], Bq[0]) && h16_ok(A[1], Bq[1]) && h16_ok(A[2], Bq[2])) {   /* f16 slabs */
            double lo[3], hi[3], b[3];
            for (int ax = 0; ax < 3; ax++) h16_axis(A[ax], Bq[ax], &lo[ax], &hi[ax], &b[ax]);
            const double tmn = hround(tmin, -1), tmx = hround(*hitT, 1);
            for (int s = 0; s < 8; s++) {
                const int w = s < 4 ? 0 : 1; double tn = tmn, tf = tmx;
                for (int ax = 0; ax < 3; ax++) {
                    const unsigned qlo = byte_of(q[2 * ax + w], s), qhi = byte_of(q[6 + 2 * ax + w], s);
                    const double n = hfma(1024.0 + (flip[ax] ? qhi : qlo), b[ax], lo[ax]), f = hfma(1024.0 + (flip[ax] ? qlo : qhi), b[ax], hi[ax]);
                    tn = fmax(tn, n); tf = fmin(tf, f);
                }
                if (tn <= tf) boxHit |= 1u << s;
            }
        } else {   /* FP32 slabs, widened */
            float lo[3], hi[3], b[3];
            for (int ax = 0; ax < 3; ax++) f32_axis(A[ax], Bq[ax], &lo[ax], &hi[ax], &b[ax]);
            for (int s = 0; s < 8; s++) {
                const int w = s < 4 ? 0 : 1; float n3[3], f3[3];
                for (int ax = 0; ax < 3; ax++) {
                    const unsigned qlo = byte_of(q[2 * ax + w], s), qhi = byte_of(q[6 + 2 * ax + w], s);
                    n3[ax] = fmaf((float)(flip[ax] ? qhi : qlo), b[ax], lo[ax]); f3[ax] = fmaf((float)(flip[ax] ? qlo : qhi), b[ax], hi[ax]);
                }
                const float tn = fmaxf(fmaxf(n3[0], n3[1]), fmaxf(n3[2], tmin)), tf = fminf(fminf(f3[0], f3[1]), fminf(f3[2], *hitT));
                if (tn <= tf) boxHit |= 1u << s;
            }
        }
        unsigned hits = 0;
        for (int s = 0; s < 8; s++) {
            if (!(boxHit & (1u << s))) continue;
            const unsigned m = byte_of(s < 4 ? m0 : m1, s);
            if (m & 0x80u) {
                if (wt_leaf(vt, triBase + (int)(m & 31u), (int)((m >> 5) & 3u) + 1, o, &wt, tmin, any, hitT, hitTri, hu, hv, st) && any) return 1;
            }
        }
        for (int s = 0; s < 8; s++) if ((boxHit & imask) & (1u << s)) hits |= 1u << (s ^ oct);
        if (hits) { if (hm) { if (sp == 40) return -1; stk[sp][0] = cb; stk[sp][1] = (im << 8) | hm; sp++; } cb = (unsigned)childBase; im = imask; hm = hits; }
        while (hm == 0) { if (sp == 0) return *hitTri >= 0; sp--; cb = stk[sp][0]; im = stk[sp][1] >> 8; hm = stk[sp][1] & 255u; }
        const unsigned k = (unsigned)__builtin_ctz(hm); hm &= hm - 1;
        node = (int)cb + __builtin_popcount(im & ((1u << (k ^ oct)) - 1u));
    }
}
long orc_trace_prec(const float* nodes, const float* vt, const float* ro, const float* rd, long n, int any, float* hits, int* occ, long long* stats) {
    long bad = 0; Stats st = { 0, 0 };
    for (long i = 0; i < n; i++) {
        const V3 o = v3(ro[4 * i], ro[4 * i + 1], ro[4 * i + 2]), d = v3(rd[4 * i], rd[4 * i + 1], rd[4 * i + 2]);
        float t = rd[4 * i + 3], u = 0.f, v = 0.f; int tri = -1;
        if (trav_prec((const V4*)nodes, (const V4*)vt, o, d, ro[4 * i + 3], any, &t, &tri, &u, &v, stats ? &st : NULL) < 0) bad++;
        if (any) occ[i] = tri;
        else { hits[4 * i] = t; hits[4 * i + 1] = u; hits[4 * i + 2] = v; memcpy(&hits[4 * i + 3], &tri, 4); }
    }
    if (stats) { stats[0] = st.nodes; stats[1] = st.tris; }
    return bad;
}

/* ------------------------------------------------------------------ two-level scenes (batched form)
 * Not a reference function: restates the CUDA batched form's traversal (accel/traverse_inst.cuh:10-41 is its model):
 * per ray, the TLAS of its scene (BVH2, leaves = one instance, nearer child first, leaves pushed like inner nodes and
 * entered when they come up), the instance's BLAS (width 2, 4 or 8, root = its mesh) with the ray brought into object
 * space by the instance's world->object rows (t shared), Moller-Trumbore triangles. inst: 28 floats per instance
 * (inv rows, fwd rows, root, mesh, det sign, pad as in cwp_instance). Closest: hits float4 + hit instance; any:
 * first occluder (hits may be NULL) + its instance. Returns the number of rays that hit a stack bound. */
static int trav_blas(int width, const V4* nodes, const V4* tv, V3 o, V3 d, float tmin, int any, float* t, int* h, float* u, float* v, int root) {
    if (width == 2) return trav2r(nodes, tv, o, d, tmin, any, 0, t, h, u, v, NULL, root);
    if (width == 4) return trav4r(nodes, tv, o, d, tmin, any, 0, t, h, u, v, NULL, root);
    return trav8r(nodes, tv, o, d, tmin, any, 0, t, h, u, v, NULL, root);
}
/* visit counters of the two-level traversal: TLAS nodes, instance entries, BLAS nodes, triangle tests (enabled by
 * orc_inst_stats; for cost studies) */
static long long g_inst_stats[4]; static int g_inst_stats_on;
void orc_inst_stats(int on, long long* out) { if (out) memcpy(out, g_inst_stats, sizeof g_inst_stats); memset(g_inst_stats, 0, sizeof g_inst_stats); g_inst_stats_on = on; }
/* One TLAS node of width 4 (8 float4: lo x, hi x, lo y, hi y, lo z, hi z of four children, child references,
 * counts; count 1 = an instance, 0 = an inner node, reference -1 = empty): the hit children sorted by entry distance
 * with the batched form's sorting network, the nearest returned and the others pushed far to near (instances as
 * ~index). Returns 1 when it chose an entry (*go), 0 when nothing was hit, -1 on a stack bound. */
static int o_tlas4_visit(const V4* T, int node, float idx, float idy, float idz, float ox, float oy, float oz, float tmin, float t,
                         int* stack, int* sp, int* go) {
    const float INF = 3.4e38f;
    const V4* nb = T + 8 * (size_t)node;
    const float LX[4] = { nb[0].x, nb[0].y, nb[0].z, nb[0].w }, HX[4] = { nb[1].x, nb[1].y, nb[1].z, nb[1].w };
    const float LY[4] = { nb[2].x, nb[2].y, nb[2].z, nb[2].w }, HY[4] = { nb[3].x, nb[3].y, nb[3].z, nb[3].w };
    const float LZ[4] = { nb[4].x, nb[4].y, nb[4].z, nb[4].w }, HZ[4] = { nb[5].x, nb[5].y, nb[5].z, nb[5].w };
    const int CC[4] = { fi(nb[6].x), fi(nb[6].y), fi(nb[6].z), fi(nb[6].w) }, KK[4] = { fi(nb[7].x), fi(nb[7].y), fi(nb[7].z), fi(nb[7].w) };
    float ht[4]; int he[4];
    for (int j = 0; j < 4; j++) {
        const float x0 = fmaf(LX[j], idx, ox), x1 = fmaf(HX[j], idx, ox), y0 = fmaf(LY[j], idy, oy), y1 = fmaf(HY[j], idy, oy), z0 = fmaf(LZ[j], idz, oz), z1 = fmaf(HZ[j], idz, oz);
        const float tn = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
        const float tf = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), t));
        ht[j] = CC[j] >= 0 && tn <= tf ? tn : INF;
        he[j] = KK[j] > 0 ? ~CC[j] : CC[j];
    }
#define O_CSWAP(a, b) { if (ht[b] < ht[a]) { float q_ = ht[a]; ht[a] = ht[b]; ht[b] = q_; int r_ = he[a]; he[a] = he[b]; he[b] = r_; } }
    O_CSWAP(0, 1) O_CSWAP(2, 3) O_CSWAP(0, 2) O_CSWAP(1, 3) O_CSWAP(1, 2)
#undef O_CSWAP
    if (ht[0] == INF) return 0;
    if (*sp + 3 > 64) return -1;
    if (ht[3] < INF) stack[(*sp)++] = he[3];
    if (ht[2] < INF) stack[(*sp)++] = he[2];
    if (ht[1] < INF) stack[(*sp)++] = he[1];
    *go = he[0];
    return 1;
}

/* one ray through one two-level scene (root = its TLAS root, < 0 for an empty scene); tlas_width 2 (BVH2 nodes) or
 * 4 (o_tlas4_visit); returns -1 on a stack bound */
static int o_inst1(int width, int tlas_width, int any, const float* blas, const float* tris, const V4* T, int root, const float* inst, V3 o, V3 d, float tmin,
                   float* pt, int* ph, float* pu, float* pv, int* phi) {
    float t = *pt, u = 0.f, v = 0.f; int h = -1, hi = -1, done = 0, bad = 0;
    if (root >= 0) {
        const float idx = safe_rcp(d.x), idy = safe_rcp(d.y), idz = safe_rcp(d.z), ox = -o.x * idx, oy = -o.y * idy, oz = -o.z * idz;
        int stack[64], sp = 0, next = root;
        while (!done) {
            if (g_inst_stats_on) g_inst_stats[0]++;
            int go;
            if (tlas_width == 4) {
                const int r = o_tlas4_visit(T, next, idx, idy, idz, ox, oy, oz, tmin, t, stack, &sp, &go);
                if (r < 0) { bad = 1; break; }
                if (r == 0) { if (sp == 0) break; go = stack[--sp]; }
            } else {
            const V4 n0 = T[4 * next], n1 = T[4 * next + 1], nz = T[4 * next + 2], mt = T[4 * next + 3];
            const int c0 = fi(mt.x), c1 = fi(mt.y), k0 = fi(mt.z), k1 = fi(mt.w);
            const float a0 = fmaf(n0.x, idx, ox), a1 = fmaf(n0.y, idx, ox), a2 = fmaf(n0.z, idy, oy), a3 = fmaf(n0.w, idy, oy), a4 = fmaf(nz.x, idz, oz), a5 = fmaf(nz.y, idz, oz);
            const float b0 = fmaf(n1.x, idx, ox), b1 = fmaf(n1.y, idx, ox), b2 = fmaf(n1.z, idy, oy), b3 = fmaf(n1.w, idy, oy), b4 = fmaf(nz.z, idz, oz), b5 = fmaf(nz.w, idz, oz);
            const float t0n = fmaxf(fmaxf(fminf(a0, a1), fminf(a2, a3)), fmaxf(fminf(a4, a5), tmin));
            const float t0f = fminf(fminf(fmaxf(a0, a1), fmaxf(a2, a3)), fminf(fmaxf(a4, a5), t));
            const float t1n = fmaxf(fmaxf(fminf(b0, b1), fminf(b2, b3)), fmaxf(fminf(b4, b5), tmin));
            const float t1f = fminf(fminf(fmaxf(b0, b1), fmaxf(b2, b3)), fminf(fmaxf(b4, b5), t));
            const int h0 = c0 >= 0 && t0n <= t0f, h1 = c1 >= 0 && t1n <= t1f;
            int e0 = k0 > 0 ? ~c0 : c0, e1 = k1 > 0 ? ~c1 : c1;
            if (h0 && h1) { if (t1n < t0n) { int q = e0; e0 = e1; e1 = q; } if (sp == 64) { bad = 1; break; } stack[sp++] = e1; go = e0; }
            else if (h0 || h1) go = h0 ? e0 : e1;
            else { if (sp == 0) break; go = stack[--sp]; }
            }
            while (go < 0) {   /* an instance: its BLAS in object space, then the next TLAS entry */
                const float* I = inst + 28 * (size_t)(~go);
                const V3 lo = v3(I[0] * o.x + I[1] * o.y + I[2] * o.z + I[3], I[4] * o.x + I[5] * o.y + I[6] * o.z + I[7], I[8] * o.x + I[9] * o.y + I[10] * o.z + I[11]);
                const V3 ld = v3(I[0] * d.x + I[1] * d.y + I[2] * d.z, I[4] * d.x + I[5] * d.y + I[6] * d.z, I[8] * d.x + I[9] * d.y + I[10] * d.z);
                int iroot; memcpy(&iroot, &I[24], 4);
                float bt = t, bu = 0.f, bv = 0.f; int bh = -1;
                Stats bs = { 0, 0 };
                if (g_inst_stats_on) g_inst_stats[1]++;
                if ((width == 2 ? trav2r((const V4*)blas, (const V4*)tris, lo, ld, tmin, any, 0, &bt, &bh, &bu, &bv, g_inst_stats_on ? &bs : NULL, iroot)
                     : width == 4 ? trav4r((const V4*)blas, (const V4*)tris, lo, ld, tmin, any, 0, &bt, &bh, &bu, &bv, g_inst_stats_on ? &bs : NULL, iroot)
                     : trav8r((const V4*)blas, (const V4*)tris, lo, ld, tmin, any, 0, &bt, &bh, &bu, &bv, g_inst_stats_on ? &bs : NULL, iroot)) < 0) { bad = 1; done = 1; break; }
                g_inst_stats[2] += bs.nodes; g_inst_stats[3] += bs.tris;
                if (bh >= 0 && bt < t) { t = bt; h = bh; u = bu; v = bv; hi = ~go; }
                if (any && h >= 0) { done = 1; break; }
                if (sp == 0) { done = 1; break; }
                go = stack[--sp];
            }
            if (!done) next = go;
        }
    }
    *pt = t; *ph = h; *pu = u; *pv = v; *phi = hi;
    return bad ? -1 : 0;
}
long orc_trace_inst(int width, int tlas_width, int any, const float* blas, const float* tris, const float* tlas, const int* scene_root, int n_scenes, const float* inst,
                    const float* ro, const float* rd, const int* scene_of, long n, float* hits, int* hit_inst) {
    long bad = 0;
    for (long i = 0; i < n; i++) {
        const V3 o = v3(ro[4 * i], ro[4 * i + 1], ro[4 * i + 2]), d = v3(rd[4 * i], rd[4 * i + 1], rd[4 * i + 2]);
        float t = rd[4 * i + 3], u, v; int h, hi;
        const int sc = scene_of[i], root = sc >= 0 && sc < n_scenes ? scene_root[sc] : -1;
        if (o_inst1(width, tlas_width, any, blas, tris, (const V4*)tlas, root, inst, o, d, ro[4 * i + 3], &t, &h, &u, &v, &hi) < 0) bad++;
        if (hits) { hits[4 * i] = t; hits[4 * i + 1] = u; hits[4 * i + 2] = v; hits[4 * i + 3] = iff(h); }
        hit_inst[i] = hi;
    }
    return bad;
}

/* ------------------------------------------------------------------ OpenPBR-subset BSDF (render/bsdf.h:17-220)
 * Local frame: z = shading normal, wo.z > 0. Material = 16 floats in the cwp_material / Material layout
 * (scene/material.h:12-17): base[3], metallic, spec[3], roughness, emission[3], ior, spec_weight, transmission, pad[2].
 * Written from the same papers as render/bsdf.h (GGX / height-correlated Smith, Dupuy-Benyoub visible normals,
 * exact dielectric Fresnel, F82-tinted Schlick). */
typedef struct { float base[3], metallic, spec[3], roughness, emission[3], ior, ws, transmission, pad0, pad1; } OMat;
#define O_PI 3.14159265f
#define O_DELTA 1e-3f
static float o_lum(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
static float o_d(float cm, float a2) { if (cm <= 0.f) return 0.f; float c2 = cm * cm, k = c2 * (a2 - 1.f) + 1.f; return a2 / (O_PI * k * k); }
static float o_lambda(float cw, float a2) { float c2 = cw * cw; if (c2 < 1e-12f) return 1e12f; return 0.5f * (sqrtf(1.f + a2 * (1.f - c2) / c2) - 1.f); }
static float o_g1(float c, float a2) { return 1.f / (1.f + o_lambda(c, a2)); }
static float o_g2(float co, float ci, float a2) { return 1.f / (1.f + o_lambda(co, a2) + o_lambda(ci, a2)); }
static float o_vpdf(V3 wo, V3 m, float a2) { float om = dot3(wo, m); if (om <= 0.f || m.z <= 0.f) return 0.f; return o_g1(wo.z, a2) * om * o_d(m.z, a2) / wo.z; }
static V3 o_vsample(V3 wo, float a, float u1, float u2) {
    V3 v = normz(v3(a * wo.x, a * wo.y, wo.z)); float ph = 6.2831853f * u1, z = (1.f - u2) * (1.f + v.z) - v.z;
    float s = sqrtf(fminf(fmaxf(1.f - z * z, 0.f), 1.f));
    V3 h = v3(s * cosf(ph) + v.x, s * sinf(ph) + v.y, z + v.z);
    return normz(v3(a * h.x, a * h.y, fmaxf(h.z, 0.f)));
}
static float o_fd(float ci, float eta) {
    float s2 = (1.f - ci * ci) / (eta * eta); if (s2 >= 1.f) return 1.f;
    float ct = sqrtf(1.f - s2), rs = (ci - eta * ct) / (ci + eta * ct), rp = (eta * ci - ct) / (eta * ci + ct);
    return 0.5f * (rs * rs + rp * rp);
}
static V3 o_f82(V3 F0, V3 tint, float mu) {
    mu = fminf(fmaxf(mu, 0.f), 1.f);
    float q = 1.f - mu, q2 = q * q, q5 = q2 * q2 * q, q6 = q5 * q, mb = 1.f / 7.f, qb = 6.f / 7.f, qb2 = qb * qb, qb5 = qb2 * qb2 * qb, qb6 = qb5 * qb;
    float c[3] = { F0.x, F0.y, F0.z }, t[3] = { tint.x, tint.y, tint.z }, o[3];
    for (int i = 0; i < 3; i++) {
        float s = c[i] + (1.f - c[i]) * q5, sb = c[i] + (1.f - c[i]) * qb5, b = sb * (1.f - t[i]) * (1.f / (mb * qb6));
        float F = s - b * (mu * q6); o[i] = fminf(fmaxf(F, 0.f), 1.f);
    }
    return v3(o[0], o[1], o[2]);
}
static V3 o_cos_dir(float u0, float u1) {   /* cosine hemisphere about +z (core/sampling.h:19-22) */
    V3 n = v3(0.f, 0.f, 1.f), t, b; onb(n, &t, &b);
    float r = sqrtf(u0), ph = 6.2831853f * u1;
    return normz(add(add(muls(t, r * cosf(ph)), muls(b, r * sinf(ph))), muls(n, sqrtf(fmaxf(0.f, 1.f - u0)))));
}
typedef struct { V3 f; float pdf; } OEval;
/* glossy-diffuse (bsdf.h:84-124) */
typedef struct { V3 base; float ws, eta, a, a2, Fo, pSpec, kd; int delta; V3 nr; } OGd;
/* bump-terminator shadowing of the diffuse lobe (Chiang, Li, Burley, SIGGRAPH 2019 talk; bsdf.h:67-75): nr = the
 * unperturbed normal in the frame of the mapped shading normal, g = (nr . wi) / (wi.z nr.z), G = g + g^2 - g^3 on
 * [0, 1), 1 above, 0 below; nr = +z: G = 1 */
static float o_bump(V3 nr, V3 wi) {
    if (nr.z >= 1.f) return 1.f;
    const float g = dot3(nr, wi) / (wi.z * nr.z);
    if (g >= 1.f) return 1.f;
    if (g < 0.f) return 0.f;
    return g + g * g - g * g * g;
}
static OGd o_gd(const OMat* m, V3 wo, int energy, float ux1, float ux2) {
    OGd g; g.base = v3(m->base[0], m->base[1], m->base[2]); g.ws = m->ws; g.eta = m->ior; g.a = m->roughness * m->roughness; g.a2 = g.a * g.a; g.delta = g.a < O_DELTA;
    g.Fo = g.ws > 0.f ? g.ws * o_fd(wo.z, g.eta) : 0.f;
    float pd = (1.f - g.Fo) * o_lum(g.base); g.pSpec = g.Fo + pd > 0.f ? g.Fo / (g.Fo + pd) : 0.f;
    g.kd = 1.f - g.Fo;
    if (energy && g.ws > 0.f && !g.delta) {
        V3 mm = o_vsample(wo, g.a, ux1, ux2); float om = dot3(wo, mm); V3 wr = sub(muls(mm, 2.f * om), wo);
        float X = (om > 0.f && wr.z > 0.f) ? g.ws * o_fd(om, g.eta) * o_g2(wo.z, wr.z, g.a2) / o_g1(wo.z, g.a2) : 0.f;
        g.kd = 1.f - X;
    }
    g.kd = fmaxf(g.kd, 0.f); g.nr = v3(0.f, 0.f, 1.f);
    return g;
}
static OEval o_gd_eval(const OGd* g, V3 wo, V3 wi) {
    OEval r = { v3(0.f, 0.f, 0.f), 0.f };
    if (wi.z <= 0.f) return r;
    r.f = muls(g->base, g->kd * 0.31830989f * o_bump(g->nr, wi)); r.pdf = (1.f - g->pSpec) * wi.z * 0.31830989f;
    if (!g->delta && g->Fo > 0.f) {
        V3 m = normz(add(wo, wi)); float om = dot3(wo, m);
        if (om > 0.f) {
            float s = g->ws * o_fd(om, g->eta) * o_d(m.z, g->a2) * o_g2(wo.z, wi.z, g->a2) / (4.f * wo.z * wi.z);
            r.f = add(r.f, v3(s, s, s)); r.pdf += g->pSpec * o_vpdf(wo, m, g->a2) / (4.f * om);
        }
    }
    return r;
}
static int o_gd_sample(const OGd* g, V3 wo, float u, float u1, float u2, V3* wi, V3* w, float* pdf) {
    if (u < g->pSpec) {
        if (g->delta) { *wi = v3(-wo.x, -wo.y, wo.z); float s = g->Fo / g->pSpec; *w = v3(s, s, s); *pdf = 0.f; return 1; }
        V3 m = o_vsample(wo, g->a, u1, u2); *wi = sub(muls(m, 2.f * dot3(wo, m)), wo);
        if (wi->z <= 0.f) return 0;
    } else { *wi = o_cos_dir(u1, u2); if (wi->z <= 0.f) return 0; }
    OEval e = o_gd_eval(g, wo, *wi); if (e.pdf <= 0.f) return 0;
    *w = muls(e.f, wi->z / e.pdf); *pdf = e.pdf; return 1;
}
/* conductor (bsdf.h:127-148) */
static OEval o_cond_eval(const OMat* m, V3 wo, V3 wi) {
    OEval r = { v3(0.f, 0.f, 0.f), 0.f }; float a = m->roughness * m->roughness, a2 = a * a;
    if (a < O_DELTA || wi.z <= 0.f) return r;
    V3 h = normz(add(wo, wi)); float om = dot3(wo, h); if (om <= 0.f) return r;
    r.f = muls(o_f82(v3(m->base[0], m->base[1], m->base[2]), v3(m->spec[0], m->spec[1], m->spec[2]), om), m->ws * o_d(h.z, a2) * o_g2(wo.z, wi.z, a2) / (4.f * wo.z * wi.z));
    r.pdf = o_vpdf(wo, h, a2) / (4.f * om);
    return r;
}
static int o_cond_sample(const OMat* m, V3 wo, float u1, float u2, V3* wi, V3* w, float* pdf) {
    float a = m->roughness * m->roughness, a2 = a * a; V3 F0 = v3(m->base[0], m->base[1], m->base[2]), tint = v3(m->spec[0], m->spec[1], m->spec[2]);
    if (a < O_DELTA) { *wi = v3(-wo.x, -wo.y, wo.z); *w = muls(o_f82(F0, tint, wo.z), m->ws); *pdf = 0.f; return 1; }
    V3 h = o_vsample(wo, a, u1, u2); float om = dot3(wo, h); *wi = sub(muls(h, 2.f * om), wo);
    if (wi->z <= 0.f || om <= 0.f) return 0;
    *w = muls(o_f82(F0, tint, om), m->ws * o_g2(wo.z, wi->z, a2) / o_g1(wo.z, a2));
    *pdf = o_vpdf(wo, h, a2) / (4.f * om); return 1;
}
/* rough dielectric (bsdf.h:151-192) */
static OEval o_diel_eval(const OMat* m, float eta, V3 wo, V3 wi) {
    OEval r = { v3(0.f, 0.f, 0.f), 0.f }; float a = m->roughness * m->roughness, a2 = a * a;
    if (a < O_DELTA) return r;
    if (wi.z > 0.f) {
        V3 h = normz(add(wo, wi)); float om = dot3(wo, h); if (om <= 0.f) return r;
        float F = o_fd(om, eta), s = F * o_d(h.z, a2) * o_g2(wo.z, wi.z, a2) / (4.f * wo.z * wi.z);
        r.f = v3(s, s, s); r.pdf = F * o_vpdf(wo, h, a2) / (4.f * om);
    } else if (wi.z < 0.f) {
        V3 h = normz(add(wo, muls(wi, eta))); if (h.z < 0.f) h = neg(h);
        float om = dot3(wo, h), im = dot3(wi, h); if (om <= 0.f || im >= 0.f) return r;
        float F = o_fd(om, eta); if (F >= 1.f) return r;
        float den = om + eta * im, j = eta * eta * (-im) / (den * den);
        float s = (1.f - F) * o_d(h.z, a2) * o_g2(wo.z, -wi.z, a2) * om * j / (wo.z * -wi.z);
        r.f = muls(v3(m->base[0], m->base[1], m->base[2]), s); r.pdf = (1.f - F) * o_vpdf(wo, h, a2) * j;
    }
    return r;
}
static int o_diel_sample(const OMat* m, float eta, V3 wo, float u, float u1, float u2, V3* wi, V3* w, float* pdf) {
    float a = m->roughness * m->roughness; int delta = a < O_DELTA;
    V3 h = delta ? v3(0.f, 0.f, 1.f) : o_vsample(wo, a, u1, u2);
    float om = dot3(wo, h); if (om <= 0.f) return 0;
    float F = o_fd(om, eta);
    if (u < F) { *wi = sub(muls(h, 2.f * om), wo); if (wi->z <= 0.f) return 0; if (delta) { *w = v3(1.f, 1.f, 1.f); *pdf = 0.f; return 1; } }
    else {
        float ct = sqrtf(fmaxf(1.f - (1.f - om * om) / (eta * eta), 0.f));
        *wi = add(muls(wo, -1.f / eta), muls(h, om / eta - ct)); if (wi->z >= 0.f) return 0;
        *wi = normz(*wi);
        if (delta) { *w = v3(m->base[0], m->base[1], m->base[2]); *pdf = 0.f; return 1; }
    }
    OEval e = o_diel_eval(m, eta, wo, *wi); if (e.pdf <= 0.f) return 0;
    *w = muls(e.f, fabsf(wi->z) / e.pdf); *pdf = e.pdf; return 1;
}
static void o_weights(const OMat* m, float* wM, float* wT, float* wD) { *wM = m->metallic; *wT = (1.f - m->metallic) * m->transmission; *wD = (1.f - m->metallic) * (1.f - m->transmission); }
static int o_non_delta(const OMat* m) {
    float wM, wT, wD; o_weights(m, &wM, &wT, &wD); int rough = m->roughness * m->roughness >= O_DELTA;
    return (wD > 0.f && (o_lum(v3(m->base[0], m->base[1], m->base[2])) > 0.f || rough)) || ((wM > 0.f || wT > 0.f) && rough);
}
static OEval o_bsdf_eval(const OMat* m, V3 wo, V3 wi, float eta, int gd, float ux1, float ux2, V3 nr) {
    float wM, wT, wD; o_weights(m, &wM, &wT, &wD); OEval r = { v3(0.f, 0.f, 0.f), 0.f };
    if (wM > 0.f) { OEval e = o_cond_eval(m, wo, wi); r.f = add(r.f, muls(e.f, wM)); r.pdf += wM * e.pdf; }
    if (wT > 0.f) { OEval e = o_diel_eval(m, eta, wo, wi); r.f = add(r.f, muls(e.f, wT)); r.pdf += wT * e.pdf; }
    if (wD > 0.f) { OGd g = o_gd(m, wo, gd, ux1, ux2); g.nr = nr; OEval e = o_gd_eval(&g, wo, wi); r.f = add(r.f, muls(e.f, wD)); r.pdf += wD * e.pdf; }
    return r;
}
static int o_bsdf_sample(const OMat* m, V3 wo, float eta, int gd, float ux1, float ux2, float u, float u1, float u2, V3* wi, V3* w, float* pdf, V3 nr) {
    float wM, wT, wD; o_weights(m, &wM, &wT, &wD); int ok;
    if (u < wM) ok = o_cond_sample(m, wo, u1, u2, wi, w, pdf);
    else if (u < wM + wT) ok = o_diel_sample(m, eta, wo, fminf((u - wM) / wT, 0.99999994f), u1, u2, wi, w, pdf);
    else { OGd g = o_gd(m, wo, gd, ux1, ux2); g.nr = nr; ok = o_gd_sample(&g, wo, fminf(wD > 0.f ? (u - wM - wT) / wD : 0.f, 0.99999994f), u1, u2, wi, w, pdf); }
    if (!ok) return 0;
    if (*pdf <= 0.f) return 1;
    if (wM == 1.f || wT == 1.f || wD == 1.f) return 1;
    OEval e = o_bsdf_eval(m, wo, *wi, eta, gd, ux1, ux2, nr); if (e.pdf <= 0.f) return 0;
    *w = muls(e.f, fabsf(wi->z) / e.pdf); *pdf = e.pdf; return 1;
}
/* nr: an unperturbed normal per case (the bump-terminator term), or NULL: +z (off) */
void orc_bsdf_eval(const float* mats, const int* mat, const float* wo, const float* wi, const float* eta, int gd, const float* ux, float* f, float* pdf, long n,
                   const float* nr) {
    for (long i = 0; i < n; i++) {
        OEval e = o_bsdf_eval((const OMat*)(mats + 16 * (size_t)mat[i]), a3(wo + 3 * i), a3(wi + 3 * i), eta[i], gd, ux[2 * i], ux[2 * i + 1],
                              nr ? a3(nr + 3 * i) : v3(0.f, 0.f, 1.f));
        f[3 * i] = e.f.x; f[3 * i + 1] = e.f.y; f[3 * i + 2] = e.f.z; pdf[i] = e.pdf;
    }
}
void orc_bsdf_sample(const float* mats, const int* mat, const float* wo, const float* eta, int gd, const float* ux, const float* uvw, float* wi, float* w, float* pdf, int* ok, long n,
                     const float* nr) {
    for (long i = 0; i < n; i++) {
        V3 a = v3(0.f, 0.f, 0.f), b = a; float p = 0.f;
        ok[i] = o_bsdf_sample((const OMat*)(mats + 16 * (size_t)mat[i]), a3(wo + 3 * i), eta[i], gd, ux[2 * i], ux[2 * i + 1], uvw[3 * i], uvw[3 * i + 1], uvw[3 * i + 2], &a, &b, &p,
                              nr ? a3(nr + 3 * i) : v3(0.f, 0.f, 1.f));
        wi[3 * i] = a.x; wi[3 * i + 1] = a.y; wi[3 * i + 2] = a.z; w[3 * i] = b.x; w[3 * i + 1] = b.y; w[3 * i + 2] = b.z; pdf[i] = p;
    }
}

/* ------------------------------------------------------------------ serving form: one request on the host
 * Not a reference function as a whole: restates the CUDA serving loop's per-path arithmetic (camera ray with a box
 * filter, render/wavefront.cu:42-58; shading = shadeFull<INST>, render/wavefront.cu:223-356: one light sample per
 * vertex over the sun, the emissive triangles and an environment map with the power heuristic, light modes, Russian
 * roulette) over the two-level scene above and the BSDF restatement. Paths [j0, j1) of the request
 * in the CUDA path order (pixel = tile order of j mod N, sample j / N); accum = w * h float4 sums, counts[0] closest
 * rays, counts[1] shadow rays. */
typedef struct { float pos[3], ax[3], ay[3], az[3], fx, fy, px, py; int w, h; float lens_r, focus_d; } OCam;
typedef struct { int scene, frame; OCam cam; int spp, max_depth; unsigned seed; float sun_to[3], sun_e[3], sky[3], sun_cos, eps; int env; float env_rot_deg;
                 int light_mode, rr, rr_depth, env_uniform, bump_shadow; float near_clip; int filter_bh; } OReq;
/* concentric disk map (Shirley & Chiu 1997; core/sampling.h:46-52) */
static void o_disk(float u0, float u1, float* x, float* y) {
    const float a = 2.f * u0 - 1.f, b = 2.f * u1 - 1.f;
    if (a == 0.f && b == 0.f) { *x = *y = 0.f; return; }
    float r, ph;
    if (fabsf(a) > fabsf(b)) { r = a; ph = 0.78539816f * (b / a); } else { r = b; ph = 1.57079633f - 0.78539816f * (a / b); }
    *x = r * cosf(ph); *y = r * sinf(ph);
}
enum { O_LIGHT_MIS = 0, O_LIGHT_NEE = 1, O_LIGHT_BSDF = 2 };   /* render/params.h:23 */

/* Emissive-triangle light tables of one frame (SceneSetup::frameData, app/scene_setup.cpp:274-299). soup: 12 floats
 * per triangle of every mesh in mesh order, (v0, face id), (v1, face material), (v2, 0); triangle material =
 * mesh_mat[mesh] + face material clamped to the table; emissive when an emission component is > 0. Instances in
 * order, each one's emissive triangles in mesh order: corners by the float 3x4 rows, area 0.5 |e1 x e2| in float,
 * power luminance x area summed in double. em_tris: 12 floats per triangle, (w0, global id), (e1, material), (e2, 0);
 * em_cdf n + 1 floats; mat_pdf n_mats floats = luminance / total power. Returns n (0 when the total power is 0);
 * em_tris NULL: the count only. */
long orc_emissive_tables(const float* soup, const int* mesh_first, int n_mesh, const int* mesh_mat, const float* mats, int n_mats,
                         const float* xf, const int* inst_mesh, long n_inst, float* em_tris, float* em_cdf, float* mat_pdf) {
    const OMat* M = (const OMat*)mats;
    long n = 0; double tot = 0.0;
    double* pw = NULL; float* rec = NULL; long cap = 0;   /* records staged here: the caller's array holds only what is returned */
    for (long i = 0; i < n_inst; i++) {
        const float* m = xf + 12 * i; const int mesh = inst_mesh[i];
        for (int g = mesh_first[mesh]; g < mesh_first[mesh + 1]; g++) {
            const float* r = soup + 12 * (size_t)g;
            int mid = mesh_mat[mesh] + fi(r[7]); mid = mid < 0 ? 0 : mid >= n_mats ? n_mats - 1 : mid;
            if (!(M[mid].emission[0] > 0.f || M[mid].emission[1] > 0.f || M[mid].emission[2] > 0.f)) continue;
            float w[3][3];
            for (int c = 0; c < 3; c++) for (int k = 0; k < 3; k++)
                w[c][k] = m[4 * k] * r[4 * c] + m[4 * k + 1] * r[4 * c + 1] + m[4 * k + 2] * r[4 * c + 2] + m[4 * k + 3];
            const V3 e1 = v3(w[1][0] - w[0][0], w[1][1] - w[0][1], w[1][2] - w[0][2]), e2 = v3(w[2][0] - w[0][0], w[2][1] - w[0][1], w[2][2] - w[0][2]);
            const V3 cr = cross3(e1, e2);
            const double area = 0.5 * sqrtf(dot3(cr, cr));
            double pwr = o_lum(v3(M[mid].emission[0], M[mid].emission[1], M[mid].emission[2])) * area; pwr = pwr > 0 ? pwr : 0;
            if (n == cap) { cap = cap ? 2 * cap : 256; pw = (double*)realloc(pw, sizeof(double) * (size_t)cap); rec = (float*)realloc(rec, sizeof(float) * 12 * (size_t)cap); }
            pw[n] = pwr; tot += pwr;
            {
                float* t = rec + 12 * (size_t)n;
                t[0] = w[0][0]; t[1] = w[0][1]; t[2] = w[0][2]; memcpy(&t[3], &g, 4);
                t[4] = e1.x; t[5] = e1.y; t[6] = e1.z; memcpy(&t[7], &mid, 4);
                t[8] = e2.x; t[9] = e2.y; t[10] = e2.z; t[11] = 0.f;
            }
            n++;
        }
    }
    if (!(tot > 0)) n = 0;
    if (em_tris) {
        for (int j = 0; j < n_mats; j++) mat_pdf[j] = 0.f;
        if (n) {
            memcpy(em_tris, rec, sizeof(float) * 12 * (size_t)n);
            double c = 0.0; em_cdf[0] = 0.f;
            for (long e = 0; e < n; e++) { c += pw[e]; em_cdf[e + 1] = (float)(c / tot); }
            em_cdf[n] = 1.f;
            for (int j = 0; j < n_mats; j++)
                if (M[j].emission[0] > 0.f || M[j].emission[1] > 0.f || M[j].emission[2] > 0.f) mat_pdf[j] = (float)(o_lum(v3(M[j].emission[0], M[j].emission[1], M[j].emission[2])) / tot);
        }
    }
    free(pw); free(rec);
    return n;
}

/* Environment map tables (scene/environment.cpp:7-38): texels = rgb x strength (float4), marg = CDF over rows (h + 1),
 * cond = CDF within each row (h rows of w + 1); texel weight luminance x sin(theta), sums in double. */
void orc_envmap_build(const float* rgb, int w, int h, float strength, float* texels, float* marg, float* cond) {
    const double pi = 3.14159265358979323846;
    double* row = (double*)malloc(sizeof(double) * (size_t)(w + 1));
    double* rs = (double*)malloc(sizeof(double) * (size_t)h);
    for (int y = 0; y < h; y++) {
        const double st = sin(pi * (y + 0.5) / h);
        row[0] = 0.0;
        for (int x = 0; x < w; x++) {
            const float* c = rgb + ((size_t)y * w + x) * 3;
            float* t = texels + 4 * ((size_t)y * w + x);
            t[0] = c[0] * strength; t[1] = c[1] * strength; t[2] = c[2] * strength; t[3] = 0.f;
            const double lum = 0.2126 * t[0] + 0.7152 * t[1] + 0.0722 * t[2];
            row[x + 1] = row[x] + (lum > 0 ? lum : 0.0) * st;
        }
        rs[y] = row[w];
        for (int x = 0; x <= w; x++) cond[(size_t)y * (w + 1) + x] = rs[y] > 0 ? (float)(row[x] / rs[y]) : (float)x / w;
        cond[(size_t)y * (w + 1) + w] = 1.f;
    }
    double acc = 0.0, tot = 0.0;
    for (int y = 0; y < h; y++) tot += rs[y];
    marg[0] = 0.f;
    for (int y = 0; y < h; y++) { acc += rs[y]; marg[y + 1] = tot > 0 ? (float)(acc / tot) : (float)(y + 1) / h; }
    marg[h] = 1.f;
    free(row); free(rs);
}

/* environment lookups of the serving integrator (render/wavefront.cu:177-197): equirectangular, row 0 = +z, centre
 * column +x, rotated by rot about +z */
typedef struct { const float* tex; const float* marg; const float* cond; int w, h; float rot; } OEnv;
static void o_env_texel(const OEnv* E, V3 d, int* x, int* y, float* v) {
    float u = 0.5f - (atan2f(d.y, d.x) - E->rot) * (1.f / 6.2831853f); u -= floorf(u);
    *v = acosf(fminf(fmaxf(d.z, -1.f), 1.f)) * 0.31830989f;
    *x = (int)(u * E->w); if (*x > E->w - 1) *x = E->w - 1;
    *y = (int)(*v * E->h); if (*y > E->h - 1) *y = E->h - 1;
}
static float o_env_pdf_texel(const OEnv* E, int x, int y, float v) {
    const float* cr = E->cond + (size_t)y * (E->w + 1);
    const float puv = (E->marg[y + 1] - E->marg[y]) * (cr[x + 1] - cr[x]) * E->w * E->h;
    const float st = sinf(v * 3.14159265f);
    return st > 0.f ? puv / (2.f * 3.14159265f * 3.14159265f * st) : 0.f;
}
/* Material textures (render/wavefront.cu:198-204, 252-270; scene/texture.h). A lookup restates the texture unit's
 * documented linear filtering of 8-bit RGBA images with normalised coordinates and wrap addressing: coordinate
 * frac(u) * w - 0.5, the four texels around it weighted by the fractional parts kept to 8 bits, channels read as
 * value / 255 and, for colour images, decoded from sRGB before the weighting. Images top row first, looked up at
 * (u, 1 - v). OTex and OMTex have the layouts of cwp_texture and cwp_material_textures. */
typedef struct { const unsigned char* rgba; int w, h, srgb, nearest; } OTex;
typedef struct { int base_color, emission, normal, metallic, roughness, metallic_ch, roughness_ch; float normal_scale; } OMTex;
static float o_srgb(float c) { return c <= 0.04045f ? c / 12.92f : powf((c + 0.055f) / 1.055f, 2.4f); }
static void o_tex(const OTex* T, float u, float v, float out[4]) {
    if (T->nearest) {   /* point sampling: the texel containing (frac(u) w, frac(v) h) */
        int i = (int)floorf((u - floorf(u)) * T->w), j = (int)floorf((v - floorf(v)) * T->h);
        i = i < T->w ? i : T->w - 1; j = j < T->h ? j : T->h - 1;
        const unsigned char* p = T->rgba + 4 * ((size_t)j * T->w + i);
        for (int c = 0; c < 4; c++) { float x8 = p[c] / 255.f; if (T->srgb && c < 3) x8 = o_srgb(x8); out[c] = x8; }
        return;
    }
    const float x = (u - floorf(u)) * T->w - 0.5f, y = (v - floorf(v)) * T->h - 0.5f;
    const float fx = floorf(x), fy = floorf(y);
    const float a = rintf((x - fx) * 256.f) / 256.f, b = rintf((y - fy) * 256.f) / 256.f;
    const int i0 = (int)fx, j0 = (int)fy;
    for (int c = 0; c < 4; c++) out[c] = 0.f;
    for (int k = 0; k < 4; k++) {
        int i = i0 + (k & 1), j = j0 + (k >> 1);
        i %= T->w; if (i < 0) i += T->w; j %= T->h; if (j < 0) j += T->h;
        const float wgt = ((k & 1) ? a : 1.f - a) * ((k >> 1) ? b : 1.f - b);
        const unsigned char* p = T->rgba + 4 * ((size_t)j * T->w + i);
        for (int c = 0; c < 4; c++) { float x8 = p[c] / 255.f; if (T->srgb && c < 3) x8 = o_srgb(x8); out[c] += wgt * x8; }
    }
}
void orc_texture_sample(const void* tex, const int* id, const float* uv, float* rgba, long n) {
    const OTex* T = (const OTex*)tex;
    for (long i = 0; i < n; i++) o_tex(&T[id[i]], uv[2 * i], 1.f - uv[2 * i + 1], rgba + 4 * i);
}

static int o_cdf_find(const float* cdf, int n, float u) { int lo = 0, hi = n; while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (cdf[mid] <= u) lo = mid; else hi = mid; } return lo; }
static float o_mis(float a, float b) { const float a2 = a * a; return a2 / (a2 + b * b); }
static int o_tile_pixel(int j, int w, int h) {
    if ((w & 7) | (h & 3)) return j;
    const int t = j >> 5, r = j & 31, tilesX = w >> 3;
    return ((t / tilesX) * 4 + (r >> 3)) * w + (t % tilesX) * 8 + (r & 7);
}
long orc_render_request(const void* reqp, int width, int tlas_width, const float* blas, const float* tris, const float* tlas, int root, const float* inst,
                        const float* mats, int n_mats, const int* mesh_mat, int gd, long j0, long j1, float* accum, long long* counts,
                        const float* env_tex, const float* env_marg, const float* env_cond, int env_w, int env_h,
                        const void* tex, const void* mtex, int n_mtex, const float* uvs, const float* tans, const int* mesh_first,
                        const float* em_tris, const float* em_cdf, const float* mat_pdf, long n_em, const float* nrm, const float* ftab) {
    const OTex* TX = (const OTex*)tex; const OMTex* MX = (const OMTex*)mtex;
    const OReq* R = (const OReq*)reqp; const OCam* C = &R->cam;
    const int N = C->w * C->h; long bad = 0;
    const OEnv E = { env_tex, env_marg, env_cond, env_w, env_h, R->env_rot_deg * 3.14159265f / 180.f };
    const int hasEnv = R->env >= 0 && env_tex != NULL;
    const V3 sunTo = v3(R->sun_to[0], R->sun_to[1], R->sun_to[2]), sunE = v3(R->sun_e[0], R->sun_e[1], R->sun_e[2]), sky = v3(R->sky[0], R->sky[1], R->sky[2]);
    const OMat* MT = (const OMat*)mats;
    /* light-type probabilities (render/wavefront.cu:531-533): equal over the sun (luminance > 0), the emissive
     * triangles and the map, the latter two not in BSDF mode */
    const int sunOn = o_lum(sunE) > 0.f, triOn = n_em > 0 && R->light_mode != O_LIGHT_BSDF, envOn = hasEnv && R->light_mode != O_LIGHT_BSDF;
    const int nt = sunOn + triOn + envOn;
    const float pSun = sunOn ? 1.f / nt : 0.f, pTri = triOn ? 1.f / nt : 0.f, pEnv = envOn ? 1.f / nt : 0.f;
    for (long j = j0; j < j1; j++) {
        const int pix = o_tile_pixel((int)(j % N), C->w, C->h); const unsigned smp = (unsigned)(j / N), seed = R->seed;
        const int x = pix % C->w, y = pix / C->w;
        /* camera ray (render/wavefront.cu:42-58): box or Blackman-Harris filter, thin lens, near clip */
        const float u0 = orc_rng(pix, smp, 0, 0, seed), u1 = orc_rng(pix, smp, 0, 1, seed);
        float jx, jy;
        if (R->filter_bh) { jx = table_lookup(ftab, 64, u0); jy = table_lookup(ftab, 64, u1); } else { jx = u0 - 0.5f; jy = u1 - 0.5f; }
        const float dx = (x + 0.5f + jx - C->px) / C->fx, dy = -(y + 0.5f + jy - C->py) / C->fy;
        const V3 cax = v3(C->ax[0], C->ax[1], C->ax[2]), cay = v3(C->ay[0], C->ay[1], C->ay[2]), caz = v3(C->az[0], C->az[1], C->az[2]);
        const V3 pos = v3(C->pos[0], C->pos[1], C->pos[2]), pin = sub(add(muls(cax, dx), muls(cay, dy)), caz);
        V3 o = pos, d = normz(pin);
        if (C->lens_r > 0.f) {
            float lx, ly; o_disk(orc_rng(pix, smp, 0, 2, seed), orc_rng(pix, smp, 0, 3, seed), &lx, &ly);
            const V3 pf = add(pos, muls(pin, C->focus_d));
            o = add(add(pos, muls(cax, lx * C->lens_r)), muls(cay, ly * C->lens_r));
            d = normz(sub(pf, o));
        }
        float tmin0 = R->near_clip;
        V3 T = v3(1.f, 1.f, 1.f);
        float lastPdf = 0.f;   /* pdf of the last BSDF sample (0: camera ray; <= 0: a delta lobe) */
        float* A = accum + 4 * (size_t)pix;
        for (int depth = 0;; depth++) {
            float t = 1e30f, u, v; int tri, hi;
            if (o_inst1(width, tlas_width, 0, blas, tris, (const V4*)tlas, root, inst, o, d, depth == 0 ? tmin0 : 0.f, &t, &tri, &u, &v, &hi) < 0) bad++;
            counts[0]++;
            if (tri < 0) {   /* miss: the environment weighted against its light sampling, or the constant sky */
                V3 L = sky;
                if (hasEnv) {
                    int ex, ey; float ev; o_env_texel(&E, d, &ex, &ey, &ev);
                    const float* tx4 = E.tex + 4 * ((size_t)ey * E.w + ex); L = v3(tx4[0], tx4[1], tx4[2]);
                    if (lastPdf > 0.f) {
                        if (R->light_mode == O_LIGHT_NEE) L = v3(0.f, 0.f, 0.f);
                        else if (R->light_mode == O_LIGHT_MIS) L = muls(L, o_mis(lastPdf, pEnv * (R->env_uniform ? 0.25f * 0.31830989f : o_env_pdf_texel(&E, ex, ey, ev))));
                    }
                }
                A[0] += T.x * L.x; A[1] += T.y * L.y; A[2] += T.z * L.z; break;
            }
            const float* I = inst + 28 * (size_t)hi;
            const V4* TR = (const V4*)tris;
            const V3 e1 = xyz4(TR[3 * tri + 1]), e2 = xyz4(TR[3 * tri + 2]), no = cross3(e1, e2);
            const V3 nw = v3(I[0] * no.x + I[4] * no.y + I[8] * no.z, I[1] * no.x + I[5] * no.y + I[9] * no.z, I[2] * no.x + I[6] * no.y + I[10] * no.z);
            int imesh; memcpy(&imesh, &I[25], 4);
            const V3 ng0 = muls(normz(nw), I[26]);
            int mid = mesh_mat[imesh] + fi(TR[3 * tri + 1].w); mid = mid < 0 ? 0 : mid >= n_mats ? n_mats - 1 : mid;
            OMat Mc = *(const OMat*)(mats + 16 * (size_t)mid); const OMat* M = &Mc;
            V3 nsw = ng0;
            if (nrm) {   /* corner normals (12 floats per triangle in mesh order) by the inverse transpose (wavefront.cu:245-249) */
                const float* n0 = nrm + 12 * ((size_t)mesh_first[imesh] + fi(TR[3 * tri].w));
                const float w0 = 1.f - u - v;
                const V3 nn = add(add(muls(v3(n0[0], n0[1], n0[2]), w0), muls(v3(n0[4], n0[5], n0[6]), u)), muls(v3(n0[8], n0[9], n0[10]), v));
                const V3 nt = v3(I[0] * nn.x + I[4] * nn.y + I[8] * nn.z, I[1] * nn.x + I[5] * nn.y + I[9] * nn.z, I[2] * nn.x + I[6] * nn.y + I[10] * nn.z);
                const float l = sqrtf(dot3(nt, nt));
                if (l > 0.f) nsw = muls(nt, 1.f / l);
                if (dot3(nsw, ng0) < 0.f) nsw = neg(nsw);
            }
            const V3 nsU0 = nsw; int mapped = 0;   /* the normal before a normal image, for the bump-terminator term */
            if (MX && mid < n_mtex && (MX[mid].base_color >= 0 || MX[mid].emission >= 0 || MX[mid].normal >= 0 || MX[mid].metallic >= 0 || MX[mid].roughness >= 0)) {
                const OMTex X = MX[mid];
                const long ti = (long)mesh_first[imesh] + fi(TR[3 * tri].w);
                const float* q = uvs + 8 * (size_t)ti; const float b0 = 1.f - u - v;
                const float tu = q[0] * b0 + q[2] * u + q[4] * v, tv = q[1] * b0 + q[3] * u + q[5] * v;
                float c[4];
                if (X.base_color >= 0) { o_tex(&TX[X.base_color], tu, 1.f - tv, c); Mc.base[0] *= c[0]; Mc.base[1] *= c[1]; Mc.base[2] *= c[2]; }
                if (X.emission >= 0) { o_tex(&TX[X.emission], tu, 1.f - tv, c); Mc.emission[0] *= c[0]; Mc.emission[1] *= c[1]; Mc.emission[2] *= c[2]; }
                if (X.metallic >= 0) { o_tex(&TX[X.metallic], tu, 1.f - tv, c); Mc.metallic *= c[X.metallic_ch]; }
                if (X.roughness >= 0) { o_tex(&TX[X.roughness], tu, 1.f - tv, c); Mc.roughness *= c[X.roughness_ch]; }
                if (X.normal >= 0 && tans) {   /* tangent-space normal: n = T x + B y + N z, B = sign (N x T) */
                    const float* t0 = tans + 12 * (size_t)ti; const float w0 = 1.f - u - v;
                    V3 tg = v3(t0[0] * w0 + t0[4] * u + t0[8] * v, t0[1] * w0 + t0[5] * u + t0[9] * v, t0[2] * w0 + t0[6] * u + t0[10] * v);
                    const float sg = ((t0[3] * w0 + t0[7] * u + t0[11] * v) < 0.f ? -1.f : 1.f) * I[26];
                    const float* F = I + 12;
                    tg = v3(F[0] * tg.x + F[1] * tg.y + F[2] * tg.z, F[4] * tg.x + F[5] * tg.y + F[6] * tg.z, F[8] * tg.x + F[9] * tg.y + F[10] * tg.z);
                    tg = sub(tg, muls(nsw, dot3(nsw, tg)));
                    const float tl = sqrtf(dot3(tg, tg));
                    if (tl > 0.f) {
                        tg = muls(tg, 1.f / tl);
                        const V3 bt = muls(cross3(nsw, tg), sg);
                        o_tex(&TX[X.normal], tu, 1.f - tv, c);
                        const V3 nm = add(add(muls(tg, (2.f * c[0] - 1.f) * X.normal_scale), muls(bt, (2.f * c[1] - 1.f) * X.normal_scale)), muls(nsw, 2.f * c[2] - 1.f));
                        const float nl = sqrtf(dot3(nm, nm));
                        if (nl > 0.f) { nsw = muls(nm, 1.f / nl); mapped = 1; }
                    }
                }
            }
            const V3 p = add(o, muls(d, t));
            if (M->emission[0] > 0.f || M->emission[1] > 0.f || M->emission[2] > 0.f) {   /* MIS against light sampling of this triangle */
                float w = 1.f;
                if (lastPdf > 0.f) {
                    if (R->light_mode == O_LIGHT_NEE) w = 0.f;
                    else if (R->light_mode == O_LIGHT_MIS) {
                        const float cl = fabsf(dot3(ng0, d)), pa = n_em > 0 ? mat_pdf[mid] : 0.f;
                        w = o_mis(lastPdf, cl > 0.f ? pTri * pa * t * t / cl : 0.f);
                    }
                }
                if (w > 0.f) { A[0] += T.x * M->emission[0] * w; A[1] += T.y * M->emission[1] * w; A[2] += T.z * M->emission[2] * w; }
            }
            if (depth > R->max_depth) break;
            if (R->rr && depth >= R->rr_depth) {   /* Russian roulette */
                const float qs = fminf(fmaxf(fmaxf(T.x, fmaxf(T.y, T.z)), 0.05f), 1.f);
                if (orc_rng(pix, smp, (unsigned)depth + 1u, 6, seed) >= qs) break;
                T = muls(T, 1.f / qs);
            }
            const int front = dot3(ng0, d) < 0.f;
            const V3 ng = front ? ng0 : neg(ng0);
            V3 ns = front ? nsw : neg(nsw); const V3 wo = neg(d);
            if (dot3(ns, wo) <= 1e-6f) ns = ng;
            V3 tx, ty; onb(ns, &tx, &ty);
            const V3 woL = v3(dot3(wo, tx), dot3(wo, ty), dot3(wo, ns));
            V3 nrL = v3(0.f, 0.f, 1.f);
            if (R->bump_shadow && mapped) {
                const V3 nsU = front ? nsU0 : neg(nsU0);
                nrL = v3(dot3(nsU, tx), dot3(nsU, ty), dot3(nsU, ns));
                if (!(nrL.z > 0.f)) nrL = v3(0.f, 0.f, 1.f);
            }
            const float eta = front ? M->ior : 1.f / M->ior;
            const V3 up = add(p, muls(ng, R->eps)), dn = sub(p, muls(ng, R->eps));
            const unsigned dr = (unsigned)depth + 1u;
            const float ux1 = orc_rng(pix, smp, dr, 7, seed), ux2 = orc_rng(pix, smp, dr, 7, seed ^ 0x68E31DA4u);
            if (o_non_delta(M)) {
                /* one light sample (render/wavefront.cu:295-344) */
                const float us = orc_rng(pix, smp, dr, 5, seed), u2 = orc_rng(pix, smp, dr, 2, seed), u3 = orc_rng(pix, smp, dr, 3, seed);
                V3 l = v3(0.f, 0.f, 1.f), Le = v3(0.f, 0.f, 0.f); float pl = 0.f, tmax = 1e30f; int ok = 0, isSun = 0, side = 0;
                if (us < pSun) { l = cone_dir(sunTo, R->sun_cos, u2, u3); Le = sunE; pl = pSun; isSun = 1; ok = 1; }
                else if (us < pSun + pTri) {
                    const float ut = fminf((us - pSun) / pTri, 0.99999994f);
                    const int e = o_cdf_find(em_cdf, (int)n_em, ut);
                    const float* a = em_tris + 12 * (size_t)e;
                    const float su = sqrtf(u2);
                    const V3 a1 = v3(a[4], a[5], a[6]), a2 = v3(a[8], a[9], a[10]);
                    const V3 pL = add(add(v3(a[0], a[1], a[2]), muls(a1, su * (1.f - u3))), muls(a2, su * u3));
                    const V3 nL = normz(cross3(a1, a2));
                    side = dot3(ng, sub(pL, p)) > 0.f ? 1 : -1;
                    const V3 dv = sub(pL, side > 0 ? up : dn);
                    const float dist2 = dot3(dv, dv), dist = sqrtf(dist2);
                    if (dist > 0.f) {
                        l = muls(dv, 1.f / dist);
                        const float cl = fabsf(dot3(nL, l));
                        if (cl > 0.f) {
                            const int lm = fi(a[7]);
                            pl = pTri * mat_pdf[lm] * dist2 / cl; Le = v3(MT[lm].emission[0], MT[lm].emission[1], MT[lm].emission[2]); tmax = dist * (1.f - 1e-3f); ok = 1;
                            if (MX && lm < n_mtex && MX[lm].emission >= 0) {
                                const float* q = uvs + 8 * (size_t)fi(a[3]); const float b1 = su * (1.f - u3), b2 = su * u3, b0 = 1.f - b1 - b2;
                                float c[4]; o_tex(&TX[MX[lm].emission], q[0] * b0 + q[2] * b1 + q[4] * b2, 1.f - (q[1] * b0 + q[3] * b1 + q[5] * b2), c);
                                Le = v3(Le.x * c[0], Le.y * c[1], Le.z * c[2]);
                            }
                        }
                    }
                } else if (pEnv > 0.f && R->env_uniform) {
                    const float z = 1.f - 2.f * u2, r = sqrtf(fmaxf(0.f, 1.f - z * z)), ph = 6.2831853f * u3;
                    l = v3(r * cosf(ph), r * sinf(ph), z); pl = pEnv * (0.25f * 0.31830989f);
                    int ex, ey; float ev; o_env_texel(&E, l, &ex, &ey, &ev);
                    const float* t4 = E.tex + 4 * ((size_t)ey * E.w + ex); Le = v3(t4[0], t4[1], t4[2]); ok = 1;
                } else if (pEnv > 0.f) {
                    const float ue = fminf((us - pSun - pTri) / pEnv, 0.99999994f);
                    const int y = o_cdf_find(E.marg, E.h, ue);
                    const float* cr = E.cond + (size_t)y * (E.w + 1);
                    const int x = o_cdf_find(cr, E.w, u2);
                    const float v = (y + u3) / E.h, w0 = cr[x + 1] - cr[x];
                    float u = (x + 0.5f) / E.w;
                    if (w0 > 0.f) u = (x + fminf((u2 - cr[x]) / w0, 0.99999994f)) / E.w;
                    const float ph = (0.5f - u) * 6.2831853f + E.rot, th = v * 3.14159265f, st = sinf(th);
                    l = v3(st * cosf(ph), st * sinf(ph), cosf(th));
                    const float pe = o_env_pdf_texel(&E, x, y, v);
                    if (pe > 0.f) { const float* t4 = E.tex + 4 * ((size_t)y * E.w + x); pl = pEnv * pe; Le = v3(t4[0], t4[1], t4[2]); ok = 1; }
                }
                const V3 lL = v3(dot3(l, tx), dot3(l, ty), dot3(l, ns));
                const float gl = dot3(ng, l);
                if (ok && lL.z != 0.f && (gl > 0.f) == (lL.z > 0.f)) {
                    const OEval e = o_bsdf_eval(M, woL, lL, eta, gd, ux1, ux2, nrL);
                    const float wgt_l = (isSun || R->light_mode == O_LIGHT_NEE) ? 1.f : o_mis(pl, e.pdf);
                    const V3 c = muls(mulv(mulv(T, e.f), Le), fabsf(lL.z) * wgt_l / pl);
                    if (c.x > 0.f || c.y > 0.f || c.z > 0.f) {
                        float st = tmax, su, sv; int sh, shi;
                        const V3 so = (side ? side > 0 : gl > 0.f) ? up : dn;
                        if (o_inst1(width, tlas_width, 1, blas, tris, (const V4*)tlas, root, inst, so, l, 0.f, &st, &sh, &su, &sv, &shi) < 0) bad++;
                        counts[1]++;
                        if (sh < 0) { A[0] += c.x; A[1] += c.y; A[2] += c.z; }
                    }
                }
            }
            V3 wiL, wgt; float pdf;
            if (!o_bsdf_sample(M, woL, eta, gd, ux1, ux2, orc_rng(pix, smp, dr, 4, seed), orc_rng(pix, smp, dr, 0, seed), orc_rng(pix, smp, dr, 1, seed), &wiL, &wgt, &pdf, nrL)) break;
            const V3 wi = normz(add(add(muls(tx, wiL.x), muls(ty, wiL.y)), muls(ns, wiL.z)));
            const float gi = dot3(ng, wi);
            if (gi == 0.f || (gi > 0.f) != (wiL.z > 0.f)) break;
            T = mulv(T, wgt);
            if (!(fmaxf(T.x, fmaxf(T.y, T.z)) > 0.f)) break;
            o = gi > 0.f ? up : dn; d = wi; lastPdf = pdf;
        }
    }
    return bad;
}
