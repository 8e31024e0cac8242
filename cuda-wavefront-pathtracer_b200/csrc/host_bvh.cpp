// host_bvh.cpp - parallel binned-SAH builder, BVH2/BVH4/CWBVH encodings, triangle packing.
#include "host_bvh.h"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <future>
#include <thread>

namespace cwpb {

// ======================= binned SAH =======================
namespace {

struct SahRun {
    const SahOptions& o;
    int threads;
    std::vector<Box3> tb; std::vector<float3> cent; std::vector<int> idx;
    struct Part { std::vector<BNode> nodes; int maxDepth = 0; };

    static constexpr int kParGrain = 1 << 15;    // nodes with at least this many triangles bin on several threads
    static constexpr int kTaskGrain = 1 << 12;   // subtrees with at least this many triangles may run as tasks

    explicit SahRun(const SahOptions& op) : o(op) {
        threads = op.threads > 0 ? op.threads : (int)std::max(1u, std::thread::hardware_concurrency());
    }

    template <class F> void par_for(int begin, int end, int parts, F fn) {
        std::vector<std::thread> ts; int n = end - begin;
        for (int p = 1; p < parts; p++) ts.emplace_back(fn, p, begin + (int)((long)n * p / parts), begin + (int)((long)n * (p + 1) / parts));
        fn(0, begin, begin + (int)((long)n / parts));
        for (auto& t : ts) t.join();
    }

    void bounds(int begin, int end, Box3& box, Box3& cb) {
        int parts = (end - begin >= kParGrain && threads > 1) ? threads : 1;
        std::vector<Box3> pb(parts), pc(parts);
        par_for(begin, end, parts, [&](int p, int b, int e) {
            Box3 x, y; for (int i = b; i < e; i++) { x.grow(tb[idx[i]]); y.grow(cent[idx[i]]); } pb[p] = x; pc[p] = y; });
        for (int p = 0; p < parts; p++) { box.grow(pb[p]); cb.grow(pc[p]); }
    }

    static float comp(float3 v, int a) { return a == 0 ? v.x : a == 1 ? v.y : v.z; }

    // best (axis, bin) by the binned SAH, or axis -1 when every axis of the centroid box is degenerate
    void best_split(int begin, int end, const Box3& cb, int& bestAxis, int& bestBin) {
        const int NB = o.bins;
        float bestCost = FLT_MAX; bestAxis = -1; bestBin = -1;
        float3 ext = cb.extent();
        int parts = (end - begin >= kParGrain && threads > 1) ? threads : 1;
        std::vector<Box3> bb((size_t)parts * 3 * NB); std::vector<int> bc((size_t)parts * 3 * NB, 0);
        par_for(begin, end, parts, [&](int p, int b, int e) {
            for (int axis = 0; axis < 3; axis++) {
                float lo = comp(cb.lo, axis), ex = comp(ext, axis);
                if (ex <= 1e-12f) continue;
                float scale = NB / ex;
                Box3* B = &bb[((size_t)p * 3 + axis) * NB]; int* C = &bc[((size_t)p * 3 + axis) * NB];
                for (int i = b; i < e; i++) {
                    int k = (int)((comp(cent[idx[i]], axis) - lo) * scale); k = k < 0 ? 0 : k > NB - 1 ? NB - 1 : k;
                    B[k].grow(tb[idx[i]]); C[k]++;
                }
            }
        });
        std::vector<Box3> binBox(NB); std::vector<int> binCnt(NB); std::vector<float> rA(NB); std::vector<int> rC(NB);
        for (int axis = 0; axis < 3; axis++) {
            if (comp(ext, axis) <= 1e-12f) continue;
            for (int k = 0; k < NB; k++) {
                Box3 x; int c = 0;
                for (int p = 0; p < parts; p++) { x.grow(bb[((size_t)p * 3 + axis) * NB + k]); c += bc[((size_t)p * 3 + axis) * NB + k]; }
                binBox[k] = x; binCnt[k] = c;
            }
            // sweep from the right: area and count of bins (k, NB)
            Box3 acc; int cnt = 0;
            for (int k = NB - 1; k > 0; k--) { acc.grow(binBox[k]); cnt += binCnt[k]; rA[k] = acc.area(); rC[k] = cnt; }
            // sweep from the left; split after bin k
            Box3 lacc; int lcnt = 0;
            for (int k = 0; k < NB - 1; k++) {
                lacc.grow(binBox[k]); lcnt += binCnt[k];
                if (lcnt == 0 || rC[k + 1] == 0) continue;
                float cost = lacc.area() * lcnt + rA[k + 1] * rC[k + 1];
                if (cost < bestCost) { bestCost = cost; bestAxis = axis; bestBin = k; }
            }
        }
    }

    int node(int begin, int end, int depth, Part& P, int spawn) {
        int id = (int)P.nodes.size(); P.nodes.emplace_back();
        P.maxDepth = std::max(P.maxDepth, depth);
        Box3 box, cb; bounds(begin, end, box, cb);
        P.nodes[id].box = box;
        const int n = end - begin;
        if (n <= o.leafMax || depth >= o.depthCap) { P.nodes[id].first = begin; P.nodes[id].count = n; return id; }
        int axis, bin; best_split(begin, end, cb, axis, bin);
        int mid;
        if (axis < 0) mid = (begin + end) / 2;   // coincident centroids: median of the current order
        else {
            float lo = comp(cb.lo, axis), scale = o.bins / comp(cb.extent(), axis); const int NB = o.bins;
            int* p = std::partition(idx.data() + begin, idx.data() + end, [&](int t) {
                int k = (int)((comp(cent[t], axis) - lo) * scale); k = k < 0 ? 0 : k > NB - 1 ? NB - 1 : k; return k <= bin; });
            mid = (int)(p - idx.data());
            if (mid == begin || mid == end) mid = (begin + end) / 2;
        }
        if (spawn > 0 && n >= kTaskGrain) {
            Part L, R;
            auto right = std::async(std::launch::async, [&] { node(mid, end, depth + 1, R, spawn - 1); });
            node(begin, mid, depth + 1, L, spawn - 1);
            right.get();
            int lb = splice(P, L), rb = splice(P, R);
            P.nodes[id].left = lb; P.nodes[id].right = rb;
        } else {
            int l = node(begin, mid, depth + 1, P, 0);
            int r = node(mid, end, depth + 1, P, 0);
            P.nodes[id].left = l; P.nodes[id].right = r;
        }
        return id;
    }

    static int splice(Part& P, const Part& S) {
        int base = (int)P.nodes.size();
        for (BNode b : S.nodes) { if (!b.leaf() && b.left >= 0) { b.left += base; b.right += base; } P.nodes.push_back(b); }
        P.maxDepth = std::max(P.maxDepth, S.maxDepth);
        return base;
    }
};

}  // namespace

void build_sah(const Mesh& m, const SahOptions& o, BinaryBvh& out) {
    SahRun R(o);
    const size_t n = m.nt();
    R.tb.resize(n); R.cent.resize(n); R.idx.resize(n);
    for (size_t i = 0; i < n; i++) {
        Box3 b; b.grow(m.vert(m.f[3 * i])); b.grow(m.vert(m.f[3 * i + 1])); b.grow(m.vert(m.f[3 * i + 2]));
        R.tb[i] = b; R.cent[i] = (b.lo + b.hi) * 0.5f; R.idx[i] = (int)i;
    }
    int spawn = 0; while ((1 << spawn) < R.threads * 4 && spawn < 12) spawn++;
    if (R.threads <= 1) spawn = 0;
    SahRun::Part P; P.nodes.reserve(2 * n / std::max(1, o.leafMax) + 16);
    R.node(0, (int)n, 0, P, spawn);
    out.nodes.swap(P.nodes); out.prim.swap(R.idx); out.maxDepth = P.maxDepth; out.leafMax = o.leafMax;
}

// ======================= spatial splits =======================
// Binned SAH with spatial splits (Stich, Friedrich & Dietrich, "Spatial Splits in Bounding Volume Hierarchies",
// HPG 2009): a node whose best object split leaves children overlapping by more than alpha of the root's area also
// tries splitting space at bin planes, clipping the triangles that straddle a plane into both children; the cheaper
// split by the SAH wins. Leaves then reference triangles (a triangle may appear in several leaves); a spatial split
// may duplicate at most `budget` x the node's references (a local rule, so the tree does not depend on the order in
// which subtrees are built).
namespace {
struct SRef { int tri; Box3 box; };
struct SbvhRun {
    const Mesh& m; const SahOptions& o; float alphaArea = 0.f, budget = 0.f;
    struct Part { std::vector<BNode> nodes; std::vector<int> prim; int maxDepth = 0; };
    SbvhRun(const Mesh& mm, const SahOptions& oo) : m(mm), o(oo) {}
    static float comp(float3 v, int a) { return a == 0 ? v.x : a == 1 ? v.y : v.z; }
    static void setc(float3& v, int a, float x) { if (a == 0) v.x = x; else if (a == 1) v.y = x; else v.z = x; }
    static bool empty(const Box3& b) { return !(b.lo.x <= b.hi.x && b.lo.y <= b.hi.y && b.lo.z <= b.hi.z); }

    // box of the part of triangle t with lo <= p[axis] <= hi, within `within`
    Box3 chop(int t, int axis, float lo, float hi, const Box3& within) const {
        const float3 v[3] = { m.vert(m.f[3 * t]), m.vert(m.f[3 * t + 1]), m.vert(m.f[3 * t + 2]) };
        Box3 r;
        for (int i = 0; i < 3; i++) {
            const float3 a = v[i], c = v[(i + 1) % 3];
            const float pa = comp(a, axis), pc = comp(c, axis);
            if (pa >= lo && pa <= hi) r.grow(a);
            for (int q = 0; q < 2; q++) {
                const float plane = q ? hi : lo;
                if ((pa < plane && pc > plane) || (pa > plane && pc < plane)) {
                    const float s = (plane - pa) / (pc - pa);
                    float3 x = f3(a.x + (c.x - a.x) * s, a.y + (c.y - a.y) * s, a.z + (c.z - a.z) * s); setc(x, axis, plane);
                    r.grow(x);
                }
            }
        }
        r.lo = vmax(r.lo, within.lo); r.hi = vmin(r.hi, within.hi);
        return r;
    }

    int node(std::vector<SRef>& refs, int depth, Part& P, int spawn) {
        const int id = (int)P.nodes.size(); P.nodes.emplace_back();
        P.maxDepth = std::max(P.maxDepth, depth);
        Box3 box, cb;
        for (const SRef& r : refs) { box.grow(r.box); cb.grow((r.box.lo + r.box.hi) * 0.5f); }
        P.nodes[id].box = box;
        const int n = (int)refs.size();
        if (n <= o.leafMax || depth >= o.depthCap) {
            P.nodes[id].first = (int)P.prim.size(); P.nodes[id].count = n;
            for (const SRef& r : refs) P.prim.push_back(r.tri);
            return id;
        }
        const int NB = o.bins;
        // object split over the reference centroids
        float objCost = FLT_MAX; int objAxis = -1, objBin = -1; Box3 objL, objR;
        {
            const float3 ext = cb.extent();
            std::vector<Box3> bb(NB); std::vector<int> bc(NB); std::vector<Box3> rB(NB); std::vector<int> rC(NB);
            for (int axis = 0; axis < 3; axis++) {
                const float lo = comp(cb.lo, axis), ex = comp(ext, axis);
                if (ex <= 1e-12f) continue;
                const float scale = NB / ex;
                std::fill(bb.begin(), bb.end(), Box3()); std::fill(bc.begin(), bc.end(), 0);
                for (const SRef& r : refs) { int k = (int)((comp((r.box.lo + r.box.hi) * 0.5f, axis) - lo) * scale); k = k < 0 ? 0 : k > NB - 1 ? NB - 1 : k; bb[k].grow(r.box); bc[k]++; }
                Box3 acc; int cnt = 0;
                for (int k = NB - 1; k > 0; k--) { acc.grow(bb[k]); cnt += bc[k]; rB[k] = acc; rC[k] = cnt; }
                Box3 la; int lc = 0;
                for (int k = 0; k < NB - 1; k++) {
                    la.grow(bb[k]); lc += bc[k];
                    if (lc == 0 || rC[k + 1] == 0) continue;
                    const float c = la.area() * lc + rB[k + 1].area() * rC[k + 1];
                    if (c < objCost) { objCost = c; objAxis = axis; objBin = k; objL = la; objR = rB[k + 1]; }
                }
            }
        }
        // spatial split, when the object split's children overlap enough and the reference budget allows
        float spCost = FLT_MAX; int spAxis = -1; float spPos = 0.f;
        if (objAxis >= 0) {
            Box3 ov; ov.lo = vmax(objL.lo, objR.lo); ov.hi = vmin(objL.hi, objR.hi);
            if (!empty(ov) && ov.area() > alphaArea) {
                std::vector<Box3> bb(NB); std::vector<int> enter(NB), leave(NB); std::vector<Box3> rB(NB); std::vector<int> rC(NB);
                for (int axis = 0; axis < 3; axis++) {
                    const float lo = comp(box.lo, axis), ex = comp(box.extent(), axis);
                    if (ex <= 1e-12f) continue;
                    const float w = ex / NB;
                    std::fill(bb.begin(), bb.end(), Box3()); std::fill(enter.begin(), enter.end(), 0); std::fill(leave.begin(), leave.end(), 0);
                    for (const SRef& r : refs) {
                        int b0 = (int)((comp(r.box.lo, axis) - lo) / w), b1 = (int)((comp(r.box.hi, axis) - lo) / w);
                        b0 = std::min(std::max(b0, 0), NB - 1); b1 = std::min(std::max(b1, b0), NB - 1);
                        if (b0 == b1) bb[b0].grow(r.box);
                        else for (int k = b0; k <= b1; k++) {
                            const Box3 c = chop(r.tri, axis, k == b0 ? -FLT_MAX : lo + k * w, k == b1 ? FLT_MAX : lo + (k + 1) * w, r.box);
                            if (!empty(c)) bb[k].grow(c);
                        }
                        enter[b0]++; leave[b1]++;
                    }
                    Box3 acc; int cnt = 0;
                    for (int k = NB - 1; k > 0; k--) { acc.grow(bb[k]); cnt += leave[k]; rB[k] = acc; rC[k] = cnt; }
                    Box3 la; int lc = 0;
                    for (int k = 0; k < NB - 1; k++) {
                        la.grow(bb[k]); lc += enter[k];
                        if (lc == 0 || rC[k + 1] == 0 || lc + rC[k + 1] > n + budget * n) continue;
                        const float c = la.area() * lc + rB[k + 1].area() * rC[k + 1];
                        if (c < spCost) { spCost = c; spAxis = axis; spPos = lo + (k + 1) * w; }
                    }
                }
            }
        }
        std::vector<SRef> L, R;
        if (spAxis >= 0 && spCost < objCost) {
            for (const SRef& r : refs) {
                if (comp(r.box.hi, spAxis) <= spPos) L.push_back(r);
                else if (comp(r.box.lo, spAxis) >= spPos) R.push_back(r);
                else {
                    const Box3 a = chop(r.tri, spAxis, -FLT_MAX, spPos, r.box), b = chop(r.tri, spAxis, spPos, FLT_MAX, r.box);
                    const bool ea = empty(a), eb = empty(b);
                    if (!ea) L.push_back({ r.tri, a });
                    if (!eb) R.push_back({ r.tri, b });
                    if (ea && eb) L.push_back(r);
                }
            }
            if (L.empty() || R.empty()) { L.clear(); R.clear(); spAxis = -1; }
        }
        if (L.empty() && R.empty()) {
            if (objAxis < 0) {   // coincident centroids: halves of the current order
                L.assign(refs.begin(), refs.begin() + n / 2); R.assign(refs.begin() + n / 2, refs.end());
            } else {
                const float lo = comp(cb.lo, objAxis), scale = NB / comp(cb.extent(), objAxis);
                for (const SRef& r : refs) {
                    int k = (int)((comp((r.box.lo + r.box.hi) * 0.5f, objAxis) - lo) * scale); k = k < 0 ? 0 : k > NB - 1 ? NB - 1 : k;
                    (k <= objBin ? L : R).push_back(r);
                }
                if (L.empty() || R.empty()) { L.assign(refs.begin(), refs.begin() + n / 2); R.assign(refs.begin() + n / 2, refs.end()); }
            }
        }
        std::vector<SRef>().swap(refs);
        if (spawn > 0 && n >= (1 << 12)) {
            Part PL, PR;
            auto right = std::async(std::launch::async, [&] { node(R, depth + 1, PR, spawn - 1); });
            node(L, depth + 1, PL, spawn - 1);
            right.get();
            const int lb = splice(P, PL), rb = splice(P, PR);
            P.nodes[id].left = lb; P.nodes[id].right = rb;
        } else {
            const int l = node(L, depth + 1, P, 0);
            const int r = node(R, depth + 1, P, 0);
            P.nodes[id].left = l; P.nodes[id].right = r;
        }
        return id;
    }
    static int splice(Part& P, const Part& S) {
        const int base = (int)P.nodes.size(), pbase = (int)P.prim.size();
        for (BNode b : S.nodes) { if (b.leaf()) b.first += pbase; else if (b.left >= 0) { b.left += base; b.right += base; } P.nodes.push_back(b); }
        P.prim.insert(P.prim.end(), S.prim.begin(), S.prim.end());
        P.maxDepth = std::max(P.maxDepth, S.maxDepth);
        return base;
    }
};
}  // namespace

void build_sbvh(const Mesh& m, const SahOptions& o, float alpha, float budget, BinaryBvh& out) {
    SbvhRun R(m, o);
    const size_t n = m.nt();
    std::vector<SRef> refs(n);
    Box3 root;
    for (size_t i = 0; i < n; i++) {
        Box3 b; b.grow(m.vert(m.f[3 * i])); b.grow(m.vert(m.f[3 * i + 1])); b.grow(m.vert(m.f[3 * i + 2]));
        refs[i] = { (int)i, b }; root.grow(b);
    }
    R.alphaArea = alpha * root.area(); R.budget = budget;
    const int threads = o.threads > 0 ? o.threads : (int)std::max(1u, std::thread::hardware_concurrency());
    int spawn = 0; while ((1 << spawn) < threads * 4 && spawn < 12) spawn++;
    if (threads <= 1) spawn = 0;
    SbvhRun::Part P;
    R.node(refs, 0, P, spawn);
    out.nodes.swap(P.nodes); out.prim.swap(P.prim); out.maxDepth = P.maxDepth; out.leafMax = o.leafMax;
}

// Binary tree of a one-mesh H-PLOC build (2n - 1 nodes of 2 float4: (lo, left), (hi, right); leaves [0, n) hold one
// primitive in `left`; children have smaller ids than their parent; root 2n - 2) with its leaves collapsed where that
// lowers the SAH cost: a subtree of at most leafMax triangles becomes one leaf when A x count <= A + cost(left) +
// cost(right), leaf cost = area x triangles, inner cost = area + the children's (the dynamic programme of the
// reference's treeFromHploc, accel/bvh_tools.cpp:12-38). The result is numbered in pre-order, left subtree first.
void tree_from_hploc(const std::vector<float4>& hn, int64_t n, int leafMax, BinaryBvh& out) {
    const int64_t tot = 2 * n - 1;
    std::vector<int> L((size_t)tot), R((size_t)tot), cnt((size_t)tot);
    std::vector<double> cost((size_t)tot); std::vector<char> asLeaf((size_t)tot); std::vector<Box3> box((size_t)tot);
    for (int64_t h = 0; h < tot; h++) {   // ids increase from children to parents: one pass visits children first
        box[h].lo = xyz(hn[2 * h]); box[h].hi = xyz(hn[2 * h + 1]);
        L[h] = bits_i(hn[2 * h].w); R[h] = bits_i(hn[2 * h + 1].w);
        const double A = box[h].area();
        if (h < n) { cnt[h] = 1; cost[h] = A; asLeaf[h] = 1; continue; }
        cnt[h] = cnt[L[h]] + cnt[R[h]];
        const double inner = A + cost[L[h]] + cost[R[h]], leaf = cnt[h] <= leafMax ? A * cnt[h] : 1e300;
        asLeaf[h] = leaf <= inner;
        cost[h] = leaf <= inner ? leaf : inner;
    }
    out = BinaryBvh(); out.leafMax = leafMax;
    out.nodes.reserve((size_t)tot); out.prim.reserve((size_t)n);
    struct Item { int64_t h; int parent; bool right; int depth; };
    std::vector<Item> todo{ { tot - 1, -1, false, 0 } };
    std::vector<int64_t> gather;
    while (!todo.empty()) {
        const Item it = todo.back(); todo.pop_back();
        const int id = (int)out.nodes.size();
        out.nodes.push_back(BNode()); out.nodes[id].box = box[it.h];
        if (it.parent >= 0) (it.right ? out.nodes[it.parent].right : out.nodes[it.parent].left) = id;
        out.maxDepth = std::max(out.maxDepth, it.depth);
        if (asLeaf[it.h]) {   // the subtree's primitives, left to right
            out.nodes[id].first = (int)out.prim.size();
            gather.assign(1, it.h);
            while (!gather.empty()) {
                const int64_t g = gather.back(); gather.pop_back();
                if (g < n) out.prim.push_back(L[g]); else { gather.push_back(R[g]); gather.push_back(L[g]); }
            }
            out.nodes[id].count = (int)out.prim.size() - out.nodes[id].first;
        } else {
            todo.push_back({ R[it.h], id, true, it.depth + 1 });
            todo.push_back({ L[it.h], id, false, it.depth + 1 });
        }
    }
}

double sah_cost(const BinaryBvh& B, double cNode, double cPrim) {
    double s = 0, a0 = B.nodes[0].box.area();
    if (!(a0 > 0)) return 0;
    for (const BNode& n : B.nodes) s += n.leaf() ? n.box.area() * n.count * cPrim : n.box.area() * cNode;
    return s / a0;
}

// ======================= BVH2 / BVH4 =======================
namespace {
inline float fbits(int i) { return bits_f(i); }
inline int ibits(float f) { return bits_i(f); }

void wrap_leaf_root(BinaryBvh& B) {   // a root leaf becomes the single child of a new internal root
    BNode r; r.box = B.nodes[0].box; r.left = 0; r.right = -1;
    B.nodes.push_back(r);
}

int emit2(const BinaryBvh& B, int bn, std::vector<float4>& out) {
    const BNode& nd = B.nodes[bn];
    int id = (int)(out.size() / 4); out.resize(out.size() + 4);
    int ch[2] = { nd.left, nd.right }, c[2], k[2]; Box3 bx[2];
    for (int j = 0; j < 2; j++) {
        if (ch[j] < 0) { c[j] = -1; k[j] = 0; bx[j].lo = bx[j].hi = f3(kEmptyBox, kEmptyBox, kEmptyBox); continue; }
        const BNode& cn = B.nodes[ch[j]]; bx[j] = cn.box;
        if (cn.leaf()) { c[j] = cn.first; k[j] = cn.count; } else { k[j] = 0; c[j] = emit2(B, ch[j], out); }
    }
    float4* n = &out[(size_t)id * 4];
    n[0] = make_float4(bx[0].lo.x, bx[0].hi.x, bx[0].lo.y, bx[0].hi.y);
    n[1] = make_float4(bx[1].lo.x, bx[1].hi.x, bx[1].lo.y, bx[1].hi.y);
    n[2] = make_float4(bx[0].lo.z, bx[0].hi.z, bx[1].lo.z, bx[1].hi.z);
    n[3] = make_float4(fbits(c[0]), fbits(c[1]), fbits(k[0]), fbits(k[1]));
    return id;
}

int emit4(const BinaryBvh& B, int bn, std::vector<float4>& out) {
    const std::vector<BNode>& N = B.nodes;
    int id = (int)(out.size() / 8); out.resize(out.size() + 8);
    std::vector<int> ch = { N[bn].left, N[bn].right };
    while (ch.size() < 4) {   // open the largest-area internal child
        int best = -1; float bestA = -1;
        for (size_t j = 0; j < ch.size(); j++) if (ch[j] >= 0 && !N[ch[j]].leaf()) { float a = N[ch[j]].box.area(); if (a > bestA) { bestA = a; best = (int)j; } }
        if (best < 0) break;
        int nb = ch[best]; ch[best] = N[nb].left; ch.push_back(N[nb].right);
    }
    int c[4], k[4]; Box3 bx[4];
    for (int j = 0; j < 4; j++) {
        if (j >= (int)ch.size() || ch[j] < 0) { c[j] = -1; k[j] = 0; bx[j].lo = bx[j].hi = f3(kEmptyBox, kEmptyBox, kEmptyBox); continue; }
        const BNode& cn = N[ch[j]]; bx[j] = cn.box;
        if (cn.leaf()) { c[j] = cn.first; k[j] = cn.count; } else { k[j] = 0; c[j] = emit4(B, ch[j], out); }
    }
    float4* n = &out[(size_t)id * 8];
    n[0] = make_float4(bx[0].lo.x, bx[1].lo.x, bx[2].lo.x, bx[3].lo.x);
    n[1] = make_float4(bx[0].hi.x, bx[1].hi.x, bx[2].hi.x, bx[3].hi.x);
    n[2] = make_float4(bx[0].lo.y, bx[1].lo.y, bx[2].lo.y, bx[3].lo.y);
    n[3] = make_float4(bx[0].hi.y, bx[1].hi.y, bx[2].hi.y, bx[3].hi.y);
    n[4] = make_float4(bx[0].lo.z, bx[1].lo.z, bx[2].lo.z, bx[3].lo.z);
    n[5] = make_float4(bx[0].hi.z, bx[1].hi.z, bx[2].hi.z, bx[3].hi.z);
    n[6] = make_float4(fbits(c[0]), fbits(c[1]), fbits(c[2]), fbits(c[3]));
    n[7] = make_float4(fbits(k[0]), fbits(k[1]), fbits(k[2]), fbits(k[3]));
    return id;
}
}  // namespace

void layout_bvh2(BinaryBvh& B, std::vector<float4>& nodes) {
    nodes.clear();
    if (B.nodes[0].leaf()) { wrap_leaf_root(B); emit2(B, (int)B.nodes.size() - 1, nodes); }
    else emit2(B, 0, nodes);
}
void layout_bvh4(BinaryBvh& B, std::vector<float4>& nodes) {
    nodes.clear();
    if (B.nodes[0].leaf()) { wrap_leaf_root(B); emit4(B, (int)B.nodes.size() - 1, nodes); }
    else emit4(B, 0, nodes);
}

// ======================= 8-wide quantised nodes =======================
namespace {
// smallest power-of-two exponent e with lo + 255 * 2^e >= hi (-100 for a flat axis); bvh_tools.cpp:58-63
int quant_exponent(float ext, float lo, float hi) {
    if (!(ext > 0.f)) return -100;
    int e = (int)ceilf(log2f(ext / 255.f)); if (e < -100) e = -100;
    while (lo + 255.f * ldexpf(1.f, e) < hi) e++;
    return e;
}
int quant(float v, float origin, float scale, bool up) {
    float f = (v - origin) / scale; int i = up ? (int)ceilf(f) : (int)floorf(f);
    return i < 0 ? 0 : i > 255 ? 255 : i;
}
unsigned pack_bytes(const int* q, int b) { return (unsigned)q[b] | ((unsigned)q[b + 1] << 8) | ((unsigned)q[b + 2] << 16) | ((unsigned)q[b + 3] << 24); }

// writes one 80 B node: box = node bounds, childBox[s] = child bounds of slot s (valid where meta[s] != 0)
void write_wide_node(float4* o, const Box3& box, const Box3* childBox, const int* meta, unsigned imask, int childBase, int triBase) {
    float3 ext = box.extent();
    int ex = quant_exponent(ext.x, box.lo.x, box.hi.x), ey = quant_exponent(ext.y, box.lo.y, box.hi.y), ez = quant_exponent(ext.z, box.lo.z, box.hi.z);
    float sx = ldexpf(1.f, ex), sy = ldexpf(1.f, ey), sz = ldexpf(1.f, ez);
    int q[6][8];
    for (int s = 0; s < 8; s++) {
        if (!meta[s]) { for (int a = 0; a < 6; a++) q[a][s] = 0; continue; }
        const Box3& cb = childBox[s];
        q[0][s] = quant(cb.lo.x, box.lo.x, sx, false); q[3][s] = quant(cb.hi.x, box.lo.x, sx, true);
        q[1][s] = quant(cb.lo.y, box.lo.y, sy, false); q[4][s] = quant(cb.hi.y, box.lo.y, sy, true);
        q[2][s] = quant(cb.lo.z, box.lo.z, sz, false); q[5][s] = quant(cb.hi.z, box.lo.z, sz, true);
    }
    unsigned ew = (unsigned)(ex + 127) | ((unsigned)(ey + 127) << 8) | ((unsigned)(ez + 127) << 16) | (imask << 24);
    o[0] = make_float4(box.lo.x, box.lo.y, box.lo.z, fbits((int)ew));
    o[1] = make_float4(fbits(childBase), fbits(triBase), fbits((int)pack_bytes(meta, 0)), fbits((int)pack_bytes(meta, 4)));
    unsigned u[12];
    for (int a = 0; a < 6; a++) { u[2 * a] = pack_bytes(q[a], 0); u[2 * a + 1] = pack_bytes(q[a], 4); }
    for (int j = 0; j < 3; j++) o[2 + j] = make_float4(fbits((int)u[4 * j]), fbits((int)u[4 * j + 1]), fbits((int)u[4 * j + 2]), fbits((int)u[4 * j + 3]));
}

// ---- SAH collapse working tree and dynamic programme ----
struct Collapse {
    std::vector<Box3> box; std::vector<int> L, R, first, cnt, p;   // binary tree; leaves have L = R = -1
    std::vector<float> C; std::vector<unsigned char> D, K8;       // C[n*8+i]: best cost of n as i wide-tree roots
    const std::vector<int>* prim = nullptr;
    enum : unsigned char { kLeaf = 0, kNode = 1, kPrev = 2, kDist = 10 };

    bool is_leaf(int n) const { return L[n] < 0 || D[(size_t)n * 8 + 1] == kLeaf; }
    // the i subtrees that stand for node n when it is expanded into i roots
    void roots(int n, int i, std::vector<int>& out) const {
        for (;;) {
            if (i == 1) { out.push_back(n); return; }
            unsigned char d = D[(size_t)n * 8 + i];
            if (d == kPrev) { i--; continue; }
            int k = d - kDist; roots(L[n], k, out); roots(R[n], i - k, out); return;
        }
    }
    void leaf_prims(int n, std::vector<int>& out) const {
        std::vector<int> st(1, n);
        while (!st.empty()) {
            int h = st.back(); st.pop_back();
            if (L[h] < 0) { for (int t = 0; t < cnt[h]; t++) out.push_back((*prim)[first[h] + t]); }
            else { st.push_back(R[h]); st.push_back(L[h]); }
        }
    }
};
}  // namespace

void collapse_cwbvh(const BinaryBvh& B, WideBvh& out) {
    const int pMax = 3; const float cNode = 1.f, cPrim = 0.3f, INF = 3e38f;
    Collapse w; w.prim = &B.prim;
    const size_t N0 = B.nodes.size();
    w.box.resize(N0); w.L.resize(N0); w.R.resize(N0); w.first.resize(N0); w.cnt.resize(N0);
    for (size_t i = 0; i < N0; i++) {
        const BNode& b = B.nodes[i]; bool lf = b.leaf();
        w.box[i] = b.box; w.L[i] = lf ? -1 : b.left; w.R[i] = lf ? -1 : b.right; w.first[i] = b.first; w.cnt[i] = lf ? b.count : 0;
    }
    // leaves above pMax triangles are split into halves with the parent's box (new nodes are appended, and split again
    // if still too large)
    for (size_t i = 0; i < w.box.size(); i++) {
        if (w.L[i] >= 0 || w.cnt[i] <= pMax) continue;
        int h = w.cnt[i] / 2, a = (int)w.box.size();
        Box3 bx = w.box[i];
        w.box.push_back(bx); w.box.push_back(bx);
        w.L.push_back(-1); w.L.push_back(-1); w.R.push_back(-1); w.R.push_back(-1);
        w.first.push_back(w.first[i]); w.cnt.push_back(h); w.first.push_back(w.first[i] + h); w.cnt.push_back(w.cnt[i] - h);
        w.L[i] = a; w.R[i] = a + 1; w.cnt[i] = 0;
    }
    const size_t N = w.box.size();
    w.C.assign(N * 8, 0.f); w.D.assign(N * 8, 0); w.K8.assign(N, 1); w.p.assign(N, 0);
    for (size_t ii = N; ii-- > 0;) {   // children have larger ids than parents: decreasing id is a post-order
        const int n = (int)ii; const float A = w.box[n].area();
        float* c = &w.C[(size_t)n * 8]; unsigned char* d = &w.D[(size_t)n * 8];
        if (w.L[n] < 0) {
            w.p[n] = w.cnt[n]; float cl = A * w.p[n] * cPrim;
            for (int i = 1; i < 8; i++) { c[i] = cl; d[i] = i == 1 ? Collapse::kLeaf : Collapse::kPrev; }
            continue;
        }
        const int l = w.L[n], r = w.R[n]; w.p[n] = w.p[l] + w.p[r];
        const float* cl = &w.C[(size_t)l * 8]; const float* cr = &w.C[(size_t)r * 8];
        float dist[9]; int dk[9];
        for (int j = 2; j <= 8; j++) {
            dist[j] = INF; dk[j] = 1;
            for (int k = 1; k < j; k++) { float v = cl[k] + cr[j - k]; if (v < dist[j]) { dist[j] = v; dk[j] = k; } }
        }
        float cLeaf = w.p[n] <= pMax ? A * w.p[n] * cPrim : INF, cInt = dist[8] + A * cNode;
        if (cLeaf <= cInt) { c[1] = cLeaf; d[1] = Collapse::kLeaf; } else { c[1] = cInt; d[1] = Collapse::kNode; }
        w.K8[n] = (unsigned char)dk[8];
        for (int i = 2; i < 8; i++) {
            if (dist[i] < c[i - 1]) { c[i] = dist[i]; d[i] = (unsigned char)(Collapse::kDist + dk[i]); }
            else { c[i] = c[i - 1]; d[i] = Collapse::kPrev; }
        }
    }
    out.nodes.clear(); out.order.clear(); out.order.reserve(B.prim.size()); out.maxLeafTris = 0;
    const int root = 0; const float Ar = w.box[root].area();
    const bool rootLeaf = w.is_leaf(root);
    if (rootLeaf) out.sah = Ar > 0 ? (Ar * w.p[root] * cPrim + Ar * cNode) / Ar : 0;
    else {
        float d8 = INF; int l = w.L[root], r = w.R[root];
        for (int k = 1; k < 8; k++) d8 = std::min(d8, w.C[(size_t)l * 8 + k] + w.C[(size_t)r * 8 + 8 - k]);
        out.sah = Ar > 0 ? (d8 + Ar * cNode) / Ar : 0;
    }
    struct Job { int bn, slot; bool asLeaf; };
    std::vector<Job> jobs{ { root, 0, rootLeaf } };
    out.nodes.resize(5);
    std::vector<int> ch, pr;
    while (!jobs.empty()) {
        const Job jb = jobs.back(); jobs.pop_back();
        const int n = jb.bn;
        ch.clear();
        if (jb.asLeaf) ch.push_back(n); else { w.roots(w.L[n], w.K8[n], ch); w.roots(w.R[n], 8 - w.K8[n], ch); }
        const Box3 box = w.box[n]; const float3 pc = (box.lo + box.hi) * 0.5f;
        // greedy slot assignment: repeatedly take the (child, free slot) pair with the lowest cost, where slot s
        // costs -dot(child centre - node centre, octant direction of s) (bit set = negative axis)
        int slotChild[8]; for (int s = 0; s < 8; s++) slotChild[s] = -1;
        float cost[8][8]; bool used[8] = { false };
        for (size_t c = 0; c < ch.size(); c++) {
            float3 cc = (w.box[ch[c]].lo + w.box[ch[c]].hi) * 0.5f - pc;
            for (int s = 0; s < 8; s++) cost[c][s] = -(cc.x * (s & 1 ? -1.f : 1.f) + cc.y * (s & 2 ? -1.f : 1.f) + cc.z * (s & 4 ? -1.f : 1.f));
        }
        for (size_t it = 0; it < ch.size(); it++) {
            float bc = INF; int bi = -1, bs = -1;
            for (size_t c = 0; c < ch.size(); c++) if (!used[c]) for (int s = 0; s < 8; s++) if (slotChild[s] < 0 && cost[c][s] < bc) { bc = cost[c][s]; bi = (int)c; bs = s; }
            if (bi < 0) for (size_t c = 0; c < ch.size() && bi < 0; c++) if (!used[c]) for (int s = 0; s < 8; s++) if (slotChild[s] < 0) { bi = (int)c; bs = s; break; }
            used[bi] = true; slotChild[bs] = ch[bi];
        }
        int meta[8] = { 0 }; Box3 cbx[8]; bool childLeaf[8] = { false };
        const int triBase = (int)out.order.size(); unsigned imask = 0; int nInt = 0;
        for (int s = 0; s < 8; s++) {
            int cn = slotChild[s]; if (cn < 0) continue;
            cbx[s] = w.box[cn];
            if (jb.asLeaf || w.is_leaf(cn)) {
                pr.clear(); w.leaf_prims(cn, pr);
                int off = (int)out.order.size() - triBase, cnt = (int)pr.size();
                out.order.insert(out.order.end(), pr.begin(), pr.end());
                meta[s] = 0x80 | ((cnt - 1) << 5) | off;
                out.maxLeafTris = std::max(out.maxLeafTris, cnt);
                childLeaf[s] = true;
            } else { meta[s] = 0x40; imask |= 1u << s; nInt++; }
        }
        const int childBase = (int)(out.nodes.size() / 5);
        out.nodes.resize(out.nodes.size() + 5 * (size_t)nInt);
        write_wide_node(&out.nodes[(size_t)jb.slot * 5], box, cbx, meta, imask, childBase, triBase);
        int ord = 0;
        for (int s = 0; s < 8; s++) if (slotChild[s] >= 0 && !childLeaf[s]) { jobs.push_back({ slotChild[s], childBase + ord, false }); ord++; }
    }
}

namespace {
struct Greedy8 {
    const BinaryBvh* B; WideBvh* out;
    void emit(int bn, int slot) {
        const std::vector<BNode>& N = B->nodes;
        std::vector<int> ch; if (N[bn].left >= 0) ch.push_back(N[bn].left); if (N[bn].right >= 0) ch.push_back(N[bn].right);
        while (ch.size() < 8) {
            int best = -1; float bestA = -1;
            for (size_t j = 0; j < ch.size(); j++) if (!N[ch[j]].leaf()) { float a = N[ch[j]].box.area(); if (a > bestA) { bestA = a; best = (int)j; } }
            if (best < 0) break;
            int nb = ch[best]; ch[best] = N[nb].left; ch.push_back(N[nb].right);
        }
        // slot by octant of the child centre relative to the node centre, nearest free slot by Hamming distance
        const Box3 box = N[bn].box; const float3 c = (box.lo + box.hi) * 0.5f;
        int slotChild[8]; for (int s = 0; s < 8; s++) slotChild[s] = -1;
        for (int cn : ch) {
            const Box3& cb = N[cn].box; float3 cc = (cb.lo + cb.hi) * 0.5f;
            int want = (cc.x < c.x ? 1 : 0) | (cc.y < c.y ? 2 : 0) | (cc.z < c.z ? 4 : 0), pick = -1, bestD = 99;
            for (int s = 0; s < 8; s++) if (slotChild[s] < 0) { int d = __builtin_popcount((unsigned)(s ^ want)); if (d < bestD) { bestD = d; pick = s; } }
            slotChild[pick] = cn;
        }
        int meta[8] = { 0 }; Box3 cbx[8];
        const int triBase = (int)out->order.size(); unsigned imask = 0; int nInt = 0;
        for (int s = 0; s < 8; s++) {
            int cn = slotChild[s]; if (cn < 0) continue;
            cbx[s] = N[cn].box;
            if (N[cn].leaf()) {
                int off = (int)out->order.size() - triBase, cnt = N[cn].count;
                for (int t = 0; t < cnt; t++) out->order.push_back(B->prim[N[cn].first + t]);
                meta[s] = 0x80 | ((cnt - 1) << 5) | off;
                out->maxLeafTris = std::max(out->maxLeafTris, cnt);
            } else { meta[s] = 0x40; imask |= 1u << s; nInt++; }
        }
        const int childBase = (int)(out->nodes.size() / 5);
        out->nodes.resize(out->nodes.size() + 5 * (size_t)nInt);
        write_wide_node(&out->nodes[(size_t)slot * 5], box, cbx, meta, imask, childBase, triBase);
        int ord = 0;
        for (int s = 0; s < 8; s++) if (slotChild[s] >= 0 && !N[slotChild[s]].leaf()) { emit(slotChild[s], childBase + ord); ord++; }
    }
};
}  // namespace

void collapse_greedy8(BinaryBvh& B, WideBvh& out) {
    out.nodes.clear(); out.order.clear(); out.order.reserve(B.prim.size()); out.maxLeafTris = 0;
    out.sah = sah_cost(B, 1, 1);
    int root = 0;
    if (B.nodes[0].leaf()) { wrap_leaf_root(B); root = (int)B.nodes.size() - 1; }
    out.nodes.resize(5);
    Greedy8 g{ &B, &out }; g.emit(root, 0);
}

int append_bvh2(std::vector<float4>& all, const std::vector<float4>& blas, int triBase) {
    int base = (int)(all.size() / 4);
    for (size_t i = 0; i < blas.size(); i += 4) {
        float4 m = blas[i + 3]; int c0 = ibits(m.x), c1 = ibits(m.y), k0 = ibits(m.z), k1 = ibits(m.w);
        if (k0 > 0) c0 += triBase; else if (c0 >= 0) c0 += base;
        if (k1 > 0) c1 += triBase; else if (c1 >= 0) c1 += base;
        all.push_back(blas[i]); all.push_back(blas[i + 1]); all.push_back(blas[i + 2]); all.push_back(make_float4(fbits(c0), fbits(c1), m.z, m.w));
    }
    return base;
}
int append_bvh8(std::vector<float4>& all, const std::vector<float4>& blas, int triBase) {
    int base = (int)(all.size() / 5);
    for (size_t i = 0; i < blas.size(); i += 5) {
        float4 a = blas[i + 1];
        all.push_back(blas[i]);
        all.push_back(make_float4(fbits(ibits(a.x) + base), fbits(ibits(a.y) + triBase), a.z, a.w));
        all.push_back(blas[i + 2]); all.push_back(blas[i + 3]); all.push_back(blas[i + 4]);
    }
    return base;
}

// ======================= triangles =======================
void pack_tris(const Mesh& m, const std::vector<int>& order, std::vector<float4>& tris, std::vector<float4>& nrm) {
    const size_t n = order.size(); tris.resize(3 * n); nrm.clear(); if (m.hasN()) nrm.resize(3 * n);
    for (size_t k = 0; k < n; k++) {
        const int t = order[k]; const int* f = &m.f[3 * (size_t)t];
        float3 v0 = m.vert(f[0]), e1 = m.vert(f[1]) - v0, e2 = m.vert(f[2]) - v0;
        int mat = m.fm.empty() ? 0 : m.fm[t];
        tris[3 * k] = f4(v0, fbits(t)); tris[3 * k + 1] = f4(e1, fbits(mat)); tris[3 * k + 2] = f4(e2, 0.f);
        if (m.hasN()) for (int c = 0; c < 3; c++) nrm[3 * k + c] = make_float4(m.n[3 * (size_t)f[c]], m.n[3 * (size_t)f[c] + 1], m.n[3 * (size_t)f[c] + 2], 0.f);
    }
}

// Woop unit-triangle rows: M = [e1 e2 n]^-1 (adjugate / determinant in FP64, the cofactor expressions in the
// reference's order so the rounded floats agree, tri_pack.cpp:18-38), row r = (M[r][0..2], -M[r] . v0)
void pack_woop(const Mesh& m, const std::vector<int>& order, std::vector<float4>& w) {
    const size_t n = order.size(); w.resize(3 * n);
    for (size_t k = 0; k < n; k++) {
        const int* f = &m.f[3 * (size_t)order[k]];
        float3 v0 = m.vert(f[0]), e1 = m.vert(f[1]) - v0, e2 = m.vert(f[2]) - v0, nn = cross(e1, e2);
        double a[3][3] = { { e1.x, e2.x, nn.x }, { e1.y, e2.y, nn.y }, { e1.z, e2.z, nn.z } };
        double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) + a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
        double iv[3][3] = { { 0 } };
        if (!(fabs(det) < 1e-300)) {
            double id = 1.0 / det;
            iv[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) * id; iv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) * id; iv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) * id;
            iv[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) * id; iv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * id; iv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) * id;
            iv[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) * id; iv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) * id; iv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * id;
        }
        for (int r = 0; r < 3; r++) {
            double t = -(iv[r][0] * v0.x + iv[r][1] * v0.y + iv[r][2] * v0.z);
            w[3 * k + r] = make_float4((float)iv[r][0], (float)iv[r][1], (float)iv[r][2], (float)t);
        }
    }
}

void pack_verts(const Mesh& m, const std::vector<int>& order, std::vector<float4>& v) {
    const size_t n = order.size(); v.resize(3 * n);
    for (size_t k = 0; k < n; k++) {
        const int* f = &m.f[3 * (size_t)order[k]];
        for (int c = 0; c < 3; c++) v[3 * k + c] = f4(m.vert(f[c]), 0.f);
    }
}

}  // namespace cwpb
