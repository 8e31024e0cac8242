// host_bvh.h - host BVH construction and the GPU node / triangle encodings.
//
// The encodings are the reference's, byte for byte, so that buffers built here and buffers built by the reference
// are interchangeable (accel/bvh_layouts.h, accel/bvh_tools.h, accel/tri_pack.h):
//   BVH2 (64 B/node):  (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y), (same for c1), (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z),
//                      (c0, c1, cnt0, cnt1) as int bits; cnt > 0: leaf of cnt triangles from c; cnt == 0: node c
//                      (c = -1: empty slot with EMPTY_BOX bounds).
//   BVH4 (128 B/node): SoA child boxes lo.x, hi.x, lo.y, hi.y, lo.z, hi.z (one float4 each), child int4, count int4.
//   CWBVH (80 B/node): origin xyz + (exponents x, y, z biased by 127, imask << 24); childBase, triBase, meta[0..7];
//                      8-bit quantised child boxes lo.x[8], lo.y[8], lo.z[8], hi.x[8], hi.y[8], hi.z[8].
//   Triangles, leaf order: (v0, original id), (e1, material), (e2, 0); Woop rows: inverse of [e1 e2 e1xe2] with
//   translation, 3 float4 per triangle, computed in FP64 and rounded.
#pragma once
#include "host_scene.h"
#include <cfloat>
#include <vector>

namespace cwpb {

static const float kEmptyBox = 3e37f;

struct Box3 {
    float3 lo, hi;
    Box3() : lo(f3(FLT_MAX, FLT_MAX, FLT_MAX)), hi(f3(-FLT_MAX, -FLT_MAX, -FLT_MAX)) {}
    void grow(float3 p) { lo = vmin(lo, p); hi = vmax(hi, p); }
    void grow(const Box3& b) { lo = vmin(lo, b.lo); hi = vmax(hi, b.hi); }
    // surface area; 0 for an empty box (accel/aabb.h:11)
    float area() const { if (hi.x < lo.x) return 0.f; float3 d = hi - lo; return 2.f * (d.x * d.y + d.y * d.z + d.z * d.x); }
    float3 extent() const { return hi - lo; }
};

struct BNode { Box3 box; int left = -1, right = -1, first = 0, count = 0; bool leaf() const { return count > 0; } };

// Binary BVH: nodes[0] is the root, nodes are numbered in pre-order (left subtree first); prim is the triangle order
// that leaves index into.
struct BinaryBvh { std::vector<BNode> nodes; std::vector<int> prim; int maxDepth = 0; int leafMax = 4; };

struct SahOptions {
    int bins = 16;       // SAH bins per axis (the reference uses 16)
    int leafMax = 4;     // leaves hold at most leafMax triangles
    int depthCap = 62;   // nodes at this depth become leaves
    int threads = 0;     // 0 = all hardware threads; 1 = serial. The result does not depend on it.
};

// Binned-SAH BVH2 over the triangles of m (the algorithm of accel/bvh_builder.cpp:5-68 with a configurable bin
// count). Independent subtrees and the binning of large nodes run on several threads; the tree is renumbered to
// pre-order at the end, so the output is identical for any thread count and, at 16 bins, to the reference builder.
void build_sah(const Mesh& m, const SahOptions& o, BinaryBvh& out);

// Binned SAH with spatial splits (SBVH): prim then holds triangle references, a triangle possibly in several leaves.
// alpha: relative overlap area above which a node tries spatial splits (1e-5 typical); budget: cap on the extra
// references as a fraction of the triangle count. Parallel subtrees; the result does not depend on the thread count.
void build_sbvh(const Mesh& m, const SahOptions& o, float alpha, float budget, BinaryBvh& out);

// Binary BVH from a one-mesh GPU H-PLOC build (hploc.h: hploc_build_mesh) with SAH-optimal leaf collapse to at
// most leafMax triangles per leaf; numbered in pre-order like build_sah's trees.
void tree_from_hploc(const std::vector<float4>& hn, int64_t n, int leafMax, BinaryBvh& out);

// SAH cost normalised by the root area: internal nodes cost cNode, leaves cPrim per triangle (bvh_tools.cpp:40-44).
double sah_cost(const BinaryBvh& B, double cNode, double cPrim);

// Layouts. build may append a wrapper root when the root is a leaf (as the reference does).
void layout_bvh2(BinaryBvh& B, std::vector<float4>& nodes);
void layout_bvh4(BinaryBvh& B, std::vector<float4>& nodes);
struct WideBvh { std::vector<float4> nodes; std::vector<int> order; int maxLeafTris = 0; double sah = 0; };
// SAH-optimal 8-wide collapse (Ylitie et al. 2017; c_node 1, c_prim 0.3, leaves <= 3), bvh_tools.cpp:75-168
void collapse_cwbvh(const BinaryBvh& B, WideBvh& out);
// greedy 8-wide collapse (largest-area child opened first), bvh_layouts.cpp:65-134
void collapse_greedy8(BinaryBvh& B, WideBvh& out);

// concatenation of per-mesh layouts with absolute indices (bvh_tools.cpp:170-189); returns the root node index
int append_bvh2(std::vector<float4>& all, const std::vector<float4>& blas, int triBase);
int append_bvh8(std::vector<float4>& all, const std::vector<float4>& blas, int triBase);

void pack_tris(const Mesh& m, const std::vector<int>& order, std::vector<float4>& tris, std::vector<float4>& nrm);
void pack_woop(const Mesh& m, const std::vector<int>& order, std::vector<float4>& w);
// exact corner positions in leaf order, (v0, 0), (v1, 0), (v2, 0): the watertight triangle test needs the shared
// vertices of neighbouring triangles bit for bit (v0 + e1 would be rounded)
void pack_verts(const Mesh& m, const std::vector<int>& order, std::vector<float4>& v);

}  // namespace cwpb
