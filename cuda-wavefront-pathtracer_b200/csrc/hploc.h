// hploc.h - GPU BVH construction for many primitive sets at once.
//
// Every primitive (a box) belongs to one segment (one mesh, or one scene's instances); segments are contiguous ranges
// of the primitive array. One build runs, for all segments together:
//   1. per-segment centroid bounds (warp-reduced atomics),
//   2. 64-bit keys = segment id (10 bits) above an 18-bit-per-axis Morton code of the centroid in its segment's
//      bounds, paired with the primitive index,
//   3. one radix sort of all pairs (CUB, bundled with the CUDA toolkit),
//   4. ONE hierarchical-PLOC launch (Benthin, Meister, Barczak & Grimm, "H-PLOC", HPG 2024): one thread per sorted
//      primitive climbs the implicit LBVH of its segment bottom-up (Apetrei 2014: a node's parent lies on the side of
//      the smaller key difference, the second thread to reach a parent carries on with the union range; equal keys
//      are ordered by position), and wherever a range holds more than kPlocT clusters - or is its segment's root -
//      the warp merges the clusters of both children by PLOC (nearest neighbour by merged-box surface area within
//      kPlocR positions, mutual pairs merge) down to kPlocT (1 at the root). A segment never crosses into another.
// Output: per segment s with m prims, 2m - 1 binary nodes in the region starting at 2 first(s) - s: the m leaves in
// sorted order, then the m - 1 internal nodes; node = (lo.xyz, left), (hi.xyz, right) as int bits, leaves have
// left = primitive index and right = -1; count[node] = primitives below. The root is the region's last node.
#pragma once
#include "runtime.h"
#include <cstdint>
#include <vector>

namespace cwpb {

static constexpr int kSegBits = 10;          // up to 1024 segments per build
static constexpr int kMortonBits = 54;       // 18 bits per axis

struct SegBuilder {
    int device = 0;
    int64_t capPrims = 0; int capSegs = 0;
    float4* nodes = nullptr;                  // 2 float4 per node, 2 n - nSeg nodes
    int* count = nullptr;                     // primitives under each node
    unsigned long long *keys = nullptr, *keysSorted = nullptr;
    int *vals = nullptr, *valsSorted = nullptr;
    int *clusters = nullptr, *bounds = nullptr;
    int* segFirst = nullptr;                  // device copy, nSeg + 1 entries
    int* counters = nullptr;                  // next internal node id per segment
    unsigned* cbox = nullptr;                 // 6 ordered-uint bounds per segment
    void* tmp = nullptr; size_t tmpBytes = 0;

    int reserve(int64_t n, int nSeg);
    // lo / hi: n boxes (device, float4 xyz); segFirst: host array of nSeg + 1 offsets. Stream-ordered. Returns CWP_OK
    // or an error code; the roots are segRoot(s) below.
    int build(const float4* lo, const float4* hi, int64_t n, const int* segFirstHost, int nSeg, cudaStream_t st);
    void release();
    static int64_t regionBase(int64_t first, int s) { return 2 * first - s; }
};

// One mesh (v: 3 floats per vertex, f: 3 ints per triangle) built on `device` with one segment: the triangle boxes
// are made on the host, a warm-up build runs, then a CUDA-event-timed build (gpuMs: bounds, keys, sort, H-PLOC);
// nodesOut receives its 2 nt - 1 binary nodes (2 float4 each, leaves [0, nt) in sorted order, root last).
int hploc_build_mesh(const float* v, const int* f, int64_t nt, int device, std::vector<float4>& nodesOut, double& gpuMs);

}  // namespace cwpb
