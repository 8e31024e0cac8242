// wide_emit.h - GPU encodings of segmented H-PLOC trees: BVH2 (64 B), BVH4 (128 B) and CWBVH (80 B) nodes plus
// Moller-Trumbore triangle records for every mesh of a build, and the per-scene TLAS (BVH2 over instances).
#pragma once
#include "hploc.h"

namespace cwpb {

// One layout of every BLAS of a build. Node i < nSeg is the root of mesh i; all child / triangle indices are absolute.
struct WideLayout {
    int width = 0;                       // 2, 4 or 8
    float4* nodes = nullptr; int64_t nNodes = 0, capNodes = 0;
    float4* tris = nullptr;              // 3 float4 per triangle, leaf order: (v0, mesh-local id), (e1, material), (e2, 0)
    int stride() const { return width == 2 ? 4 : width == 4 ? 8 : 5; }
};

// Emits one layout from the binary trees of B (built over the triangles triV: 3 float4 per triangle with the
// mesh-local id in v0.w and the material in v1.w, as int bits). Deterministic: nodes are numbered level by level in
// the order of their parents, whatever order the H-PLOC build allocated its binary nodes in. Synchronises the stream
// once per tree level. leafMax: triangles per leaf (<= 3 for width 8).
int emit_wide(const SegBuilder& B, const int* segFirstHost, int nSeg, const float4* triV, int width, int leafMax, WideLayout& out,
              cudaStream_t st);
void free_wide(WideLayout& w);

// Per-scene TLAS from a segmented build over instance boxes: BVH2 nodes (leaves hold one instance, count 1) in the
// region [first(s), first(s) + m) of scene s's instances; root(s) = first + m - 2 (first when m == 1). With tlas4,
// also the width-4 form (8 float4 per node, same indices and roots: each node's children are the BVH2 node's
// grandchildren). With dstFirstDev, the build ran over a compact copy and segment s's nodes and instance references go
// to the region that starts at dstFirstDev[s] instead of first(s).
void emit_tlas(const SegBuilder& B, int nInst, const int* segFirstDev, int nSeg, float4* tlas, cudaStream_t st, const int* dstFirstDev = nullptr,
               float4* tlas4 = nullptr);

// World boxes of instances (the 8 corners of their mesh's root box through the object -> world rows).
void instance_boxes(const cwp_instance* inst, int nInst, const float4* meshBox, float4* lo, float4* hi, cudaStream_t st);

// Triangle boxes (for the BLAS build) and the mesh root boxes after it.
void triangle_boxes(const float4* triV, int64_t n, float4* lo, float4* hi, cudaStream_t st);
void root_boxes(const SegBuilder& B, const int* segFirstDev, int nSeg, float4* meshBox, cudaStream_t st);

// Reference checks run after every build (CWP_ERR_INVALID if a child, triangle or instance index is out of range, or
// an inner child does not come after its parent); dBad is one device int of scratch. Synchronise the stream.
int check_wide(const WideLayout& w, int64_t nTris, int* dBad, cudaStream_t st);
int check_tlas(const float4* tlas, int nInst, const int* segFirstDev, int nSeg, int* dBad, cudaStream_t st, const int* dstFirstDev = nullptr,
               const float4* tlas4 = nullptr);

}  // namespace cwpb
