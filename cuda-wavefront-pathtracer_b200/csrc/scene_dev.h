// scene_dev.h - device copy of a scene's nodes and triangles, shared by the ray-batch and renderer entry points.
#pragma once
#include "runtime.h"
#include <cstdint>
#include <vector>

namespace cwpb {

struct DeviceScene {
    int device = 0, variant = 2, tri = 1;
    float4* nodes = nullptr; int64_t nNodes = 0;     // nodes in units of one node (stride float4 each)
    float4* tris = nullptr; int64_t nTris = 0;       // (v0, id), (e1, mat), (e2, 0)
    float4* woop = nullptr;                          // Woop rows or nullptr
    float4* nrm = nullptr;                           // per-corner normals or nullptr
    float4* verts = nullptr;                         // exact corners (precision form) or nullptr
    bool precise = false;                            // ray batches use the precision form (FP16 slabs + watertight)
    float3* albedo = nullptr; int nAlbedo = 0;
    size_t bytes = 0;
    void* arena = nullptr; size_t hotBytes = 0;     // one allocation; its first hotBytes hold nodes, leaf rows, triangles, corners
    // CWBVH: the device copy is numbered breadth first (same tree, same child order), so the nodes of levels 0..L are
    // the first levelEnd[L] nodes - the ones the frame kernels can stage in shared memory
    int levelEnd[4] = { 0, 0, 0, 0 };
    const float4* leafData() const { return precise ? verts : tri == 1 ? woop : tris; }
};

// Checks every child and leaf reference of the node array against the buffer sizes (so that no traversal can read
// out of bounds), then uploads. variant comes from the node stride (4 -> BVH2, 8 -> BVH4, 5 -> CWBVH).
int upload_scene(const cwp_scene_buffers* s, int tri, int device, DeviceScene& out);
void free_scene(DeviceScene& s);
int validate_nodes(const float* nodes, int64_t nF4, int stride, int64_t nTris, int* variantOut);
// Breadth-first renumbering of a validated CWBVH (5 float4 per node, root 0): every node keeps its children, in slot
// order and contiguous; only the node indices (and each node's child base) change. levelEnd[L] = number of nodes in
// levels 0..L. False when the nodes do not form one tree rooted at node 0.
bool cwbvh_breadth_first(const float* in, int64_t nNodes, std::vector<float>& out, int levelEnd[4]);

}  // namespace cwpb
