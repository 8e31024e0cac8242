// lights.h - emissive triangles as area lights of instanced scenes: which triangles of which mesh emit (once per
// material table), and per frame their world-space corners and the power CDF that light sampling draws from.
#pragma once
#include "cwp_b200.h"
#include <vector>

namespace cwpb {

struct EmissiveTri { int mat; int gtri; float v[9]; };   // material, global triangle id, object-space corners

// emissive triangles of every mesh, in mesh order: mesh m owns tris[first[m], first[m + 1])
struct EmissiveSet {
    std::vector<int> first;
    std::vector<EmissiveTri> tris;
    bool empty() const { return tris.empty(); }
};

inline bool is_emissive(const cwp_material& m) { return m.emission[0] > 0.f || m.emission[1] > 0.f || m.emission[2] > 0.f; }

// soup: 12 floats per triangle ((v0, face id), (v1, face material), (v2, 0)) of nMesh meshes, mesh m's triangles
// [meshFirst[m], meshFirst[m + 1]); triangle material = meshMat[m] + face material, clamped to the table
void emissive_set(const float* soup, const int* meshFirst, int nMesh, const int* meshMat, const cwp_material* mats, int nMats, EmissiveSet& out);

// the light tables of one frame: emT 12 floats per emissive instance triangle, emC nEm + 1 floats, mlp nMats floats;
// emT, emC empty when the scene has no emissive triangle or their total power is 0
void frame_lights(const EmissiveSet& S, const float* xf, const int* instMesh, int64_t nInst, const cwp_material* mats, int nMats,
                  std::vector<float>& emT, std::vector<float>& emC, std::vector<float>& mlp);

}  // namespace cwpb
