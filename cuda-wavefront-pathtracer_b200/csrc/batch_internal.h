// batch_internal.h - what the serving loop uses of a cwp_batch: the scene-tagged trace on a caller's stream with the
// batch's tuning, and the device arrays that shading reads (triangle records of the traced layout, instances).
#pragma once
#include "cwp_b200.h"
#include <cuda_runtime.h>

namespace cwpb {
// nDev: the ray count read on the device at launch (n is then ignored), so a count produced by an earlier kernel needs no
// host round trip
int batch_trace_dev(cwp_batch* b, bool any, const float4* o, const float4* d, const int* sc, float4* hits, int* inst, int64_t n, cudaStream_t st,
                    const int* nDev = nullptr);
const float4* batch_tris(const cwp_batch* b);          // triangle records (v0, id), (e1, material), (e2, 0) of the tuned width
const cwp_instance* batch_instances(const cwp_batch* b);
int batch_mesh_count(const cwp_batch* b);
int batch_device(const cwp_batch* b);
const int* batch_mesh_first(const cwp_batch* b);       // device: nMesh + 1 offsets of each mesh's triangles in mesh order
int64_t batch_tri_count(const cwp_batch* b);            // triangles of all meshes
const float4* batch_tri_soup(const cwp_batch* b);     // device: the input triangles, (v0, face id), (v1, face material), (v2, 0) in mesh order
const int* batch_mesh_first_host(const cwp_batch* b);  // host: nMesh + 1 offsets
const float4* batch_normals(const cwp_batch* b);      // device: corner normals, 3 float4 per triangle in mesh order, or null
}  // namespace cwpb
