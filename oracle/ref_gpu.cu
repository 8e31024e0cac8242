// ref_gpu.cu - TEST INFRASTRUCTURE ONLY: the reference's own device traversal (accel/traverse.cuh trav<V,ANY,TRI>)
// in a one-ray-per-thread batch kernel shaped like the reference's k_trace / k_shadow (render/wavefront.cu:61-82:
// 128-thread blocks, __launch_bounds__(128, 12) as the default MINB = 12 build, --use_fast_math). Built by
// oracle/Makefile into oracle/_ref/libcwpref_gpu.so; the GPU parity tests compare the library's hits with it on
// identical ray batches.
#include "accel/traverse.cuh"
#include <cstdint>

template <int V, bool ANY, int TRI>
__global__ void __launch_bounds__(128, 12) ref_k_batch(const float4* __restrict__ nodes, const float4* __restrict__ tv, const float4* __restrict__ ro,
                                                       const float4* __restrict__ rd, float4* hits, int* occ, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x; if (i >= n) return;
    float4 O = ro[i], D = rd[i]; float t = D.w, u = 0.f, v = 0.f; int tri = -1;
    trav<V, ANY, TRI>(nodes, tv, xyz(O), xyz(D), O.w, t, tri, u, v);
    if (ANY) occ[i] = tri; else hits[i] = make_float4(t, u, v, __int_as_float(tri));
}

// device pointers; returns a cudaError_t value (0 = success)
extern "C" int ref_gpu_trace(int variant, int any, int tri, const float* nodes, const float* tv, const float* ro, const float* rd, long n,
                             float* hits, int* occ, void* stream) {
    if (n <= 0) return 0;
    int g = (int)((n + 127) / 128); cudaStream_t s = (cudaStream_t)stream;
    const float4 *N = (const float4*)nodes, *T = (const float4*)tv, *O = (const float4*)ro, *D = (const float4*)rd; float4* H = (float4*)hits;
#define RL(VV) do { if (any) { if (tri) ref_k_batch<VV, true, 1><<<g, 128, 0, s>>>(N, T, O, D, H, occ, (int)n); else ref_k_batch<VV, true, 0><<<g, 128, 0, s>>>(N, T, O, D, H, occ, (int)n); } \
                    else { if (tri) ref_k_batch<VV, false, 1><<<g, 128, 0, s>>>(N, T, O, D, H, occ, (int)n); else ref_k_batch<VV, false, 0><<<g, 128, 0, s>>>(N, T, O, D, H, occ, (int)n); } } while (0)
    if (variant == 2) RL(2); else if (variant == 4) RL(4); else RL(8);
#undef RL
    return (int)cudaGetLastError();
}

// The reference's GPU BVH construction for a static mesh, as its --builder hploc runs it (app/scene_setup.cpp:76-83):
// hplocBuildHost (accel/hploc.cu:195-209: upload, one warm-up build, one CUDA-event-timed build, download) on the
// triangle boxes lo / hi (n float4 each, host), then treeFromHploc (accel/bvh_tools.cpp:12-38: SAH-optimal leaf
// collapse to leafMax) and sahCost (bvh_tools.cpp:40-44, c_node = c_prim = 1). Returns the SAH cost; *gpu_ms = the
// timed device build; *n_nodes / *max_depth of the collapsed binary tree.
#include "accel/hploc.h"
#include "accel/bvh_tools.h"
#include <vector>
extern "C" double ref_hploc_tree(const float* lo, const float* hi, int n, int leafMax, double* gpu_ms, int* n_nodes, int* max_depth) {
    std::vector<float4> L((size_t)n), H((size_t)n), nodes;
    for (int i = 0; i < n; i++) { L[i] = make_float4(lo[4 * i], lo[4 * i + 1], lo[4 * i + 2], 0.f); H[i] = make_float4(hi[4 * i], hi[4 * i + 1], hi[4 * i + 2], 0.f); }
    double ms = 0;
    const int root = hplocBuildHost(L, H, nodes, ms);
    BVHBuilder B; treeFromHploc(nodes, n, root, leafMax, B);
    *gpu_ms = ms; *n_nodes = (int)B.nodes.size(); *max_depth = B.maxDepth;
    return sahCost(B, 1, 1);
}
