// probe.cu - on-chip read-bandwidth probe: the denominator of the traversal kernels' on-chip roofline. Traversal
// reads nodes and triangles that stay resident in L2 (a scene's acceleration structure is far smaller than the
// 126 MB L2), so the bandwidth it can draw on is L2's, not HBM's. The probe reads an L2-resident buffer from every SM
// with 16-byte ld.global.cg loads (cached in L2, not L1), several passes per launch, and reports bytes per second.
#include "cwp_b200.h"
#include "runtime.h"
#include <algorithm>

namespace cwpb {

__global__ void __launch_bounds__(256) k_l2_read(const float4* __restrict__ buf, int64_t n4, int reps, float* sink) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x, t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float acc = 0.f;
    for (int r = 0; r < reps; r++) {
        int64_t i = t0;
        for (; i + 3 * stride < n4; i += 4 * stride) {   // four independent loads in flight per thread
            const float4 a = __ldcg(buf + i), b = __ldcg(buf + i + stride), c = __ldcg(buf + i + 2 * stride), d = __ldcg(buf + i + 3 * stride);
            acc += (a.x + b.y) + (c.z + d.w);
        }
        for (; i < n4; i += stride) { const float4 a = __ldcg(buf + i); acc += a.x; }
    }
    if (acc == 1.2345e-30f) sink[0] = acc;   // keeps the loads; the buffer holds zeros, so this store never happens
}

}  // namespace cwpb

extern "C" int cwp_measure_l2_read(int64_t bytes, int32_t reps, int32_t device, double* gbs) {
    CWPB_CHECK(gbs && bytes >= (1 << 20) && bytes <= (int64_t(96) << 20) && (bytes & 15) == 0 && reps >= 1 && reps <= 1000, CWP_ERR_INVALID,
               "bad probe arguments (bytes %lld in [1 MiB, 96 MiB] and a multiple of 16, reps %d in [1, 1000])", (long long)bytes, reps);
    CWPB_CUDA(cudaSetDevice(device));
    int sms = 0; CWPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    float4* buf = nullptr; float* sink = nullptr; cudaStream_t st = nullptr; cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = CWP_OK; double best = 0.0;
    auto ok = [&](cudaError_t e) { if (e != cudaSuccess && rc == CWP_OK) rc = cwpb::set_error(CWP_ERR_CUDA, "%s (L2 probe)", cudaGetErrorString(e)); return rc == CWP_OK; };
    if (ok(cudaMalloc(&buf, (size_t)bytes)) && ok(cudaMalloc(&sink, sizeof(float))) && ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) &&
        ok(cudaEventCreate(&e0)) && ok(cudaEventCreate(&e1)) && ok(cudaMemsetAsync(buf, 0, (size_t)bytes, st))) {
        const int64_t n4 = bytes / 16;
        for (int it = 0; it < 6 && rc == CWP_OK; it++) {   // the first launch warms L2; the best of the other five counts
            ok(cudaEventRecord(e0, st));
            cwpb::k_l2_read<<<sms * 8, 256, 0, st>>>(buf, n4, reps, sink);
            ok(cudaGetLastError()); ok(cudaEventRecord(e1, st)); ok(cudaEventSynchronize(e1));
            float ms = 0.f;
            if (ok(cudaEventElapsedTime(&ms, e0, e1)) && it > 0 && ms > 0.f) best = std::max(best, (double)bytes * reps / (ms * 1e-3) / 1e9);
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    if (buf) cudaFree(buf);
    if (sink) cudaFree(sink);
    if (rc == CWP_OK) *gbs = best;
    return rc;
}
