// display.cu - headless display transform: accumulated radiance sums -> 8-bit sRGB RGBA on the device, so tone-mapped
// frames can be served from the accumulation buffer without a graphics stack. Mode 0 is the PNG transform of the batch
// renderer (divide by spp, clip to [0, 1], sRGB OETF, x * 255 + 0.5 truncated); modes 1 and 2 are the Reinhard curve
// x / (1 + x) and the ACES filmic fit of Narkowicz (2015), applied before the OETF. Exposure scales by 2^EV.
#include "cwp_b200.h"
#include "runtime.h"

namespace cwpb {

// sRGB OETF (IEC 61966-2-1) of a clipped value, rounded as the PNG writer rounds
__device__ __forceinline__ unsigned char srgb8(float x) {
    x = fminf(fmaxf(x, 0.f), 1.f);
    x = x <= 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.f / 2.4f) - 0.055f;
    return (unsigned char)(x * 255.f + 0.5f);
}
__device__ __forceinline__ float tone(float x, int mode) {
    if (mode == 1) return x / (1.f + x);
    if (mode == 2) { const float a = 0.6f * x; return (a * (2.51f * a + 0.03f)) / (a * (2.43f * a + 0.59f) + 0.14f); }
    return x;
}
__global__ void k_display(const float4* __restrict__ acc, uchar4* __restrict__ out, int64_t n, float spp, float scale, int mode) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = acc[i];
    float r = a.x / spp, g = a.y / spp, b = a.z / spp;
    if (scale != 1.f) { r *= scale; g *= scale; b *= scale; }
    if (mode != 0) { r = tone(fmaxf(r, 0.f), mode); g = tone(fmaxf(g, 0.f), mode); b = tone(fmaxf(b, 0.f), mode); }
    out[i] = make_uchar4(srgb8(r), srgb8(g), srgb8(b), 255);
}

}  // namespace cwpb

extern "C" int cwp_display(const float* d_accum, uint8_t* d_rgba, int64_t n, int32_t spp, float exposure_ev, int32_t mode, void* stream) {
    CWPB_CHECK(n >= 0 && spp >= 0 && mode >= 0 && mode <= 2, CWP_ERR_INVALID, "bad display arguments (n %lld, spp %d, mode %d)", (long long)n, spp, mode);
    if (n == 0) return CWP_OK;
    CWPB_CHECK(d_accum && d_rgba, CWP_ERR_INVALID, "NULL buffer");
    const float scale = exposure_ev == 0.f ? 1.f : exp2f(exposure_ev);
    cwpb::k_display<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>((const float4*)d_accum, (uchar4*)d_rgba, n, (float)(spp > 0 ? spp : 1), scale, mode);
    CWPB_CUDA(cudaGetLastError());
    return CWP_OK;
}
