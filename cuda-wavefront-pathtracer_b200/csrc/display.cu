// display.cu - headless display transform: accumulated radiance sums -> 8-bit sRGB RGBA on the device, so that
// tone-mapped frames can be served straight from the accumulation buffer without a graphics stack.
//
// Per pixel: mean radiance (sum / spp, IEEE division), times the exposure 2^EV, through a tone curve, clipped to
// [0, 1], sRGB-encoded and quantised to 8 bits the way the batch renderer's PNG writer quantises. The curves (mode):
//   0  none: exactly the PNG transform of the batch renderer (the reference's io/image.cpp tonemapSRGB8);
//   1  Reinhard's global operator x / (1 + x) (Reinhard, Stark, Shirley, Ferwerda, SIGGRAPH 2002);
//   2  the ACES filmic curve fit of Narkowicz (2015), x (2.51 x + 0.03) / (x (2.43 x + 0.59) + 0.14), evaluated at
//      0.6 x (the exposure the fit was made for; the reference's viewer applies the same).
// The curve is a template parameter, so each launch runs one branch-free instantiation.
#include "cwp_b200.h"
#include "runtime.h"

namespace cwpb {
namespace {

// IEC 61966-2-1 encoding of a linear value (linear segment below 0.0031308, else the 1/2.4 power segment), then
// x * 255 + 0.5 truncated; device code is compiled without contraction, so this rounds as the host writer does
__device__ __forceinline__ unsigned encode_srgb8(float linear) {
    const float x = fminf(fmaxf(linear, 0.f), 1.f);
    const float e = x > 0.0031308f ? 1.055f * powf(x, 1.f / 2.4f) - 0.055f : 12.92f * x;
    return (unsigned)(e * 255.f + 0.5f);
}

template <int MODE>
__device__ __forceinline__ float tone_curve(float x) {
    if (MODE == 1) { x = fmaxf(x, 0.f); return x / (1.f + x); }
    if (MODE == 2) { const float v = 0.6f * fmaxf(x, 0.f); return v * (2.51f * v + 0.03f) / (v * (2.43f * v + 0.59f) + 0.14f); }
    return x;
}

// grid-stride over the pixels; one 16-byte streaming load and one packed 32-bit store (R, G, B, 255 in byte order)
template <int MODE>
__global__ void __launch_bounds__(256) k_display(const float4* __restrict__ acc, unsigned* __restrict__ rgba, int64_t n, float spp, float scale) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 s = __ldcs(acc + i);
        const unsigned r = encode_srgb8(tone_curve<MODE>(s.x / spp * scale));
        const unsigned g = encode_srgb8(tone_curve<MODE>(s.y / spp * scale));
        const unsigned b = encode_srgb8(tone_curve<MODE>(s.z / spp * scale));
        __stcs(rgba + i, r | (g << 8) | (b << 16) | 0xff000000u);
    }
}

}  // namespace
}  // namespace cwpb

extern "C" int cwp_display(const float* d_accum, uint8_t* d_rgba, int64_t n, int32_t spp, float exposure_ev, int32_t mode, void* stream) {
    CWPB_CHECK(n >= 0 && spp >= 0 && mode >= 0 && mode <= 2, CWP_ERR_INVALID, "bad display arguments (n %lld, spp %d, mode %d)", (long long)n, spp, mode);
    if (n == 0) return CWP_OK;
    CWPB_CHECK(d_accum && d_rgba, CWP_ERR_INVALID, "NULL buffer");
    CWPB_CHECK(((uintptr_t)d_accum & 15) == 0 && ((uintptr_t)d_rgba & 3) == 0, CWP_ERR_INVALID, "buffers must be 16-byte (accum) and 4-byte (rgba) aligned");
    const float scale = exposure_ev == 0.f ? 1.f : exp2f(exposure_ev);   // x * 1 is exact: exposure 0 changes nothing
    const float s = (float)(spp > 0 ? spp : 1);
    const int64_t want = (n + 255) / 256;
    const unsigned grid = (unsigned)(want < 4096 ? want : 4096);
    const float4* a = (const float4*)d_accum; unsigned* o = (unsigned*)d_rgba; cudaStream_t st = (cudaStream_t)stream;
    if (mode == 0) cwpb::k_display<0><<<grid, 256, 0, st>>>(a, o, n, s, scale);
    else if (mode == 1) cwpb::k_display<1><<<grid, 256, 0, st>>>(a, o, n, s, scale);
    else cwpb::k_display<2><<<grid, 256, 0, st>>>(a, o, n, s, scale);
    CWPB_CUDA(cudaGetLastError());
    return CWP_OK;
}
