// vecmath.h - float3 arithmetic, the stateless sample hash and the sampling warps shared by host and device code.
//
// Arithmetic contract: device code is compiled with --fmad=false, host code without FMA contraction, so every
// expression below rounds identically on the CPU and on the GPU. Fused multiply-adds appear only where written
// as fmaf(); the CPU oracle uses the same fused forms, which makes traversal results bit-identical between them.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#define CWPB_HD __host__ __device__ __forceinline__

namespace cwpb {

CWPB_HD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
CWPB_HD float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
CWPB_HD float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
CWPB_HD float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
CWPB_HD float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
CWPB_HD float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
CWPB_HD float3 operator*(float s, float3 a) { return f3(a.x * s, a.y * s, a.z * s); }
CWPB_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
CWPB_HD float3 cross(float3 a, float3 b) { return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
CWPB_HD float length(float3 a) { return sqrtf(dot(a, a)); }
CWPB_HD float3 normalize(float3 a) { float l = length(a); return l > 0.f ? a * (1.0f / l) : a; }
CWPB_HD float3 vmin(float3 a, float3 b) { return f3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
CWPB_HD float3 vmax(float3 a, float3 b) { return f3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
CWPB_HD float maxc(float3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
CWPB_HD float3 xyz(float4 a) { return f3(a.x, a.y, a.z); }
CWPB_HD float4 f4(float3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
// fused dot product used by the triangle tests: ((a.x b.x) + a.y b.y) + a.z b.z with two fused steps
CWPB_HD float fdot(float3 a, float3 b) { return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)); }
// fused affine row: w + a.x r.x + a.y r.y + a.z r.z
CWPB_HD float frow(float4 r, float3 a) { return fmaf(a.z, r.z, fmaf(a.y, r.y, fmaf(a.x, r.x, r.w))); }

CWPB_HD float bits_f(int i) {
#ifdef __CUDA_ARCH__
    return __int_as_float(i);
#else
    union { int i; float f; } u; u.i = i; return u.f;
#endif
}
CWPB_HD int bits_i(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_int(f);
#else
    union { int i; float f; } u; u.f = f; return u.i;
#endif
}
CWPB_HD unsigned bits_u(float f) { return (unsigned)bits_i(f); }
CWPB_HD float bits_fu(unsigned u) { return bits_f((int)u); }

// ---- stateless sample hash ----
// Every random number of a path is a pure function of (pixel, sample, depth, dimension, seed). The mixing function
// and its constants are those of the reference (core/rng.h:6-12): the sample streams must be the same for rendered
// frames to agree sample by sample.
CWPB_HD unsigned mix32(unsigned x) { x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16; return x; }
CWPB_HD float sample01(unsigned pix, unsigned smp, unsigned depth, unsigned dim, unsigned seed) {
    unsigned h = mix32(pix * 0x9E3779B1U ^ mix32(smp * 0x85EBCA77U ^ mix32((depth * 8u + dim) * 0xC2B2AE3DU ^ seed)));
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}

#define CWPB_TWO_PI 6.2831853f
#define CWPB_INV_PI 0.31830989f

// orthonormal frame around a unit normal (Duff et al., JCGT 2017), as core/sampling.h:13-16
CWPB_HD void frame_of(float3 n, float3& t, float3& b) {
    float s = n.z >= 0.f ? 1.f : -1.f; float a = -1.f / (s + n.z); float c = n.x * n.y * a;
    t = f3(1.f + s * n.x * n.x * a, s * c, -s * n.x); b = f3(c, s + n.y * n.y * a, -n.y);
}
// cos and sin of 2 pi u for u in [0, 1)
CWPB_HD void turn(float u, float& c, float& s) { const float ph = CWPB_TWO_PI * u; c = cosf(ph); s = sinf(ph); }
// cosine-weighted hemisphere direction (pdf cos/pi), as core/sampling.h:19-22
CWPB_HD float3 cosine_dir(float3 n, float u0, float u1) {
    float r = sqrtf(u0), c, s; turn(u1, c, s); float3 t, b; frame_of(n, t, b);
    return normalize(t * (r * c) + b * (r * s) + n * sqrtf(fmaxf(0.f, 1.f - u0)));
}
// uniform direction in a cone of half-angle acos(cosMax), as core/sampling.h:25-29
CWPB_HD float3 cone_dir(float3 axis, float cosMax, float u0, float u1) {
    float cz = 1.f - u0 * (1.f - cosMax); float sz = sqrtf(fmaxf(0.f, 1.f - cz * cz)), c, s; turn(u1, c, s);
    float3 t, b; frame_of(axis, t, b);
    return normalize(axis * cz + t * (sz * c) + b * (sz * s));
}
// piecewise-linear inverse-CDF lookup of n+1 entries, as core/sampling.h:32-34
CWPB_HD float table_lookup(const float* tab, int n, float u) {
    float f = u * n; int k = (int)f; k = k < n - 1 ? k : n - 1; float t = f - k; return tab[k] * (1.f - t) + tab[k + 1] * t;
}
// concentric disk map (Shirley & Chiu 1997), as core/sampling.h:46-52
CWPB_HD void disk_map(float u0, float u1, float& x, float& y) {
    float a = 2.f * u0 - 1.f, b = 2.f * u1 - 1.f;
    if (a == 0.f && b == 0.f) { x = y = 0.f; return; }
    float r, ph;
    if (fabsf(a) > fabsf(b)) { r = a; ph = 0.78539816f * (b / a); } else { r = b; ph = 1.57079633f - 0.78539816f * (a / b); }
    x = r * cosf(ph); y = r * sinf(ph);
}

}  // namespace cwpb
