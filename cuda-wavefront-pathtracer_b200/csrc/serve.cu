// serve.cu - the serving form: a request loop with continuous batching over the resident scenes of a cwp_batch.
//
// Requests wait in a FIFO queue and are admitted into one of max_requests slots when a slot is free and the device has
// room for the request's image (cudaMemGetInfo, less hbm_reserve). Every step:
//   1. admission, and when it admitted anything, one TLAS update of the admitted slots (slot k's scene animated to its
//      frame; every slot owns a fixed TLAS region, so the other slots' TLAS stay untouched);
//   2. new camera paths for the admitted requests, up to the path capacity, shared evenly between the requests that
//      still have samples to issue (so small requests are not stuck behind large ones);
//   3. one scene-tagged closest-hit launch over every queued ray, whatever request it belongs to;
//   4. shading (OpenPBR-subset BSDFs, one light sample per vertex over the sun, the emissive triangles and an
//      environment map, MIS with BSDF sampling, Russian roulette): continuations into the next queue, shadow rays into
//      the shadow queue, per-slot counts of traced, shadow and finished paths;
//   5. one any-hit launch over the shadow queue and the accumulation of the unoccluded contributions;
//   6. completion: a request whose paths were all issued and have all finished is done.
// A request's image depends only on its own inputs: every random number is keyed by (pixel, sample, depth, dimension,
// request seed), and shading reads only its own slot's parameters. max_requests = 1 gives the plain form (one request
// on the GPU at a time, the same kernels).
#include "batch_internal.h"
#include "bsdf.cuh"
#include "cwp_b200.h"
#include "lights.h"
#include "runtime.h"
#include "trav.cuh"
#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <vector>

namespace cwpb {

struct SlotParams {
    cwp_camera cam;
    float3 sunTo, sunE, sky; float sunCos, eps;
    unsigned seed; int maxDepth, N; float4* accum;
    // the request's environment map (envTex null: the constant sky): texels, CDF over rows, CDF within each row
    const float4* envTex; const float* envMarg; const float* envCond; int envW, envH; float envRot;
    // light sampling: light-type probabilities, mode (CWP_LIGHT_*), Russian roulette, uniform environment samples; the
    // scene's emissive triangles at the request's frame (nEm = 0: none): 3 float4 each, power CDF, area density by material
    float pSun, pTri, pEnv; int lightMode, rr, rrDepth, envUniform, nEm, bumpShadow;
    float nearClip; int filterBh;
    const float4* emTris; const float* emCdf; const float* matPdf;
};

// ---------------- environment map (scene/environment.h orientation; render/wavefront.cu:177-197, 319-331) ----------
// equirectangular, row 0 = +z, the centre column facing +x, u growing toward -y; rotated by envRot about +z
__device__ __forceinline__ void env_uv(const SlotParams& S, float3 d, float& u, float& v) {
    u = 0.5f - (atan2f(d.y, d.x) - S.envRot) * (1.f / CWPB_TWO_PI); u -= floorf(u);
    v = acosf(fminf(fmaxf(d.z, -1.f), 1.f)) * CWPB_INV_PI;
}
__device__ __forceinline__ float3 env_dir(const SlotParams& S, float u, float v) {
    const float ph = (0.5f - u) * CWPB_TWO_PI + S.envRot, th = v * CWPB_PI, st = sinf(th);
    return f3(st * cosf(ph), st * sinf(ph), cosf(th));
}
__device__ __forceinline__ void env_texel(const SlotParams& S, float3 d, int& x, int& y, float& v) {
    float u; env_uv(S, d, u, v);
    x = min((int)(u * S.envW), S.envW - 1); y = min((int)(v * S.envH), S.envH - 1);
}
// solid-angle density of sampling texel (x, y) at polar coordinate v: its probability over its solid angle
__device__ __forceinline__ float env_pdf_texel(const SlotParams& S, int x, int y, float v) {
    const float* cr = S.envCond + (size_t)y * (S.envW + 1);
    const float puv = (S.envMarg[y + 1] - S.envMarg[y]) * (cr[x + 1] - cr[x]) * S.envW * S.envH;
    const float st = sinf(v * CWPB_PI);
    return st > 0.f ? puv / (2.f * CWPB_PI * CWPB_PI * st) : 0.f;
}
__device__ __forceinline__ float3 env_radiance(const SlotParams& S, float3 d) {
    int x, y; float v; env_texel(S, d, x, y, v);
    const float4 t = S.envTex[(size_t)y * S.envW + x];
    return f3(t.x, t.y, t.z);
}
__device__ __forceinline__ float3 uniform_sphere(float u0, float u1) {   // core/sampling.h:55-58
    const float z = 1.f - 2.f * u0, r = sqrtf(fmaxf(0.f, 1.f - z * z)), ph = CWPB_TWO_PI * u1;
    return f3(r * cosf(ph), r * sinf(ph), z);
}
// largest i in [0, n) with cdf[i] <= u (cdf: n + 1 entries from 0 to 1)
__device__ __forceinline__ int cdf_find(const float* cdf, int n, float u) {
    int lo = 0, hi = n;
    while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (cdf[mid] <= u) lo = mid; else hi = mid; }
    return lo;
}

// queue entry k: o = (origin, tmin), d = (direction, tmax), scene id = slot, T = (throughput, pdf of the last BSDF
// sample or 0), info = (slot, pixel, sample, depth)
struct RayQueue { float4* o; float4* d; int* sc; float4* T; int4* info; };
// shadow entry: o, d, scene id = slot, c = (contribution, pixel bits), slot
struct ShadowQueue { float4* o; float4* d; int* sc; float4* c; };
// per-slot counters: [0] closest rays shaded, [1] shadow rays, [2] paths finished
static constexpr int kSlotCounters = 4;

__device__ __forceinline__ unsigned lanes_lt() { unsigned m; asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m)); return m; }
__device__ __forceinline__ float rnd_s(unsigned seed, unsigned pix, unsigned smp, unsigned depth, unsigned dim) { return sample01(pix, smp, depth, dim, seed); }

// paths j of a request: pixel (8 x 4 tiles when the image allows, else row-major) = j mod N, sample = j / N
__device__ __forceinline__ int serve_pixel(int j, int w, int h) {
    if ((w & 7) | (h & 3)) return j;
    const int t = j >> 5, r = j & 31, tilesX = w >> 3;
    return ((t / tilesX) * 4 + (r >> 3)) * w + (t % tilesX) * 8 + (r & 7);
}

// chunk c: slot, first path index, count, queue position of its first path (ascending). Camera rays as k_raygen
// (render/wavefront.cu:42-58): box or Blackman-Harris pixel filter (ftab: its inverse CDF), thin lens, near clip.
__global__ void k_serve_raygen(const int4* __restrict__ chunks, int nChunks, int total, const SlotParams* __restrict__ slots, RayQueue q, int base,
                               const float* __restrict__ ftab) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    int lo = 0, hi = nChunks - 1;
    while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (__ldg(&chunks[mid].w) <= t) lo = mid; else hi = mid - 1; }
    const int4 c = chunks[lo];
    const int slot = c.x, j = c.y + (t - c.w);
    const SlotParams& S = slots[slot];
    const cwp_camera& C = S.cam;
    const int pix = serve_pixel(j % S.N, C.w, C.h); const unsigned smp = (unsigned)(j / S.N);
    const int x = pix % C.w, y = pix / C.w;
    const float u0 = rnd_s(S.seed, pix, smp, 0, 0), u1 = rnd_s(S.seed, pix, smp, 0, 1);
    float jx, jy;
    if (S.filterBh) { jx = table_lookup(ftab, CWP_FILTER_TABLE, u0); jy = table_lookup(ftab, CWP_FILTER_TABLE, u1); }
    else { jx = u0 - 0.5f; jy = u1 - 0.5f; }
    const float dx = (x + 0.5f + jx - C.px) / C.fx, dy = -(y + 0.5f + jy - C.py) / C.fy;
    const float3 ax = f3(C.ax[0], C.ax[1], C.ax[2]), ay = f3(C.ay[0], C.ay[1], C.ay[2]), az = f3(C.az[0], C.az[1], C.az[2]), pos = f3(C.pos[0], C.pos[1], C.pos[2]);
    float3 d = normalize(ax * dx + ay * dy - az), o = pos;
    if (C.lens_r > 0.f) {   // thin lens: origin on the lens disk, aimed at the pinhole ray's point on the focal plane
        float lx, ly; disk_map(rnd_s(S.seed, pix, smp, 0, 2), rnd_s(S.seed, pix, smp, 0, 3), lx, ly);
        const float3 pf = pos + (ax * dx + ay * dy - az) * C.focus_d;
        o = pos + ax * (lx * C.lens_r) + ay * (ly * C.lens_r);
        d = normalize(pf - o);
    }
    const int k = base + t;
    q.o[k] = make_float4(o.x, o.y, o.z, S.nearClip); q.d[k] = make_float4(d.x, d.y, d.z, 1e30f); q.sc[k] = slot;
    q.T[k] = make_float4(1.f, 1.f, 1.f, 0.f); q.info[k] = make_int4(slot, pix, (int)smp, 0);
}

struct ShadeArgs {
    int n; RayQueue in, out; ShadowQueue sq;
    const float4* hits; const int* hinst; const cwp_instance* inst; const float4* tris;
    const cwp_material* mats; int nMats; const int* meshMat; const SlotParams* slots; int gdEnergy;
    // material textures (mtex null: none): texture objects, bindings per material, per-triangle uvs / tangents by
    // mesh-local index from each mesh's first triangle
    const cudaTextureObject_t* texObj; const cwp_material_textures* mtex; int nMtex; const float4* uvs; const float4* tans; const int* meshFirst;
    const float4* nrm;   // corner normals by global triangle id (3 float4 each), or null: flat shading
    int* cnt;          // [0] next queue length, [1] shadow queue length
    int* slotCnt;      // kSlotCounters per slot
};

// per-slot counts of this warp's lanes: lanes are grouped by slot, and each group's lowest lane adds the group's counts
__device__ __forceinline__ void slot_counts(int* slotCnt, int slot, bool valid, bool traced, bool shadow, bool ended) {
    const unsigned peers = __match_any_sync(0xffffffffu, valid ? slot : -1);
    const unsigned hasT = __ballot_sync(0xffffffffu, traced) & peers, hasS = __ballot_sync(0xffffffffu, shadow) & peers, hasE = __ballot_sync(0xffffffffu, ended) & peers;
    if (valid && (int)(threadIdx.x & 31) == __ffs(peers) - 1) {
        if (hasT) atomicAdd(&slotCnt[kSlotCounters * slot + 0], __popc(hasT));
        if (hasS) atomicAdd(&slotCnt[kSlotCounters * slot + 1], __popc(hasS));
        if (hasE) atomicAdd(&slotCnt[kSlotCounters * slot + 2], __popc(hasE));
    }
}

__device__ __forceinline__ int warp_slot(int* counter, bool want) {
    const unsigned m = __ballot_sync(0xffffffffu, want);
    if (!m) return -1;
    const int leader = __ffs(m) - 1, lane = threadIdx.x & 31;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    return want ? base + __popc(m & lanes_lt()) : -1;
}

__device__ __forceinline__ void add_rgb(float4* accum, int pix, float3 c) { atomicAdd(accum + pix, make_float4(c.x, c.y, c.z, 0.f)); }

// ---------------- material textures (render/wavefront.cu:198-204, 252-270) ----------------
// (u, v) of a hit from the corner uvs: b1, b2 = barycentric weights of corners 1 and 2
__device__ __forceinline__ float2 tri_uv(const float4* uvs, int64_t t, float b1, float b2) {
    const float4 p = uvs[2 * t], q = uvs[2 * t + 1]; const float b0 = 1.f - b1 - b2;
    return make_float2(p.x * b0 + p.z * b1 + q.x * b2, p.y * b0 + p.w * b1 + q.y * b2);
}
// images are stored top row first and uvs have v up
__device__ __forceinline__ float4 tex_rgba(cudaTextureObject_t o, float2 uv) { return tex2D<float4>(o, uv.x, 1.f - uv.y); }
__device__ __forceinline__ float tex_ch(float4 c, int ch) { return ch == 0 ? c.x : ch == 1 ? c.y : ch == 2 ? c.z : c.w; }
__device__ __forceinline__ float3 xf_vec(const float* m, float3 v) {   // the linear part of 3x4 rows m
    return f3(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[4] * v.x + m[5] * v.y + m[6] * v.z, m[8] * v.x + m[9] * v.y + m[10] * v.z);
}

// The material of a hit with its textures applied (glTF semantics: the images multiply the factors), and the shading
// normal ns (in: the geometric normal ng0; out: perturbed by a normal image in the corner tangents' frame).
// Returns whether a normal image perturbed ns.
__device__ __forceinline__ bool apply_textures(const ShadeArgs& a, int mid, const cwp_instance& I, int tri, float hu, float hv, cwp_material& M, float3& ns) {
    if (!a.mtex || mid >= a.nMtex) return false;
    const cwp_material_textures X = a.mtex[mid];
    if (X.base_color < 0 && X.emission < 0 && X.normal < 0 && X.metallic < 0 && X.roughness < 0) return false;
    const int64_t t = (int64_t)__ldg(a.meshFirst + I.mesh) + __float_as_int(__ldg(a.tris + 3 * (size_t)tri).w);   // mesh-local triangle id
    const float2 uv = tri_uv(a.uvs, t, hu, hv);
    if (X.base_color >= 0) { const float4 c = tex_rgba(a.texObj[X.base_color], uv); M.base_color[0] *= c.x; M.base_color[1] *= c.y; M.base_color[2] *= c.z; }
    if (X.emission >= 0) { const float4 c = tex_rgba(a.texObj[X.emission], uv); M.emission[0] *= c.x; M.emission[1] *= c.y; M.emission[2] *= c.z; }
    if (X.metallic >= 0) M.metallic *= tex_ch(tex_rgba(a.texObj[X.metallic], uv), X.metallic_ch);
    if (X.roughness >= 0) M.roughness *= tex_ch(tex_rgba(a.texObj[X.roughness], uv), X.roughness_ch);
    if (X.normal >= 0 && a.tans) {   // tangent-space normal: n = T x + B y + N z, B = sign * (N x T)
        const float w0 = 1.f - hu - hv;
        const float4 t0 = a.tans[3 * t], t1 = a.tans[3 * t + 1], t2 = a.tans[3 * t + 2];
        float3 tg = f3(t0.x, t0.y, t0.z) * w0 + f3(t1.x, t1.y, t1.z) * hu + f3(t2.x, t2.y, t2.z) * hv;
        const float sg = ((t0.w * w0 + t1.w * hu + t2.w * hv) < 0.f ? -1.f : 1.f) * I.det_sign;
        tg = xf_vec(I.fwd, tg);
        tg = tg - ns * dot(ns, tg);
        const float tl = length(tg);
        if (tl > 0.f) {
            tg = tg * (1.f / tl);
            const float3 bt = cross(ns, tg) * sg;
            const float4 c = tex_rgba(a.texObj[X.normal], uv);
            const float3 nm = tg * ((2.f * c.x - 1.f) * X.normal_scale) + bt * ((2.f * c.y - 1.f) * X.normal_scale) + ns * (2.f * c.z - 1.f);
            const float nl = length(nm);
            if (nl > 0.f) { ns = nm * (1.f / nl); return true; }
        }
    }
    return false;
}

// 8 resident blocks per SM (64 registers, a few spills): the kernel stalls on instruction fetch under divergence, and
// more warps hide it; measured 17% faster than the 96-register form on the mixed request stream
#ifndef CWPB_SHADE_MINB
#define CWPB_SHADE_MINB 8
#endif
__global__ void __launch_bounds__(128, CWPB_SHADE_MINB) k_serve_shade(const ShadeArgs a) {
    const int stride = gridDim.x * blockDim.x;
    for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < a.n; base += stride) {
        const int k = base + (threadIdx.x & 31);
        const bool valid = k < a.n;
        int slot = 0, pix = 0, depth = 0; unsigned smp = 0;
        bool ended = false, wantShadow = false, wantCont = false;
        float3 T = f3(0.f, 0.f, 0.f), so = T, sd = T, contrib = T, co = T, cd = T; float cpdf = 0.f, stmax = 1e30f;
        if (valid) {
            const int4 info = a.in.info[k];
            slot = info.x; pix = info.y; smp = (unsigned)info.z; depth = info.w;
            const float4 T4 = a.in.T[k]; T = f3(T4.x, T4.y, T4.z);
            const SlotParams& S = a.slots[slot];
            const float4 O = a.in.o[k], D = a.in.d[k], H = a.hits[k];
            const float3 d = f3(D.x, D.y, D.z);
            const int tri = __float_as_int(H.w);
            if (tri < 0) {   // miss: the environment, weighted against its light sampling, or the constant sky
                float3 L = S.sky;
                if (S.envTex) {
                    int x, y; float v; env_texel(S, d, x, y, v);
                    const float4 t4 = S.envTex[(size_t)y * S.envW + x];
                    L = f3(t4.x, t4.y, t4.z);
                    if (T4.w > 0.f) {   // T.w: pdf of the last BSDF sample (0: camera ray or a delta lobe, counted fully)
                        if (S.lightMode == CWP_LIGHT_NEE) L = f3(0.f, 0.f, 0.f);
                        else if (S.lightMode == CWP_LIGHT_MIS) L = L * mis_power(T4.w, S.pEnv * (S.envUniform ? 0.25f * CWPB_INV_PI : env_pdf_texel(S, x, y, v)));
                    }
                }
                add_rgb(S.accum, pix, T * L);
                ended = true;
            } else {
                const cwp_instance& I = a.inst[a.hinst[k]];
                const float4 e1 = __ldg(a.tris + 3 * (size_t)tri + 1), e2 = __ldg(a.tris + 3 * (size_t)tri + 2);
                const float3 no = cross(f3(e1.x, e1.y, e1.z), f3(e2.x, e2.y, e2.z));
                // object -> world normal: inverse transpose, orientation by the sign of det(fwd)
                const float3 nw = f3(I.inv[0] * no.x + I.inv[4] * no.y + I.inv[8] * no.z, I.inv[1] * no.x + I.inv[5] * no.y + I.inv[9] * no.z,
                                     I.inv[2] * no.x + I.inv[6] * no.y + I.inv[10] * no.z);
                const float3 ng0 = normalize(nw) * I.det_sign;
                const int mid = min(max(__ldg(a.meshMat + I.mesh) + __float_as_int(e1.w), 0), a.nMats - 1);
                cwp_material M = a.mats[mid];
                float3 nsw = ng0;   // shading normal before orientation
                if (a.nrm) {   // interpolated corner normals by the inverse transpose, turned to the geometric normal's side
                    const int64_t t = (int64_t)__ldg(a.meshFirst + I.mesh) + __float_as_int(__ldg(a.tris + 3 * (size_t)tri).w);
                    const float4 n0 = __ldg(a.nrm + 3 * t), n1 = __ldg(a.nrm + 3 * t + 1), n2 = __ldg(a.nrm + 3 * t + 2);
                    const float3 nn = f3(n0.x, n0.y, n0.z) * (1.f - H.y - H.z) + f3(n1.x, n1.y, n1.z) * H.y + f3(n2.x, n2.y, n2.z) * H.z;
                    const float3 nt = f3(I.inv[0] * nn.x + I.inv[4] * nn.y + I.inv[8] * nn.z, I.inv[1] * nn.x + I.inv[5] * nn.y + I.inv[9] * nn.z,
                                         I.inv[2] * nn.x + I.inv[6] * nn.y + I.inv[10] * nn.z);
                    const float l = length(nt);
                    if (l > 0.f) nsw = nt * (1.f / l);
                    if (dot(nsw, ng0) < 0.f) nsw = -nsw;
                }
                const float3 nsU = nsw;   // the normal before a normal image (the bump-terminator term)
                const bool mapped = apply_textures(a, mid, I, tri, H.y, H.z, M, nsw);
                const float3 p = f3(O.x, O.y, O.z) + d * H.x;
                const float3 em = mat_v3(M.emission);
                if (em.x > 0.f || em.y > 0.f || em.z > 0.f) {   // two-sided emission, weighted against light sampling of this triangle
                    float w = 1.f;
                    if (T4.w > 0.f) {
                        if (S.lightMode == CWP_LIGHT_NEE) w = 0.f;
                        else if (S.lightMode == CWP_LIGHT_MIS) {
                            const float cl = fabsf(dot(ng0, d)), pa = S.nEm > 0 ? __ldg(S.matPdf + mid) : 0.f;
                            w = mis_power(T4.w, cl > 0.f ? S.pTri * pa * H.x * H.x / cl : 0.f);
                        }
                    }
                    if (w > 0.f) add_rgb(S.accum, pix, T * em * w);
                }
                bool alive = depth <= S.maxDepth;
                if (alive && S.rr && depth >= S.rrDepth) {   // Russian roulette: survive with max(T) in [0.05, 1]
                    const float qs = fminf(fmaxf(maxc(T), 0.05f), 1.f);
                    if (rnd_s(S.seed, pix, smp, (unsigned)depth + 1u, 6) >= qs) alive = false;
                    else T = T * (1.f / qs);
                }
                if (!alive) ended = true;
                else {
                    const bool front = dot(ng0, d) < 0.f;
                    const float3 ng = front ? ng0 : -ng0;
                    float3 ns = front ? nsw : -nsw;
                    const float3 wo = -d;
                    if (dot(ns, wo) <= 1e-6f) ns = ng;
                    float3 tx, ty; frame_of(ns, tx, ty);
                    const float3 woL = f3(dot(wo, tx), dot(wo, ty), dot(wo, ns));
                    float3 nrL = f3(0.f, 0.f, 1.f);   // the unperturbed normal in the shading frame: bump-terminator shadowing
                    if (S.bumpShadow && mapped) {
                        const float3 nu = front ? nsU : -nsU;
                        nrL = f3(dot(nu, tx), dot(nu, ty), dot(nu, ns));
                        if (!(nrL.z > 0.f)) nrL = f3(0.f, 0.f, 1.f);
                    }
                    const float eta = front ? M.ior : 1.f / M.ior;
                    const float3 up = p + ng * S.eps, dn = p - ng * S.eps;
                    const unsigned dr = (unsigned)depth + 1u;
                    const float ux1 = rnd_s(S.seed, pix, smp, dr, 7), ux2 = sample01(pix, smp, dr, 7, S.seed ^ 0x68E31DA4u);
                    if (has_non_delta(M)) {
                        // one light sample: the light type by its probability, a triangle by power (a uniform point on
                        // it), an environment texel by luminance x sin(theta); weighted against BSDF sampling by the
                        // power heuristic (the sun, a near-delta cone, and NEE mode: weight 1)
                        const float us = rnd_s(S.seed, pix, smp, dr, 5), u2 = rnd_s(S.seed, pix, smp, dr, 2), u3 = rnd_s(S.seed, pix, smp, dr, 3);
                        float3 l = f3(0.f, 0.f, 1.f), Le = f3(0.f, 0.f, 0.f); float pl = 0.f, tmax = 1e30f; bool isSun = false, ok = false;
                        int side = 0;   // +1 / -1: the origin side fixed by a triangle sample
                        if (us < S.pSun) { l = cone_dir(S.sunTo, S.sunCos, u2, u3); Le = S.sunE; pl = S.pSun; isSun = true; ok = true; }
                        else if (us < S.pSun + S.pTri) {
                            const int e = cdf_find(S.emCdf, S.nEm, fminf((us - S.pSun) / S.pTri, 0.99999994f));
                            const float4 a0 = S.emTris[3 * e], a1 = S.emTris[3 * e + 1], a2 = S.emTris[3 * e + 2];
                            const float su = sqrtf(u2);
                            const float3 pL = f3(a0.x, a0.y, a0.z) + f3(a1.x, a1.y, a1.z) * (su * (1.f - u3)) + f3(a2.x, a2.y, a2.z) * (su * u3);
                            const float3 nL = normalize(cross(f3(a1.x, a1.y, a1.z), f3(a2.x, a2.y, a2.z)));
                            // connect from the shadow ray's own offset origin, so that tmax ends just short of the point
                            side = dot(ng, pL - p) > 0.f ? 1 : -1;
                            const float3 dv = pL - (side > 0 ? up : dn);
                            const float dist2 = dot(dv, dv), dist = sqrtf(dist2);
                            if (dist > 0.f) {
                                l = dv * (1.f / dist);
                                const float cl = fabsf(dot(nL, l));
                                if (cl > 0.f) {
                                    const int lm = __float_as_int(a1.w);
                                    pl = S.pTri * __ldg(S.matPdf + lm) * dist2 / cl; Le = mat_v3(a.mats[lm].emission); tmax = dist * (1.f - 1e-3f); ok = true;
                                    if (a.mtex && lm < a.nMtex && a.mtex[lm].emission >= 0) {
                                        const float4 c = tex_rgba(a.texObj[a.mtex[lm].emission], tri_uv(a.uvs, __float_as_int(a0.w), su * (1.f - u3), su * u3));
                                        Le = Le * f3(c.x, c.y, c.z);
                                    }
                                }
                            }
                        } else if (S.pEnv > 0.f && S.envUniform) {
                            l = uniform_sphere(u2, u3); pl = S.pEnv * (0.25f * CWPB_INV_PI); Le = env_radiance(S, l); ok = true;
                        } else if (S.pEnv > 0.f) {
                            const float ue = fminf((us - S.pSun - S.pTri) / S.pEnv, 0.99999994f);
                            const int y = cdf_find(S.envMarg, S.envH, ue);
                            const float* cr = S.envCond + (size_t)y * (S.envW + 1);
                            const int x = cdf_find(cr, S.envW, u2);
                            const float v = (y + u3) / S.envH, w0 = cr[x + 1] - cr[x];
                            float u = (x + 0.5f) / S.envW;
                            if (w0 > 0.f) u = (x + fminf((u2 - cr[x]) / w0, 0.99999994f)) / S.envW;   // the rest of u2 within the texel
                            l = env_dir(S, u, v);
                            const float pe = env_pdf_texel(S, x, y, v);
                            if (pe > 0.f) { pl = S.pEnv * pe; const float4 t4 = S.envTex[(size_t)y * S.envW + x]; Le = f3(t4.x, t4.y, t4.z); ok = true; }
                        }
                        const float3 lL = f3(dot(l, tx), dot(l, ty), dot(l, ns));
                        const float gl = dot(ng, l);
                        if (ok && lL.z != 0.f && (gl > 0.f) == (lL.z > 0.f)) {
                            const BsdfValue e = bsdf_eval(M, woL, lL, eta, a.gdEnergy, ux1, ux2, nrL);
                            const float w = (isSun || S.lightMode == CWP_LIGHT_NEE) ? 1.f : mis_power(pl, e.pdf);
                            contrib = T * e.f * Le * (fabsf(lL.z) * w / pl);
                            if (contrib.x > 0.f || contrib.y > 0.f || contrib.z > 0.f) {
                                wantShadow = true; so = (side ? side > 0 : gl > 0.f) ? up : dn; sd = l; stmax = tmax;
                            }
                        }
                    }
                    float3 wiL, wgt; float pdf;
                    if (bsdf_sample(M, woL, eta, a.gdEnergy, ux1, ux2, rnd_s(S.seed, pix, smp, dr, 4), rnd_s(S.seed, pix, smp, dr, 0), rnd_s(S.seed, pix, smp, dr, 1), wiL, wgt, pdf, nrL)) {
                        const float3 wi = normalize(tx * wiL.x + ty * wiL.y + ns * wiL.z);
                        const float gi = dot(ng, wi);
                        if (gi != 0.f && (gi > 0.f) == (wiL.z > 0.f)) {
                            T = T * wgt;
                            if (maxc(T) > 0.f) { wantCont = true; co = gi > 0.f ? up : dn; cd = wi; cpdf = pdf; }
                        }
                    }
                    if (!wantCont) ended = true;
                }
            }
        }
        slot_counts(a.slotCnt, slot, valid, valid, wantShadow, ended);
        const int sp = warp_slot(a.cnt + 1, wantShadow);
        if (sp >= 0) {
            a.sq.o[sp] = make_float4(so.x, so.y, so.z, 0.f); a.sq.d[sp] = make_float4(sd.x, sd.y, sd.z, stmax); a.sq.sc[sp] = slot;
            a.sq.c[sp] = make_float4(contrib.x, contrib.y, contrib.z, __int_as_float(pix));
        }
        const int cp = warp_slot(a.cnt, wantCont);
        if (cp >= 0) {
            a.out.o[cp] = make_float4(co.x, co.y, co.z, 0.f); a.out.d[cp] = make_float4(cd.x, cd.y, cd.z, 1e30f); a.out.sc[cp] = slot;
            a.out.T[cp] = make_float4(T.x, T.y, T.z, cpdf); a.out.info[cp] = make_int4(slot, pix, (int)smp, depth + 1);
        }
    }
}

// unoccluded shadow rays add their contributions; the count is read on the device (grid-stride)
__global__ void k_serve_shadow_accum(const int* nDev, ShadowQueue sq, const int* __restrict__ occ, const SlotParams* __restrict__ slots) {
    const int n = *nDev;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        if (occ[k] >= 0) continue;
        const float4 c = sq.c[k];
        add_rgb(slots[sq.sc[k]].accum, __float_as_int(c.w), f3(c.x, c.y, c.z));
    }
}

// ---------------- regrouping the queue by request ----------------
// The continuations of a step come out interleaved across requests; a counting sort by slot (histogram, scan,
// scatter of the 68-byte entries, counts read on the device) makes the rays a warp fetches belong to one scene, so the
// traversal of a step touches one scene's TLAS and BLAS at a time instead of all of them at once.
__global__ void __launch_bounds__(256) k_slot_hist(const int* __restrict__ nDev, const int4* __restrict__ info, int* hist, int nSlots) {
    extern __shared__ int h[];
    for (int i = threadIdx.x; i < nSlots; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const int n = *nDev;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) atomicAdd_block(&h[__ldg(&info[k].x)], 1);
    __syncthreads();
    for (int i = threadIdx.x; i < nSlots; i += blockDim.x) if (h[i]) atomicAdd(&hist[i], h[i]);
}
__global__ void __launch_bounds__(1024) k_slot_scan(int* hist, int* cursor, int nSlots) {   // one block, nSlots <= 1024
    __shared__ int v[1024];
    const int i = threadIdx.x, x = i < nSlots ? hist[i] : 0;
    v[i] = x; __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) { const int y = i >= off ? v[i - off] : 0; __syncthreads(); v[i] += y; __syncthreads(); }
    if (i < nSlots) cursor[i] = v[i] - x;
}
__global__ void __launch_bounds__(256) k_slot_scatter(const int* __restrict__ nDev, RayQueue src, RayQueue dst, int* cursor) {
    const int n = *nDev, lane = threadIdx.x & 31;
    for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < n; base += gridDim.x * blockDim.x) {
        const int k = base + lane; const bool ok = k < n;
        const int4 info = ok ? src.info[k] : make_int4(-1, 0, 0, 0);
        const unsigned peers = __match_any_sync(0xffffffffu, info.x);
        const int leader = __ffs(peers) - 1;
        int pos = 0;
        if (ok && lane == leader) pos = atomicAdd(&cursor[info.x], __popc(peers));
        pos = __shfl_sync(0xffffffffu, pos, leader) + __popc(peers & lanes_lt());
        if (ok) { dst.o[pos] = src.o[k]; dst.d[pos] = src.d[k]; dst.sc[pos] = src.sc[k]; dst.T[pos] = src.T[k]; dst.info[pos] = info; }
    }
}

// ---------------- BSDF test kernels ----------------
__global__ void k_bsdf_eval(const cwp_material* mats, const int* mat, const float3* wo, const float3* wi, const float* eta, int gd, const float2* ux,
                            const float3* nr, float4* f, float* pdf, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const BsdfValue e = bsdf_eval(mats[mat[i]], wo[i], wi[i], eta[i], gd, ux[i].x, ux[i].y, nr ? nr[i] : f3(0.f, 0.f, 1.f));
    f[i] = make_float4(e.f.x, e.f.y, e.f.z, 0.f); pdf[i] = e.pdf;
}
__global__ void k_bsdf_sample(const cwp_material* mats, const int* mat, const float3* wo, const float* eta, int gd, const float2* ux, const float3* uvw,
                              const float3* nr, float3* wi, float3* w, float* pdf, int* ok, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 a = f3(0.f, 0.f, 0.f), b = a; float p = 0.f;
    ok[i] = bsdf_sample(mats[mat[i]], wo[i], eta[i], gd, ux[i].x, ux[i].y, uvw[i].x, uvw[i].y, uvw[i].z, a, b, p, nr ? nr[i] : f3(0.f, 0.f, 1.f)) ? 1 : 0;
    wi[i] = a; w[i] = b; pdf[i] = p;
}

}  // namespace cwpb

using namespace cwpb;

struct ServeRequest {
    cwp_request r; int64_t id; int slot = -1;
    double submitMs = 0, admitMs = 0, doneMs = 0;
    int64_t total = 0, issued = 0, finished = 0; double rays = 0, shadow = 0;
    float4* accum = nullptr; bool done = false;
    void* lights = nullptr;   // the request's emissive-triangle tables (pool memory), freed at completion
    // host data prepared at submission (so that admission, on the step's critical path, only copies): the scene's
    // instances at the request's frame and its emissive-triangle tables
    std::vector<cwp_instance> inst; std::vector<float> emT, emC, mlp;
};

struct cwp_server {
    cwp_batch* batch = nullptr; int device = 0;
    cwp_server_options O{};
    cwp_material* mats = nullptr; int nMats = 0; int* meshMat = nullptr;
    std::vector<cwp_material> hMats; EmissiveSet em;   // host materials; the meshes' emissive triangles (object space)
    // scenes: instance descriptors per scene (host)
    std::vector<cwp_instance_desc> desc; std::vector<int> sceneFirst;
    std::vector<float> xf; std::vector<int32_t> xfFirst, xfCount;   // per descriptor: matrices by frame (count 0: animated)
    // per slot: request id or -1, its instances (host) for the TLAS rebuild
    std::vector<int64_t> slotReq; std::vector<std::vector<cwp_instance>> slotInst; std::vector<int> admitted;   // slots admitted since the last TLAS update
    struct EnvMap { float4* tex = nullptr; float* marg = nullptr; float* cond = nullptr; int w = 0, h = 0; };
    std::vector<EnvMap> envs;   // environment maps the requests may name
    // material textures: images (CUDA arrays + texture objects) and the device tables shading reads
    std::vector<cudaArray_t> texArrays; std::vector<cudaTextureObject_t> texObjs;
    cudaTextureObject_t* dTexObj = nullptr; cwp_material_textures* dMtex = nullptr; int nMtex = 0; float4* dUvs = nullptr; float4* dTans = nullptr;
    SlotParams* dSlots = nullptr; int* slotCnt = nullptr; std::vector<int> hSlotCnt;
    float* ftab = nullptr;   // Blackman-Harris pixel-filter inverse CDF (CWP_FILTER_TABLE + 1 floats)
    RayQueue q[2]{}; RayQueue qs{}; int* slotBins = nullptr; ShadowQueue sq{}; float4* hits = nullptr; int* hinst = nullptr; int* occ = nullptr; int* cnt = nullptr; int4* dChunks = nullptr;
    int* hcnt = nullptr;   // pinned: [0..1] counts, then slot counters
    SlotParams* hSlots = nullptr; int4* hChunks = nullptr; bool slotsDirty = false;   // pinned mirrors of dSlots and dChunks
    cudaMemPool_t pool = nullptr;   // request images: freed memory stays in the pool for the next admissions
    double freeAt = -1e30; int64_t freeB = 0; uint64_t freeReserved = 0;   // last device free-memory query and the pool size then
    int cur = 0; int64_t nCur = 0;
    std::deque<int64_t> pending; std::map<int64_t, ServeRequest> reqs; std::vector<int64_t> completed;
    int64_t nextId = 1;
    cudaStream_t st = nullptr;
    cudaStream_t cst = nullptr;   // result copies: completed images, read while the next step runs
    std::chrono::steady_clock::time_point t0;
    std::vector<void*> allocs;
    cudaEvent_t ev[6] = {};   // raygen start, closest start, shade start, shadow start, shadow end, accumulation start
    cwp_server_info info{};
    bool overlap = true;        // a step returns with its launches queued; the next call takes its results
    bool inflight = false; int64_t inflightN = 0; double inflightStart = 0;   // the queued step: rays traced, host start time
};

// one CUDA array and texture object per image: bilinear filtering, wrap addressing, normalised coordinates, 8-bit
// channels read as [0, 1] floats, colour images decoded from sRGB by the texture unit (render/wavefront.cu:535-546)
static void free_textures(std::vector<cudaArray_t>& arrays, std::vector<cudaTextureObject_t>& objs) {
    for (cudaTextureObject_t o : objs) cudaDestroyTextureObject(o);
    for (cudaArray_t a : arrays) cudaFreeArray(a);
    objs.clear(); arrays.clear();
}
static int make_textures(const cwp_texture* tex, int n, std::vector<cudaArray_t>& arrays, std::vector<cudaTextureObject_t>& objs) {
    for (int i = 0; i < n; i++) {
        const cwp_texture& T = tex[i];
        CWPB_CHECK(T.rgba && T.w > 0 && T.h > 0 && T.w <= 32768 && T.h <= 32768 && (T.srgb == 0 || T.srgb == 1) && (T.nearest == 0 || T.nearest == 1),
                   CWP_ERR_INVALID, "texture %d: %dx%d, srgb %d, nearest %d", i, T.w, T.h, T.srgb, T.nearest);
    }
    for (int i = 0; i < n; i++) {
        const cwp_texture& T = tex[i];
        const cudaChannelFormatDesc cd = cudaCreateChannelDesc<uchar4>();
        cudaArray_t arr = nullptr;
        cudaError_t e = cudaMallocArray(&arr, &cd, T.w, T.h);
        if (e == cudaSuccess) arrays.push_back(arr);
        if (e == cudaSuccess) e = cudaMemcpy2DToArray(arr, 0, 0, T.rgba, (size_t)T.w * 4, (size_t)T.w * 4, T.h, cudaMemcpyHostToDevice);
        cudaTextureObject_t o = 0;
        if (e == cudaSuccess) {
            cudaResourceDesc rd; memset(&rd, 0, sizeof rd); rd.resType = cudaResourceTypeArray; rd.res.array.array = arr;
            cudaTextureDesc td; memset(&td, 0, sizeof td);
            td.addressMode[0] = td.addressMode[1] = cudaAddressModeWrap; td.filterMode = T.nearest ? cudaFilterModePoint : cudaFilterModeLinear;
            td.readMode = cudaReadModeNormalizedFloat; td.normalizedCoords = 1; td.sRGB = T.srgb;
            e = cudaCreateTextureObject(&o, &rd, &td, nullptr);
        }
        if (e != cudaSuccess) { free_textures(arrays, objs); return set_error(e == cudaErrorMemoryAllocation ? CWP_ERR_NOMEM : CWP_ERR_CUDA, "texture %d: %s", i, cudaGetErrorString(e)); }
        objs.push_back(o);
    }
    return CWP_OK;
}

static double now_ms(const cwp_server* s) { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - s->t0).count(); }

extern "C" double cwp_server_clock_ms(const cwp_server* s) { return s ? now_ms(s) : 0.0; }

extern "C" void cwp_server_destroy(cwp_server* s) {
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->st) cudaStreamSynchronize(s->st);   // a queued step included
    if (s->cst) cudaStreamSynchronize(s->cst);
    for (auto& kv : s->reqs) {
        if (kv.second.accum) cudaFreeAsync(kv.second.accum, s->st);
        if (kv.second.lights) cudaFreeAsync(kv.second.lights, s->st);
    }
    if (s->st) cudaStreamSynchronize(s->st);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    for (auto& e : s->envs) { cudaFree(e.tex); cudaFree(e.marg); cudaFree(e.cond); }
    free_textures(s->texArrays, s->texObjs);
    cudaFree(s->dTexObj); cudaFree(s->dMtex); cudaFree(s->dUvs); cudaFree(s->dTans);
    for (void* p : s->allocs) cudaFree(p);
    if (s->hcnt) cudaFreeHost(s->hcnt);
    if (s->hSlots) cudaFreeHost(s->hSlots);
    if (s->hChunks) cudaFreeHost(s->hChunks);
    for (cudaEvent_t e : s->ev) if (e) cudaEventDestroy(e);
    if (s->st) cudaStreamDestroy(s->st);
    if (s->cst) cudaStreamDestroy(s->cst);
    delete s;
}

static int server_create(cwp_batch* b, const cwp_material* mats, int n, const int* meshBase, const cwp_server_options* o, cwp_server* s) {
    s->batch = b; s->device = batch_device(b);
    s->O.max_paths = o && o->max_paths > 0 ? o->max_paths : (8ll << 20);
    s->O.max_requests = o && o->max_requests > 0 ? o->max_requests : 64;
    s->O.gd_energy = o ? o->gd_energy : 1;
    s->O.hbm_reserve = o && o->hbm_reserve > 0 ? o->hbm_reserve : (1ll << 30);
    s->O.regroup = o && o->regroup < 0 ? -1 : 1;
    s->O.policy = o ? o->policy : 0;
    s->overlap = !(o && o->overlap < 0);
    CWPB_CHECK(s->O.policy == 0 || s->O.policy == 1, CWP_ERR_INVALID, "policy %d is not 0 or 1", s->O.policy);
    CWPB_CHECK(s->O.max_paths < (1ll << 30), CWP_ERR_INVALID, "max_paths %lld above 2^30", (long long)s->O.max_paths);
    CWPB_CHECK(s->O.max_requests <= 1024, CWP_ERR_INVALID, "max_requests %d above 1024", s->O.max_requests);
    CWPB_CHECK(mats && n >= 1 && meshBase, CWP_ERR_INVALID, "no materials");
    const int nMesh = batch_mesh_count(b);
    for (int m = 0; m < nMesh; m++) CWPB_CHECK(meshBase[m] >= 0 && meshBase[m] < n, CWP_ERR_INVALID, "mesh %d material base %d out of range", m, meshBase[m]);
    for (int i = 0; i < n; i++) CWPB_CHECK(mats[i].ior > 0.f && mats[i].roughness >= 0.f && mats[i].metallic >= 0.f && mats[i].metallic <= 1.f &&
                                           mats[i].transmission >= 0.f && mats[i].transmission <= 1.f, CWP_ERR_INVALID, "material %d out of range", i);
    CWPB_CUDA(cudaSetDevice(s->device));
    CWPB_CUDA(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
    CWPB_CUDA(cudaStreamCreateWithFlags(&s->cst, cudaStreamNonBlocking));
    for (cudaEvent_t& e : s->ev) CWPB_CUDA(cudaEventCreate(&e));
    auto alloc = [&](void** p, size_t bytes) -> int { CWPB_CUDA(cudaMalloc(p, bytes)); s->allocs.push_back(*p); return CWP_OK; };
    const size_t P = (size_t)s->O.max_paths, R = (size_t)s->O.max_requests;
    int rc = alloc((void**)&s->mats, (size_t)n * sizeof(cwp_material));
    if (!rc) rc = alloc((void**)&s->meshMat, (size_t)nMesh * sizeof(int));
    for (int k = 0; k < 2 && !rc; k++) {
        rc = alloc((void**)&s->q[k].o, P * 16); if (!rc) rc = alloc((void**)&s->q[k].d, P * 16); if (!rc) rc = alloc((void**)&s->q[k].sc, P * 4);
        if (!rc) rc = alloc((void**)&s->q[k].T, P * 16); if (!rc) rc = alloc((void**)&s->q[k].info, P * 16);
    }
    if (!rc) { rc = alloc((void**)&s->qs.o, P * 16); if (!rc) rc = alloc((void**)&s->qs.d, P * 16); if (!rc) rc = alloc((void**)&s->qs.sc, P * 4);
               if (!rc) rc = alloc((void**)&s->qs.T, P * 16); if (!rc) rc = alloc((void**)&s->qs.info, P * 16); }
    if (!rc) rc = alloc((void**)&s->slotBins, 2 * R * sizeof(int));
    if (!rc) rc = alloc((void**)&s->sq.o, P * 16); if (!rc) rc = alloc((void**)&s->sq.d, P * 16); if (!rc) rc = alloc((void**)&s->sq.sc, P * 4);
    if (!rc) rc = alloc((void**)&s->sq.c, P * 16);
    if (!rc) rc = alloc((void**)&s->hits, P * 16); if (!rc) rc = alloc((void**)&s->hinst, P * 4); if (!rc) rc = alloc((void**)&s->occ, P * 4);
    if (!rc) rc = alloc((void**)&s->cnt, 4 * sizeof(int));
    if (!rc) rc = alloc((void**)&s->dSlots, R * sizeof(SlotParams));
    if (!rc) rc = alloc((void**)&s->slotCnt, R * kSlotCounters * sizeof(int));
    if (!rc) rc = alloc((void**)&s->dChunks, (R + 1) * sizeof(int4));
    if (!rc) rc = alloc((void**)&s->ftab, (CWP_FILTER_TABLE + 1) * sizeof(float));
    if (rc) return rc;
    {
        cwp_params pd;
        if (int r2 = cwp_params_defaults(&pd)) return r2;
        CWPB_CUDA(cudaMemcpy(s->ftab, pd.ftab, (CWP_FILTER_TABLE + 1) * sizeof(float), cudaMemcpyHostToDevice));
    }
    CWPB_CUDA(cudaMallocHost(&s->hcnt, (4 + R * kSlotCounters) * sizeof(int)));
    CWPB_CUDA(cudaMallocHost(&s->hSlots, R * sizeof(SlotParams))); memset(s->hSlots, 0, R * sizeof(SlotParams));
    CWPB_CUDA(cudaMallocHost(&s->hChunks, (R + 1) * sizeof(int4)));
    {
        cudaMemPoolProps pp{};
        pp.allocType = cudaMemAllocationTypePinned; pp.location.type = cudaMemLocationTypeDevice; pp.location.id = s->device;
        CWPB_CUDA(cudaMemPoolCreate(&s->pool, &pp));
        uint64_t keep = UINT64_MAX;   // never hand freed images back to the driver between steps
        CWPB_CUDA(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    CWPB_CUDA(cudaMemcpy(s->mats, mats, (size_t)n * sizeof(cwp_material), cudaMemcpyHostToDevice));
    CWPB_CUDA(cudaMemcpy(s->meshMat, meshBase, (size_t)nMesh * sizeof(int), cudaMemcpyHostToDevice));
    CWPB_CUDA(cudaMemset(s->slotCnt, 0, R * kSlotCounters * sizeof(int)));
    s->nMats = n; s->hMats.assign(mats, mats + n);
    if (std::any_of(mats, mats + n, is_emissive)) {   // emissive triangles of every mesh, from the batch's input triangles
        std::vector<float4> soup((size_t)3 * batch_tri_count(b));
        CWPB_CUDA(cudaMemcpy(soup.data(), batch_tri_soup(b), soup.size() * sizeof(float4), cudaMemcpyDeviceToHost));
        emissive_set((const float*)soup.data(), batch_mesh_first_host(b), nMesh, meshBase, mats, n, s->em);
    }
    s->slotReq.assign(R, -1); s->slotInst.assign(R, {}); s->hSlotCnt.assign(R * kSlotCounters, 0);
    s->t0 = std::chrono::steady_clock::now();
    return CWP_OK;
}

extern "C" int cwp_server_create(cwp_batch* b, const cwp_material* mats, int32_t n, const int32_t* meshBase, const cwp_server_options* o, cwp_server** out) {
    CWPB_CHECK(b && out, CWP_ERR_INVALID, "NULL argument");
    *out = nullptr;
    cwp_server* s = new cwp_server();
    if (int rc = server_create(b, mats, n, meshBase, o, s)) { cwp_server_destroy(s); return rc; }
    *out = s;
    return CWP_OK;
}

extern "C" int cwp_server_set_scenes(cwp_server* s, const cwp_instance_desc* desc, int64_t n, const int32_t* first, int32_t nScenes) {
    CWPB_CHECK(s && first && nScenes >= 1 && (n == 0 || desc), CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(first[0] == 0 && first[nScenes] == n, CWP_ERR_INVALID, "scene offsets do not cover the %lld descriptors", (long long)n);
    for (int k = 0; k < nScenes; k++) CWPB_CHECK(first[k + 1] >= first[k], CWP_ERR_INVALID, "scene offsets decrease at %d", k);
    const int nMesh = batch_mesh_count(s->batch);
    for (int64_t i = 0; i < n; i++) CWPB_CHECK(desc[i].mesh >= 0 && desc[i].mesh < nMesh, CWP_ERR_INVALID, "descriptor %lld: mesh %d out of range", (long long)i, desc[i].mesh);
    CWPB_CHECK(s->reqs.empty(), CWP_ERR_STATE, "scenes change only while no request is queued or running");
    int cap = 1;
    for (int k = 0; k < nScenes; k++) cap = std::max(cap, first[k + 1] - first[k]);
    // one TLAS region per slot, sized for the largest scene: admissions rebuild only the admitted slots' TLAS
    if (int rc = cwp_batch_reserve_scenes(s->batch, s->O.max_requests, cap)) return rc;
    s->desc.assign(desc, desc + n); s->sceneFirst.assign(first, first + nScenes + 1);
    s->xf.clear(); s->xfFirst.clear(); s->xfCount.clear();
    return CWP_OK;
}

extern "C" int cwp_server_set_instance_xforms(cwp_server* s, const float* xforms, const int32_t* firstXf, const int32_t* nXf, int64_t n) {
    CWPB_CHECK(s, CWP_ERR_INVALID, "server is NULL");
    CWPB_CHECK(s->reqs.empty(), CWP_ERR_STATE, "instance matrices change only while no request is queued or running");
    if (!firstXf || !nXf) { s->xf.clear(); s->xfFirst.clear(); s->xfCount.clear(); return CWP_OK; }
    CWPB_CHECK(n == (int64_t)s->desc.size(), CWP_ERR_INVALID, "%lld matrix ranges for %zu descriptors", (long long)n, s->desc.size());
    int64_t total = 0;
    for (int64_t i = 0; i < n; i++) {
        CWPB_CHECK(firstXf[i] >= 0 && nXf[i] >= 0 && (nXf[i] == 0 || xforms), CWP_ERR_INVALID, "descriptor %lld: matrix range %d + %d", (long long)i, firstXf[i], nXf[i]);
        total = std::max<int64_t>(total, (int64_t)firstXf[i] + nXf[i]);
    }
    for (int64_t k = 0; k < 12 * total; k++) CWPB_CHECK(std::isfinite(xforms[k]), CWP_ERR_INVALID, "matrix entry %lld is not finite", (long long)k);
    s->xf.assign(xforms, xforms + 12 * total); s->xfFirst.assign(firstXf, firstXf + n); s->xfCount.assign(nXf, nXf + n);
    return CWP_OK;
}

extern "C" int cwp_server_set_envmaps(cwp_server* s, const cwp_envmap* maps, int32_t n) {
    CWPB_CHECK(s && n >= 0 && (n == 0 || maps), CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(s->reqs.empty(), CWP_ERR_STATE, "environment maps change only while no request is queued or running");
    CWPB_CUDA(cudaSetDevice(s->device));
    std::vector<cwp_server::EnvMap> built;
    auto drop = [&]() { for (auto& e : built) { cudaFree(e.tex); cudaFree(e.marg); cudaFree(e.cond); } };
    for (int i = 0; i < n; i++) {
        const cwp_envmap& m = maps[i];
        CWPB_CHECK(m.rgb && m.w > 0 && m.h > 0 && (int64_t)m.w * m.h < (1ll << 28), CWP_ERR_INVALID, "environment map %d: %dx%d", i, m.w, m.h);
        const size_t nt = (size_t)m.w * m.h;
        std::vector<float> tex(4 * nt), marg((size_t)m.h + 1), cond((size_t)m.h * (m.w + 1));
        if (int rc = cwp_envmap_build(m.rgb, m.w, m.h, m.strength, tex.data(), marg.data(), cond.data())) { drop(); return rc; }
        cwp_server::EnvMap E; E.w = m.w; E.h = m.h;
        cudaError_t e = cudaMalloc(&E.tex, nt * sizeof(float4));
        if (e == cudaSuccess) e = cudaMalloc(&E.marg, marg.size() * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&E.cond, cond.size() * sizeof(float));
        if (e == cudaSuccess) e = cudaMemcpy(E.tex, tex.data(), nt * sizeof(float4), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(E.marg, marg.data(), marg.size() * sizeof(float), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(E.cond, cond.data(), cond.size() * sizeof(float), cudaMemcpyHostToDevice);
        built.push_back(E);
        if (e != cudaSuccess) { drop(); return set_error(e == cudaErrorMemoryAllocation ? CWP_ERR_NOMEM : CWP_ERR_CUDA, "environment map %d: %s", i, cudaGetErrorString(e)); }
    }
    for (auto& e : s->envs) { cudaFree(e.tex); cudaFree(e.marg); cudaFree(e.cond); }
    s->envs = built;
    return CWP_OK;
}

extern "C" int cwp_server_set_textures(cwp_server* s, const cwp_texture* tex, int32_t nTex, const cwp_material_textures* mtex, int32_t nMtex,
                                       const float* uvs, const float* tans) {
    CWPB_CHECK(s && nTex >= 0 && nMtex >= 0 && (nTex == 0 || tex) && (nMtex == 0 || mtex), CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(s->reqs.empty(), CWP_ERR_STATE, "textures change only while no request is queued or running");
    bool used = false;
    for (int m = 0; m < nMtex; m++) {
        const cwp_material_textures& X = mtex[m];
        const int ids[5] = { X.base_color, X.emission, X.normal, X.metallic, X.roughness };
        for (int id : ids) { CWPB_CHECK(id >= -1 && id < nTex, CWP_ERR_INVALID, "material %d: texture %d out of range (%d images)", m, id, nTex); used |= id >= 0; }
        CWPB_CHECK(X.metallic_ch >= 0 && X.metallic_ch < 4 && X.roughness_ch >= 0 && X.roughness_ch < 4, CWP_ERR_INVALID, "material %d: channel out of range", m);
        CWPB_CHECK(std::isfinite(X.normal_scale), CWP_ERR_INVALID, "material %d: normal scale is not finite", m);
    }
    CWPB_CHECK(!used || uvs, CWP_ERR_INVALID, "texture bindings without uvs");
    CWPB_CUDA(cudaSetDevice(s->device));
    std::vector<cudaArray_t> arrays; std::vector<cudaTextureObject_t> objs;
    if (int rc = make_textures(tex, nTex, arrays, objs)) return rc;
    const int64_t nt = batch_tri_count(s->batch);
    cudaTextureObject_t* dObj = nullptr; cwp_material_textures* dM = nullptr; float4* dU = nullptr; float4* dT = nullptr;
    cudaError_t e = cudaSuccess;
    if (nTex) { e = cudaMalloc(&dObj, nTex * sizeof(cudaTextureObject_t)); if (e == cudaSuccess) e = cudaMemcpy(dObj, objs.data(), nTex * sizeof(cudaTextureObject_t), cudaMemcpyHostToDevice); }
    if (e == cudaSuccess && nMtex) { e = cudaMalloc(&dM, nMtex * sizeof(cwp_material_textures)); if (e == cudaSuccess) e = cudaMemcpy(dM, mtex, nMtex * sizeof(cwp_material_textures), cudaMemcpyHostToDevice); }
    if (e == cudaSuccess && used) { e = cudaMalloc(&dU, (size_t)nt * 2 * sizeof(float4)); if (e == cudaSuccess) e = cudaMemcpy(dU, uvs, (size_t)nt * 2 * sizeof(float4), cudaMemcpyHostToDevice); }
    if (e == cudaSuccess && used && tans) { e = cudaMalloc(&dT, (size_t)nt * 3 * sizeof(float4)); if (e == cudaSuccess) e = cudaMemcpy(dT, tans, (size_t)nt * 3 * sizeof(float4), cudaMemcpyHostToDevice); }
    if (e != cudaSuccess) {
        cudaFree(dObj); cudaFree(dM); cudaFree(dU); cudaFree(dT); free_textures(arrays, objs);
        return set_error(e == cudaErrorMemoryAllocation ? CWP_ERR_NOMEM : CWP_ERR_CUDA, "textures: %s", cudaGetErrorString(e));
    }
    free_textures(s->texArrays, s->texObjs);
    cudaFree(s->dTexObj); cudaFree(s->dMtex); cudaFree(s->dUvs); cudaFree(s->dTans);
    s->texArrays = arrays; s->texObjs = objs; s->dTexObj = dObj; s->dMtex = dM; s->nMtex = used ? nMtex : 0; s->dUvs = dU; s->dTans = dT;
    return CWP_OK;
}

__global__ void k_tex_sample(const cudaTextureObject_t* obj, const int* id, const float2* uv, float4* out, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = tex_rgba(obj[id[i]], uv[i]);
}

extern "C" int cwp_texture_sample_batch(const cwp_texture* tex, int32_t nTex, const int32_t* id, const float* uv, float* rgba, int64_t n) {
    CWPB_CHECK(tex && nTex > 0 && id && uv && rgba && n >= 0, CWP_ERR_INVALID, "NULL argument");
    for (int64_t i = 0; i < n; i++) CWPB_CHECK(id[i] >= 0 && id[i] < nTex, CWP_ERR_INVALID, "lookup %lld: texture %d out of range", (long long)i, id[i]);
    if (n == 0) return CWP_OK;
    std::vector<cudaArray_t> arrays; std::vector<cudaTextureObject_t> objs;
    if (int rc = make_textures(tex, nTex, arrays, objs)) return rc;
    cudaTextureObject_t* dObj = nullptr; int* dId = nullptr; float2* dUv = nullptr; float4* dOut = nullptr;
    cudaError_t e = cudaMalloc(&dObj, nTex * sizeof(cudaTextureObject_t));
    if (e == cudaSuccess) e = cudaMalloc(&dId, n * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&dUv, n * sizeof(float2));
    if (e == cudaSuccess) e = cudaMalloc(&dOut, n * sizeof(float4));
    if (e == cudaSuccess) e = cudaMemcpy(dObj, objs.data(), nTex * sizeof(cudaTextureObject_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dId, id, n * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dUv, uv, n * sizeof(float2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) { k_tex_sample<<<(unsigned)((n + 255) / 256), 256>>>(dObj, dId, dUv, dOut, n); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = cudaMemcpy(rgba, dOut, n * sizeof(float4), cudaMemcpyDeviceToHost);
    cudaFree(dObj); cudaFree(dId); cudaFree(dUv); cudaFree(dOut); free_textures(arrays, objs);
    if (e != cudaSuccess) return set_error(CWP_ERR_CUDA, "texture lookups: %s", cudaGetErrorString(e));
    return CWP_OK;
}

// A request's host data, prepared at submission: the instances of its scene at its frame, and (unless it samples the
// BSDF only) the emissive-triangle tables there. Scenes and instance matrices change only while no request is queued,
// so the data stays valid until admission.
static int prepare_request(const cwp_server* s, ServeRequest& q) {
    std::vector<float> xf; std::vector<int> im;
    q.inst.clear();
    for (int i = s->sceneFirst[q.r.scene]; i < s->sceneFirst[q.r.scene + 1]; i++) {
        float m[12]; cwp_instance rec;
        if (!s->xfCount.empty() && s->xfCount[i] > 0) {   // a matrix per frame, the last one held
            const float* x = s->xf.data() + 12 * ((size_t)s->xfFirst[i] + std::min(std::max(q.r.frame, 0), s->xfCount[i] - 1));
            std::copy(x, x + 12, m);
        } else if (int rc = cwp_xform_animate(&s->desc[i], q.r.frame, m)) return rc;
        if (int rc = cwp_instance_from_xform(m, s->desc[i].mesh, &rec)) return rc;
        q.inst.push_back(rec); xf.insert(xf.end(), m, m + 12); im.push_back(s->desc[i].mesh);
    }
    q.emT.clear(); q.emC.clear(); q.mlp.clear();
    if (!s->em.empty() && q.r.light_mode != CWP_LIGHT_BSDF)
        frame_lights(s->em, xf.data(), im.data(), (int64_t)im.size(), s->hMats.data(), s->nMats, q.emT, q.emC, q.mlp);
    return CWP_OK;
}

extern "C" int cwp_server_submit(cwp_server* s, const cwp_request* r, int64_t* id) {
    CWPB_CHECK(s && r && id, CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(!s->sceneFirst.empty(), CWP_ERR_STATE, "no scenes (cwp_server_set_scenes)");
    CWPB_CHECK(r->scene >= 0 && r->scene + 1 < (int)s->sceneFirst.size(), CWP_ERR_INVALID, "scene %d out of range", r->scene);
    CWPB_CHECK(r->env >= -1 && r->env < (int)s->envs.size(), CWP_ERR_INVALID, "environment map %d out of range (%d maps)", r->env, (int)s->envs.size());
    CWPB_CHECK(std::isfinite(r->env_rot_deg), CWP_ERR_INVALID, "environment rotation is not finite");
    CWPB_CHECK(r->light_mode >= CWP_LIGHT_MIS && r->light_mode <= CWP_LIGHT_BSDF && (r->rr == 0 || r->rr == 1) && r->rr_depth >= 0 && (r->env_uniform == 0 || r->env_uniform == 1) &&
               (r->bump_shadow == 0 || r->bump_shadow == 1) && (r->filter_bh == 0 || r->filter_bh == 1) && std::isfinite(r->near_clip) && r->near_clip >= 0.f &&
               std::isfinite(r->cam.lens_r) && r->cam.lens_r >= 0.f && (r->cam.lens_r == 0.f || (std::isfinite(r->cam.focus_d) && r->cam.focus_d > 0.f)),
               CWP_ERR_INVALID, "light mode %d, rr %d, rr_depth %d, env_uniform %d, bump_shadow %d, filter_bh %d, near %g, lens %g / %g", r->light_mode, r->rr, r->rr_depth,
               r->env_uniform, r->bump_shadow, r->filter_bh, r->near_clip, r->cam.lens_r, r->cam.focus_d);
    CWPB_CHECK(r->cam.w > 0 && r->cam.h > 0 && r->spp > 0 && r->max_depth >= 0 && r->max_depth <= 64, CWP_ERR_INVALID, "bad request size");
    const int64_t total = (int64_t)r->cam.w * r->cam.h * r->spp;
    CWPB_CHECK(total < (1ll << 31), CWP_ERR_INVALID, "%lld paths in one request (limit 2^31)", (long long)total);
    ServeRequest q; q.r = *r; q.submitMs = now_ms(s); q.total = total;
    if (int rc = prepare_request(s, q)) return rc;
    q.id = s->nextId++;
    const int64_t qid = q.id;
    s->reqs[qid] = std::move(q); s->pending.push_back(qid);
    *id = qid;
    return CWP_OK;
}

// TLAS of the slots admitted since the last update (their previous requests' rays are no longer in flight)
static int rebuild_tlas(cwp_server* s) {
    std::vector<cwp_instance> all; std::vector<int> counts;
    for (int k : s->admitted) { all.insert(all.end(), s->slotInst[k].begin(), s->slotInst[k].end()); counts.push_back((int)s->slotInst[k].size()); }
    const int rc = cwp_batch_update_scenes(s->batch, s->admitted.data(), (int)s->admitted.size(), all.data(), counts.data());
    s->admitted.clear();
    return rc;
}

// device bytes an admission may use: free memory plus what the image pool holds unused, less the reserve. The
// device query (milliseconds) runs at most every 50 ms; in between, the pool's own growth is taken off its answer.
static int admission_budget(cwp_server* s, int64_t& avail) {
    uint64_t reserved = 0, used = 0;
    CWPB_CUDA(cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
    CWPB_CUDA(cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrUsedMemCurrent, &used));
    const double t = now_ms(s);
    if (t - s->freeAt > 50.0) {
        size_t freeB = 0, totalB = 0;
        CWPB_CUDA(cudaMemGetInfo(&freeB, &totalB));
        s->freeB = (int64_t)freeB; s->freeReserved = reserved; s->freeAt = t;
    }
    const int64_t freeNow = s->freeB - ((int64_t)reserved - (int64_t)s->freeReserved);
    avail = freeNow + (int64_t)(reserved > used ? reserved - used : 0) - s->O.hbm_reserve;
    return CWP_OK;
}

static int admit(cwp_server* s, bool& changed) {
    changed = false;
    if (s->pending.empty()) return CWP_OK;
    int64_t avail = 0;
    bool queried = false;
    while (!s->pending.empty()) {
        int slot = -1;
        for (int k = 0; k < s->O.max_requests; k++) if (s->slotReq[k] < 0) { slot = k; break; }
        if (slot < 0) break;
        if (!queried) { if (int rc = admission_budget(s, avail)) return rc; queried = true; }   // one query per step
        ServeRequest& q = s->reqs[s->pending.front()];
        const int64_t bytes = (int64_t)q.r.cam.w * q.r.cam.h * (int64_t)sizeof(float4);
        if (avail < bytes) break;   // admission by free device memory
        const cudaError_t e = cudaMallocFromPoolAsync((void**)&q.accum, (size_t)bytes, s->pool, s->st);   // stream-ordered, pooled
        if (e == cudaErrorMemoryAllocation) { cudaGetLastError(); q.accum = nullptr; break; }   // fragmentation: wait for frees
        CWPB_CUDA(e);
        avail -= bytes;
        CWPB_CUDA(cudaMemsetAsync(q.accum, 0, (size_t)bytes, s->st));
        SlotParams& P = s->hSlots[slot];
        P = SlotParams{};
        P.cam = q.r.cam; P.sunTo = f3(q.r.sun_to[0], q.r.sun_to[1], q.r.sun_to[2]); P.sunE = f3(q.r.sun_e[0], q.r.sun_e[1], q.r.sun_e[2]);
        P.sky = f3(q.r.sky[0], q.r.sky[1], q.r.sky[2]); P.sunCos = q.r.sun_cos; P.eps = q.r.eps; P.seed = q.r.seed; P.maxDepth = q.r.max_depth;
        P.N = q.r.cam.w * q.r.cam.h; P.accum = q.accum;
        if (q.r.env >= 0) {
            const cwp_server::EnvMap& E = s->envs[q.r.env];
            P.envTex = E.tex; P.envMarg = E.marg; P.envCond = E.cond; P.envW = E.w; P.envH = E.h; P.envRot = q.r.env_rot_deg * 3.14159265f / 180.f;
        }
        // the scene's instances at the request's frame, and its emissive triangles there (prepared at submission)
        if (!q.emT.empty()) {
            const std::vector<float>& emT = q.emT; const std::vector<float>& emC = q.emC; const std::vector<float>& mlp = q.mlp;
            {
                const size_t bT = emT.size() * sizeof(float), bC = (emC.size() * sizeof(float) + 15) & ~(size_t)15, bM = mlp.size() * sizeof(float);
                const cudaError_t e2 = (int64_t)(bT + bC + bM) <= avail ? cudaMallocFromPoolAsync(&q.lights, bT + bC + bM, s->pool, s->st) : cudaErrorMemoryAllocation;
                if (e2 == cudaErrorMemoryAllocation) {   // no room for the tables: the request waits with its image freed
                    cudaGetLastError(); q.lights = nullptr;
                    CWPB_CUDA(cudaFreeAsync(q.accum, s->st)); q.accum = nullptr;
                    break;
                }
                CWPB_CUDA(e2);
                avail -= (int64_t)(bT + bC + bM);
                char* base = (char*)q.lights;   // pageable sources: staged before the calls return
                CWPB_CUDA(cudaMemcpyAsync(base, emT.data(), bT, cudaMemcpyHostToDevice, s->st));
                CWPB_CUDA(cudaMemcpyAsync(base + bT, emC.data(), emC.size() * sizeof(float), cudaMemcpyHostToDevice, s->st));
                CWPB_CUDA(cudaMemcpyAsync(base + bT + bC, mlp.data(), bM, cudaMemcpyHostToDevice, s->st));
                P.emTris = (const float4*)base; P.emCdf = (const float*)(base + bT); P.matPdf = (const float*)(base + bT + bC); P.nEm = (int)(emT.size() / 12);
            }
        }
        // light-type probabilities (render/wavefront.cu:531-533): equal over the enabled types
        const float sunL = 0.2126f * P.sunE.x + 0.7152f * P.sunE.y + 0.0722f * P.sunE.z;
        const bool sunOn = sunL > 0.f, triOn = P.nEm > 0 && q.r.light_mode != CWP_LIGHT_BSDF, envOn = q.r.env >= 0 && q.r.light_mode != CWP_LIGHT_BSDF;
        const int nt = (int)sunOn + (int)triOn + (int)envOn;
        P.pSun = sunOn ? 1.f / nt : 0.f; P.pTri = triOn ? 1.f / nt : 0.f; P.pEnv = envOn ? 1.f / nt : 0.f;
        P.lightMode = q.r.light_mode; P.rr = q.r.rr; P.rrDepth = q.r.rr_depth; P.envUniform = q.r.env_uniform; P.bumpShadow = q.r.bump_shadow;
        P.nearClip = q.r.near_clip; P.filterBh = q.r.filter_bh;
        s->slotInst[slot].swap(q.inst); q.inst.clear(); q.inst.shrink_to_fit();
        s->slotsDirty = true;
        CWPB_CUDA(cudaMemsetAsync(s->slotCnt + kSlotCounters * slot, 0, kSlotCounters * sizeof(int), s->st));
        q.slot = slot; q.admitMs = now_ms(s); s->info.admissions++; s->admitted.push_back(slot);
        s->slotReq[slot] = q.id; s->hSlotCnt[kSlotCounters * slot + 2] = 0;
        s->pending.pop_front();
        changed = true;
    }
    if (s->slotsDirty) {   // every admitted slot's parameters in one copy (the previous step's copies have completed)
        CWPB_CUDA(cudaMemcpyAsync(s->dSlots, s->hSlots, (size_t)s->O.max_requests * sizeof(SlotParams), cudaMemcpyHostToDevice, s->st));
        s->slotsDirty = false;
    }
    return CWP_OK;
}

// takes the results of the queued step: waits for its launches (the step's one host round trip), reads the queue
// lengths and per-request counts, adds its timings and completes the requests whose paths have all finished
static int finish_step(cwp_server* s) {
    if (!s->inflight) return CWP_OK;
    s->inflight = false;
    const int R = s->O.max_requests; const int64_t n = s->inflightN;
    CWPB_CUDA(cudaStreamSynchronize(s->st));
    int64_t nNext = 0, nShadow = 0;
    if (n > 0) { nNext = s->hcnt[0]; nShadow = s->hcnt[1]; }
    {
        float a = 0, b = 0, c = 0, d = 0;
        CWPB_CUDA(cudaEventElapsedTime(&a, s->ev[0], s->ev[1])); CWPB_CUDA(cudaEventElapsedTime(&b, s->ev[1], s->ev[2]));
        CWPB_CUDA(cudaEventElapsedTime(&c, s->ev[2], s->ev[3])); CWPB_CUDA(cudaEventElapsedTime(&d, s->ev[3], s->ev[4]));
        float e = 0; CWPB_CUDA(cudaEventElapsedTime(&e, s->ev[5], s->ev[4]));
        s->info.raygen_ms += a; s->info.closest_ms += b; s->info.shade_ms += c; s->info.shadow_ms += d; s->info.accum_ms += e;
        s->info.steps++; s->info.rays += n; s->info.shadow_rays += nShadow;
    }
    if ((s->info.steps & 63) == 0 || nNext == 0) { if (int rc = cwp_batch_status(s->batch)) return rc; }   // traversal bounds: checked every 64 steps and when the queue drains
    s->cur ^= 1; s->nCur = nNext;
    const double t = now_ms(s);
    for (int k = 0; k < R; k++) {
        if (s->slotReq[k] < 0) continue;
        ServeRequest& q = s->reqs[s->slotReq[k]];
        const int* c = s->hcnt + 4 + kSlotCounters * k;
        q.rays = c[0]; q.shadow = c[1]; q.finished = c[2];
        if (q.issued == q.total && q.finished == q.total) {
            q.done = true; q.doneMs = t; s->completed.push_back(q.id); s->slotReq[k] = -1; q.slot = -1;
            if (q.lights) { CWPB_CUDA(cudaFreeAsync(q.lights, s->st)); q.lights = nullptr; }
        }
    }
    return CWP_OK;
}

// queues one step's launches: new camera paths, closest hits, shading, regrouping, shadow rays, accumulation, and
// the copies of the counts the host reads when it takes the step's results
static int launch_step(cwp_server* s) {
    // new camera paths: free capacity shared evenly by the slots with samples left to issue, oldest first
    const int R = s->O.max_requests;
    std::vector<int> needy;
    for (int k = 0; k < R; k++) if (s->slotReq[k] >= 0) { const ServeRequest& q = s->reqs[s->slotReq[k]]; if (q.issued < q.total) needy.push_back(k); }
    std::sort(needy.begin(), needy.end(), [&](int a, int b) { return s->reqs[s->slotReq[a]].admitMs < s->reqs[s->slotReq[b]].admitMs; });
    int64_t freeCap = s->O.max_paths - s->nCur;
    int nChunks = 0; int64_t added = 0;
    for (size_t i = 0; i < needy.size() && freeCap > 0; i++) {
        ServeRequest& q = s->reqs[s->slotReq[needy[i]]];
        // even share: what is left split over the requests not yet served; oldest first: all that is left
        const int64_t share = s->O.policy == 1 ? freeCap : freeCap / (int64_t)(needy.size() - i);
        const int64_t take = std::min(q.total - q.issued, std::max<int64_t>(share, 1));
        if (take <= 0) continue;
        s->hChunks[nChunks++] = make_int4(needy[i], (int)q.issued, (int)take, (int)added);
        q.issued += take; added += take; freeCap -= take;
    }
    RayQueue& in = s->q[s->cur]; RayQueue& out = s->q[s->cur ^ 1];
    CWPB_CUDA(cudaEventRecord(s->ev[0], s->st));
    if (added > 0) {
        CWPB_CUDA(cudaMemcpyAsync(s->dChunks, s->hChunks, (size_t)nChunks * sizeof(int4), cudaMemcpyHostToDevice, s->st));
        k_serve_raygen<<<(unsigned)((added + 255) / 256), 256, 0, s->st>>>(s->dChunks, nChunks, (int)added, s->dSlots, in, (int)s->nCur, s->ftab);
        CWPB_CUDA(cudaGetLastError());
    }
    const int64_t n = s->nCur + added;
    CWPB_CUDA(cudaEventRecord(s->ev[1], s->st));
    CWPB_CUDA(cudaEventRecord(s->ev[2], s->st));
    CWPB_CUDA(cudaEventRecord(s->ev[3], s->st));
    CWPB_CUDA(cudaEventRecord(s->ev[5], s->st));
    if (n > 0) {
        if (int rc = batch_trace_dev(s->batch, false, in.o, in.d, in.sc, s->hits, s->hinst, n, s->st)) return rc;
        CWPB_CUDA(cudaEventRecord(s->ev[2], s->st));
        CWPB_CUDA(cudaMemsetAsync(s->cnt, 0, 4 * sizeof(int), s->st));
        ShadeArgs a{};
        a.n = (int)n; a.in = in; a.out = out; a.sq = s->sq; a.hits = s->hits; a.hinst = s->hinst; a.inst = batch_instances(s->batch); a.tris = batch_tris(s->batch);
        a.mats = s->mats; a.nMats = s->nMats; a.meshMat = s->meshMat; a.slots = s->dSlots; a.gdEnergy = s->O.gd_energy; a.cnt = s->cnt; a.slotCnt = s->slotCnt;
        a.texObj = s->dTexObj; a.mtex = s->nMtex ? s->dMtex : nullptr; a.nMtex = s->nMtex; a.uvs = s->dUvs; a.tans = s->dTans; a.meshFirst = batch_mesh_first(s->batch);
        a.nrm = batch_normals(s->batch);
        const unsigned g = (unsigned)std::min<int64_t>((n + 127) / 128, 148 * 16);
        k_serve_shade<<<g, 128, 0, s->st>>>(a);
        CWPB_CUDA(cudaGetLastError());
        CWPB_CUDA(cudaEventRecord(s->ev[3], s->st));
        if (R > 1 && s->O.regroup >= 0) {   // regroup the next step's rays by request (continuous batching interleaves them)
            CWPB_CUDA(cudaMemsetAsync(s->slotBins, 0, 2 * R * sizeof(int), s->st));
            k_slot_hist<<<148 * 4, 256, R * sizeof(int), s->st>>>(s->cnt, out.info, s->slotBins, R);
            k_slot_scan<<<1, 1024, 0, s->st>>>(s->slotBins, s->slotBins + R, R);
            k_slot_scatter<<<148 * 8, 256, 0, s->st>>>(s->cnt, out, s->qs, s->slotBins + R);
            CWPB_CUDA(cudaGetLastError());
            std::swap(s->q[s->cur ^ 1], s->qs);   // the regrouped copy is the next step's input
        }
        // shadow rays: count on the device, no host round trip before the any-hit launch
        if (int rc = batch_trace_dev(s->batch, true, s->sq.o, s->sq.d, s->sq.sc, nullptr, s->occ, 0, s->st, s->cnt + 1)) return rc;
        CWPB_CUDA(cudaEventRecord(s->ev[5], s->st));
        k_serve_shadow_accum<<<148 * 8, 256, 0, s->st>>>(s->cnt + 1, s->sq, s->occ, s->dSlots);
        CWPB_CUDA(cudaGetLastError());
    }
    CWPB_CUDA(cudaEventRecord(s->ev[4], s->st));
    if (n > 0) CWPB_CUDA(cudaMemcpyAsync(s->hcnt, s->cnt, 2 * sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CWPB_CUDA(cudaMemcpyAsync(s->hcnt + 4, s->slotCnt, (size_t)R * kSlotCounters * sizeof(int), cudaMemcpyDeviceToHost, s->st));
    s->inflight = true; s->inflightN = n;
    return CWP_OK;
}

// One step: the results of the queued step (overlapped form), admissions, the TLAS update for new requests, and
// the next step's launches; with overlap -1 the call waits for them before returning. In the overlapped form the
// device runs a step while the caller submits, polls and reads results; admissions still wait for the step before
// them (free slots are known only then), so the device idles for the admission and TLAS update only.
extern "C" int cwp_server_step(cwp_server* s, int32_t* nActive, int32_t* nPending) {
    CWPB_CHECK(s, CWP_ERR_INVALID, "server is NULL");
    CWPB_CUDA(cudaSetDevice(s->device));
    const double stepStart = now_ms(s);
    if (int rc = finish_step(s)) return rc;
    const double admitStart = now_ms(s);
    bool changed = false;
    if (int rc = admit(s, changed)) return rc;
    s->info.admit_ms += now_ms(s) - admitStart;
    if (changed) {
        CWPB_CUDA(cudaStreamSynchronize(s->st));
        const double t = now_ms(s);
        if (int rc = rebuild_tlas(s)) return rc;
        s->info.tlas_ms += now_ms(s) - t; s->info.tlas_rebuilds++;
        cwp_batch_info bi{}; if (cwp_batch_info_of(s->batch, &bi) == CWP_OK) s->info.tlas_device_ms += bi.tlas_build_ms;
    }
    const int R = s->O.max_requests;
    bool any = false;
    for (int k = 0; k < R; k++) any |= s->slotReq[k] >= 0;
    if (any) {
        if (int rc = launch_step(s)) return rc;
        if (!s->overlap) { if (int rc = finish_step(s)) return rc; }
    }
    s->info.step_ms += now_ms(s) - stepStart;
    if (nActive) { int a = 0; for (int k = 0; k < R; k++) a += s->slotReq[k] >= 0; *nActive = a; }
    if (nPending) *nPending = (int)s->pending.size();
    return CWP_OK;
}

extern "C" int cwp_server_poll(cwp_server* s, int64_t* ids, int32_t cap, int32_t* n) {
    CWPB_CHECK(s && n && (cap == 0 || ids), CWP_ERR_INVALID, "NULL argument");
    const int k = (int)std::min<size_t>(s->completed.size(), (size_t)std::max(cap, 0));
    for (int i = 0; i < k; i++) ids[i] = s->completed[i];
    s->completed.erase(s->completed.begin(), s->completed.begin() + k);
    *n = k;
    return CWP_OK;
}

extern "C" int cwp_server_result(cwp_server* s, int64_t id, float* accum, cwp_request_stats* st) {
    CWPB_CHECK(s, CWP_ERR_INVALID, "server is NULL");
    auto it = s->reqs.find(id);
    CWPB_CHECK(it != s->reqs.end(), CWP_ERR_INVALID, "unknown request %lld", (long long)id);
    ServeRequest& q = it->second;
    CWPB_CHECK(q.done, CWP_ERR_STATE, "request %lld is not complete", (long long)id);
    CWPB_CUDA(cudaSetDevice(s->device));
    if (accum) {   // the image's last writes completed before its step's results were taken; a queued step may be running
        CWPB_CUDA(cudaMemcpyAsync(accum, q.accum, (size_t)q.r.cam.w * q.r.cam.h * sizeof(float4), cudaMemcpyDeviceToHost, s->cst));
        CWPB_CUDA(cudaStreamSynchronize(s->cst));
    }
    if (st) {
        st->submit_ms = q.submitMs; st->admit_ms = q.admitMs; st->done_ms = q.doneMs; st->rays = q.rays; st->shadow_rays = q.shadow;
        st->w = q.r.cam.w; st->h = q.r.cam.h; st->spp = q.r.spp; st->pad = 0;
    }
    CWPB_CUDA(cudaFreeAsync(q.accum, s->st));
    s->reqs.erase(it);
    return CWP_OK;
}

extern "C" int cwp_bsdf_eval_batch(const cwp_material* mats, int32_t nm, const int32_t* mat, const float* wo, const float* wi, const float* eta, int32_t gd,
                                   const float* ux, float* f, float* pdf, int64_t n, const float* nr) {
    CWPB_CHECK(mats && nm > 0 && mat && wo && wi && eta && ux && f && pdf && n >= 0, CWP_ERR_INVALID, "NULL argument");
    for (int64_t i = 0; i < n; i++) CWPB_CHECK(mat[i] >= 0 && mat[i] < nm, CWP_ERR_INVALID, "material index %d out of range", mat[i]);
    if (n == 0) return CWP_OK;
    cwp_material* dm; int* dmat; float3 *dwo, *dwi; float* deta; float2* dux; float4* df; float* dpdf;
    CWPB_CUDA(cudaMalloc(&dm, nm * sizeof(cwp_material))); CWPB_CUDA(cudaMalloc(&dmat, n * 4)); CWPB_CUDA(cudaMalloc(&dwo, n * 12)); CWPB_CUDA(cudaMalloc(&dwi, n * 12));
    CWPB_CUDA(cudaMalloc(&deta, n * 4)); CWPB_CUDA(cudaMalloc(&dux, n * 8)); CWPB_CUDA(cudaMalloc(&df, n * 16)); CWPB_CUDA(cudaMalloc(&dpdf, n * 4));
    cudaMemcpy(dm, mats, nm * sizeof(cwp_material), cudaMemcpyHostToDevice); cudaMemcpy(dmat, mat, n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dwo, wo, n * 12, cudaMemcpyHostToDevice); cudaMemcpy(dwi, wi, n * 12, cudaMemcpyHostToDevice); cudaMemcpy(deta, eta, n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dux, ux, n * 8, cudaMemcpyHostToDevice);
    float3* dnr = nullptr;
    if (nr) { CWPB_CUDA(cudaMalloc(&dnr, n * 12)); cudaMemcpy(dnr, nr, n * 12, cudaMemcpyHostToDevice); }
    k_bsdf_eval<<<(unsigned)((n + 127) / 128), 128>>>(dm, dmat, dwo, dwi, deta, gd, dux, dnr, df, dpdf, n);
    cudaError_t e = cudaGetLastError();
    std::vector<float4> hf(n);
    if (e == cudaSuccess) e = cudaMemcpy(hf.data(), df, n * 16, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(pdf, dpdf, n * 4, cudaMemcpyDeviceToHost);
    for (int64_t i = 0; i < n && e == cudaSuccess; i++) { f[3 * i] = hf[i].x; f[3 * i + 1] = hf[i].y; f[3 * i + 2] = hf[i].z; }
    cudaFree(dm); cudaFree(dmat); cudaFree(dwo); cudaFree(dwi); cudaFree(deta); cudaFree(dux); cudaFree(df); cudaFree(dpdf); cudaFree(dnr);
    CWPB_CUDA(e);
    return CWP_OK;
}

extern "C" int cwp_bsdf_sample_batch(const cwp_material* mats, int32_t nm, const int32_t* mat, const float* wo, const float* eta, int32_t gd, const float* ux,
                                     const float* uvw, float* wi, float* weight, float* pdf, int32_t* ok, int64_t n, const float* nr) {
    CWPB_CHECK(mats && nm > 0 && mat && wo && eta && ux && uvw && wi && weight && pdf && ok && n >= 0, CWP_ERR_INVALID, "NULL argument");
    for (int64_t i = 0; i < n; i++) CWPB_CHECK(mat[i] >= 0 && mat[i] < nm, CWP_ERR_INVALID, "material index %d out of range", mat[i]);
    if (n == 0) return CWP_OK;
    cwp_material* dm; int *dmat, *dok; float3 *dwo, *duvw, *dwi, *dw; float *deta, *dpdf; float2* dux;
    CWPB_CUDA(cudaMalloc(&dm, nm * sizeof(cwp_material))); CWPB_CUDA(cudaMalloc(&dmat, n * 4)); CWPB_CUDA(cudaMalloc(&dwo, n * 12)); CWPB_CUDA(cudaMalloc(&deta, n * 4));
    CWPB_CUDA(cudaMalloc(&dux, n * 8)); CWPB_CUDA(cudaMalloc(&duvw, n * 12)); CWPB_CUDA(cudaMalloc(&dwi, n * 12)); CWPB_CUDA(cudaMalloc(&dw, n * 12));
    CWPB_CUDA(cudaMalloc(&dpdf, n * 4)); CWPB_CUDA(cudaMalloc(&dok, n * 4));
    cudaMemcpy(dm, mats, nm * sizeof(cwp_material), cudaMemcpyHostToDevice); cudaMemcpy(dmat, mat, n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dwo, wo, n * 12, cudaMemcpyHostToDevice); cudaMemcpy(deta, eta, n * 4, cudaMemcpyHostToDevice); cudaMemcpy(dux, ux, n * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(duvw, uvw, n * 12, cudaMemcpyHostToDevice);
    float3* dnr = nullptr;
    if (nr) { CWPB_CUDA(cudaMalloc(&dnr, n * 12)); cudaMemcpy(dnr, nr, n * 12, cudaMemcpyHostToDevice); }
    k_bsdf_sample<<<(unsigned)((n + 127) / 128), 128>>>(dm, dmat, dwo, deta, gd, dux, duvw, dnr, dwi, dw, dpdf, dok, n);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(wi, dwi, n * 12, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(weight, dw, n * 12, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(pdf, dpdf, n * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(ok, dok, n * 4, cudaMemcpyDeviceToHost);
    cudaFree(dm); cudaFree(dmat); cudaFree(dwo); cudaFree(deta); cudaFree(dux); cudaFree(duvw); cudaFree(dwi); cudaFree(dw); cudaFree(dpdf); cudaFree(dok); cudaFree(dnr);
    CWPB_CUDA(e);
    return CWP_OK;
}

extern "C" int cwp_server_info_of(const cwp_server* s, cwp_server_info* out) {
    CWPB_CHECK(s && out, CWP_ERR_INVALID, "NULL argument");
    *out = s->info;
    return CWP_OK;
}
