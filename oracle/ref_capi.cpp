// ref_capi.cpp - TEST INFRASTRUCTURE ONLY: a C wrapper around the reference's own host code, compiled from the
// reference's sources by oracle/Makefile into oracle/_ref/libcwpref.so. Used to pin the oracle and the library
// against the reference (byte-identical BVH buffers, same traversal results) and as the timed CPU baseline.
//   builder / layouts ... accel/bvh_builder.cpp, accel/bvh_layouts.cpp, accel/bvh_tools.cpp, accel/tri_pack.cpp
//   traversal ........... accel/traverse.cuh trav<V, ANY, TRI> compiled as host C++ through ref_shim.h
//   instance transforms . scene/instances.cpp invertXform / instanceXform (with io/json.cpp, which it links)
//   two-level traversal . accel/traverse_inst.cuh travInst<V, ANY, TRI> compiled as host C++ through ref_shim.h
//   materials ........... render/bsdf.h bsdfEval / bsdfSample (host + device code, compiled for the host)
// The harness (threads, argument marshalling) is ours; the arithmetic is the reference's.
#include "ref_shim.h"
#include "accel/bvh_builder.h"
#include "accel/bvh_layouts.h"
#include "accel/bvh_tools.h"
#include "accel/tri_pack.h"
#include "accel/traverse.cuh"
#include "accel/traverse_inst.cuh"
#include "core/rng.h"
#include "scene/instances.h"
#include "scene/environment.h"
#include "scene/synthetic.h"
#include "scene/camera.h"
#include "io/hdr_image.h"
#include "render/bsdf.h"
#include "core/sampling.h"
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

static Mesh to_mesh(const float* v, long nv, const int* f, const int* fm, long nt) {
    Mesh m;
    for (long i = 0; i < nv; i++) m.v.push_back(make_float3(v[3 * i], v[3 * i + 1], v[3 * i + 2]));
    for (long i = 0; i < nt; i++) { m.f.push_back(make_int3(f[3 * i], f[3 * i + 1], f[3 * i + 2])); m.fm.push_back(fm ? fm[i] : 0); }
    m.kd.push_back(make_float3(0.8f, 0.8f, 0.8f));
    return m;
}

// Builds like setupScene's layout step (app/scene_setup.cpp:190-222): variant 2 / 4 / 8, collapse 0 = SAH (CWBVH,
// built from leaf-1 trees), 1 = greedy BVH8. Writes nodes (float4s, up to cap_f4), leaf order, packed triangles and
// Woop rows (3 float4 per triangle each). Returns the node count in float4 units, or -1 if cap_f4 is too small.
extern "C" long ref_build(const float* v, long nv, const int* f, const int* fm, long nt, int variant, int leaf, int collapse,
                          float* nodes_out, long cap_f4, int* order_out, float* tris_out, float* woop_out, int* max_depth, double* sah, double* build_ms) {
    Mesh m = to_mesh(v, nv, f, fm, nt);
    auto t0 = std::chrono::steady_clock::now();
    const bool cw = variant == 8 && collapse == 0;
    BVHBuilder B; B.leafMax = cw ? 1 : (variant == 8 && leaf > 4) ? 4 : leaf; B.build(m);
    std::vector<float4> nodes; std::vector<int> order;
    if (variant == 2) { *sah = sahCost(B, 1, 1); BVH2Flat F; F.build(B); nodes.swap(F.nodes); order = B.idx; }
    else if (variant == 4) { *sah = sahCost(B, 1, 1); BVH4Flat F; F.build(B); nodes.swap(F.nodes); order = B.idx; }
    else if (cw) { CWBVH C; C.build(B); nodes.swap(C.nodes); order.swap(C.order); *sah = C.sah; }
    else { *sah = sahCost(B, 1, 1); BVH8Flat F; F.build(B); nodes.swap(F.nodes); order.swap(F.order); }
    *build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    *max_depth = B.maxDepth;
    if ((long)nodes.size() > cap_f4) return -1;
    memcpy(nodes_out, nodes.data(), nodes.size() * 16);
    memcpy(order_out, order.data(), order.size() * 4);
    std::vector<float4> tris, nrm, woop;
    packTriangles(m, order, tris, nrm); packWoop(m, order, woop);
    memcpy(tris_out, tris.data(), tris.size() * 16); memcpy(woop_out, woop.data(), woop.size() * 16);
    return (long)nodes.size();
}

// The reference's binned-SAH build alone (single thread, as the reference runs it), for the CPU-baseline timing.
extern "C" double ref_build_ms(const float* v, long nv, const int* f, long nt, int leaf) {
    Mesh m = to_mesh(v, nv, f, nullptr, nt);
    auto t0 = std::chrono::steady_clock::now();
    BVHBuilder B; B.leafMax = leaf; B.build(m);
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

template <int V, bool ANY, int TRI>
static void run(const float4* nodes, const float4* tv, const float4* ro, const float4* rd, float4* hits, int* occ, long b, long e) {
    for (long i = b; i < e; i++) {
        float4 O = ro[i], D = rd[i]; float t = D.w, u = 0.f, vv = 0.f; int tri = -1;
        trav<V, ANY, TRI>(nodes, tv, xyz(O), xyz(D), O.w, t, tri, u, vv);
        if (ANY) occ[i] = tri; else hits[i] = make_float4(t, u, vv, __int_as_float(tri));
    }
}

// The reference's traversal over a ray batch on `threads` host threads (0 = all): closest hits as float4 (t, u, v,
// tri bits) like traceOne (render/wavefront.cu:62-66), any-hit as the first occluder index or -1. Returns seconds.
extern "C" double ref_trace(int variant, int any, int tri, const float* nodes, const float* tv, const float* ro, const float* rd, long n, float* hits, int* occ, int threads) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    auto fn = [&](long b, long e) {
        const float4 *N = (const float4*)nodes, *T = (const float4*)tv, *O = (const float4*)ro, *D = (const float4*)rd; float4* H = (float4*)hits;
#define REF_RUN(VV) do { if (any) { if (tri) run<VV, true, 1>(N, T, O, D, H, occ, b, e); else run<VV, true, 0>(N, T, O, D, H, occ, b, e); } \
                         else { if (tri) run<VV, false, 1>(N, T, O, D, H, occ, b, e); else run<VV, false, 0>(N, T, O, D, H, occ, b, e); } } while (0)
        if (variant == 2) REF_RUN(2); else if (variant == 4) REF_RUN(4); else REF_RUN(8);
#undef REF_RUN
    };
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> ts;
    for (int k = 0; k < threads; k++) ts.emplace_back(fn, n * k / threads, n * (k + 1) / threads);
    for (auto& t : ts) t.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// ---------------------------------------------------------------------------------------------------------------
// The legacy diffuse frame on host threads, for the CPU baseline of the frame metric. The reference has no CPU
// renderer (its shading runs only as CUDA kernels), so this harness strings together the reference's own
// host-compilable code - rng4 (core/rng.h), sampleUniformCone / sampleCosineHemisphere / onb (core/sampling.h), the
// float3 helpers (core/vec.h) and trav<V, ANY, TRI> (accel/traverse.cuh) - with the per-vertex logic of k_raygen and
// shadeOne (render/wavefront.cu:42-58, 94-136) restated around them. Paths are traced one after another per thread.
// P points at a cwp_params-layout struct (include/cwp_b200.h). Pixels [pix0, pix1), samples [s_base, s_base + spp);
// returns seconds, adds radiance sums to accum (float4 per pixel) and ray counts to counts[0..1].
struct RefParams {
    float pos[3], ax[3], ay[3], az[3]; float fx, fy, px, py; int w, h; float lens_r, focus_d;
    float sun_to[3], sun_e[3], sky[3]; float sun_cos; int max_b; unsigned seed; float eps, near_clip; int has_n, filter_bh; float ftab[65];
};

// The frame parameters the reference's CLI sets up for a look-at camera with a horizontal field of view
// (app/scene_setup.cpp:172-185): the camera from its own lookAtC2W / focalFromHfov / makeCamera (scene/camera.cpp),
// the normalised sun direction, the sun cone's cosine, the ray offset eps_scale x extent and its Blackman-Harris
// table. out: one RefParams (the cwp_params layout), ref_params_size() bytes.
extern "C" int ref_params_size(void) { return (int)sizeof(RefParams); }
extern "C" void ref_frame_params(const float* pos, const float* tgt, const float* up, float hfov_deg, int w, int h, const float* sun_to, const float* sun_e,
                                 const float* sky, float sun_angle_deg, int max_b, unsigned seed, float eps_scale, float extent, void* out) {
    float c2w[16];
    lookAtC2W(make_float3(pos[0], pos[1], pos[2]), make_float3(tgt[0], tgt[1], tgt[2]), make_float3(up[0], up[1], up[2]), c2w);
    const float fx = focalFromHfov(w, hfov_deg);
    const Cam c = makeCamera(c2w, fx, fx, w, h);
    RefParams& P = *(RefParams*)out;
    memset(&P, 0, sizeof P);
    const float3 v3[4] = { c.pos, c.ax, c.ay, c.az };
    float* dst[4] = { P.pos, P.ax, P.ay, P.az };
    for (int k = 0; k < 4; k++) { dst[k][0] = v3[k].x; dst[k][1] = v3[k].y; dst[k][2] = v3[k].z; }
    P.fx = c.fx; P.fy = c.fy; P.px = c.px; P.py = c.py; P.w = c.w; P.h = c.h; P.lens_r = c.lensR; P.focus_d = c.focusD;
    const float3 s = normalize(make_float3(sun_to[0], sun_to[1], sun_to[2]));
    P.sun_to[0] = s.x; P.sun_to[1] = s.y; P.sun_to[2] = s.z;
    for (int k = 0; k < 3; k++) { P.sun_e[k] = sun_e[k]; P.sky[k] = sky[k]; }
    P.sun_cos = cosf(0.5f * sun_angle_deg * 3.14159265f / 180.f);
    P.max_b = max_b; P.seed = seed; P.eps = eps_scale * extent; P.near_clip = 0.f; P.has_n = 0; P.filter_bh = 0;
    buildBlackmanHarrisTable(P.ftab, 64, 1.5);
}

template <int V, int TRI>
static void ref_paths(const RefParams& P, const float4* nodes, const float4* tv, const float4* tris, const float3* albedo, int bounces,
                      int spp, int sBase, long pix0, long pix1, float* accum, long long* nClosest, long long* nShadow) {
    const float3 ax = make_float3(P.ax[0], P.ax[1], P.ax[2]), ay = make_float3(P.ay[0], P.ay[1], P.ay[2]), az = make_float3(P.az[0], P.az[1], P.az[2]);
    const float3 pos = make_float3(P.pos[0], P.pos[1], P.pos[2]), sunTo = make_float3(P.sun_to[0], P.sun_to[1], P.sun_to[2]);
    const float3 sunE = make_float3(P.sun_e[0], P.sun_e[1], P.sun_e[2]), sky = make_float3(P.sky[0], P.sky[1], P.sky[2]);
    const int depths = bounces + 2;
    for (long pix = pix0; pix < pix1; pix++) {
        const int x = (int)(pix % P.w), y = (int)(pix / P.w);
        for (int smp = sBase; smp < sBase + spp; smp++) {
            float u0 = rng4(pix, smp, 0, 0, P.seed), u1 = rng4(pix, smp, 0, 1, P.seed), jx, jy;
            if (P.filter_bh) { jx = sampleTable(P.ftab, 64, u0); jy = sampleTable(P.ftab, 64, u1); } else { jx = u0 - 0.5f; jy = u1 - 0.5f; }
            float dx = (x + 0.5f + jx - P.px) / P.fx, dy = -(y + 0.5f + jy - P.py) / P.fy;
            float3 d = normalize(ax * dx + ay * dy - az), o = pos, T = make_float3(1.f, 1.f, 1.f); float tmin = P.near_clip;
            for (int depth = 0; depth < depths; depth++) {
                (*nClosest)++;
                float t = 1e30f, u = 0.f, v = 0.f; int tri = -1;
                trav<V, false, TRI>(nodes, tv, o, d, tmin, t, tri, u, v);
                if (tri < 0) { float3 c = T * sky; accum[4 * pix] += c.x; accum[4 * pix + 1] += c.y; accum[4 * pix + 2] += c.z; break; }
                if (depth > P.max_b) break;
                float3 p = o + d * t; float4 b = tris[3 * tri + 1], c4 = tris[3 * tri + 2];
                float3 ng = normalize(cross(xyz(b), xyz(c4))), ns = ng;
                if (dot(ng, d) > 0.f) { ng = -ng; ns = -ns; }
                float3 alb = albedo[__float_as_int(b.w)];
                float3 po = p + ng * P.eps;
                float3 l = sampleUniformCone(sunTo, P.sun_cos, rng4(pix, smp, depth + 1, 2, P.seed), rng4(pix, smp, depth + 1, 3, P.seed));
                float cl = dot(ns, l);
                if (cl > 0.f && dot(ng, l) > 0.f) {
                    float3 contrib = T * alb * sunE * (cl * CWP_INV_PI); (*nShadow)++;
                    float st = 1e30f, su, sv; int stri = -1;
                    if (!trav<V, true, TRI>(nodes, tv, po, l, 0.f, st, stri, su, sv)) { accum[4 * pix] += contrib.x; accum[4 * pix + 1] += contrib.y; accum[4 * pix + 2] += contrib.z; }
                }
                float3 nd = sampleCosineHemisphere(ns, rng4(pix, smp, depth + 1, 0, P.seed), rng4(pix, smp, depth + 1, 1, P.seed));
                if (dot(nd, ng) <= 0.f) break;
                T = T * alb; o = po; d = nd; tmin = 0.f;
            }
        }
    }
}

extern "C" double ref_render_cpu(const void* params, int variant, int tri, const float* nodes, const float* tv, const float* tris, const float* albedo,
                                 int bounces, int spp, int s_base, long pix0, long pix1, float* accum, long long* counts, int threads) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    const RefParams& P = *(const RefParams*)params;
    std::vector<long long> nc(threads, 0), ns(threads, 0);
    auto fn = [&](int k) {
        long b = pix0 + (pix1 - pix0) * k / threads, e = pix0 + (pix1 - pix0) * (k + 1) / threads;
        const float4 *N = (const float4*)nodes, *T = (const float4*)tv, *TR = (const float4*)tris; const float3* A = (const float3*)albedo;
        if (variant == 2) { if (tri) ref_paths<2, 1>(P, N, T, TR, A, bounces, spp, s_base, b, e, accum, &nc[k], &ns[k]); else ref_paths<2, 0>(P, N, T, TR, A, bounces, spp, s_base, b, e, accum, &nc[k], &ns[k]); }
        else if (variant == 4) { if (tri) ref_paths<4, 1>(P, N, T, TR, A, bounces, spp, s_base, b, e, accum, &nc[k], &ns[k]); else ref_paths<4, 0>(P, N, T, TR, A, bounces, spp, s_base, b, e, accum, &nc[k], &ns[k]); }
        else { if (tri) ref_paths<8, 1>(P, N, T, TR, A, bounces, spp, s_base, b, e, accum, &nc[k], &ns[k]); else ref_paths<8, 0>(P, N, T, TR, A, bounces, spp, s_base, b, e, accum, &nc[k], &ns[k]); }
    };
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> ts;
    for (int k = 0; k < threads; k++) ts.emplace_back(fn, k);
    for (auto& t : ts) t.join();
    double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int k = 0; k < threads; k++) { counts[0] += nc[k]; counts[1] += ns[k]; }
    return sec;
}

// scene/instances.cpp:64-79
extern "C" void ref_xform_invert(const float* m, float* inv, float* det_sign) {
    Xform M, I; for (int i = 0; i < 12; i++) M.m[i] = m[i];
    invertXform(M, I, *det_sign);
    for (int i = 0; i < 12; i++) inv[i] = I.m[i];
}
// scene/instances.cpp:48-62 (parametric instance: translate, axis, angle, scale and their per-frame velocities)
extern "C" void ref_xform_animate(const float* translate, const float* translate_vel, const float* axis, float angle_deg, float angle_vel,
                                  const float* scale, const float* scale_vel, int frame, float* m) {
    InstanceDesc d;
    d.translate = make_float3(translate[0], translate[1], translate[2]); d.translateVel = make_float3(translate_vel[0], translate_vel[1], translate_vel[2]);
    d.axis = make_float3(axis[0], axis[1], axis[2]); d.angleDeg = angle_deg; d.angleVel = angle_vel;
    d.scale = make_float3(scale[0], scale[1], scale[2]); d.scaleVel = make_float3(scale_vel[0], scale_vel[1], scale_vel[2]);
    const Xform X = instanceXform(d, frame);
    for (int i = 0; i < 12; i++) m[i] = X.m[i];
}

// The reference's two-level traversal (accel/traverse_inst.cuh:10-41) over a scene-tagged ray batch on `threads` host
// threads: TLAS = BVH2 nodes with instance leaves, roots per scene, DevInstance records (accel/instance.h:7, the same
// 112-byte layout as cwp_instance), BLAS nodes / triangles with absolute indices. Returns seconds.
extern "C" double ref_trace_inst(int variant, int any, int tri, const float* blas, const float* tv, const float* tlas, const int* scene_root, int n_scenes,
                                 const void* inst, const float* ro, const float* rd, const int* scene_of, long n, float* hits, int* hit_inst, int threads) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    auto fn = [&](long b, long e) {
        const float4 *N = (const float4*)blas, *T = (const float4*)tv, *TL = (const float4*)tlas, *O = (const float4*)ro, *D = (const float4*)rd;
        const DevInstance* I = (const DevInstance*)inst;
        for (long i = b; i < e; i++) {
            const float4 o = O[i], d = D[i]; float t = d.w, u = 0.f, v = 0.f; int h = -1, hi = -1;
            const int sc = scene_of[i], root = sc >= 0 && sc < n_scenes ? scene_root[sc] : -1;
            if (root >= 0) {
#define REF_INST(VV) do { if (any) { if (tri) travInst<VV, true, 1>(TL, root, I, N, T, xyz(o), xyz(d), o.w, t, h, u, v, hi); else travInst<VV, true, 0>(TL, root, I, N, T, xyz(o), xyz(d), o.w, t, h, u, v, hi); } \
                         else { if (tri) travInst<VV, false, 1>(TL, root, I, N, T, xyz(o), xyz(d), o.w, t, h, u, v, hi); else travInst<VV, false, 0>(TL, root, I, N, T, xyz(o), xyz(d), o.w, t, h, u, v, hi); } } while (0)
                if (variant == 2) REF_INST(2); else if (variant == 4) REF_INST(4); else REF_INST(8);
#undef REF_INST
            }
            if (hits) { hits[4 * i] = t; hits[4 * i + 1] = u; hits[4 * i + 2] = v; hits[4 * i + 3] = __int_as_float(h); }
            hit_inst[i] = hi;
        }
    };
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> ts;
    for (int k = 0; k < threads; k++) ts.emplace_back(fn, n * k / threads, n * (k + 1) / threads);
    for (auto& t : ts) t.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// render/bsdf.h:196-220 for n (material, wo, wi) triples; mats: Material records (scene/material.h:12-17, 64 B)
extern "C" void ref_bsdf_eval(const void* mats, const int* mat, const float* wo, const float* wi, const float* eta, int gd, const float* ux, float* f, float* pdf, long n) {
    const Material* M = (const Material*)mats;
    for (long i = 0; i < n; i++) {
        BsdfEval e = bsdfEval(M[mat[i]], make_float3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), make_float3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), eta[i], gd, ux[2 * i], ux[2 * i + 1]);
        f[3 * i] = e.f.x; f[3 * i + 1] = e.f.y; f[3 * i + 2] = e.f.z; pdf[i] = e.pdf;
    }
}
extern "C" void ref_bsdf_sample(const void* mats, const int* mat, const float* wo, const float* eta, int gd, const float* ux, const float* uvw, float* wi, float* w, float* pdf, int* ok, long n) {
    const Material* M = (const Material*)mats;
    for (long i = 0; i < n; i++) {
        float3 a = make_float3(0.f, 0.f, 0.f), b = a; float p = 0.f;
        ok[i] = bsdfSample(M[mat[i]], make_float3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), eta[i], gd, ux[2 * i], ux[2 * i + 1], uvw[3 * i], uvw[3 * i + 1], uvw[3 * i + 2], a, b, p) ? 1 : 0;
        wi[3 * i] = a.x; wi[3 * i + 1] = a.y; wi[3 * i + 2] = a.z; w[3 * i] = b.x; w[3 * i + 1] = b.y; w[3 * i + 2] = b.z; pdf[i] = p;
    }
}
// the same with an unperturbed normal nr per triple (the bump-terminator term of the diffuse lobe, render/bsdf.h:67-75)
extern "C" void ref_bsdf_eval_nr(const void* mats, const int* mat, const float* wo, const float* wi, const float* eta, int gd, const float* ux, const float* nr,
                                 float* f, float* pdf, long n) {
    const Material* M = (const Material*)mats;
    for (long i = 0; i < n; i++) {
        BsdfEval e = bsdfEval(M[mat[i]], make_float3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), make_float3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), eta[i], gd, ux[2 * i], ux[2 * i + 1],
                              make_float3(nr[3 * i], nr[3 * i + 1], nr[3 * i + 2]));
        f[3 * i] = e.f.x; f[3 * i + 1] = e.f.y; f[3 * i + 2] = e.f.z; pdf[i] = e.pdf;
    }
}
extern "C" void ref_bsdf_sample_nr(const void* mats, const int* mat, const float* wo, const float* eta, int gd, const float* ux, const float* uvw, const float* nr,
                                   float* wi, float* w, float* pdf, int* ok, long n) {
    const Material* M = (const Material*)mats;
    for (long i = 0; i < n; i++) {
        float3 a = make_float3(0.f, 0.f, 0.f), b = a; float p = 0.f;
        ok[i] = bsdfSample(M[mat[i]], make_float3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), eta[i], gd, ux[2 * i], ux[2 * i + 1], uvw[3 * i], uvw[3 * i + 1], uvw[3 * i + 2], a, b, p,
                           make_float3(nr[3 * i], nr[3 * i + 1], nr[3 * i + 2])) ? 1 : 0;
        wi[3 * i] = a.x; wi[3 * i + 1] = a.y; wi[3 * i + 2] = a.z; w[3 * i] = b.x; w[3 * i + 1] = b.y; w[3 * i + 2] = b.z; pdf[i] = p;
    }
}
extern "C" int ref_material_size(void) { return (int)sizeof(Material); }
// the pixel-filter inverse CDF of setupScene (core/sampling.h:38-43, app/scene_setup.cpp:185): n + 1 entries
extern "C" void ref_bh_table(float* tab, int n, double width) { buildBlackmanHarrisTable(tab, n, width); }

// the reference's loadHDR + buildEnvMap on a Radiance file: sizes first (texels/marg/cond NULL), then the tables
extern "C" int ref_env_build(const char* path, float strength, int* w, int* h, float* rgb, float* texels, float* marg, float* cond) {
    EnvMapHost E;
    if (!buildEnvMap(path, strength, E)) return -1;
    *w = E.w; *h = E.h;
    if (rgb) { int ww, hh; std::vector<float> v; if (!loadHDR(path, ww, hh, v)) return -1; memcpy(rgb, v.data(), v.size() * sizeof(float)); }
    if (texels) for (size_t i = 0; i < E.texels.size(); i++) { texels[4 * i] = E.texels[i].x; texels[4 * i + 1] = E.texels[i].y; texels[4 * i + 2] = E.texels[i].z; texels[4 * i + 3] = E.texels[i].w; }
    if (marg) memcpy(marg, E.marg.data(), E.marg.size() * sizeof(float));
    if (cond) memcpy(cond, E.cond.data(), E.cond.size() * sizeof(float));
    return 0;
}

// the reference's makeSynthetic + syntheticCamera: counts first (v/f/fm/kd NULL), then the arrays; c2w may be NULL
extern "C" void ref_synthetic(int grid, int nu, int nv, int gs, long* nverts, long* ntris, float* v, int* f, int* fm, float* kd, float* c2w) {
    Mesh M;
    makeSynthetic(M, grid, nu, nv, gs);
    *nverts = (long)M.v.size(); *ntris = (long)M.f.size();
    if (v) for (size_t i = 0; i < M.v.size(); i++) { v[3 * i] = M.v[i].x; v[3 * i + 1] = M.v[i].y; v[3 * i + 2] = M.v[i].z; }
    if (f) for (size_t i = 0; i < M.f.size(); i++) { f[3 * i] = M.f[i].x; f[3 * i + 1] = M.f[i].y; f[3 * i + 2] = M.f[i].z; }
    if (fm) memcpy(fm, M.fm.data(), M.fm.size() * sizeof(int));
    if (kd) for (size_t i = 0; i < M.kd.size(); i++) { kd[3 * i] = M.kd[i].x; kd[3 * i + 1] = M.kd[i].y; kd[3 * i + 2] = M.kd[i].z; }
    if (c2w) syntheticCamera(c2w);
}
