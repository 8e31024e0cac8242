// capi.cpp - C entry points: errors, meshes, host BVH builds, camera and parameter helpers.
#include "host_bvh.h"
#include "hploc.h"
#include "runtime.h"
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

namespace cwpb {
static thread_local std::string g_err;
int set_error(int code, const char* fmt, ...) {
    char buf[1024]; va_list ap; va_start(ap, fmt); vsnprintf(buf, sizeof buf, fmt, ap); va_end(ap);
    g_err = buf; return code;
}
void clear_error() { g_err.clear(); }
}  // namespace cwpb

using namespace cwpb;

extern "C" const char* cwp_last_error(void) { return g_err.c_str(); }
extern "C" int32_t cwp_version(void) { return 1; }

// ---------------- meshes ----------------
struct cwp_mesh { Mesh m; };

extern "C" int cwp_mesh_box_field(int32_t n_boxes, uint64_t seed, cwp_mesh** out) {
    CWPB_CHECK(out, CWP_ERR_INVALID, "out is NULL");
    CWPB_CHECK(n_boxes >= 0 && n_boxes <= (1 << 26), CWP_ERR_INVALID, "box count %d out of range", n_boxes);
    cwp_mesh* h = new cwp_mesh();
    box_field(n_boxes, seed, 20.f, 0.2f, 3.f, h->m);
    *out = h; return CWP_OK;
}

extern "C" int cwp_mesh_sphere_grid(int32_t grid, int32_t nu, int32_t nv, int32_t ground, cwp_mesh** out) {
    CWPB_CHECK(out, CWP_ERR_INVALID, "out is NULL");
    CWPB_CHECK(grid >= 0 && grid <= 64 && nu >= 3 && nu <= 4096 && nv >= 2 && nv <= 4096 && ground >= 1 && ground <= 8192,
               CWP_ERR_INVALID, "sphere grid %d, %d x %d quads, ground %d out of range", grid, nu, nv, ground);
    CWPB_CHECK((int64_t)grid * grid * nu * (nv + 1) + (int64_t)(ground + 1) * (ground + 1) < (1ll << 31), CWP_ERR_INVALID,
               "sphere grid has more than 2^31 vertices");
    cwp_mesh* h = new cwp_mesh();
    sphere_grid(grid, nu, nv, ground, h->m);
    *out = h; return CWP_OK;
}

extern "C" void cwp_sphere_grid_c2w(float c2w[16]) { if (c2w) sphere_grid_c2w(c2w); }

extern "C" int cwp_mesh_load(const char* path, cwp_mesh** out) {
    CWPB_CHECK(path && out, CWP_ERR_INVALID, "NULL argument");
    cwp_mesh* h = new cwp_mesh(); std::string err;
    if (!load_mesh(path, h->m, &err)) { delete h; return set_error(CWP_ERR_IO, "%s: %s", path, err.c_str()); }
    *out = h; return CWP_OK;
}

extern "C" int cwp_mesh_from_view(const cwp_mesh_view* v, cwp_mesh** out) {
    CWPB_CHECK(v && out, CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(v->n_verts >= 0 && v->n_tris >= 0 && (v->n_verts == 0 || v->verts) && (v->n_tris == 0 || v->faces), CWP_ERR_INVALID, "bad mesh view");
    cwp_mesh* h = new cwp_mesh(); Mesh& m = h->m;
    m.v.assign(v->verts, v->verts + 3 * v->n_verts);
    m.f.assign(v->faces, v->faces + 3 * v->n_tris);
    if (v->face_mat) m.fm.assign(v->face_mat, v->face_mat + v->n_tris); else m.fm.assign(v->n_tris, 0);
    if (v->normals) m.n.assign(v->normals, v->normals + 3 * v->n_verts);
    if (v->albedo && v->n_albedo > 0) m.kd.assign(v->albedo, v->albedo + 3 * v->n_albedo); else m.kd = { 0.8f, 0.8f, 0.8f };
    for (int x : m.f) if (x < 0 || (int64_t)x >= v->n_verts) { delete h; return set_error(CWP_ERR_INVALID, "face index %d out of range", x); }
    for (int x : m.fm) if (x < 0) { delete h; return set_error(CWP_ERR_INVALID, "negative material id"); }
    *out = h; return CWP_OK;
}

extern "C" int cwp_mesh_view_of(const cwp_mesh* h, cwp_mesh_view* out) {
    CWPB_CHECK(h && out, CWP_ERR_INVALID, "NULL argument");
    const Mesh& m = h->m;
    out->verts = m.v.data(); out->n_verts = (int64_t)m.nv(); out->faces = m.f.data(); out->n_tris = (int64_t)m.nt();
    out->face_mat = m.fm.empty() ? nullptr : m.fm.data(); out->normals = m.hasN() ? m.n.data() : nullptr;
    out->albedo = m.kd.data(); out->n_albedo = (int32_t)(m.kd.size() / 3);
    return CWP_OK;
}

extern "C" int cwp_mesh_write_ply(const cwp_mesh* h, const char* path) {
    CWPB_CHECK(h && path, CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(write_ply(path, h->m), CWP_ERR_IO, "cannot write %s", path);
    return CWP_OK;
}

extern "C" void cwp_mesh_free(cwp_mesh* h) { delete h; }

// ---------------- host BVH ----------------
struct cwp_bvh {
    std::vector<float4> nodes, tris, nrm, woop, verts; std::vector<int> order;
    int stride = 4, maxDepth = 0, maxLeafTris = 0; double sah = 0, ms = 0;
};

extern "C" int cwp_bvh_build(const cwp_mesh* h, const cwp_build_options* o, cwp_bvh** out) {
    CWPB_CHECK(h && o && out, CWP_ERR_INVALID, "NULL argument");
    *out = nullptr;
    const Mesh& m = h->m;
    CWPB_CHECK(m.nt() > 0, CWP_ERR_INVALID, "mesh has no triangles");
    CWPB_CHECK(m.nt() < (1u << 30), CWP_ERR_INVALID, "too many triangles");
    CWPB_CHECK(o->variant == 2 || o->variant == 4 || o->variant == 8, CWP_ERR_INVALID, "variant %d is not 2, 4 or 8", o->variant);
    CWPB_CHECK(o->bins >= 2 && o->bins <= 256, CWP_ERR_INVALID, "bins %d out of [2, 256]", o->bins);
    CWPB_CHECK(o->leaf >= 1 && o->leaf <= 64, CWP_ERR_INVALID, "leaf %d out of [1, 64]", o->leaf);
    CWPB_CHECK(o->collapse == 0 || o->collapse == 1, CWP_ERR_INVALID, "collapse must be 0 (SAH) or 1 (greedy)");
    auto t0 = std::chrono::steady_clock::now();
    const bool cw = o->variant == 8 && o->collapse == 0;
    SahOptions so; so.bins = o->bins; so.threads = o->threads;
    // leaf size rules of setupScene (scene_setup.cpp:192-193): the SAH collapse starts from single-triangle leaves,
    // the greedy 8-wide layout caps leaves at 4 (3 bits of count in the meta byte)
    so.leafMax = cw ? 1 : (o->variant == 8 && o->leaf > 4) ? 4 : o->leaf;
    CWPB_CHECK(o->variant == 8 || so.leafMax <= 64, CWP_ERR_INVALID, "leaf too large");
    CWPB_CHECK(o->spatial >= 0.f && o->spatial < 1.f, CWP_ERR_INVALID, "spatial %g out of [0, 1)", o->spatial);
    CWPB_CHECK(o->builder == 0 || o->builder == 1, CWP_ERR_INVALID, "builder %d is not 0 (host SAH) or 1 (GPU H-PLOC)", o->builder);
    CWPB_CHECK(o->builder == 0 || o->spatial == 0.f, CWP_ERR_INVALID, "spatial splits need the host builder");
    BinaryBvh B;
    double gpuMs = -1.0;
    if (o->builder == 1) {
        std::vector<float4> hn;
        if (int rc = hploc_build_mesh(m.v.data(), m.f.data(), (int64_t)m.nt(), o->device, hn, gpuMs)) return rc;
        tree_from_hploc(hn, (int64_t)m.nt(), so.leafMax, B);
    } else if (o->spatial > 0.f) build_sbvh(m, so, o->spatial, 0.3f, B);
    else build_sah(m, so, B);
    cwp_bvh* r = new cwp_bvh();
    r->maxDepth = B.maxDepth;
    if (o->variant == 2) { r->sah = sah_cost(B, 1, 1); layout_bvh2(B, r->nodes); r->order = B.prim; r->stride = 4; }
    else if (o->variant == 4) { r->sah = sah_cost(B, 1, 1); layout_bvh4(B, r->nodes); r->order = B.prim; r->stride = 8; }
    else {
        WideBvh W;
        if (cw) collapse_cwbvh(B, W); else collapse_greedy8(B, W);
        r->nodes.swap(W.nodes); r->order.swap(W.order); r->sah = W.sah; r->maxLeafTris = W.maxLeafTris; r->stride = 5;
    }
    if (o->variant != 8) { int mx = 0; for (const BNode& n : B.nodes) if (n.leaf()) mx = n.count > mx ? n.count : mx; r->maxLeafTris = mx; }
    pack_tris(m, r->order, r->tris, r->nrm);
    pack_woop(m, r->order, r->woop);
    pack_verts(m, r->order, r->verts);
    r->ms = gpuMs >= 0.0 ? gpuMs : std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (o->variant != 8 && B.maxDepth > 63) { delete r; return set_error(CWP_ERR_INVALID, "BVH depth %d exceeds the traversal stack (64)", B.maxDepth); }
    *out = r; return CWP_OK;
}

extern "C" int cwp_bvh_data_of(const cwp_bvh* b, cwp_bvh_data* out) {
    CWPB_CHECK(b && out, CWP_ERR_INVALID, "NULL argument");
    out->nodes = (const float*)b->nodes.data(); out->n_node_float4 = (int64_t)b->nodes.size(); out->node_stride = b->stride;
    out->order = b->order.data(); out->n_tris = (int64_t)b->order.size();
    out->tris = (const float*)b->tris.data(); out->nrm = b->nrm.empty() ? nullptr : (const float*)b->nrm.data(); out->woop = (const float*)b->woop.data();
    out->max_depth = b->maxDepth; out->max_leaf_tris = b->maxLeafTris; out->sah = b->sah; out->build_ms = b->ms;
    out->verts = (const float*)b->verts.data();
    return CWP_OK;
}

extern "C" void cwp_bvh_free(cwp_bvh* b) { delete b; }

// ---------------- camera / params ----------------
extern "C" int cwp_camera_from_c2w(const float c2w[16], float fx, float fy, int32_t w, int32_t h, cwp_camera* c) {
    CWPB_CHECK(c2w && c, CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(w > 0 && h > 0 && fx > 0 && fy > 0, CWP_ERR_INVALID, "bad intrinsics");
    memset(c, 0, sizeof *c);
    c->pos[0] = c2w[3]; c->pos[1] = c2w[7]; c->pos[2] = c2w[11];
    for (int i = 0; i < 3; i++) { c->ax[i] = c2w[4 * i]; c->ay[i] = c2w[4 * i + 1]; c->az[i] = c2w[4 * i + 2]; }
    c->fx = fx; c->fy = fy; c->px = w * 0.5f; c->py = h * 0.5f; c->w = w; c->h = h; c->lens_r = 0.f; c->focus_d = 1.f;
    return CWP_OK;
}

extern "C" int cwp_camera_look_at(const float pos[3], const float tgt[3], const float up[3], float hfov, int32_t w, int32_t h, cwp_camera* c) {
    CWPB_CHECK(pos && tgt && up && c, CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(hfov > 0.f && hfov < 180.f, CWP_ERR_INVALID, "hfov %g out of (0, 180)", hfov);
    const float3 p = f3(pos[0], pos[1], pos[2]), t = f3(tgt[0], tgt[1], tgt[2]), u = f3(up[0], up[1], up[2]);
    const float3 f = normalize(t - p), r = normalize(cross(f, u)), uu = cross(r, f), az = -f;
    float m[16] = { 0 }; m[15] = 1.f;
    const float3 cols[3] = { r, uu, az };
    for (int col = 0; col < 3; col++) { m[col] = cols[col].x; m[4 + col] = cols[col].y; m[8 + col] = cols[col].z; }
    m[3] = p.x; m[7] = p.y; m[11] = p.z;
    const float fx = (w * 0.5f) / tanf(hfov * 0.5f * 3.14159265f / 180.f);   // camera.cpp:15
    return cwp_camera_from_c2w(m, fx, fx, w, h, c);
}

extern "C" int cwp_params_defaults(cwp_params* p) {
    CWPB_CHECK(p, CWP_ERR_INVALID, "NULL argument");
    memset(p, 0, sizeof *p);
    p->sun_to[0] = 0.3f; p->sun_to[1] = -0.5f; p->sun_to[2] = 0.8f;
    for (int i = 0; i < 3; i++) { p->sun_e[i] = 3.f; p->sky[i] = 0.3f; }
    p->max_b = 8; p->seed = 1000; p->filter_bh = 0;
    return cwp_params_finish(p, 0.526f, 1e-4f, 1.f);
}

// Blackman-Harris inverse CDF over a window of the given width in pixels at n+1 points (core/sampling.h:38-43)
static void bh_table(float* tab, int n, double width) {
    const int NS = 4096; std::vector<double> cdf(NS + 1, 0.0);
    for (int i = 0; i < NS; i++) {
        double t = (i + 0.5) / NS;
        double f = 0.35875 - 0.48829 * cos(2 * M_PI * t) + 0.14128 * cos(4 * M_PI * t) - 0.01168 * cos(6 * M_PI * t);
        cdf[i + 1] = cdf[i] + fmax(f, 0.0);
    }
    for (int i = 0; i <= NS; i++) cdf[i] /= cdf[NS];
    for (int k = 0; k <= n; k++) {
        double u = (double)k / n; int j = 0;
        while (j < NS - 1 && cdf[j + 1] < u) j++;
        double t = cdf[j + 1] > cdf[j] ? (u - cdf[j]) / (cdf[j + 1] - cdf[j]) : 0.0;
        tab[k] = (float)(((j + t) / NS - 0.5) * width);
    }
}

extern "C" int cwp_params_finish(cwp_params* p, float sunAngleDeg, float epsScale, float extent) {
    CWPB_CHECK(p, CWP_ERR_INVALID, "NULL argument");
    float3 s = normalize(f3(p->sun_to[0], p->sun_to[1], p->sun_to[2]));
    p->sun_to[0] = s.x; p->sun_to[1] = s.y; p->sun_to[2] = s.z;
    p->sun_cos = cosf(0.5f * sunAngleDeg * 3.14159265f / 180.f);   // scene_setup.cpp:182
    p->eps = epsScale * extent;                                      // scene_setup.cpp:183
    bh_table(p->ftab, CWP_FILTER_TABLE, 1.5);
    return CWP_OK;
}
