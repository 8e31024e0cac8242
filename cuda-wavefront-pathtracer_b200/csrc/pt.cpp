// pt.cpp - batch renderer command line: the reference CLI's flags and per-frame JSON statistics (app/pt.cpp:13-53,
// app/scene_setup.cpp:27-57, 85-271) on top of the C ABI of libcwpb200.so. Loads a mesh (PLY / OBJ) or generates the
// box field, reads camera and lighting JSON files, builds the BVH on the host, renders on the GPU, prints one JSON
// line per timed frame and writes <out>.png (sRGB) and <out>.pfm (linear radiance).
//   Covered: the legacy diffuse integrator (Lambert + sun + constant sky), BVH2 / BVH4 / CWBVH, Woop and
//   Moller-Trumbore triangles, CUDA-graph or host-loop frames. Flags of the reference that select paths this
//   build does not have (full integrator, environment maps, textures, scene files, viewer) are refused with a message.
#include "cwp_b200.h"
#include "host_scene.h"
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using cwpb::Json;

namespace {

struct Args {
    std::string mesh, camera, out = "out", variant = "bvh2", c2wKey = "c2w_blender_zup", tri = "mt", c2w, lighting, integrator = "auto";
    std::string builder = "sah", collapse = "sah";
    int fuse = -1, leaf = 4, batch = 64, boxes = 0, frame = 0, w = 512, h = 512, spp = 256, bounces = 8, persistent = 0, filterBH = 1, smooth = 1;
    int warm = 8, yupToZup = -1, reps = 1, devloop = 0, sort = 0, graph = -1, bins = 16, threads = 0;
    float fx = 0, fy = 0, hfov = 0, epsScale = 1e-4f, nearClip = 0.f, sunAngleDeg = 0.526f, aperture = -1.f, focusDist = -1.f;
    unsigned seed = 1000;
    float sunTo[3] = { 0.3f, -0.5f, 0.8f }, sunE[3] = { 3.f, 3.f, 3.f }, sky[3] = { 0.3f, 0.3f, 0.3f }, albedo[3] = { -1.f, 0.f, 0.f };
};

bool parse(int argc, char** argv, Args& A) {
    for (int i = 1; i < argc; i++) {
        std::string k = argv[i];
        auto need = [&](int n) { if (i + n >= argc) { fprintf(stderr, "%s needs %d value(s)\n", k.c_str(), n); exit(1); } };
        auto S = [&]() { need(1); return std::string(argv[++i]); };
        auto I = [&]() { need(1); return atoi(argv[++i]); };
        auto F = [&]() { need(1); return (float)atof(argv[++i]); };
        auto F3 = [&](float* v) { need(3); for (int j = 0; j < 3; j++) v[j] = (float)atof(argv[++i]); };
        if (k == "--mesh") A.mesh = S(); else if (k == "--camera") A.camera = S(); else if (k == "--out") A.out = S();
        else if (k == "--variant") A.variant = S(); else if (k == "--c2w_key") A.c2wKey = S(); else if (k == "--c2w") A.c2w = S(); else if (k == "--tri") A.tri = S();
        else if (k == "--boxes") A.boxes = I(); else if (k == "--frame") A.frame = I(); else if (k == "--width") A.w = I(); else if (k == "--height") A.h = I();
        else if (k == "--spp") A.spp = I(); else if (k == "--bounces") A.bounces = I(); else if (k == "--persistent") A.persistent = I();
        else if (k == "--filter") A.filterBH = S() == "bh"; else if (k == "--smooth") A.smooth = I(); else if (k == "--warm") A.warm = I();
        else if (k == "--yup_to_zup") A.yupToZup = I(); else if (k == "--reps") A.reps = I(); else if (k == "--batch") A.batch = I();
        else if (k == "--devloop") A.devloop = I(); else if (k == "--sort") A.sort = I(); else if (k == "--fuse") A.fuse = I(); else if (k == "--leaf") A.leaf = I();
        else if (k == "--fx") A.fx = F(); else if (k == "--fy") A.fy = F(); else if (k == "--hfov") A.hfov = F(); else if (k == "--seed") A.seed = (unsigned)I();
        else if (k == "--sun_to") F3(A.sunTo); else if (k == "--sun_rgb") F3(A.sunE); else if (k == "--sky") F3(A.sky); else if (k == "--albedo") F3(A.albedo);
        else if (k == "--sun_angle") A.sunAngleDeg = F(); else if (k == "--eps") A.epsScale = F(); else if (k == "--near") A.nearClip = F();
        else if (k == "--lighting") A.lighting = S(); else if (k == "--integrator") A.integrator = S(); else if (k == "--graph") A.graph = I();
        else if (k == "--builder") A.builder = S(); else if (k == "--collapse") A.collapse = S(); else if (k == "--bins") A.bins = I(); else if (k == "--threads") A.threads = I();
        else if (k == "--aperture") A.aperture = F(); else if (k == "--focus_dist") A.focusDist = F();
        else if (k == "--synthetic" || k == "--scene" || k == "--materials" || k == "--env" || k == "--env_strength" || k == "--env_rot" ||
                 k == "--light_sampling" || k == "--rr" || k == "--rr_depth" || k == "--gd_energy" || k == "--bump_shadow" || k == "--tex_filter" ||
                 k == "--textures" || k == "--loader" || k == "--env_sampling" || k == "--frames" || k == "--frame_start" || k == "--flatten") {
            fprintf(stderr, "%s selects the full integrator, scene files or the sphere scene, which this build does not provide (diffuse benchmark path only)\n", k.c_str());
            return false;
        } else { fprintf(stderr, "unknown arg %s\n", argv[i]); return false; }
    }
    if (A.integrator == "full") { fprintf(stderr, "--integrator full is not provided by this build\n"); return false; }
    if (A.integrator != "auto" && A.integrator != "legacy") { fprintf(stderr, "--integrator must be auto, legacy or full\n"); return false; }
    if (A.builder != "sah") { fprintf(stderr, "--builder %s: only the host binned-SAH builder is available\n", A.builder.c_str()); return false; }
    if (A.collapse != "sah" && A.collapse != "greedy") { fprintf(stderr, "--collapse must be sah or greedy\n"); return false; }
    if (A.variant != "bvh2" && A.variant != "bvh4" && A.variant != "bvh8") { fprintf(stderr, "--variant must be bvh2, bvh4 or bvh8\n"); return false; }
    return true;
}

std::vector<double> numbers_of(const Json& j, const char* key) { return j.numbers(key); }

int fail(const char* what) { fprintf(stderr, "%s: %s\n", what, cwp_last_error()); return 1; }

bool write_png(const std::string& path, int w, int h, const std::vector<uint8_t>& rgb) {
    // stored (uncompressed) deflate blocks, as io/image.cpp:16-37
    static uint32_t tab[256]; static bool init = false;
    if (!init) { for (uint32_t n = 0; n < 256; n++) { uint32_t c = n; for (int k = 0; k < 8; k++) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1; tab[n] = c; } init = true; }
    auto crc = [&](const std::vector<uint8_t>& b) { uint32_t c = 0xFFFFFFFFu; for (uint8_t x : b) c = tab[(c ^ x) & 0xFF] ^ (c >> 8); return c ^ 0xFFFFFFFFu; };
    auto be32 = [](std::vector<uint8_t>& v, uint32_t x) { v.push_back(x >> 24); v.push_back(x >> 16); v.push_back(x >> 8); v.push_back(x); };
    FILE* fp = fopen(path.c_str(), "wb"); if (!fp) return false;
    auto chunk = [&](const char* type, const std::vector<uint8_t>& data) {
        std::vector<uint8_t> len, td(type, type + 4), c; be32(len, (uint32_t)data.size()); td.insert(td.end(), data.begin(), data.end()); be32(c, crc(td));
        fwrite(len.data(), 1, 4, fp); fwrite(td.data(), 1, td.size(), fp); fwrite(c.data(), 1, 4, fp);
    };
    const uint8_t sig[8] = { 137, 80, 78, 71, 13, 10, 26, 10 }; fwrite(sig, 1, 8, fp);
    std::vector<uint8_t> ihdr; be32(ihdr, w); be32(ihdr, h); ihdr.insert(ihdr.end(), { 8, 2, 0, 0, 0 }); chunk("IHDR", ihdr);
    std::vector<uint8_t> raw; raw.reserve((size_t)h * (3 * w + 1));
    for (int y = 0; y < h; y++) { raw.push_back(0); raw.insert(raw.end(), rgb.begin() + (size_t)y * w * 3, rgb.begin() + (size_t)(y + 1) * w * 3); }
    std::vector<uint8_t> z = { 0x78, 0x01 }; uint32_t a = 1, b = 0;
    for (uint8_t x : raw) { a = (a + x) % 65521; b = (b + a) % 65521; }
    for (size_t pos = 0; pos < raw.size();) {
        size_t n = std::min<size_t>(65535, raw.size() - pos); bool last = pos + n == raw.size();
        z.insert(z.end(), { (uint8_t)last, (uint8_t)(n & 255), (uint8_t)(n >> 8), (uint8_t)(~n & 255), (uint8_t)((~n >> 8) & 255) });
        z.insert(z.end(), raw.begin() + pos, raw.begin() + pos + n); pos += n;
    }
    be32(z, (b << 16) | a); chunk("IDAT", z); chunk("IEND", {});
    return fclose(fp) == 0;
}

}  // namespace

int main(int argc, char** argv) {
    Args A;
    if (!parse(argc, argv, A)) return 1;
    auto t0 = std::chrono::steady_clock::now();
    // ---- scene ----
    cwp_mesh* mesh = nullptr;
    if (A.boxes > 0) { if (cwp_mesh_box_field(A.boxes, 1, &mesh)) return fail("box field"); }
    else if (!A.mesh.empty()) { if (cwp_mesh_load(A.mesh.c_str(), &mesh)) return fail("mesh"); }
    else { fprintf(stderr, "no scene: give --mesh PATH or --boxes N\n"); return 1; }
    cwp_mesh_view mv; cwp_mesh_view_of(mesh, &mv);
    std::vector<float> v(mv.verts, mv.verts + 3 * mv.n_verts), nrm, kd(mv.albedo, mv.albedo + 3 * mv.n_albedo);
    if (mv.normals) nrm.assign(mv.normals, mv.normals + 3 * mv.n_verts);
    std::vector<int> f(mv.faces, mv.faces + 3 * mv.n_tris), fm(mv.n_tris, 0);
    if (mv.face_mat) fm.assign(mv.face_mat, mv.face_mat + mv.n_tris);
    std::string ext = A.mesh.size() > 5 ? A.mesh.substr(A.mesh.size() - 5) : "";
    if (A.yupToZup == 1) {   // y-up -> z-up: (x, y, z) -> (x, -z, y), scene_setup.cpp:65-67
        for (size_t i = 0; i < v.size(); i += 3) { float y = v[i + 1], z = v[i + 2]; v[i + 1] = -z; v[i + 2] = y; }
        for (size_t i = 0; i < nrm.size(); i += 3) { float y = nrm[i + 1], z = nrm[i + 2]; nrm[i + 1] = -z; nrm[i + 2] = y; }
    }
    if (!A.smooth) nrm.clear();
    Json L;
    if (!A.lighting.empty()) {
        std::string err;
        if (!cwpb::parse_json(cwpb::read_text(A.lighting), L, &err)) { fprintf(stderr, "lighting file %s: %s\n", A.lighting.c_str(), err.c_str()); return 1; }
        std::vector<double> x = L.numbers("sun_dir_to_light_world_zup"); if (x.size() == 3) for (int j = 0; j < 3; j++) A.sunTo[j] = (float)x[j];
        if (const Json* e = L.at("sun_irradiance_W_m2")) if (e->kind == Json::Num) for (int j = 0; j < 3; j++) A.sunE[j] = (float)e->num;
        if (const Json* e = L.at("sun_angle_rad")) if (e->kind == Json::Num) A.sunAngleDeg = (float)(e->num * 180.0 / M_PI);
        x = L.numbers("sky_radiance_rgb_linear"); if (x.size() == 3) for (int j = 0; j < 3; j++) A.sky[j] = (float)x[j];
        x = L.numbers("albedo_rgb_linear_by_material_index");
        if (x.size() >= 3) { kd.clear(); for (size_t j = 0; j + 2 < x.size(); j += 3) for (int c = 0; c < 3; c++) kd.push_back((float)x[j + c]); }
        if (L.at("env_map")) { fprintf(stderr, "lighting file %s: environment maps are not provided by this build\n", A.lighting.c_str()); return 1; }
    }
    int maxMat = 0; for (int m : fm) maxMat = m > maxMat ? m : maxMat;
    while ((int)(kd.size() / 3) <= maxMat) { kd.push_back(0.8f); kd.push_back(0.8f); kd.push_back(0.8f); }
    if (A.albedo[0] >= 0.f) for (size_t j = 0; j < kd.size(); j += 3) for (int c = 0; c < 3; c++) kd[j + c] = A.albedo[c];
    cwp_mesh_free(mesh); mesh = nullptr;
    cwp_mesh_view nv{ v.data(), (int64_t)(v.size() / 3), f.data(), (int64_t)(f.size() / 3), fm.data(), nrm.empty() ? nullptr : nrm.data(), kd.data(), (int32_t)(kd.size() / 3) };
    if (cwp_mesh_from_view(&nv, &mesh)) return fail("mesh");
    float lo[3] = { 1e30f, 1e30f, 1e30f }, hi[3] = { -1e30f, -1e30f, -1e30f };
    for (size_t i = 0; i < v.size(); i += 3) for (int c = 0; c < 3; c++) { lo[c] = fminf(lo[c], v[i + c]); hi[c] = fmaxf(hi[c], v[i + c]); }
    const float extent = fmaxf(hi[0] - lo[0], fmaxf(hi[1] - lo[1], hi[2] - lo[2]));
    double loadS = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    fprintf(stderr, "mesh: %zu verts %zu tris, normals=%d, mats=%zu, extent=%.3f load %.2fs\n", v.size() / 3, f.size() / 3, !nrm.empty(), kd.size() / 3, extent, loadS);
    // ---- camera ----
    float c2w[16] = { 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1 }; bool haveC2w = false;
    if (!A.camera.empty()) {
        Json C; std::string err;
        if (!cwpb::parse_json(cwpb::read_text(A.camera), C, &err)) { fprintf(stderr, "camera file %s: %s\n", A.camera.c_str(), err.c_str()); return 1; }
        if (A.fx == 0 && C.at("fx")) {   // fx / fy from the file when its image size matches, else its hfov (scene_files.cpp:57-67)
            if ((int)C.number("width", 0) == A.w && (int)C.number("height", 0) == A.h) { A.fx = (float)C.number("fx", 0); A.fy = (float)C.number("fy", 0); }
            else if (A.hfov == 0 && C.at("hfov_deg")) A.hfov = (float)C.number("hfov_deg", 0);
        }
        std::vector<double> m = C.numbers(A.c2wKey.c_str());
        size_t off = m.size() == 16 ? 0 : (size_t)A.frame * 16;
        if (m.size() < 16 || off + 16 > m.size()) { fprintf(stderr, "no matrix %s[%d] in camera file\n", A.c2wKey.c_str(), A.frame); return 1; }
        for (int j = 0; j < 16; j++) c2w[j] = (float)m[off + j];
        haveC2w = true;
        if (A.aperture < 0.f && C.at("aperture_radius")) A.aperture = (float)C.number("aperture_radius", 0);
        if (A.focusDist < 0.f && C.at("focus_distance")) A.focusDist = (float)C.number("focus_distance", 0);
    }
    if (!A.c2w.empty()) { std::string s = A.c2w; for (char& ch : s) if (ch == ',') ch = ' '; const char* p = s.c_str(); char* e; for (int j = 0; j < 16; j++) { c2w[j] = (float)strtod(p, &e); p = e; } haveC2w = true; }
    if (!haveC2w && A.boxes > 0) {   // box field without a camera: the benchmark view
        const float pos[3] = { 0.f, -34.f, 22.f }, tgt[3] = { 0.f, 0.f, 0.f }, up[3] = { 0.f, 0.f, 1.f }; cwp_camera c;
        if (A.hfov == 0 && A.fx == 0) A.hfov = 45.f;
        cwp_camera_look_at(pos, tgt, up, 45.f, A.w, A.h, &c);
        for (int i = 0; i < 3; i++) { c2w[4 * i] = c.ax[i]; c2w[4 * i + 1] = c.ay[i]; c2w[4 * i + 2] = c.az[i]; c2w[4 * i + 3] = c.pos[i]; }
        haveC2w = true;
    }
    if (!haveC2w) { fprintf(stderr, "no camera\n"); return 1; }
    if (A.fx == 0) { if (A.hfov == 0) A.hfov = 50.f; A.fx = (A.w * 0.5f) / tanf(A.hfov * 0.5f * 3.14159265f / 180.f); }
    if (A.fy == 0) A.fy = A.fx;
    cwp_params P; cwp_params_defaults(&P);
    if (cwp_camera_from_c2w(c2w, A.fx, A.fy, A.w, A.h, &P.cam)) return fail("camera");
    if (A.aperture > 0.f) {
        if (!(A.focusDist > 0.f)) { fprintf(stderr, "thin lens: --aperture needs --focus_dist (or \"focus_distance\" in the camera file)\n"); return 1; }
        P.cam.lens_r = A.aperture; P.cam.focus_d = A.focusDist;
    }
    for (int j = 0; j < 3; j++) { P.sun_to[j] = A.sunTo[j]; P.sun_e[j] = A.sunE[j]; P.sky[j] = A.sky[j]; }
    P.max_b = A.bounces; P.seed = A.seed; P.near_clip = A.nearClip; P.has_n = nrm.empty() ? 0 : 1; P.filter_bh = A.filterBH;
    cwp_params_finish(&P, A.sunAngleDeg, A.epsScale, extent);
    // ---- BVH ----
    const int V = A.variant == "bvh4" ? 4 : A.variant == "bvh8" ? 8 : 2, TRI = A.tri == "woop" ? 1 : 0;
    const bool cw = V == 8 && A.collapse == "sah";
    cwp_build_options bo{ V, A.bins, A.leaf, cw ? 0 : 1, A.threads };
    cwp_bvh* bvh = nullptr;
    auto tb = std::chrono::steady_clock::now();
    if (cwp_bvh_build(mesh, &bo, &bvh)) return fail("BVH");
    double bvhS = std::chrono::duration<double>(std::chrono::steady_clock::now() - tb).count();
    cwp_bvh_data bd; cwp_bvh_data_of(bvh, &bd);
    const int reportLeaf = cw ? 3 : (V == 8 && A.leaf > 4) ? 4 : A.leaf;
    fprintf(stderr, "BVH%d (sah, %d bins%s): %lld nodes (%.1f MB), depth %d, SAH %.3f, build %.2fs, tri=%s\n", V, A.bins, V == 8 ? (cw ? ", SAH collapse" : ", greedy collapse") : "",
            (long long)(bd.n_node_float4 / bd.node_stride), bd.n_node_float4 * 16 / 1e6, bd.max_depth, bd.sah, bvhS, A.tri.c_str());
    // ---- render ----
    const int K = A.batch < 1 ? 1 : A.batch;
    if (A.spp % K) { fprintf(stderr, "spp must be a multiple of batch\n"); return 1; }
    if (A.graph < 0) A.graph = 1;
    if (A.devloop || A.sort || A.persistent) fprintf(stderr, "note: --devloop/--sort/--persistent are ablation variants of the reference; frames here always use persistent kernels\n");
    cwp_scene_buffers sb{ bd.nodes, bd.n_node_float4, bd.node_stride, bd.tris, bd.n_tris, bd.nrm, bd.woop, kd.data(), (int32_t)(kd.size() / 3) };
    cwp_render_options ro{}; ro.variant = V; ro.tri = TRI; ro.batch = K; ro.bounces = A.bounces; ro.graph = A.graph;
    cwp_renderer* R = nullptr; cwp_renderer_create(&R);
    if (cwp_renderer_init(R, &P, &sb, &ro)) return fail("init");
    cwp_renderer_info info; cwp_renderer_info_of(R, &info);
    cwp_frame_stats W{};
    if (A.warm > 0) { if (cwp_renderer_render(R, ((A.warm + K - 1) / K) * K, &W, 0, 1)) return fail("render"); }
    fprintf(stderr, "warmup: %.1f ms, %.1f Mrays/s\n", W.frame_ms, W.frame_ms > 0 ? (W.rays + W.shadow_rays) / (W.frame_ms * 1e3) : 0.0);
    const int N = A.w * A.h;
    for (int r = 0; r < A.reps; r++) {
        cwp_frame_stats st;
        if (cwp_renderer_render(R, A.spp, &st, 0, 1)) return fail("render");
        double tot = st.rays + st.shadow_rays;
        printf("{\"rep\":%d,\"variant\":\"bvh%d\",\"tri\":\"%s\",\"persistent\":%d,\"devloop\":%d,\"sort\":%d,\"fuse\":%d,\"leaf\":%d,\"batch\":%d,\"minb\":0,\"scene\":\"%s\",\"tris\":%lld,"
               "\"bvh_nodes\":%lld,\"bvh_bytes\":%lld,\"bvh_depth\":%d,\"bvh_build_s\":%.2f,\"w\":%d,\"h\":%d,\"spp\":%d,\"bounces\":%d,\"rays_closest\":%.0f,\"rays_shadow\":%.0f,"
               "\"rays_total\":%.0f,\"t_trace_ms\":%.2f,\"t_frame_ms\":%.2f,\"mrays_s_trace\":%.1f,\"mrays_s_e2e\":%.1f,\"avg_path_len\":%.3f,\"vram_MB\":%.0f,\"pt_blocks\":%d,"
               "\"gpu\":\"%s\",\"filter\":\"%s\",\"smooth\":%d,\"seed\":%u,\"integrator\":\"legacy\",\"lens_r\":%.4f,\"focus_d\":%.4f,\"env_sampling\":\"importance\",\"textures\":0,"
               "\"builder\":\"sah\",\"collapse\":\"%s\",\"bvh_tree_ms\":%.2f,\"bvh_post_ms\":0.00,\"bvh_sah\":%.4f,\"graph\":%d,\"instances\":0,\"flatten\":0,\"frame\":%d,\"tlas_ms\":0.000,\"bins\":%d}\n",
               r, V, A.tri.c_str(), A.persistent, A.devloop, A.sort, A.fuse < 0 ? 1 : A.fuse, reportLeaf, K, A.boxes > 0 ? "boxes" : A.mesh.c_str(), (long long)bd.n_tris,
               (long long)(bd.n_node_float4 / bd.node_stride), (long long)(bd.n_node_float4 * 16), bd.max_depth, bvhS, A.w, A.h, A.spp, A.bounces, st.rays, st.shadow_rays,
               tot, st.trace_ms, st.frame_ms, tot / (st.trace_ms * 1e3), tot / (st.frame_ms * 1e3), st.rays / ((double)N * A.spp), info.vram_mb, info.pt_blocks, info.gpu_name,
               A.filterBH ? "blackman-harris1.5" : "box", P.has_n, A.seed, P.cam.lens_r, P.cam.focus_d, V == 8 ? A.collapse.c_str() : "-", bd.build_ms, bd.sah, A.graph, A.frame, A.bins);
        fflush(stdout);
    }
    std::vector<float> acc((size_t)N * 4), lin((size_t)N * 3); std::vector<uint8_t> rgb((size_t)N * 3);
    if (cwp_renderer_read_accum(R, acc.data())) return fail("readback");
    for (int i = 0; i < N; i++) for (int c = 0; c < 3; c++) lin[3 * i + c] = acc[4 * (size_t)i + c] / A.spp;
    for (size_t i = 0; i < lin.size(); i++) {   // clip [0, 1] + sRGB OETF, exposure 0 (io/image.cpp:45-50)
        float x = fminf(fmaxf(lin[i], 0.f), 1.f); x = x <= 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.f / 2.4f) - 0.055f;
        rgb[i] = (uint8_t)(x * 255.f + 0.5f);
    }
    write_png(A.out + ".png", A.w, A.h, rgb);
    FILE* fp = fopen((A.out + ".pfm").c_str(), "wb");
    if (fp) { fprintf(fp, "PF\n%d %d\n-1.0\n", A.w, A.h); for (int y = A.h - 1; y >= 0; y--) fwrite(&lin[(size_t)y * A.w * 3], 4, (size_t)A.w * 3, fp); fclose(fp); }
    fprintf(stderr, "wrote %s.png / .pfm (tonemap: clip[0,1] + sRGB OETF, exposure 0)\n", A.out.c_str());
    cwp_renderer_destroy(R); cwp_bvh_free(bvh); cwp_mesh_free(mesh);
    return 0;
}
