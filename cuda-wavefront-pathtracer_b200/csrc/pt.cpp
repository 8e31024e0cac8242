// pt.cpp - batch renderer command line: the reference CLI's flags and per-frame JSON statistics (app/pt.cpp:13-53,
// app/scene_setup.cpp:27-57, 85-271) on top of the C ABI of libcwpb200.so. Loads a mesh (PLY / OBJ) or generates the
// box field, reads camera and lighting JSON files, builds the BVH on the host, renders on the GPU, prints one JSON
// line per timed frame and writes <out>.png (sRGB) and <out>.pfm (linear radiance).
//   Covered: the legacy diffuse integrator (Lambert + sun + constant sky), BVH2 / BVH4 / CWBVH, Woop and
//   Moller-Trumbore triangles, CUDA-graph or host-loop frames; and the full integrator (setupScene's rule: scene
//   files, materials files with non-Lambertian or emissive entries, environment maps, Russian roulette, or
//   --integrator full) through the library's serving form: instanced scene files with animated instances and per-mesh
//   materials files, or one mesh as a single identity instance, one request per frame. --synthetic N generates the
//   reference's sphere-grid scene (N x N spheres, 200 x 100 quads each, 200 x 200 ground) with its default view. Not
//   provided: the Assimp loader and the image textures it reads (a third-party library), the viewer.
#include "cwp_b200.h"
#include "host_scene.h"
#include <algorithm>
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
    std::string scene, materials, env, lightSampling = "mis", texFilter = "linear", envSampling = "importance", loader = "auto";
    int frames = 0, frameStart = 0, flatten = 0, rr = 0, rrDepth = 3, gdEnergy = 1, bumpShadow = 0;
    float envStrength = -1.f, envRot = -1e30f;
    int fuse = -1, leaf = 4, batch = 64, boxes = 0, synthetic = 0, frame = 0, w = 512, h = 512, spp = 256, bounces = 8, persistent = 0, filterBH = 1, smooth = 1;
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
        else if (k == "--scene") A.scene = S(); else if (k == "--materials") A.materials = S(); else if (k == "--env") A.env = S();
        else if (k == "--env_strength") A.envStrength = F(); else if (k == "--env_rot") A.envRot = F(); else if (k == "--light_sampling") A.lightSampling = S();
        else if (k == "--rr") A.rr = I(); else if (k == "--rr_depth") A.rrDepth = I(); else if (k == "--gd_energy") A.gdEnergy = I(); else if (k == "--bump_shadow") A.bumpShadow = I();
        else if (k == "--tex_filter") A.texFilter = S(); else if (k == "--textures") S(); else if (k == "--loader") A.loader = S(); else if (k == "--env_sampling") A.envSampling = S();
        else if (k == "--frames") A.frames = I(); else if (k == "--frame_start") A.frameStart = I(); else if (k == "--flatten") A.flatten = I();
        else if (k == "--synthetic") A.synthetic = I();
        else { fprintf(stderr, "unknown arg %s\n", argv[i]); return false; }
    }
    if (A.integrator != "auto" && A.integrator != "legacy" && A.integrator != "full") { fprintf(stderr, "--integrator must be auto, legacy or full\n"); return false; }
    if (A.lightSampling != "mis" && A.lightSampling != "nee" && A.lightSampling != "bsdf") { fprintf(stderr, "--light_sampling must be mis, nee or bsdf\n"); return false; }
    if (A.loader != "auto" && A.loader != "builtin") { fprintf(stderr, "--loader %s: only the built-in PLY / OBJ loader is available\n", A.loader.c_str()); return false; }
    if (A.envSampling != "importance" && A.envSampling != "uniform") { fprintf(stderr, "--env_sampling must be importance or uniform\n"); return false; }
    if (A.texFilter != "linear" && A.texFilter != "nearest") { fprintf(stderr, "--tex_filter must be linear or nearest\n"); return false; }
    // the reference builds the sphere grid and then still reads the scene file's box for the ray offset
    // (scene_setup.cpp:92-154): an ill-defined mix, refused here
    if (!A.scene.empty() && A.synthetic > 0) { fprintf(stderr, "--synthetic and --scene cannot be combined\n"); return false; }
    if (!A.scene.empty() && !A.materials.empty()) { fprintf(stderr, "--materials is per mesh in scene files (\"materials\" key)\n"); return false; }
    if (A.builder != "sah" && A.builder != "hploc") { fprintf(stderr, "--builder must be sah or hploc\n"); return false; }
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

// ---------------- full integrator: scene files and materials through the serving form ----------------
cwp_material lambert(const float* kd) {   // scene/material.h:20-24
    cwp_material m{}; for (int c = 0; c < 3; c++) { m.base_color[c] = kd[c]; m.specular_color[c] = 1.f; }
    m.metallic = 0.f; m.roughness = 1.f; m.ior = 1.5f; m.specular_weight = 0.f; m.transmission = 0.f;
    return m;
}
bool is_lambert(const cwp_material& m) { return m.metallic == 0.f && m.transmission == 0.f && m.specular_weight == 0.f; }
bool is_emissive(const cwp_material& m) { return m.emission[0] > 0.f || m.emission[1] > 0.f || m.emission[2] > 0.f; }

// a materials file (io/scene_files.cpp:28-55): entries by position, or by name against the mesh's material names;
// ids the file does not give keep their Lambertian kd
bool load_materials(const std::string& path, const cwpb::Mesh& mesh, std::vector<cwp_material>& mats) {
    Json J; std::string err;
    if (!cwpb::parse_json(cwpb::read_text(path), J, &err)) { fprintf(stderr, "materials file %s: %s\n", path.c_str(), err.c_str()); return false; }
    const Json* arr = J.at("materials");
    if (!arr || arr->kind != Json::Arr) { fprintf(stderr, "materials file %s: no \"materials\" array\n", path.c_str()); return false; }
    const float gray[3] = { 0.8f, 0.8f, 0.8f };
    mats.clear(); std::vector<bool> set; int pos = 0;
    auto v3 = [](const Json& o, const char* k, const float* def, float* out) {
        std::vector<double> v = o.numbers(k);
        for (int c = 0; c < 3; c++) out[c] = v.size() == 3 ? (float)v[c] : def[c];
    };
    for (const Json& o : arr->arr) {
        cwp_material m = lambert(gray); m.roughness = 0.5f; m.specular_weight = 1.f;   // defaultMaterial()
        float tmp[3];
        v3(o, "base_color", m.base_color, tmp); for (int c = 0; c < 3; c++) m.base_color[c] = tmp[c];
        m.metallic = (float)o.number("metallic", m.metallic); m.roughness = (float)o.number("roughness", m.roughness);
        m.ior = (float)o.number("ior", m.ior); m.specular_weight = (float)o.number("specular_weight", m.specular_weight);
        v3(o, "specular_color", m.specular_color, tmp); for (int c = 0; c < 3; c++) m.specular_color[c] = tmp[c];
        m.transmission = (float)o.number("transmission", m.transmission);
        const float one[3] = { 1.f, 1.f, 1.f }; v3(o, "emission_color", one, tmp);
        const float st = (float)o.number("emission_strength", 0.0);
        for (int c = 0; c < 3; c++) m.emission[c] = tmp[c] * st;
        int id = pos++;
        const Json* nm = o.at("name");
        if (nm && nm->kind == Json::Str && !nm->str.empty())
            for (size_t j = 0; j < mesh.matName.size(); j++) if (mesh.matName[j] == nm->str) { id = (int)j; break; }
        if ((int)mats.size() <= id) { mats.resize((size_t)id + 1, lambert(gray)); set.resize((size_t)id + 1, false); }
        mats[id] = m; set[id] = true;
    }
    for (size_t j = 0; j < mats.size(); j++) if (!set[j]) mats[j] = lambert(3 * j + 2 < mesh.kd.size() ? &mesh.kd[3 * j] : gray);
    return true;
}

// a mesh's material table (normalizeMaterials, scene/instances.cpp:81-88): file entries, else Lambertian kd
std::vector<cwp_material> mesh_materials(const cwpb::Mesh& m, const std::vector<cwp_material>& fileMats) {
    int maxMat = 0; for (int t : m.fm) maxMat = t > maxMat ? t : maxMat;
    const size_t nm = std::max(std::max(m.kd.size() / 3, fileMats.size()), (size_t)maxMat + 1);
    const float gray[3] = { 0.8f, 0.8f, 0.8f };
    std::vector<cwp_material> out;
    for (size_t j = 0; j < nm; j++) out.push_back(j < fileMats.size() ? fileMats[j] : lambert(3 * j + 2 < m.kd.size() ? &m.kd[3 * j] : gray));
    return out;
}

struct FullScene {
    std::vector<cwpb::Mesh> meshes; std::vector<std::vector<cwp_material>> mats;
    std::vector<cwp_instance_desc> inst; int frames = 1;
    std::vector<std::vector<float>> xf;   // per instance: 3x4 matrices by frame ("transform" / "transforms"), or empty
};

// scene file (scene/instances.cpp:19-47): meshes with their materials files, parametric animated instances
bool load_scene(const std::string& path, const Args& A, FullScene& S) {
    Json J; std::string err;
    if (!cwpb::parse_json(cwpb::read_text(path), J, &err)) { fprintf(stderr, "scene file %s: %s\n", path.c_str(), err.c_str()); return false; }
    const std::string dir = path.find_last_of('/') == std::string::npos ? std::string() : path.substr(0, path.find_last_of('/') + 1);
    auto rel = [&](const std::string& p) { return p.empty() || p[0] == '/' ? p : dir + p; };
    S.frames = (int)J.number("frames", 1);
    const Json* ms = J.at("meshes"); const Json* is = J.at("instances");
    if (!ms || ms->kind != Json::Arr || !is || is->kind != Json::Arr) { fprintf(stderr, "scene file %s: needs \"meshes\" and \"instances\" arrays\n", path.c_str()); return false; }
    for (const Json& m : ms->arr) {
        const Json* f = m.at("file"); const Json* mt = m.at("materials"); const Json* ld = m.at("loader");
        if (!f || f->kind != Json::Str || f->str.empty()) { fprintf(stderr, "scene file: mesh without \"file\"\n"); return false; }
        if (ld && ld->kind == Json::Str && ld->str == "assimp") { fprintf(stderr, "scene file: the Assimp loader is not available\n"); return false; }
        cwpb::Mesh mesh;
        if (!cwpb::load_mesh(rel(f->str), mesh, &err)) { fprintf(stderr, "%s: %s\n", rel(f->str).c_str(), err.c_str()); return false; }
        if ((int)m.number("yup_to_zup", -1) == 1) {
            for (size_t i = 0; i < mesh.v.size(); i += 3) { float y = mesh.v[i + 1], z = mesh.v[i + 2]; mesh.v[i + 1] = -z; mesh.v[i + 2] = y; }
            for (size_t i = 0; i < mesh.n.size(); i += 3) { float y = mesh.n[i + 1], z = mesh.n[i + 2]; mesh.n[i + 1] = -z; mesh.n[i + 2] = y; }
        }
        std::vector<cwp_material> fileMats;
        if (mt && mt->kind == Json::Str && !mt->str.empty() && !load_materials(rel(mt->str), mesh, fileMats)) return false;
        S.mats.push_back(mesh_materials(mesh, fileMats)); S.meshes.push_back(std::move(mesh));
    }
    for (const Json& o : is->arr) {
        // a fixed matrix or one per frame (12 or 16 numbers each, the first 12 used; scene/instances.cpp:8-12, 36-40)
        std::vector<float> xf;
        if (o.at("transform")) {
            std::vector<double> v = o.numbers("transform");
            if (v.size() != 12 && v.size() != 16) { fprintf(stderr, "scene file: transform needs 12 or 16 numbers\n"); return false; }
            for (int k = 0; k < 12; k++) xf.push_back((float)v[k]);
        }
        if (const Json* tf = o.at("transforms")) {
            std::vector<float> per;
            for (const Json& t : tf->arr) {
                std::vector<double> v; for (const Json& x : t.arr) v.push_back(x.num);
                if (v.size() != 12 && v.size() != 16) { fprintf(stderr, "scene file: transforms entries need 12 or 16 numbers\n"); return false; }
                for (int k = 0; k < 12; k++) per.push_back((float)v[k]);
            }
            if (!per.empty()) xf = per;   // per-frame matrices take precedence over a fixed one
        }
        S.xf.push_back(xf);
        cwp_instance_desc d{}; d.mesh = (int)o.number("mesh", 0);
        if (d.mesh < 0 || d.mesh >= (int)S.meshes.size()) { fprintf(stderr, "scene file: instance mesh %d out of range\n", d.mesh); return false; }
        auto v3 = [&](const char* k, float* out, float def, bool scalar) {
            const Json* e = o.at(k);
            if (scalar && e && e->kind == Json::Num) { out[0] = out[1] = out[2] = (float)e->num; return; }
            std::vector<double> v = o.numbers(k);
            for (int c = 0; c < 3; c++) out[c] = v.size() == 3 ? (float)v[c] : def;
        };
        v3("translate", d.translate, 0.f, false); v3("translate_per_frame", d.translate_per_frame, 0.f, false);
        v3("axis", d.axis, 0.f, false); if (!o.at("axis") || o.numbers("axis").size() != 3) { d.axis[0] = d.axis[1] = 0.f; d.axis[2] = 1.f; }
        d.angle_deg = (float)o.number("angle_deg", 0.0); d.angle_deg_per_frame = (float)o.number("angle_deg_per_frame", 0.0);
        v3("scale", d.scale, 1.f, true); v3("scale_per_frame", d.scale_per_frame, 0.f, true);
        S.inst.push_back(d);
    }
    (void)A;
    return true;
}

bool write_images(const std::string& name, int w, int h, const std::vector<float>& lin);

// the camera of either path (scene_setup.cpp:158-178): a camera file, --c2w, or the box field's benchmark view
bool camera_c2w(Args& A, float c2w[16]) {
    bool haveC2w = false;
    for (int j = 0; j < 16; j++) c2w[j] = (j % 5 == 0) ? 1.f : 0.f;
    // the sphere grid sets its view and a 50 deg field before any camera file is read (scene_setup.cpp:92-95), so a
    // file's matrix replaces the view but its hfov_deg does not replace the 50 deg
    if (A.synthetic > 0) { cwp_sphere_grid_c2w(c2w); haveC2w = true; if (A.hfov == 0 && A.fx == 0) A.hfov = 50.f; }
    if (!A.camera.empty()) {
        Json C; std::string err;
        if (!cwpb::parse_json(cwpb::read_text(A.camera), C, &err)) { fprintf(stderr, "camera file %s: %s\n", A.camera.c_str(), err.c_str()); return false; }
        if (A.fx == 0 && C.at("fx")) {   // fx / fy from the file when its image size matches, else its hfov (scene_files.cpp:57-67)
            if ((int)C.number("width", 0) == A.w && (int)C.number("height", 0) == A.h) { A.fx = (float)C.number("fx", 0); A.fy = (float)C.number("fy", 0); }
            else if (A.hfov == 0 && C.at("hfov_deg")) A.hfov = (float)C.number("hfov_deg", 0);
        }
        std::vector<double> m = C.numbers(A.c2wKey.c_str());
        size_t off = m.size() == 16 ? 0 : (size_t)A.frame * 16;
        if (m.size() < 16 || off + 16 > m.size()) { fprintf(stderr, "no matrix %s[%d] in camera file\n", A.c2wKey.c_str(), A.frame); return false; }
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
    if (!haveC2w) { fprintf(stderr, "no camera\n"); return false; }
    if (A.fx == 0) { if (A.hfov == 0) A.hfov = 50.f; A.fx = (A.w * 0.5f) / tanf(A.hfov * 0.5f * 3.14159265f / 180.f); }
    if (A.fy == 0) A.fy = A.fx;
    return true;
}

// The full integrator: every mesh (or the one mesh) on the device at once, the scene's instances animated per
// frame, one request per frame and repetition. Statistics: one JSON line per rendered frame, as the legacy path.
int run_full(Args& A, const std::string& envFromLighting, float envStrengthL, float envRotL, const std::vector<float>& kdLighting) {
    FullScene S;
    const float gray[3] = { 0.8f, 0.8f, 0.8f };
    // the sphere grid wins over every mesh source, as in the reference (scene_setup.cpp:92)
    if (!A.scene.empty()) { if (!load_scene(A.scene, A, S)) return 1; }
    else {
        cwpb::Mesh mesh; std::string err;
        if (A.synthetic > 0) cwpb::sphere_grid(A.synthetic, 200, 100, 200, mesh);   // scene_setup.cpp:93
        else if (A.boxes > 0) cwpb::box_field(A.boxes, 1, 20.f, 0.2f, 3.f, mesh);   // as cwp_mesh_box_field
        else if (!cwpb::load_mesh(A.mesh, mesh, &err)) { fprintf(stderr, "%s: %s\n", A.mesh.c_str(), err.c_str()); return 1; }
        if (A.yupToZup == 1 && A.synthetic <= 0) {   // files only: the generated scenes are z-up
            for (size_t i = 0; i < mesh.v.size(); i += 3) { float y = mesh.v[i + 1], z = mesh.v[i + 2]; mesh.v[i + 1] = -z; mesh.v[i + 2] = y; }
            for (size_t i = 0; i < mesh.n.size(); i += 3) { float y = mesh.n[i + 1], z = mesh.n[i + 2]; mesh.n[i + 1] = -z; mesh.n[i + 2] = y; }
        }
        if (!kdLighting.empty()) mesh.kd = kdLighting;
        std::vector<cwp_material> fileMats;
        if (!A.materials.empty() && !load_materials(A.materials, mesh, fileMats)) return 1;
        S.mats.push_back(mesh_materials(mesh, fileMats)); S.meshes.push_back(std::move(mesh));
        cwp_instance_desc d{}; d.axis[2] = 1.f; d.scale[0] = d.scale[1] = d.scale[2] = 1.f; S.inst.push_back(d);
    }
    (void)gray;
    // combined material table, per-mesh offsets; --albedo overrides every base colour
    std::vector<cwp_material> mats; std::vector<int32_t> base;
    for (auto& m : S.mats) { base.push_back((int32_t)mats.size()); mats.insert(mats.end(), m.begin(), m.end()); }
    if (A.albedo[0] >= 0.f) for (auto& m : mats) for (int c = 0; c < 3; c++) m.base_color[c] = A.albedo[c];
    // meshes as views (normals when --smooth and the mesh has them)
    std::vector<cwp_mesh_view> views; size_t nTris = 0;
    for (auto& m : S.meshes) {
        cwp_mesh_view v{}; v.verts = m.v.data(); v.n_verts = (int64_t)m.nv(); v.faces = m.f.data(); v.n_tris = (int64_t)m.nt(); v.face_mat = m.fm.data();
        v.normals = A.smooth && m.hasN() ? m.n.data() : nullptr; views.push_back(v); nTris += m.nt();
    }
    // the frame-0 world box of every instance's vertices gives the ray offset (scene_setup.cpp:107, 153-155)
    float lo[3] = { 1e30f, 1e30f, 1e30f }, hi[3] = { -1e30f, -1e30f, -1e30f };
    for (size_t i = 0; i < S.inst.size(); i++) {
        const cwp_instance_desc& d = S.inst[i];
        float x[12];
        if (i < S.xf.size() && !S.xf[i].empty()) std::copy(S.xf[i].begin(), S.xf[i].begin() + 12, x);
        else if (cwp_xform_animate(&d, 0, x)) return fail("instance");
        const cwpb::Mesh& m = S.meshes[d.mesh];
        for (size_t i = 0; i < m.v.size(); i += 3)
            for (int r = 0; r < 3; r++) {
                const float w = x[4 * r] * m.v[i] + x[4 * r + 1] * m.v[i + 1] + x[4 * r + 2] * m.v[i + 2] + x[4 * r + 3];
                lo[r] = fminf(lo[r], w); hi[r] = fmaxf(hi[r], w);
            }
    }
    const float extent = fmaxf(hi[0] - lo[0], fmaxf(hi[1] - lo[1], hi[2] - lo[2]));
    fprintf(stderr, "full integrator: %zu meshes, %zu instances, %zu triangles, %zu materials, extent %.3f\n", S.meshes.size(), S.inst.size(), nTris, mats.size(), extent);
    float c2w[16]; if (!camera_c2w(A, c2w)) return 1;
    cwp_params P; cwp_params_defaults(&P);
    if (cwp_camera_from_c2w(c2w, A.fx, A.fy, A.w, A.h, &P.cam)) return fail("camera");
    if (A.aperture > 0.f) {
        if (!(A.focusDist > 0.f)) { fprintf(stderr, "thin lens: --aperture needs --focus_dist (or \"focus_distance\" in the camera file)\n"); return 1; }
        P.cam.lens_r = A.aperture; P.cam.focus_d = A.focusDist;
    }
    for (int j = 0; j < 3; j++) { P.sun_to[j] = A.sunTo[j]; P.sun_e[j] = A.sunE[j]; P.sky[j] = A.sky[j]; }
    cwp_params_finish(&P, A.sunAngleDeg, A.epsScale, extent);
    // device scene, server, environment map
    auto tb = std::chrono::steady_clock::now();
    // BLAS on the host (binned SAH, the reference's default --builder sah) or on the GPU (--builder hploc)
    cwp_batch_options bo{}; bo.builder = A.builder == "hploc" ? 0 : 1; cwp_batch* B = nullptr;
    if (cwp_batch_create(views.data(), (int32_t)views.size(), &bo, &B)) return fail("scene upload / BLAS build");
    cwp_server_options so{}; so.max_requests = 1; so.max_paths = std::min<int64_t>((int64_t)A.w * A.h * A.spp, 8ll << 20); so.gd_energy = A.gdEnergy;
    cwp_server* Srv = nullptr;
    if (cwp_server_create(B, mats.data(), (int32_t)mats.size(), base.data(), &so, &Srv)) return fail("server");
    const int32_t first[2] = { 0, (int32_t)S.inst.size() };
    if (cwp_server_set_scenes(Srv, S.inst.data(), (int64_t)S.inst.size(), first, 1)) return fail("scene");
    bool anyXf = false; for (auto& x : S.xf) anyXf = anyXf || !x.empty();
    if (anyXf) {
        std::vector<float> all; std::vector<int32_t> fx, nx;
        for (auto& x : S.xf) { fx.push_back((int32_t)(all.size() / 12)); nx.push_back((int32_t)(x.size() / 12)); all.insert(all.end(), x.begin(), x.end()); }
        if (cwp_server_set_instance_xforms(Srv, all.data(), fx.data(), nx.data(), (int64_t)nx.size())) return fail("instance matrices");
    }
    const std::string envPath = !A.env.empty() ? A.env : envFromLighting;
    const float envStrength = A.envStrength >= 0.f ? A.envStrength : envStrengthL, envRot = A.envRot > -1e29f ? A.envRot : envRotL;
    if (!envPath.empty()) {
        int32_t ew = 0, eh = 0;
        if (cwp_hdr_load(envPath.c_str(), &ew, &eh, nullptr)) return fail("environment map");
        std::vector<float> rgb((size_t)ew * eh * 3);
        if (cwp_hdr_load(envPath.c_str(), &ew, &eh, rgb.data())) return fail("environment map");
        cwp_envmap em{ rgb.data(), ew, eh, envStrength, 0 };
        if (cwp_server_set_envmaps(Srv, &em, 1)) return fail("environment map");
    }
    const double setupS = std::chrono::duration<double>(std::chrono::steady_clock::now() - tb).count();
    cwp_request R0{};
    R0.scene = 0; R0.cam = P.cam; R0.spp = A.spp; R0.max_depth = A.bounces; R0.seed = A.seed;
    for (int j = 0; j < 3; j++) { R0.sun_to[j] = P.sun_to[j]; R0.sun_e[j] = P.sun_e[j]; R0.sky[j] = P.sky[j]; }
    R0.sun_cos = P.sun_cos; R0.eps = P.eps; R0.env = envPath.empty() ? -1 : 0; R0.env_rot_deg = envRot;
    R0.light_mode = A.lightSampling == "nee" ? CWP_LIGHT_NEE : A.lightSampling == "bsdf" ? CWP_LIGHT_BSDF : CWP_LIGHT_MIS;
    R0.rr = A.rr ? 1 : 0; R0.rr_depth = A.rrDepth; R0.env_uniform = A.envSampling == "uniform"; R0.bump_shadow = A.bumpShadow ? 1 : 0;
    R0.near_clip = A.nearClip; R0.filter_bh = A.filterBH;
    auto render = [&](cwp_request r, std::vector<float>* acc, cwp_request_stats& st, double& ms) -> int {
        int64_t id = 0;
        const auto t = std::chrono::steady_clock::now();
        if (cwp_server_submit(Srv, &r, &id)) return fail("submit");
        for (;;) {
            int32_t act = 0, pend = 0, n = 0; int64_t done = -1;
            if (cwp_server_step(Srv, &act, &pend)) return fail("render");
            if (cwp_server_poll(Srv, &done, 1, &n)) return fail("poll");
            if (n == 1) break;
        }
        ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
        if (cwp_server_result(Srv, id, acc ? acc->data() : nullptr, &st)) return fail("result");
        return 0;
    };
    const int F = A.frames > 0 ? A.frames : S.frames, N = A.w * A.h;
    if (A.warm > 0) { cwp_request w = R0; w.spp = A.warm; w.frame = A.frameStart; cwp_request_stats st; double ms; if (int rc = render(w, nullptr, st, ms)) return rc; }
    std::vector<float> acc((size_t)N * 4), lin((size_t)N * 3);
    for (int fi = 0; fi < F; fi++) {
        const int f = A.frameStart + fi;
        for (int r = 0; r < std::max(A.reps, 1); r++) {
            cwp_request q = R0; q.frame = f; cwp_request_stats st; double ms = 0;
            if (int rc = render(q, &acc, st, ms)) return rc;
            const double tot = st.rays + st.shadow_rays;
            printf("{\"rep\":%d,\"integrator\":\"full\",\"scene\":\"%s\",\"tris\":%zu,\"instances\":%zu,\"frame\":%d,\"w\":%d,\"h\":%d,\"spp\":%d,\"bounces\":%d,"
                   "\"rays_closest\":%.0f,\"rays_shadow\":%.0f,\"rays_total\":%.0f,\"t_frame_ms\":%.2f,\"mrays_s_e2e\":%.1f,\"avg_path_len\":%.3f,\"light_sampling\":\"%s\","
                   "\"rr\":%d,\"env\":%d,\"filter\":\"%s\",\"seed\":%u,\"setup_s\":%.2f}\n",
                   r, A.scene.empty() ? (A.boxes > 0 ? "boxes" : A.synthetic > 0 ? "synthetic" : A.mesh.c_str()) : A.scene.c_str(), nTris, S.inst.size(), f, A.w, A.h, A.spp, A.bounces,
                   st.rays, st.shadow_rays, tot, ms, tot / (ms * 1e3), st.rays / ((double)N * A.spp), A.lightSampling.c_str(), R0.rr, R0.env >= 0,
                   A.filterBH ? "blackman-harris1.5" : "box", A.seed, setupS);
            fflush(stdout);
        }
        for (int i = 0; i < N; i++) for (int c = 0; c < 3; c++) lin[3 * (size_t)i + c] = acc[4 * (size_t)i + c] / A.spp;
        std::string name = A.out; if (F > 1) { char b[32]; snprintf(b, sizeof b, "_f%04d", f); name += b; }
        if (!write_images(name, A.w, A.h, lin)) { fprintf(stderr, "cannot write %s\n", name.c_str()); return 1; }
    }
    cwp_server_destroy(Srv); cwp_batch_destroy(B);
    return 0;
}

// <name>.png (clip [0, 1] + sRGB OETF, exposure 0, io/image.cpp:45-50) and <name>.pfm (linear, bottom row first)
bool write_images(const std::string& name, int w, int h, const std::vector<float>& lin) {
    std::vector<uint8_t> rgb(lin.size());
    for (size_t i = 0; i < lin.size(); i++) {
        float x = fminf(fmaxf(lin[i], 0.f), 1.f); x = x <= 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.f / 2.4f) - 0.055f;
        rgb[i] = (uint8_t)(x * 255.f + 0.5f);
    }
    if (!write_png(name + ".png", w, h, rgb)) return false;
    FILE* fp = fopen((name + ".pfm").c_str(), "wb");
    if (!fp) return false;
    fprintf(fp, "PF\n%d %d\n-1.0\n", w, h);
    for (int y = h - 1; y >= 0; y--) fwrite(&lin[(size_t)y * w * 3], 4, (size_t)w * 3, fp);
    fclose(fp);
    fprintf(stderr, "wrote %s.png / .pfm (tonemap: clip[0,1] + sRGB OETF, exposure 0)\n", name.c_str());
    return true;
}

}  // namespace

int main(int argc, char** argv) {
    Args A;
    if (!parse(argc, argv, A)) return 1;
    auto t0 = std::chrono::steady_clock::now();
    // ---- integrator (setupScene's rule, scene_setup.cpp:137-140) ----
    std::string envL; float envStrengthL = 1.f, envRotL = 0.f;
    std::vector<float> kdL;
    if (!A.lighting.empty()) {   // lighting file keys (io/scene_files.cpp:10-24), read before either path
        Json L; std::string err;
        if (!cwpb::parse_json(cwpb::read_text(A.lighting), L, &err)) { fprintf(stderr, "lighting file %s: %s\n", A.lighting.c_str(), err.c_str()); return 1; }
        std::vector<double> x = L.numbers("sun_dir_to_light_world_zup"); if (x.size() == 3) for (int j = 0; j < 3; j++) A.sunTo[j] = (float)x[j];
        if (const Json* e = L.at("sun_irradiance_W_m2")) if (e->kind == Json::Num) for (int j = 0; j < 3; j++) A.sunE[j] = (float)e->num;
        if (const Json* e = L.at("sun_angle_rad")) if (e->kind == Json::Num) A.sunAngleDeg = (float)(e->num * 180.0 / M_PI);
        x = L.numbers("sky_radiance_rgb_linear"); if (x.size() == 3) for (int j = 0; j < 3; j++) A.sky[j] = (float)x[j];
        x = L.numbers("albedo_rgb_linear_by_material_index");
        if (x.size() >= 3) for (size_t j = 0; j + 2 < x.size(); j += 3) for (int c = 0; c < 3; c++) kdL.push_back((float)x[j + c]);
        if (const Json* e = L.at("env_map")) if (e->kind == Json::Str) envL = e->str;
        envStrengthL = (float)L.number("env_strength", 1.0); envRotL = (float)L.number("env_rotation_deg", 0.0);
        A.lighting.clear();   // consumed
    }
    bool needFull = !A.scene.empty() || A.rr != 0 || !A.env.empty() || !envL.empty();
    if (!A.materials.empty()) {
        cwpb::Mesh none; std::vector<cwp_material> fm;
        if (!load_materials(A.materials, none, fm)) return 1;
        for (auto& m : fm) if (!is_lambert(m) || is_emissive(m)) needFull = true;
    }
    if (A.integrator == "legacy" && !A.scene.empty()) { fprintf(stderr, "--integrator legacy does not render scene files (use auto or full)\n"); return 1; }
    if (A.integrator == "full" || (A.integrator == "auto" && needFull)) return run_full(A, envL, envStrengthL, envRotL, kdL);
    if (needFull) fprintf(stderr, "warn: --integrator legacy ignores specular/transmissive/emissive materials, the environment map and RR\n");
    // ---- scene ----
    cwp_mesh* mesh = nullptr;
    if (A.synthetic > 0) { if (cwp_mesh_sphere_grid(A.synthetic, 200, 100, 200, &mesh)) return fail("sphere grid"); }   // first, as scene_setup.cpp:92
    else if (A.boxes > 0) { if (cwp_mesh_box_field(A.boxes, 1, &mesh)) return fail("box field"); }
    else if (!A.mesh.empty()) { if (cwp_mesh_load(A.mesh.c_str(), &mesh)) return fail("mesh"); }
    else { fprintf(stderr, "no scene: give --mesh PATH, --boxes N or --synthetic N\n"); return 1; }
    cwp_mesh_view mv; cwp_mesh_view_of(mesh, &mv);
    std::vector<float> v(mv.verts, mv.verts + 3 * mv.n_verts), nrm, kd(mv.albedo, mv.albedo + 3 * mv.n_albedo);
    if (mv.normals) nrm.assign(mv.normals, mv.normals + 3 * mv.n_verts);
    std::vector<int> f(mv.faces, mv.faces + 3 * mv.n_tris), fm(mv.n_tris, 0);
    if (mv.face_mat) fm.assign(mv.face_mat, mv.face_mat + mv.n_tris);
    std::string ext = A.mesh.size() > 5 ? A.mesh.substr(A.mesh.size() - 5) : "";
    if (A.yupToZup == 1 && A.synthetic <= 0) {   // y-up -> z-up: (x, y, z) -> (x, -z, y), scene_setup.cpp:65-67
        for (size_t i = 0; i < v.size(); i += 3) { float y = v[i + 1], z = v[i + 2]; v[i + 1] = -z; v[i + 2] = y; }
        for (size_t i = 0; i < nrm.size(); i += 3) { float y = nrm[i + 1], z = nrm[i + 2]; nrm[i + 1] = -z; nrm[i + 2] = y; }
    }
    if (!A.smooth) nrm.clear();
    if (!kdL.empty()) kd = kdL;
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
    float c2w[16];
    if (!camera_c2w(A, c2w)) return 1;
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
    // --builder hploc: the binary tree from the GPU's H-PLOC, leaves collapsed to the SAH optimum on the host, then the
    // same layouts (scene_setup.cpp:76-83)
    const int hp = A.builder == "hploc" ? 1 : 0;
    cwp_build_options bo{ V, A.bins, A.leaf, cw ? 0 : 1, A.threads, 0.f, hp, 0 };
    cwp_bvh* bvh = nullptr;
    auto tb = std::chrono::steady_clock::now();
    if (cwp_bvh_build(mesh, &bo, &bvh)) return fail("BVH");
    double bvhS = std::chrono::duration<double>(std::chrono::steady_clock::now() - tb).count();
    cwp_bvh_data bd; cwp_bvh_data_of(bvh, &bd);
    const int reportLeaf = cw ? 3 : (V == 8 && A.leaf > 4) ? 4 : A.leaf;
    const double treeMs = hp ? bd.build_ms : bvhS * 1e3, postMs = hp ? std::max(0.0, bvhS * 1e3 - bd.build_ms) : 0.0;
    fprintf(stderr, "BVH%d (%s, %d bins%s): %lld nodes (%.1f MB), depth %d, SAH %.3f, build %.2fs, tri=%s\n", V, hp ? "gpu h-ploc" : "sah", A.bins, V == 8 ? (cw ? ", SAH collapse" : ", greedy collapse") : "",
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
               "\"builder\":\"%s\",\"collapse\":\"%s\",\"bvh_tree_ms\":%.2f,\"bvh_post_ms\":%.2f,\"bvh_sah\":%.4f,\"graph\":%d,\"instances\":0,\"flatten\":0,\"frame\":%d,\"tlas_ms\":0.000,\"bins\":%d}\n",
               r, V, A.tri.c_str(), A.persistent, A.devloop, A.sort, A.fuse < 0 ? 1 : A.fuse, reportLeaf, K, A.boxes > 0 ? "boxes" : A.synthetic > 0 ? "synthetic" : A.mesh.c_str(), (long long)bd.n_tris,
               (long long)(bd.n_node_float4 / bd.node_stride), (long long)(bd.n_node_float4 * 16), bd.max_depth, bvhS, A.w, A.h, A.spp, A.bounces, st.rays, st.shadow_rays,
               tot, st.trace_ms, st.frame_ms, tot / (st.trace_ms * 1e3), tot / (st.frame_ms * 1e3), st.rays / ((double)N * A.spp), info.vram_mb, info.pt_blocks, info.gpu_name,
               A.filterBH ? "blackman-harris1.5" : "box", P.has_n, A.seed, P.cam.lens_r, P.cam.focus_d, A.builder.c_str(), V == 8 ? A.collapse.c_str() : "-", treeMs, postMs, bd.sah, A.graph, A.frame, A.bins);
        fflush(stdout);
    }
    std::vector<float> acc((size_t)N * 4), lin((size_t)N * 3);
    if (cwp_renderer_read_accum(R, acc.data())) return fail("readback");
    for (int i = 0; i < N; i++) for (int c = 0; c < 3; c++) lin[3 * i + c] = acc[4 * (size_t)i + c] / A.spp;
    if (!write_images(A.out, A.w, A.h, lin)) { fprintf(stderr, "cannot write %s\n", A.out.c_str()); return 1; }
    cwp_renderer_destroy(R); cwp_bvh_free(bvh); cwp_mesh_free(mesh);
    return 0;
}
