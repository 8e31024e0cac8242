// host_scene.cpp - box-field generator, mesh loaders/writer and a small JSON reader.
#include "host_scene.h"
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <map>

namespace cwpb {

// ---------------- box field ----------------
namespace {
struct SplitMix {
    uint64_t s;
    uint64_t next() { uint64_t z = (s += 0x9E3779B97F4A7C15ull); z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull; z = (z ^ (z >> 27)) * 0x94D049BB133111EBull; return z ^ (z >> 31); }
    double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }   // [0, 1), 53 bits
};
}  // namespace

void box_field(int nBoxes, uint64_t seed, float half, float edgeLo, float edgeHi, Mesh& m) {
    m = Mesh();
    SplitMix rng{ seed };
    auto put = [&](double x, double y, double z) { m.v.push_back((float)x); m.v.push_back((float)(-z)); m.v.push_back((float)y); };   // y-up -> z-up
    // ground plane, y = 0, counter-clockwise seen from +y
    put(-half, 0, -half); put(half, 0, -half); put(half, 0, half); put(-half, 0, half);
    const int g[6] = { 0, 2, 1, 0, 3, 2 };
    for (int k : g) m.f.push_back(k);
    m.fm.push_back(0); m.fm.push_back(0);
    const double lLo = std::log((double)edgeLo), lHi = std::log((double)edgeHi);
    // corner c: bit0 -> +x, bit1 -> +y (top), bit2 -> +z (local box frame before rotation)
    static const int quads[6][4] = { { 0, 4, 6, 2 }, { 1, 3, 7, 5 }, { 0, 1, 5, 4 }, { 2, 6, 7, 3 }, { 0, 2, 3, 1 }, { 4, 5, 7, 6 } };
    for (int b = 0; b < nBoxes; b++) {
        double cx = -half + 2.0 * half * rng.unit(), cz = -half + 2.0 * half * rng.unit();
        double ex = std::exp(lLo + (lHi - lLo) * rng.unit()), ey = std::exp(lLo + (lHi - lLo) * rng.unit()), ez = std::exp(lLo + (lHi - lLo) * rng.unit());
        double th = 2.0 * 3.14159265358979323846 * rng.unit(), c = std::cos(th), s = std::sin(th);
        int base = (int)m.nv();
        for (int k = 0; k < 8; k++) {
            double lx = (k & 1 ? 0.5 : -0.5) * ex, ly = (k & 2 ? ey : 0.0), lz = (k & 4 ? 0.5 : -0.5) * ez;
            put(cx + lx * c + lz * s, ly, cz - lx * s + lz * c);
        }
        for (auto& q : quads) {
            int t0[3] = { q[0], q[1], q[2] }, t1[3] = { q[0], q[2], q[3] };
            for (int k : t0) m.f.push_back(base + k);
            for (int k : t1) m.f.push_back(base + k);
            m.fm.push_back(0); m.fm.push_back(0);
        }
    }
    m.kd = { 0.8f, 0.8f, 0.8f };
}

// Sphere grid (scene/synthetic.cpp:6-48): the geometry must be the reference's to the bit, so every expression below
// keeps its operand order (float, left to right, no fused multiply-add on the host).
void sphere_grid(int grid, int nu, int nv, int ground, Mesh& m) {
    m = Mesh();
    m.kd = { 0.5f, 0.5f, 0.5f,  0.8f, 0.3f, 0.2f,  0.2f, 0.6f, 0.3f,  0.25f, 0.35f, 0.8f,  0.8f, 0.8f, 0.8f };
    const float half = 6.0f, pi = 3.14159265f;
    auto vert = [&](float x, float y, float z) { m.v.push_back(x); m.v.push_back(y); m.v.push_back(z); };
    auto tri = [&](int a, int b, int c, int mat) { m.f.push_back(a); m.f.push_back(b); m.f.push_back(c); m.fm.push_back(mat); };
    // ground: (ground+1)^2 vertices over [-half, half]^2 with a low ripple in z, two triangles per cell
    for (int row = 0; row <= ground; row++)
        for (int col = 0; col <= ground; col++) {
            const float x = -half + 2 * half * col / ground, y = -half + 2 * half * row / ground;
            vert(x, y, 0.05f * sinf(1.3f * x) * cosf(1.7f * y));
        }
    const int stride = ground + 1;
    for (int row = 0; row < ground; row++)
        for (int col = 0; col < ground; col++) {
            const int p00 = row * stride + col, p01 = p00 + 1, p10 = p00 + stride, p11 = p10 + 1;
            tri(p00, p01, p11, 0); tri(p00, p11, p10, 0);
        }
    // spheres: nu longitudes x (nv + 1) latitude rings each (pole rings keep nu coincident vertices), radius bumped
    // by a per-sphere phase, one of four colours in turn; the pole caps are single triangles per quad
    const float pitch = 2 * half / (grid + 1), r0 = pitch * 0.33f;
    for (int k = 0; k < grid * grid; k++) {
        const int gx = k % grid, gy = k / grid;
        const float cx = -half + pitch * (gx + 1), cy = -half + pitch * (gy + 1);
        const float cz = r0 * (1.1f + 0.3f * ((k * 7) % 5) / 4.0f);
        const float rad = r0 * (0.7f + 0.3f * ((k * 3) % 4) / 3.0f);
        const int first = (int)m.nv();
        for (int ring = 0; ring <= nv; ring++)
            for (int seg = 0; seg < nu; seg++) {
                const float th = pi * ring / nv, ph = 2 * pi * seg / nu;
                const float s = rad * (1.0f + 0.12f * sinf(6 * th + k) * cosf(5 * ph + 0.5f * k));
                const float dx = sinf(th) * cosf(ph), dy = sinf(th) * sinf(ph), dz = cosf(th);
                vert(cx + dx * s, cy + dy * s, cz + dz * s);
            }
        const int mat = 1 + k % 4;
        for (int ring = 0; ring < nv; ring++)
            for (int seg = 0; seg < nu; seg++) {
                const int next = (seg + 1) % nu;
                const int a = first + ring * nu + seg, b = first + ring * nu + next;
                const int c = a + nu, d = b + nu;
                if (ring > 0) tri(a, c, b, mat);
                if (ring < nv - 1) tri(b, c, d, mat);
            }
    }
}

void sphere_grid_c2w(float c2w[16]) {   // syntheticCamera (synthetic.cpp:50): from (0, -9.5, 6.5) at (0, 0, 0.4), z up
    const float3 pos = f3(0.f, -9.5f, 6.5f), fwd = normalize(f3(0.f, 0.f, 0.4f) - pos);
    const float3 right = normalize(cross(fwd, f3(0.f, 0.f, 1.f))), up = cross(right, fwd), back = -fwd;
    const float3 axes[3] = { right, up, back };
    for (int j = 0; j < 16; j++) c2w[j] = (j % 5 == 0) ? 1.f : 0.f;
    for (int col = 0; col < 3; col++) { c2w[col] = axes[col].x; c2w[4 + col] = axes[col].y; c2w[8 + col] = axes[col].z; }
    c2w[3] = pos.x; c2w[7] = pos.y; c2w[11] = pos.z;
}

// ---------------- PLY ----------------
namespace {
struct PlyProp { std::string name, type, countType, itemType; bool list = false; };
struct PlyElem { std::string name; long count = 0; std::vector<PlyProp> props; };
int ply_size(const std::string& t) {
    if (t == "char" || t == "uchar" || t == "int8" || t == "uint8") return 1;
    if (t == "short" || t == "ushort" || t == "int16" || t == "uint16") return 2;
    if (t == "double" || t == "float64") return 8;
    return 4;
}
double ply_bin(FILE* fp, const std::string& t, bool& ok) {
    unsigned char b[8] = { 0 }; int n = ply_size(t);
    if (fread(b, 1, n, fp) != (size_t)n) { ok = false; return 0; }
    if (t == "char" || t == "int8") return (double)(int8_t)b[0];
    if (t == "uchar" || t == "uint8") return (double)b[0];
    if (t == "short" || t == "int16") { int16_t x; memcpy(&x, b, 2); return x; }
    if (t == "ushort" || t == "uint16") { uint16_t x; memcpy(&x, b, 2); return x; }
    if (t == "uint" || t == "uint32") { uint32_t x; memcpy(&x, b, 4); return x; }
    if (t == "float" || t == "float32") { float x; memcpy(&x, b, 4); return x; }
    if (t == "double" || t == "float64") { double x; memcpy(&x, b, 8); return x; }
    int32_t x; memcpy(&x, b, 4); return x;
}
void pad_kd(Mesh& m) {
    int mx = 0; for (int t : m.fm) mx = t > mx ? t : mx;
    while ((int)(m.kd.size() / 3) <= mx) { m.kd.push_back(0.8f); m.kd.push_back(0.8f); m.kd.push_back(0.8f); }
}
}  // namespace

bool load_ply(const std::string& path, Mesh& m, std::string* err) {
    FILE* fp = fopen(path.c_str(), "rb");
    if (!fp) { if (err) *err = "cannot open " + path; return false; }
    char line[1024]; bool ascii = false, ended = false; std::vector<PlyElem> elems;
    if (!fgets(line, sizeof line, fp) || strncmp(line, "ply", 3) != 0) { fclose(fp); if (err) *err = "not a PLY file"; return false; }
    while (fgets(line, sizeof line, fp)) {
        if (!strncmp(line, "format", 6)) {
            ascii = strstr(line, "ascii") != nullptr;
            if (strstr(line, "big_endian")) { fclose(fp); if (err) *err = "big-endian PLY is not supported"; return false; }
        } else if (!strncmp(line, "element", 7)) {
            PlyElem e; char nm[256]; long c;
            if (sscanf(line + 7, "%255s %ld", nm, &c) == 2) { e.name = nm; e.count = c; elems.push_back(e); }
        } else if (!strncmp(line, "property", 8) && !elems.empty()) {
            PlyProp p; char a[64], b[64], c[64], d[64];
            int k = sscanf(line + 8, "%63s %63s %63s %63s", a, b, c, d);
            if (k >= 2 && !strcmp(a, "list") && k == 4) { p.list = true; p.countType = b; p.itemType = c; p.name = d; }
            else if (k >= 2) { p.type = a; p.name = b; }
            else continue;
            elems.back().props.push_back(p);
        } else if (!strncmp(line, "end_header", 10)) { ended = true; break; }
    }
    if (!ended) { fclose(fp); if (err) *err = "PLY header without end_header"; return false; }
    bool ok = true;
    auto rd = [&](const std::string& t) { if (ascii) { double x = 0; if (fscanf(fp, "%lf", &x) != 1) ok = false; return x; } return ply_bin(fp, t, ok); };
    const size_t v0 = m.nv();
    for (auto& e : elems) {
        if (e.name == "vertex") {
            int ix = -1, iy = -1, iz = -1, jx = -1, jy = -1, jz = -1;
            for (size_t k = 0; k < e.props.size(); k++) {
                const std::string& nm = e.props[k].name;
                if (nm == "x") ix = (int)k; else if (nm == "y") iy = (int)k; else if (nm == "z") iz = (int)k;
                else if (nm == "nx") jx = (int)k; else if (nm == "ny") jy = (int)k; else if (nm == "nz") jz = (int)k;
            }
            if (ix < 0 || iy < 0 || iz < 0) { fclose(fp); if (err) *err = "PLY vertex without x y z"; return false; }
            bool hasN = jx >= 0 && jy >= 0 && jz >= 0;
            std::vector<double> val(e.props.size());
            for (long i = 0; i < e.count && ok; i++) {
                for (size_t k = 0; k < e.props.size(); k++) {
                    const PlyProp& p = e.props[k];
                    if (p.list) { int c = (int)rd(p.countType); for (int j = 0; j < c; j++) rd(p.itemType); val[k] = 0; }
                    else val[k] = rd(p.type);
                }
                m.v.push_back((float)val[ix]); m.v.push_back((float)val[iy]); m.v.push_back((float)val[iz]);
                if (hasN) { m.n.push_back((float)val[jx]); m.n.push_back((float)val[jy]); m.n.push_back((float)val[jz]); }
            }
        } else if (e.name == "face") {
            std::vector<int> idx;
            for (long i = 0; i < e.count && ok; i++) {
                int mat = 0; idx.clear();
                for (auto& p : e.props) {
                    if (p.list) {
                        int c = (int)rd(p.countType);
                        bool isIdx = p.name == "vertex_indices" || p.name == "vertex_index";
                        for (int j = 0; j < c; j++) { int x = (int)rd(p.itemType); if (isIdx) idx.push_back(x); }
                    } else { double x = rd(p.type); if (p.name == "material_index") mat = (int)x; }
                }
                for (size_t k = 1; k + 1 < idx.size(); k++) {
                    m.f.push_back(idx[0] + (int)v0); m.f.push_back(idx[k] + (int)v0); m.f.push_back(idx[k + 1] + (int)v0); m.fm.push_back(mat);
                }
            }
        } else {
            for (long i = 0; i < e.count && ok; i++)
                for (auto& p : e.props) { if (p.list) { int c = (int)rd(p.countType); for (int j = 0; j < c; j++) rd(p.itemType); } else rd(p.type); }
        }
    }
    fclose(fp);
    if (!ok) { if (err) *err = "PLY body truncated"; return false; }
    if (!m.n.empty() && m.n.size() != m.v.size()) m.n.clear();
    for (int x : m.f) if (x < 0 || (size_t)x >= m.nv()) { if (err) *err = "PLY face index out of range"; return false; }
    if (m.kd.empty()) { m.kd = { 0.8f, 0.8f, 0.8f }; }
    pad_kd(m);
    if (m.f.empty()) { if (err) *err = "PLY without triangles"; return false; }
    return true;
}

// ---------------- OBJ ----------------
namespace {
std::string dir_of(const std::string& p) { size_t k = p.find_last_of("/\\"); return k == std::string::npos ? std::string(".") : p.substr(0, k); }
void load_mtl(const std::string& path, Mesh& m, std::map<std::string, int>& ids) {
    FILE* fp = fopen(path.c_str(), "rb"); if (!fp) return;
    char line[1024]; int cur = -1;
    while (fgets(line, sizeof line, fp)) {
        char nm[512]; float r, g, b;
        if (!strncmp(line, "newmtl", 6) && sscanf(line + 6, "%511s", nm) == 1) {
            cur = (int)(m.kd.size() / 3); ids[nm] = cur; m.kd.push_back(0.8f); m.kd.push_back(0.8f); m.kd.push_back(0.8f);
            m.matName.resize((size_t)cur + 1); m.matName[cur] = nm;
        } else if (cur >= 0 && !strncmp(line, "Kd", 2) && sscanf(line + 2, "%f %f %f", &r, &g, &b) == 3) {
            m.kd[3 * cur] = r; m.kd[3 * cur + 1] = g; m.kd[3 * cur + 2] = b;
        }
    }
    fclose(fp);
}
}  // namespace

bool load_obj(const std::string& path, Mesh& m, std::string* err) {
    FILE* fp = fopen(path.c_str(), "rb");
    if (!fp) { if (err) *err = "cannot open " + path; return false; }
    if (m.kd.empty()) m.kd = { 0.8f, 0.8f, 0.8f };
    std::vector<float> vn; std::map<std::string, int> ids; int cur = 0;
    std::vector<char> buf(1 << 16); std::vector<int> vi, ni;
    while (fgets(buf.data(), (int)buf.size(), fp)) {
        char* s = buf.data(); float x, y, z; char nm[1024];
        if (s[0] == 'v' && s[1] == ' ') { if (sscanf(s + 2, "%f %f %f", &x, &y, &z) == 3) { m.v.push_back(x); m.v.push_back(y); m.v.push_back(z); } }
        else if (s[0] == 'v' && s[1] == 'n') { if (sscanf(s + 2, "%f %f %f", &x, &y, &z) == 3) { vn.push_back(x); vn.push_back(y); vn.push_back(z); } }
        else if (s[0] == 'f' && (s[1] == ' ' || s[1] == '\t')) {
            vi.clear(); ni.clear(); char* p = s + 1;
            while (*p) {
                while (*p == ' ' || *p == '\t') p++;
                if (*p == '\n' || *p == '\r' || *p == 0) break;
                char* q = p; while (*q && *q != ' ' && *q != '\t' && *q != '\n' && *q != '\r') q++;
                int a = atoi(p), nIdx = -1;
                char* s1 = (char*)memchr(p, '/', q - p);
                if (s1) { char* s2 = (char*)memchr(s1 + 1, '/', q - s1 - 1); if (s2 && s2 + 1 < q) { int b = atoi(s2 + 1); nIdx = b > 0 ? b - 1 : (int)(vn.size() / 3) + b; } }
                vi.push_back(a > 0 ? a - 1 : (int)m.nv() + a); ni.push_back(nIdx);
                p = q;
            }
            for (size_t k = 1; k + 1 < vi.size(); k++) { m.f.push_back(vi[0]); m.f.push_back(vi[k]); m.f.push_back(vi[k + 1]); m.fm.push_back(cur); }
            for (size_t k = 0; k < vi.size(); k++)
                if (ni[k] >= 0 && ni[k] < (int)(vn.size() / 3) && vi[k] >= 0 && vi[k] < (int)m.nv()) {
                    if (m.n.size() != m.v.size()) m.n.resize(m.v.size(), 0.f);
                    for (int c = 0; c < 3; c++) m.n[3 * (size_t)vi[k] + c] = vn[3 * (size_t)ni[k] + c];
                }
        } else if (!strncmp(s, "mtllib", 6) && sscanf(s + 6, "%1023s", nm) == 1) load_mtl(dir_of(path) + "/" + nm, m, ids);
        else if (!strncmp(s, "usemtl", 6)) { cur = 0; if (sscanf(s + 6, "%1023s", nm) == 1) { auto it = ids.find(nm); if (it != ids.end()) cur = it->second; } }
    }
    fclose(fp);
    if (!m.n.empty()) { bool any = false; for (float a : m.n) if (a != 0.f) { any = true; break; } if (!any) m.n.clear(); }
    if (!m.n.empty() && m.n.size() != m.v.size()) m.n.resize(m.v.size(), 0.f);
    for (int x : m.f) if (x < 0 || (size_t)x >= m.nv()) { if (err) *err = "OBJ face index out of range"; return false; }
    pad_kd(m);
    if (m.f.empty()) { if (err) *err = "OBJ without triangles"; return false; }
    return true;
}

bool load_mesh(const std::string& path, Mesh& m, std::string* err) {
    std::string ext = path.size() > 4 ? path.substr(path.size() - 4) : std::string();
    for (auto& c : ext) c = (char)tolower((unsigned char)c);
    return ext == ".ply" ? load_ply(path, m, err) : load_obj(path, m, err);
}

bool write_ply(const std::string& path, const Mesh& m) {
    FILE* fp = fopen(path.c_str(), "wb"); if (!fp) return false;
    fprintf(fp, "ply\nformat binary_little_endian 1.0\nelement vertex %zu\nproperty float x\nproperty float y\nproperty float z\n", m.nv());
    fprintf(fp, "element face %zu\nproperty list uchar int vertex_indices\nproperty int material_index\nend_header\n", m.nt());
    fwrite(m.v.data(), sizeof(float), m.v.size(), fp);
    for (size_t t = 0; t < m.nt(); t++) {
        unsigned char c = 3; fwrite(&c, 1, 1, fp); fwrite(&m.f[3 * t], sizeof(int), 3, fp);
        int mat = m.fm.empty() ? 0 : m.fm[t]; fwrite(&mat, sizeof(int), 1, fp);
    }
    return fclose(fp) == 0;
}

// ---------------- JSON ----------------
namespace {
struct JP {
    const char* s; const char* e; std::string err;
    void ws() { while (s < e && (*s == ' ' || *s == '\t' || *s == '\n' || *s == '\r')) s++; }
    bool fail(const char* m) { if (err.empty()) err = m; return false; }
    bool str(std::string& out) {
        if (s >= e || *s != '"') return fail("expected string");
        s++;
        while (s < e && *s != '"') {
            if (*s == '\\' && s + 1 < e) { s++; char c = *s; out.push_back(c == 'n' ? '\n' : c == 't' ? '\t' : c); if (c == 'u') s += 4; s++; }
            else out.push_back(*s++);
        }
        if (s >= e) return fail("unterminated string");
        s++; return true;
    }
    bool val(Json& v, int depth) {
        if (depth > 64) return fail("nesting too deep");
        ws(); if (s >= e) return fail("unexpected end");
        if (*s == '{') {
            v.kind = Json::Obj; s++; ws();
            if (s < e && *s == '}') { s++; return true; }
            while (true) {
                ws(); std::string k; if (!str(k)) return false;
                ws(); if (s >= e || *s != ':') return fail("expected ':'"); s++;
                Json c; if (!val(c, depth + 1)) return false;
                v.obj.emplace_back(k, c); ws();
                if (s < e && *s == ',') { s++; continue; }
                if (s < e && *s == '}') { s++; return true; }
                return fail("expected ',' or '}'");
            }
        }
        if (*s == '[') {
            v.kind = Json::Arr; s++; ws();
            if (s < e && *s == ']') { s++; return true; }
            while (true) {
                Json c; if (!val(c, depth + 1)) return false;
                v.arr.push_back(c); ws();
                if (s < e && *s == ',') { s++; continue; }
                if (s < e && *s == ']') { s++; return true; }
                return fail("expected ',' or ']'");
            }
        }
        if (*s == '"') { v.kind = Json::Str; return str(v.str); }
        if (e - s >= 4 && !strncmp(s, "true", 4)) { v.kind = Json::Bool; v.b = true; s += 4; return true; }
        if (e - s >= 5 && !strncmp(s, "false", 5)) { v.kind = Json::Bool; s += 5; return true; }
        if (e - s >= 4 && !strncmp(s, "null", 4)) { v.kind = Json::Null; s += 4; return true; }
        char* q = nullptr; double x = strtod(s, &q);
        if (q == s) return fail("unexpected character");
        v.kind = Json::Num; v.num = x; s = q; return true;
    }
};
void collect(const Json& j, std::vector<double>& out) {
    if (j.kind == Json::Num) out.push_back(j.num);
    for (auto& c : j.arr) collect(c, out);
}
}  // namespace

const Json* Json::at(const std::string& k) const { for (auto& kv : obj) if (kv.first == k) return &kv.second; return nullptr; }
double Json::number(const std::string& k, double def) const { const Json* j = at(k); return j && j->kind == Num ? j->num : def; }
std::vector<double> Json::numbers(const std::string& k) const { std::vector<double> r; const Json* j = at(k); if (j) collect(*j, r); return r; }

bool parse_json(const std::string& text, Json& out, std::string* err) {
    JP p{ text.data(), text.data() + text.size(), {} };
    out = Json();
    bool ok = p.val(out, 0);
    if (ok) { p.ws(); if (p.s != p.e) ok = p.fail("trailing characters"); }
    if (!ok && err) *err = p.err;
    return ok;
}

std::string read_text(const std::string& path) {
    FILE* fp = fopen(path.c_str(), "rb"); if (!fp) return std::string();
    std::string s; char b[4096]; size_t n;
    while ((n = fread(b, 1, sizeof b, fp)) > 0) s.append(b, n);
    fclose(fp); return s;
}

}  // namespace cwpb
