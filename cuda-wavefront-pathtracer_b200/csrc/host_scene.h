// host_scene.h - meshes, the seeded box-field scene generator, PLY/OBJ input, PLY output, camera/lighting JSON.
#pragma once
#include "vecmath.h"
#include <cstdint>
#include <string>
#include <vector>

namespace cwpb {

// Indexed triangle mesh. v: 3 floats per vertex; n: optional per-vertex normals (same count as v or empty);
// f: 3 vertex indices per triangle; fm: material id per triangle; kd: 3 floats of albedo per material id.
struct Mesh {
    std::vector<float> v, n;
    std::vector<int> f, fm;
    std::vector<float> kd;
    std::vector<std::string> matName;   // material names (OBJ newmtl order), empty for other formats
    size_t nv() const { return v.size() / 3; }
    size_t nt() const { return f.size() / 3; }
    bool hasN() const { return !n.empty() && n.size() == v.size(); }
    float3 vert(int i) const { return f3(v[3 * (size_t)i], v[3 * (size_t)i + 1], v[3 * (size_t)i + 2]); }
};

// Box field on a ground plane, generated in a y-up frame and stored z-up with (x, y, z) -> (x, -z, y):
// nBoxes boxes of 12 triangles whose centres are uniform in x, z in [-half, half], edge lengths log-uniform in
// [edgeLo, edgeHi] per axis, rotation about the vertical axis uniform in [0, 2 pi), resting on the ground; plus a
// 2 half x 2 half two-triangle ground plane. Deterministic for a given seed (splitmix64 stream).
void box_field(int nBoxes, uint64_t seed, float half, float edgeLo, float edgeHi, Mesh& out);

// The reference's procedural scene (scene/synthetic.h:6-8): a ground of ground x ground quads over [-6, 6]^2 and a
// grid x grid array of bumpy spheres of nu x nv quads, 2 (ground^2 + grid^2 nu (nv - 1)) triangles, five albedos
// (ground, then four sphere colours). sphere_grid_c2w gives its default view (row-major camera-to-world).
void sphere_grid(int grid, int nu, int nv, int ground, Mesh& out);
void sphere_grid_c2w(float c2w[16]);

bool load_ply(const std::string& path, Mesh& m, std::string* err);
bool load_obj(const std::string& path, Mesh& m, std::string* err);
bool load_mesh(const std::string& path, Mesh& m, std::string* err);   // by extension
bool write_ply(const std::string& path, const Mesh& m);                // binary little endian, material_index per face

// ---- minimal JSON (objects, arrays, numbers, strings, literals) ----
struct Json {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    bool b = false; double num = 0; std::string str;
    std::vector<Json> arr; std::vector<std::pair<std::string, Json>> obj;
    const Json* at(const std::string& k) const;
    double number(const std::string& k, double def) const;
    std::vector<double> numbers(const std::string& k) const;   // every number under k, arrays flattened
};
bool parse_json(const std::string& text, Json& out, std::string* err);
std::string read_text(const std::string& path);

}  // namespace cwpb
