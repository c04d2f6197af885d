// pbrt.cpp -- PBRT scene files into scene descriptions (pt_load_pbrt), as the reference reads them.
//
// Reference: poly::pbrt_parser (src/common/parsers/pbrt_parser.cpp):
//   scan / lex            :284-640   tokens per directive, "type name" argument declarations
//   scene block           :907-1230  Sampler (pixelsamples), Film (x/yresolution), Camera
//                                    (perspective fov), LookAt and the other transforms composed
//                                    into the camera transform, Integrator (path maxdepth)
//   world block           :1232-1711 attributes, transforms, materials, lights, shapes, instances
//   Transform / Matrix4x4 :Transform.cpp:16-365, Matrix4x4.cpp:12-303 (the arithmetic restated
//                                    below in the same operation order)
//   SphereTesselator      :src/cpu/shapes/tesselators.cpp:10-84
//
// What the reference does and this loader reproduces, because it decides the world-space
// vertices and so every hit:
//   * A shape keeps a pointer to the *active transform object*, and Translate / Rotate / Scale
//     in the same attribute scope multiply into that object in place, so a transform that follows
//     a shape also moves the shapes before it in that scope (AttributeBegin / TransformBegin start
//     a new object, a copy of the current one).  Vertex normals go through the inverse stored in
//     that same object, in its final state (Mesh::intersect, mesh.cpp:397-399, calls
//     object_to_world->ApplyInPlace(Normal&), which reads the transform's Inverse matrix; the
//     mesh's own world_to_object is never used), so pt_mesh_desc::world_to_object carries it.
//   * Transform *= multiplies both the matrix and the stored inverse on the right (so the stored
//     "inverse" of a composed transform is the product of the inverses in the same order), and
//     Matrix4x4::Inverse picks pivots by integer-truncated magnitude (pivot_magnitude below).
//   * Area-light radiance objects are shared the same way: a second AreaLightSource in a scope
//     that already has one rewrites the radiance of the shapes before it.  AttributeBegin saves
//     the active material and light only when they are set; AttributeEnd restores the saved
//     material if there is one and the saved light (or none).
//   * Shape "sphere" tessellates a UV sphere with max((int)radius, 20) meridians and parallels
//     (the north pole is emitted twice, as the tessellator does) and ends with the active
//     transform, not the radius-scaled one: the radius only sets the tessellation.
//   * Inside ObjectBegin / ObjectEnd, plymesh / objmesh shapes append to the object's geometry (face indices
//     as written in each file) and a sphere replaces the block's current geometry without being
//     recorded for the object; ObjectInstance makes one shape from the object's geometry with
//     the active transform, material and light.
//   * MakeNamedMaterial "string type" "matte" makes a Lambert material of reflectance 0.5 (the
//     "rgb Kd" argument is read but not used); NamedMaterial takes the first material of that name.
//   * Radiances are the file's values x 255 (AreaLightSource L, LightSource "infinite" L).
// Where the library differs, on purpose: the Transform directive reads all 16 values (the
// reference's lexer reads 15 and then fails), and a binary PLY without normals is read with one
// vertex per file vertex (the PLY note in ply.cpp).  Not supported, with an error naming the
// directive: textures (Texture, "texture Kd"), Material "plastic" (no glossy BRDF in the render
// path), and a camera whose scene block holds more than one LookAt or any other
// transform (no LookAt is the identity camera, the same matrix as LookAt (0,0,0) (0,0,1) (0,1,0)).  Like the
// reference, unknown directives, unknown shape types and lights other than "infinite" / area
// "diffuse" are ignored.

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "pt_internal.h"

namespace pt {
namespace {

// ---- Transform arithmetic (Matrix4x4.cpp / Transform.cpp) ---------------------------------------

struct M4 {
    float m[4][4];
};

M4 identity() {
    M4 r{};
    r.m[0][0] = r.m[1][1] = r.m[2][2] = r.m[3][3] = 1.f;
    return r;
}

// Matrix4x4::operator* / operator*= : each entry summed left to right over k.
M4 mul(const M4& a, const M4& b) {
    M4 r{};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j] + a.m[i][3] * b.m[3][j];
    return r;
}

// The pivot magnitude of Matrix4x4::Inverse: its unqualified abs() resolves to the C library's
// int abs(int) there, so each entry is truncated to an integer before the comparison (a float abs
// picks other pivots and changes the low bits of most inverses; the world-to-object matrices of
// rotated shapes in the tests match the compiled reference's only with the truncation).
float pivot_magnitude(float v) {
    if (!(v > -2147483648.0f && v < 2147483648.0f)) return 2147483648.0f;  // out of int range
    return (float)std::abs((int)v);
}

// Matrix4x4::Inverse: Gauss-Jordan elimination with full pivoting (the pbrt routine).
bool inverse(const M4& in, M4& out) {
    int indxc[4] = {0, 0, 0, 0}, indxr[4] = {0, 0, 0, 0}, ipiv[4] = {0, 0, 0, 0};
    float minv[4][4];
    std::memcpy(minv, in.m, sizeof(minv));
    for (int i = 0; i < 4; i++) {
        int irow = -1, icol = -1;
        float big = 0.f;
        for (int j = 0; j < 4; j++) {
            if (ipiv[j] == 1) continue;
            for (int k = 0; k < 4; k++) {
                if (ipiv[k] == 0) {
                    if (pivot_magnitude(minv[j][k]) >= big) {
                        big = pivot_magnitude(minv[j][k]);
                        irow = j;
                        icol = k;
                    }
                } else if (ipiv[k] > 1) {
                    return false;
                }
            }
        }
        if (icol < 0) return false;
        ++ipiv[icol];
        if (irow != icol)
            for (int k = 0; k < 4; ++k) std::swap(minv[irow][k], minv[icol][k]);
        indxr[i] = irow;
        indxc[i] = icol;
        if (minv[icol][icol] == 0.f) return false;
        const float pivinv = 1.f / minv[icol][icol];
        minv[icol][icol] = 1.f;
        for (int j = 0; j < 4; j++) minv[icol][j] *= pivinv;
        for (int j = 0; j < 4; j++) {
            if (j == icol) continue;
            const float save = minv[j][icol];
            minv[j][icol] = 0;
            for (int k = 0; k < 4; k++) minv[j][k] -= minv[icol][k] * save;
        }
    }
    for (int j = 3; j >= 0; j--)
        if (indxr[j] != indxc[j])
            for (int k = 0; k < 4; k++) std::swap(minv[k][indxr[j]], minv[k][indxc[j]]);
    std::memcpy(out.m, minv, sizeof(minv));
    return true;
}

struct Xf {  // poly::Transform: the matrix and the inverse it carries
    M4 mat = identity();
    M4 inv = identity();
};

void compose(Xf& t, const Xf& rhs) {  // Transform::operator*=
    t.mat = mul(t.mat, rhs.mat);
    t.inv = mul(t.inv, rhs.inv);
}

bool xf_from_matrix(const M4& m, Xf& out) {  // Transform(const Matrix4x4&): inverse computed
    out.mat = m;
    return inverse(m, out.inv);
}

Xf xf_translate(float x, float y, float z) {
    Xf t;
    t.mat.m[0][3] = x; t.mat.m[1][3] = y; t.mat.m[2][3] = z;
    t.inv.m[0][3] = -x; t.inv.m[1][3] = -y; t.inv.m[2][3] = -z;
    return t;
}

Xf xf_scale(float x, float y, float z) {
    Xf t;
    t.mat.m[0][0] = x; t.mat.m[1][1] = y; t.mat.m[2][2] = z;
    t.inv.m[0][0] = 1.f / x; t.inv.m[1][1] = 1.f / y; t.inv.m[2][2] = 1.f / z;
    return t;
}

// rotate_directive (pbrt_parser.cpp:640-655) + Transform::Rotate (Transform.cpp:214-228).
bool xf_rotate(float deg, float x, float y, float z, Xf& out) {
    constexpr float pi_over_180 = 3.14159265358979323846 / 180.0f;
    const float angle = deg * pi_over_180;
    const float li = 1.f / std::sqrt(x * x + y * y + z * z);
    x *= li;
    y *= li;
    z *= li;
    const float s = std::sin(angle), c = std::cos(angle), omc = (1 - c);
    M4 m{};
    m.m[0][0] = c + x * x * omc;     m.m[0][1] = x * y * omc - z * s; m.m[0][2] = x * z * omc + y * s; m.m[0][3] = 0;
    m.m[1][0] = y * x * omc + z * s; m.m[1][1] = c + y * y * omc;     m.m[1][2] = y * z * omc - x * s; m.m[1][3] = 0;
    m.m[2][0] = z * x * omc - y * s; m.m[2][1] = z * y * omc + x * s; m.m[2][2] = c + z * z * omc;     m.m[2][3] = 0;
    m.m[3][0] = 0;                   m.m[3][1] = 0;                   m.m[3][2] = 0;                   m.m[3][3] = 1;
    return xf_from_matrix(m, out);
}

// ---- UV sphere (SphereTesselator::Create, tesselators.cpp:10-84) --------------------------------

struct Geometry {  // poly::mesh_geometry: packed arrays as the mesh descriptor takes them
    std::vector<float> x, y, z, nx, ny, nz;
    std::vector<uint32_t> f0, f1, f2;
};

void tessellate_sphere(unsigned meridians, unsigned parallels, Geometry& g) {
    constexpr float pi = float(3.14159265358979323846);
    constexpr float two_pi = 2.0f * pi;
    constexpr float pi_over_2 = pi / 2.0f;
    auto vert = [&g](float x, float y, float z) { g.x.push_back(x); g.y.push_back(y); g.z.push_back(z); };
    auto face = [&g](uint32_t a, uint32_t b, uint32_t c) { g.f0.push_back(a); g.f1.push_back(b); g.f2.push_back(c); };
    std::vector<unsigned> starts;
    vert(0, 1, 0);
    vert(0, 1, 0);  // the north pole twice, as the reference emits it
    starts.push_back(0);
    const float mstep = two_pi / (float)meridians;
    const float pstep = pi / (float)(parallels + 1);
    for (unsigned i = 0; i < parallels; i++) {
        const float vert_angle = pi_over_2 - (pstep * ((float)(i + 1)));
        const float y = std::sin(vert_angle);
        const float r = std::cos(vert_angle);
        starts.push_back(i * meridians + 1);
        for (unsigned j = 0; j < meridians; j++) {
            const float h = mstep * j;
            vert(std::cos(h) * r, y, std::sin(h) * r);
        }
    }
    vert(0, -1, 0);
    for (unsigned v = 1; v < meridians; v++) face(v + 1, v, 0);
    face(1, meridians, 0);
    for (unsigned p = 1; p < parallels; p++) {
        const unsigned top = starts[p], bottom = starts[p + 1];
        for (unsigned m = 1; m < meridians; m++) {
            const unsigned tr = top + m - 1, tl = top + m, bl = bottom + m - 1, br = bottom + m;
            face(br, bl, tr);
            face(tr, tl, br);
        }
        const unsigned tl = top, tr = top + meridians - 1, bl = bottom, br = bottom + meridians - 1;
        face(bl, br, tr);
        face(tr, tl, bl);
    }
    const unsigned bottom = starts[parallels];
    const uint32_t n = (uint32_t)g.x.size();
    for (unsigned v = 0; v < meridians - 1; v++) face(v + bottom, v + 1 + bottom, n - 1);
    face(n - 2, bottom, n - 1);
}

// ---- tokens and directives -----------------------------------------------------------------------

struct Arg {
    std::string type, name;
    std::vector<std::string> values;  // raw tokens (strings unquoted)
    bool quoted = false;              // values were quoted strings
};

struct Directive {
    std::string name, type;
    std::vector<std::string> bare;  // unquoted values of LookAt / Rotate / Scale / Translate / Transform
    std::vector<Arg> args;
    int line = 0;
};

struct Tok {
    std::string text;
    bool quoted;
    int line;
};

bool is_directive_name(const std::string& s) {
    static const char* names[] = {"AreaLightSource", "AttributeBegin", "AttributeEnd", "Camera", "Film", "Integrator",
                                  "LightSource", "LookAt", "MakeNamedMaterial", "Material", "NamedMaterial",
                                  "ObjectBegin", "ObjectEnd", "ObjectInstance", "PixelFilter", "Rotate", "Sampler",
                                  "Scale", "Shape", "Texture", "Transform", "TransformBegin", "TransformEnd",
                                  "Translate", "WorldBegin", "WorldEnd"};
    for (const char* n : names)
        if (s == n) return true;
    return false;
}

bool is_transform(const std::string& n) { return n == "Translate" || n == "Scale" || n == "Rotate" || n == "Transform"; }

int tokenize(const std::string& text, std::vector<Tok>& out, std::string& err) {
    int line = 1;
    size_t i = 0;
    const size_t n = text.size();
    while (i < n) {
        const char c = text[i];
        if (c == '\n') { ++line; ++i; continue; }
        if (std::isspace((unsigned char)c)) { ++i; continue; }
        if (c == '#') {
            while (i < n && text[i] != '\n') ++i;
            continue;
        }
        if (c == '[' || c == ']') {
            out.push_back({std::string(1, c), false, line});
            ++i;
            continue;
        }
        if (c == '"') {
            const size_t j = text.find('"', i + 1);
            if (j == std::string::npos) {
                err = "line " + std::to_string(line) + ": unterminated string";
                return PT_EINVAL;
            }
            std::string s = text.substr(i + 1, j - i - 1);
            out.push_back({s, true, line});
            line += (int)std::count(s.begin(), s.end(), '\n');
            i = j + 1;
            continue;
        }
        size_t j = i;
        while (j < n && !std::isspace((unsigned char)text[j]) && text[j] != '[' && text[j] != ']' && text[j] != '"' &&
               text[j] != '#')
            ++j;
        out.push_back({text.substr(i, j - i), false, line});
        i = j;
    }
    return PT_OK;
}

int parse_directives(const std::vector<Tok>& toks, std::vector<Directive>& out, std::string& err) {
    size_t i = 0;
    while (i < toks.size()) {
        const Tok& t = toks[i];
        if (t.quoted || !is_directive_name(t.text)) {
            err = "line " + std::to_string(t.line) + ": expected a directive, found [" + t.text + "]";
            return PT_EINVAL;
        }
        Directive d;
        d.name = t.text;
        d.line = t.line;
        ++i;
        // bare numbers (LookAt 9, Rotate 4, Scale 3, Translate 3, Transform [16])
        while (i < toks.size() && !toks[i].quoted && !is_directive_name(toks[i].text)) {
            if (toks[i].text != "[" && toks[i].text != "]") d.bare.push_back(toks[i].text);
            ++i;
        }
        if (!d.bare.empty() && d.name != "LookAt" && !is_transform(d.name)) {
            err = "line " + std::to_string(t.line) + ": unexpected [" + d.bare[0] + "] after " + d.name;
            return PT_EINVAL;
        }
        if (i < toks.size() && toks[i].quoted && d.bare.empty()) {  // the identifier ("type")
            if (d.name == "Texture") {
                err = "line " + std::to_string(t.line) + ": Texture is not supported (no textured materials)";
                return PT_EINVAL;
            }
            d.type = toks[i].text;
            ++i;
        }
        // "type name" [ values ] pairs
        while (i < toks.size() && toks[i].quoted) {
            Arg a;
            const std::string& decl = toks[i].text;
            std::istringstream ss(decl);
            ss >> a.type >> a.name;
            if (a.type.empty() || a.name.empty()) {
                err = "line " + std::to_string(toks[i].line) + ": bad argument declaration \"" + decl + "\"";
                return PT_EINVAL;
            }
            ++i;
            bool bracket = false;
            if (i < toks.size() && !toks[i].quoted && toks[i].text == "[") { bracket = true; ++i; }
            while (i < toks.size()) {
                if (!toks[i].quoted && toks[i].text == "]") {
                    if (bracket) { ++i; }
                    break;
                }
                if (!toks[i].quoted && is_directive_name(toks[i].text)) break;
                if (toks[i].quoted) {
                    a.quoted = true;
                    a.values.push_back(toks[i].text);
                    ++i;
                    if (!bracket) break;
                    continue;
                }
                a.values.push_back(toks[i].text);
                ++i;
                if (!bracket) break;
            }
            d.args.push_back(std::move(a));
        }
        out.push_back(std::move(d));
    }
    return PT_OK;
}

bool to_float(const std::string& s, float& v) {  // std::stof: strtof of the leading number
    char* end = nullptr;
    v = std::strtof(s.c_str(), &end);
    return end != s.c_str();
}

bool to_int(const std::string& s, int& v) {  // std::stoi
    char* end = nullptr;
    const long x = std::strtol(s.c_str(), &end, 10);
    v = (int)x;
    return end != s.c_str();
}

int floats(const Directive& d, size_t count, std::vector<float>& v, std::string& err) {
    if (d.bare.size() != count) {
        err = "line " + std::to_string(d.line) + ": " + d.name + " takes " + std::to_string(count) + " numbers";
        return PT_EINVAL;
    }
    v.resize(count);
    for (size_t k = 0; k < count; ++k)
        if (!to_float(d.bare[k], v[k])) {
            err = "line " + std::to_string(d.line) + ": " + d.name + ": [" + d.bare[k] + "] is not a number";
            return PT_EINVAL;
        }
    return PT_OK;
}

// argument types by their declared name (pbrt_argument::get_argument_type; "color" is rgb)
bool arg_is(const Arg& a, const char* type) {
    if (std::strcmp(type, "rgb") == 0) return a.type == "rgb" || a.type == "color";
    return a.type == type;
}

int arg_floats(const Directive& d, const Arg& a, std::vector<float>& v, std::string& err) {
    v.clear();
    for (const std::string& s : a.values) {
        float f;
        if (a.quoted || !to_float(s, f)) {
            err = "line " + std::to_string(d.line) + ": " + d.name + " \"" + a.name + "\": [" + s + "] is not a number";
            return PT_EINVAL;
        }
        v.push_back(f);
    }
    return PT_OK;
}

int xf_for(const Directive& d, Xf& out, std::string& err) {
    std::vector<float> v;
    int rc;
    if (d.name == "Translate") {
        if ((rc = floats(d, 3, v, err))) return rc;
        out = xf_translate(v[0], v[1], v[2]);
    } else if (d.name == "Scale") {
        if ((rc = floats(d, 3, v, err))) return rc;
        out = xf_scale(v[0], v[1], v[2]);
    } else if (d.name == "Rotate") {
        if ((rc = floats(d, 4, v, err))) return rc;
        if (!xf_rotate(v[0], v[1], v[2], v[3], out)) {
            err = "line " + std::to_string(d.line) + ": Rotate: singular matrix";
            return PT_EINVAL;
        }
    } else {  // Transform: 16 values, row-major as written (transform_directive)
        if ((rc = floats(d, 16, v, err))) return rc;
        M4 m;
        for (int k = 0; k < 16; ++k) m.m[k / 4][k % 4] = v[k];
        if (!xf_from_matrix(m, out)) {
            err = "line " + std::to_string(d.line) + ": Transform: singular matrix";
            return PT_EINVAL;
        }
    }
    return PT_OK;
}


struct Material {
    uint32_t type;
    float refl[3];
};

struct Spd {
    float rgb[3];
};

struct Shape {
    std::shared_ptr<Geometry> geometry;
    std::shared_ptr<Xf> to_world;  // the shared, possibly later-mutated transform object
    std::shared_ptr<Material> material;
    std::shared_ptr<Spd> light;
};

}  // namespace
}  // namespace pt

struct pt_pbrt_scene {
    pt_pbrt_info info{};
    std::vector<std::shared_ptr<pt::Geometry>> geometries;
    std::vector<pt_mesh_desc> meshes;
};

namespace pt {
namespace {

// plymesh / objmesh geometry appended to g (mesh_geometry's add_vertex / add_packed_face).
int read_mesh_geometry(const std::string& path, bool obj, Geometry& g, std::string& err) {
    pt_mesh_data md{};
    const int rc = obj ? pt_load_obj(path.c_str(), &md) : pt_load_ply(path.c_str(), &md);
    if (rc) {
        err = std::string(obj ? "objmesh [" : "plymesh [") + path + "]: " + pt_last_error();
        return rc;
    }
    const bool normals = md.nx && md.ny && md.nz;
    // a geometry that already has vertices without normals keeps none (mesh_geometry appends)
    const bool keep_normals = normals && g.nx.size() == g.x.size();
    g.x.insert(g.x.end(), md.x, md.x + md.num_vertices);
    g.y.insert(g.y.end(), md.y, md.y + md.num_vertices);
    g.z.insert(g.z.end(), md.z, md.z + md.num_vertices);
    if (keep_normals) {
        g.nx.insert(g.nx.end(), md.nx, md.nx + md.num_vertices);
        g.ny.insert(g.ny.end(), md.ny, md.ny + md.num_vertices);
        g.nz.insert(g.nz.end(), md.nz, md.nz + md.num_vertices);
    } else {
        g.nx.clear(); g.ny.clear(); g.nz.clear();
    }
    g.f0.insert(g.f0.end(), md.fv0, md.fv0 + md.num_faces);
    g.f1.insert(g.f1.end(), md.fv1, md.fv1 + md.num_faces);
    g.f2.insert(g.f2.end(), md.fv2, md.fv2 + md.num_faces);
    pt_mesh_data_free(&md);
    return PT_OK;
}

int load(const std::string& path, pt_pbrt_scene& out, std::string& err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        err = "cannot open [" + path + "]";
        return PT_EINVAL;
    }
    std::stringstream buf;
    buf << f.rdbuf();
    const std::string base = path.find_last_of('/') == std::string::npos ? "" : path.substr(0, path.find_last_of('/') + 1);
    std::vector<Tok> toks;
    int rc = tokenize(buf.str(), toks, err);
    if (rc) return rc;
    std::vector<Directive> ds;
    if ((rc = parse_directives(toks, ds, err))) return rc;
    size_t world = ds.size();
    for (size_t k = 0; k < ds.size(); ++k)
        if (ds[k].name == "WorldBegin") { world = k; break; }

    // ---- scene block (pbrt_parser.cpp:907-1230) ----
    pt_pbrt_info& info = out.info;
    info.spp = 8;                    // DefaultSamples
    info.width = 640;                // DefaultBoundsX
    info.height = 360;               // DefaultBoundsY
    info.max_depth = 5;
    info.camera.fov_deg = 90.f;      // DefaultCameraFOV
    int lookats = 0, other_xf = 0;
    bool sampler_seen = false, film_seen = false, integrator_seen = false, camera_seen = false;
    for (size_t k = 0; k < world; ++k) {
        const Directive& d = ds[k];
        if (d.name == "Sampler" && !sampler_seen) {
            sampler_seen = true;
            for (const Arg& a : d.args) {  // the first integer argument ends the search
                if (!arg_is(a, "integer")) continue;
                int v;
                if (a.name == "pixelsamples" && !a.values.empty() && to_int(a.values[0], v)) info.spp = (uint32_t)v;
                break;
            }
        } else if (d.name == "Film" && !film_seen) {
            film_seen = true;
            if (d.type != "image") continue;
            for (const Arg& a : d.args) {
                int v;
                if (!arg_is(a, "integer") || a.values.empty() || !to_int(a.values[0], v)) continue;
                if (a.name == "xresolution") info.width = (uint32_t)v;
                else if (a.name == "yresolution") info.height = (uint32_t)v;
            }
        } else if (d.name == "Integrator" && !integrator_seen) {
            integrator_seen = true;
            if (d.type != "path") continue;
            for (const Arg& a : d.args) {
                int v;
                if (arg_is(a, "integer") && a.name == "maxdepth" && !a.values.empty() && to_int(a.values[0], v)) {
                    info.max_depth = (uint32_t)v;
                    break;
                }
            }
        } else if (d.name == "Camera" && !camera_seen && d.type == "perspective") {
            camera_seen = true;
            for (const Arg& a : d.args) {
                std::vector<float> v;
                if (arg_is(a, "float") && a.name == "fov" && !arg_floats(d, a, v, err) && !v.empty()) info.camera.fov_deg = v[0];
            }
        } else if (d.name == "LookAt") {
            std::vector<float> v;
            if ((rc = floats(d, 9, v, err))) return rc;
            for (int c = 0; c < 3; ++c) {
                info.camera.eye[c] = v[c];
                info.camera.look_at[c] = v[3 + c];
                info.camera.up[c] = v[6 + c];
            }
            ++lookats;
        } else if (is_transform(d.name)) {
            ++other_xf;
        } else if (d.name == "Texture") {
            err = "line " + std::to_string(d.line) + ": Texture is not supported";
            return PT_EINVAL;
        }
    }
    if (lookats > 1 || other_xf != 0) {
        err = "the camera must be set by at most one LookAt and no other transform before WorldBegin "
              "(found " + std::to_string(lookats) + " LookAt and " + std::to_string(other_xf) + " other transforms)";
        return PT_EINVAL;
    }
    if (lookats == 0) {  // identity camera-to-world: exactly LookAt (0,0,0) -> (0,0,1), up (0,1,0)
        const float eye[3] = {0.f, 0.f, 0.f}, at[3] = {0.f, 0.f, 1.f}, up[3] = {0.f, 1.f, 0.f};
        std::copy(eye, eye + 3, info.camera.eye);
        std::copy(at, at + 3, info.camera.look_at);
        std::copy(up, up + 3, info.camera.up);
    }

    // ---- world block (pbrt_parser.cpp:1232-1711) ----
    std::vector<std::pair<std::string, std::shared_ptr<Material>>> named;
    std::vector<std::shared_ptr<Material>> mat_stack;
    std::vector<std::shared_ptr<Spd>> light_stack;
    std::vector<std::shared_ptr<Xf>> xf_stack;
    std::shared_ptr<Material> active_mat;
    std::shared_ptr<Spd> active_light;
    auto active_xf = std::make_shared<Xf>();
    std::unordered_map<std::string, std::shared_ptr<Geometry>> objects;
    std::shared_ptr<Geometry> current_geometry;
    bool in_object = false;
    std::vector<Shape> shapes;
    auto make_shape = [&](const std::shared_ptr<Geometry>& g) {
        Shape s;
        s.geometry = g;
        s.to_world = active_xf;
        s.material = active_mat;
        s.light = active_light;
        shapes.push_back(s);
    };
    for (size_t k = world + 1; k < ds.size(); ++k) {
        const Directive& d = ds[k];
        const std::string& n = d.name;
        if (n == "AreaLightSource") {
            if (d.type != "diffuse") continue;
            for (const Arg& a : d.args) {
                if (a.name != "L") continue;
                std::vector<float> v;
                if ((rc = arg_floats(d, a, v, err))) return rc;
                if (v.size() < 3) { err = "line " + std::to_string(d.line) + ": L needs 3 values"; return PT_EINVAL; }
                if (!active_light) active_light = std::make_shared<Spd>();
                for (int c = 0; c < 3; ++c) active_light->rgb[c] = v[c] * 255;
                break;
            }
        } else if (n == "AttributeBegin") {
            if (active_mat) mat_stack.push_back(active_mat);
            if (active_light) light_stack.push_back(active_light);
            xf_stack.push_back(active_xf);
            active_xf = std::make_shared<Xf>(*active_xf);
        } else if (n == "AttributeEnd") {
            if (!mat_stack.empty()) { active_mat = mat_stack.back(); mat_stack.pop_back(); }
            if (light_stack.empty()) active_light = nullptr;
            else { active_light = light_stack.back(); light_stack.pop_back(); }
            if (!xf_stack.empty()) { active_xf = xf_stack.back(); xf_stack.pop_back(); }
        } else if (n == "TransformBegin") {
            xf_stack.push_back(active_xf);
            active_xf = std::make_shared<Xf>(*active_xf);
        } else if (n == "TransformEnd") {
            if (!xf_stack.empty()) { active_xf = xf_stack.back(); xf_stack.pop_back(); }
        } else if (is_transform(n)) {
            Xf t;
            if ((rc = xf_for(d, t, err))) return rc;
            compose(*active_xf, t);
        } else if (n == "LightSource") {
            if (d.type != "infinite") continue;
            for (const Arg& a : d.args) {
                if (a.name != "L") continue;
                std::vector<float> v;
                if ((rc = arg_floats(d, a, v, err))) return rc;
                if (v.size() < 3) { err = "line " + std::to_string(d.line) + ": L needs 3 values"; return PT_EINVAL; }
                info.has_env = 1;
                for (int c = 0; c < 3; ++c) info.env[c] = v[c] * 255;
                break;
            }
        } else if (n == "Material") {
            auto m = std::make_shared<Material>();
            bool ok = false;
            if (d.type == "matte") {
                for (const Arg& a : d.args) {
                    if (a.name != "Kd") continue;
                    if (arg_is(a, "texture")) {
                        err = "line " + std::to_string(d.line) + ": textured Kd is not supported";
                        return PT_EINVAL;
                    }
                    if (!arg_is(a, "rgb")) continue;
                    std::vector<float> v;
                    if ((rc = arg_floats(d, a, v, err))) return rc;
                    if (v.size() < 3) { err = "line " + std::to_string(d.line) + ": Kd needs 3 values"; return PT_EINVAL; }
                    m->type = PT_MAT_LAMBERT;
                    std::copy(v.begin(), v.begin() + 3, m->refl);
                    ok = true;
                    break;
                }
            } else if (d.type == "mirror") {
                for (const Arg& a : d.args) {
                    if (a.name != "Kr" || !arg_is(a, "rgb")) continue;
                    std::vector<float> v;
                    if ((rc = arg_floats(d, a, v, err))) return rc;
                    if (v.size() < 3) { err = "line " + std::to_string(d.line) + ": Kr needs 3 values"; return PT_EINVAL; }
                    m->type = PT_MAT_MIRROR;
                    std::copy(v.begin(), v.begin() + 3, m->refl);
                    ok = true;
                    break;
                }
            } else if (d.type == "plastic") {
                err = "line " + std::to_string(d.line) + ": Material \"plastic\" is not supported (no glossy BRDF)";
                return PT_EINVAL;
            }
            active_mat = ok ? m : nullptr;  // unknown type or missing argument: no material
        } else if (n == "MakeNamedMaterial") {
            bool matte = false;
            for (const Arg& a : d.args)
                if (arg_is(a, "string") && a.name == "type" && !a.values.empty() && a.values[0] == "matte") matte = true;
            std::shared_ptr<Material> m;
            if (matte) {
                m = std::make_shared<Material>();
                m->type = PT_MAT_LAMBERT;
                m->refl[0] = m->refl[1] = m->refl[2] = 0.5f;
            }
            named.emplace_back(d.type, m);
        } else if (n == "NamedMaterial") {
            for (const auto& nm : named)
                if (nm.first == d.type) { active_mat = nm.second; break; }
        } else if (n == "ObjectBegin") {
            if (in_object) continue;  // nested: rejected by the reference, ignored
            in_object = true;
            current_geometry = std::make_shared<Geometry>();
            objects[d.type] = current_geometry;
        } else if (n == "ObjectEnd") {
            in_object = false;
            current_geometry = nullptr;
        } else if (n == "ObjectInstance") {
            auto it = objects.find(d.type);
            if (it == objects.end()) {
                err = "line " + std::to_string(d.line) + ": ObjectInstance [" + d.type + "] was not defined";
                return PT_EINVAL;
            }
            make_shape(it->second);
        } else if (n == "Shape") {
            if (d.type == "plymesh" || d.type == "objmesh") {
                std::string file;
                for (const Arg& a : d.args)
                    if (a.name == "filename" && !a.values.empty()) file = a.values[0];
                if (file.empty()) continue;  // missing filename: the reference skips the shape
                auto g = in_object ? current_geometry : std::make_shared<Geometry>();
                if ((rc = read_mesh_geometry(base + file, d.type == "objmesh", *g, err))) return rc;
                if (!in_object) make_shape(g);
            } else if (d.type == "sphere") {
                for (const Arg& a : d.args) {
                    if (!arg_is(a, "float")) continue;
                    std::vector<float> v;
                    if ((rc = arg_floats(d, a, v, err))) return rc;
                    if (v.empty()) continue;
                    // (int)radius steps per axis: a large radius would ask for an unbounded mesh (the
                    // reference tries to build it); refuse beyond 2048 (8.4 M faces)
                    if (!(v[0] < 2049.f)) {
                        err = "line " + std::to_string(d.line) + ": sphere radius " + std::to_string(v[0]) +
                              " would tessellate into more than 2048 x 2048 steps";
                        return PT_EINVAL;
                    }
                    auto g = std::make_shared<Geometry>();
                    const int sub = std::max((int)v[0], 20);
                    tessellate_sphere((unsigned)sub, (unsigned)sub, *g);
                    if (in_object) current_geometry = g;
                    else make_shape(g);
                }
            }
        } else if (n == "Texture") {
            err = "line " + std::to_string(d.line) + ": Texture is not supported";
            return PT_EINVAL;
        }
        // WorldBegin / WorldEnd / LookAt / Camera ... in the world block: ignored, as the reference does
    }

    // ---- descriptors ----
    for (const Shape& s : shapes) {
        const Geometry& g = *s.geometry;
        pt_mesh_desc m{};
        m.x = g.x.data(); m.y = g.y.data(); m.z = g.z.data();
        m.num_vertices = (uint32_t)g.x.size();
        m.fv0 = g.f0.data(); m.fv1 = g.f1.data(); m.fv2 = g.f2.data();
        m.num_faces = (uint32_t)g.f0.size();
        if (!g.nx.empty()) { m.nx = g.nx.data(); m.ny = g.ny.data(); m.nz = g.nz.data(); }
        for (int k = 0; k < 16; ++k) {
            m.object_to_world[k] = s.to_world->mat.m[k / 4][k % 4];
            m.world_to_object[k] = s.to_world->inv.m[k / 4][k % 4];  // the normals' matrix
        }
        if (s.material) {
            m.material = s.material->type;
            std::copy(s.material->refl, s.material->refl + 3, m.albedo);
        } else if (s.light) {
            m.material = PT_MAT_LAMBERT;  // an emitter's material is never sampled
        } else {
            m.material = 0;  // no material: pt_scene_create rejects it (the reference cannot shade it)
        }
        if (s.light) {
            m.is_light = 1;
            std::copy(s.light->rgb, s.light->rgb + 3, m.emission);
        }
        out.meshes.push_back(m);
        out.geometries.push_back(s.geometry);
    }
    info.num_meshes = (uint32_t)out.meshes.size();
    return PT_OK;
}

}  // namespace
}  // namespace pt

extern "C" {

int pt_load_pbrt(const char* path, pt_pbrt_scene** out) {
    if (!path || !out) return pt::fail(PT_EINVAL, "path or out is NULL");
    *out = nullptr;
    std::unique_ptr<pt_pbrt_scene> s(new pt_pbrt_scene());
    std::string err;
    int rc;
    try {
        rc = pt::load(path, *s, err);
    } catch (const std::bad_alloc&) {
        return pt::fail(PT_ENOMEM, "out of host memory reading the scene");
    }
    if (rc) return pt::fail(rc, "pt_load_pbrt: " + err);
    *out = s.release();
    return PT_OK;
}

int pt_pbrt_get_info(const pt_pbrt_scene* scene, pt_pbrt_info* info) {
    if (!scene || !info) return pt::fail(PT_EINVAL, "scene or info is NULL");
    *info = scene->info;
    return PT_OK;
}

int pt_pbrt_get_meshes(const pt_pbrt_scene* scene, const pt_mesh_desc** meshes) {
    if (!scene || !meshes) return pt::fail(PT_EINVAL, "scene or meshes is NULL");
    *meshes = scene->meshes.empty() ? nullptr : scene->meshes.data();
    return PT_OK;
}

void pt_pbrt_free(pt_pbrt_scene* scene) { delete scene; }

}  // extern "C"
