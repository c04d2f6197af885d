// ply.cpp -- scene ingest: PLY meshes (ascii, binary little / big endian) into the packed arrays
// pt_mesh_desc takes, following ply_parser::parse_header / parse_file
// (src/common/parsers/mesh_parsers.cpp:89-545): the same header grammar and checks (x, y, z
// required; normals all or none; uv both or none; face elements carry one vertex-index list of
// three entries), elements in file order, ascii numbers read with strtof / strtol like the
// reference's stof / stoi.  Two deliberate differences, both where the compiled reference
// mis-parses:
//   * binary values are read with their declared types (the reference reads every vertex property
//     as a 4-byte float and every face list as uchar + int32, mesh_parsers.cpp:418, 518-525);
//   * a binary vertex is appended once (the reference appends it twice when a file has no
//     normals, mesh_parsers.cpp:470-473, because parse_header sets has_vertex_uv for every file,
//     :321; its own test parse_ply.Binary, tests/parsers/test_ply_parser.cpp:110-133, expects one).
// The whole file is read into memory first, so binary meshes parse at memory speed.

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pt_internal.h"

namespace {

enum class PType { i8, u8, i16, u16, i32, u32, f32, f64, list, unknown };
enum class Field { x, y, z, nx, ny, nz, u, v, other };
enum class Fmt { ascii, le, be };

struct Prop {
    PType type = PType::unknown;
    PType count_type = PType::unknown, item_type = PType::unknown;  // lists
    Field field = Field::other;
};

struct Elem {
    bool vertex = false;
    long long count = 0;
    std::vector<Prop> props;
};

PType type_of(const std::string& t) {  // the token sets of get_type_for_token
    if (t == "char" || t == "int8" || t == "int_8") return PType::i8;
    if (t == "uchar" || t == "u_char" || t == "uint8" || t == "u_int8" || t == "uint_8" || t == "u_int_8") return PType::u8;
    if (t == "short" || t == "int16" || t == "int_16") return PType::i16;
    if (t == "ushort" || t == "u_short" || t == "uint16" || t == "u_int16" || t == "uint_16" || t == "u_int_16") return PType::u16;
    if (t == "int" || t == "int32" || t == "int_32") return PType::i32;
    if (t == "uint" || t == "u_int" || t == "uint32" || t == "u_int32" || t == "uint_32" || t == "u_int_32") return PType::u32;
    if (t == "float" || t == "float32" || t == "float_32") return PType::f32;
    if (t == "double" || t == "float64" || t == "float_64") return PType::f64;
    if (t == "list") return PType::list;
    return PType::unknown;
}

size_t size_of(PType t) {
    switch (t) {
        case PType::i8: case PType::u8: return 1;
        case PType::i16: case PType::u16: return 2;
        case PType::i32: case PType::u32: case PType::f32: return 4;
        case PType::f64: return 8;
        default: return 0;
    }
}

std::vector<std::string> split(const std::string& line) {
    std::vector<std::string> w;
    size_t i = 0;
    while (i < line.size()) {
        while (i < line.size() && (line[i] == ' ' || line[i] == '\t' || line[i] == '\r')) ++i;
        size_t j = i;
        while (j < line.size() && line[j] != ' ' && line[j] != '\t' && line[j] != '\r') ++j;
        if (j > i) w.push_back(line.substr(i, j - i));
        i = j;
    }
    return w;
}

struct Reader {
    const char* p;
    const char* end;
    Fmt fmt;
    bool line(std::string& out) {
        if (p >= end) return false;
        const char* q = (const char*)std::memchr(p, '\n', (size_t)(end - p));
        if (!q) q = end;
        out.assign(p, q);
        p = q < end ? q + 1 : end;
        return true;
    }
    bool bytes(void* dst, size_t n) {
        if ((size_t)(end - p) < n) return false;
        std::memcpy(dst, p, n);
        if (fmt == Fmt::be)
            for (size_t i = 0; i < n / 2; ++i) std::swap(((char*)dst)[i], ((char*)dst)[n - 1 - i]);
        p += n;
        return true;
    }
    // one binary value of type t as double (exact for every PLY scalar type)
    bool value(PType t, double& v) {
        union { int8_t i8; uint8_t u8; int16_t i16; uint16_t u16; int32_t i32; uint32_t u32; float f; double d; } u;
        if (!bytes(&u, size_of(t))) return false;
        switch (t) {
            case PType::i8: v = u.i8; break;
            case PType::u8: v = u.u8; break;
            case PType::i16: v = u.i16; break;
            case PType::u16: v = u.u16; break;
            case PType::i32: v = u.i32; break;
            case PType::u32: v = u.u32; break;
            case PType::f32: v = u.f; break;
            case PType::f64: v = u.d; break;
            default: return false;
        }
        return true;
    }
};

struct Loaded {
    std::vector<float> x, y, z, nx, ny, nz, u, v;
    std::vector<uint32_t> f0, f1, f2;
    bool normals = false, uv = false;
};

int load(const char* path, Loaded& m) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return pt::fail(PT_EINVAL, std::string("cannot open ") + path);
    std::vector<char> buf;
    char tmp[1 << 16];
    size_t n;
    while ((n = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + n);
    std::fclose(f);
    Reader rd{buf.data(), buf.data() + buf.size(), Fmt::ascii};
    const std::string where = std::string(path) + ": ";
    std::string line;
    if (!rd.line(line) || split(line).empty() || split(line)[0] != "ply") return pt::fail(PT_EINVAL, where + "missing PLY header");
    if (!rd.line(line)) return pt::fail(PT_EINVAL, where + "read error in the format line");
    {
        const auto w = split(line);
        if (w.empty() || w[0] != "format") return pt::fail(PT_EINVAL, where + "missing \"format\" header");
        if (w.size() < 2) return pt::fail(PT_EINVAL, where + "read error in the format type");
        if (w[1] == "ascii") rd.fmt = Fmt::ascii;
        else if (w[1] == "binary_little_endian") rd.fmt = Fmt::le;
        else if (w[1] == "binary_big_endian") rd.fmt = Fmt::be;
        else return pt::fail(PT_EINVAL, where + "unsupported format " + w[1]);
        if (w.size() < 3 || w[2] != "1.0") return pt::fail(PT_EINVAL, where + "unsupported format version");
    }
    std::vector<Elem> elems;
    bool has[8] = {};
    bool ended = false;
    while (rd.line(line)) {
        const auto w = split(line);
        if (w.empty()) continue;
        if (w[0] == "element") {
            if (w.size() < 3) return pt::fail(PT_EINVAL, where + "element line needs a name and a count");
            Elem e;
            if (w[1] == "vertex") e.vertex = true;
            else if (w[1] != "face") return pt::fail(PT_EINVAL, where + "element " + w[1] + " is not supported");
            char* endp = nullptr;
            errno = 0;
            e.count = std::strtoll(w[2].c_str(), &endp, 10);
            if (errno || *endp || e.count < 0) return pt::fail(PT_EINVAL, where + "bad element count " + w[2]);
            elems.push_back(e);
        } else if (w[0] == "property") {
            if (elems.empty()) return pt::fail(PT_EINVAL, where + "property with no preceding element");
            Elem& e = elems.back();
            Prop p;
            if (w.size() < 3) return pt::fail(PT_EINVAL, where + "short property line");
            p.type = type_of(w[1]);
            if (p.type == PType::unknown) return pt::fail(PT_EINVAL, where + "unrecognized property type " + w[1]);
            if (e.vertex) {
                if (p.type == PType::list) return pt::fail(PT_EINVAL, where + "list property on vertices");
                const std::string& nm = w[2];
                static const char* names[] = {"x", "y", "z", "nx", "ny", "nz"};
                p.field = Field::other;
                for (int k = 0; k < 6; ++k)
                    if (nm == names[k]) p.field = (Field)k;
                if (nm == "u" || nm == "s") p.field = Field::u;
                if (nm == "v" || nm == "t") p.field = Field::v;
                if (p.field != Field::other) has[(int)p.field] = true;
            } else {
                if (p.type != PType::list) return pt::fail(PT_EINVAL, where + "face property must be a list");
                if (w.size() < 5) return pt::fail(PT_EINVAL, where + "short face list property");
                p.count_type = type_of(w[2]);
                p.item_type = type_of(w[3]);
                if (p.count_type == PType::unknown || p.count_type == PType::list || p.item_type == PType::unknown ||
                    p.item_type == PType::list)
                    return pt::fail(PT_EINVAL, where + "face list has an unknown type");
                const std::string& nm = w[4];
                if (nm != "vertex_indices" && nm != "vertex_index" && nm != "vertices" && nm != "vertex")
                    return pt::fail(PT_EINVAL, where + "face list " + nm + " is not vertex_indices");
            }
            e.props.push_back(p);
        } else if (w[0] == "end_header") {
            ended = true;
            break;
        }
        // comment, obj_info and other header lines are skipped
    }
    if (!ended) return pt::fail(PT_EINVAL, where + "missing end_header");
    if (!has[0] || !has[1] || !has[2]) return pt::fail(PT_EINVAL, where + "vertex x, y and z properties are required");
    const int nn = has[3] + has[4] + has[5], nuv = has[6] + has[7];
    if (nn != 0 && nn != 3) return pt::fail(PT_EINVAL, where + "vertex normals need nx, ny and nz");
    if (nuv != 0 && nuv != 2) return pt::fail(PT_EINVAL, where + "vertex uv needs both u and v");
    m.normals = nn == 3;
    m.uv = nuv == 2;

    for (const Elem& e : elems) {
        if (e.vertex) {
            for (long long i = 0; i < e.count; ++i) {
                float val[9] = {};
                std::vector<std::string> w;
                if (rd.fmt == Fmt::ascii) {
                    if (!rd.line(line)) return pt::fail(PT_EINVAL, where + "error reading vertex " + std::to_string(i));
                    w = split(line);
                    if (w.size() < e.props.size()) return pt::fail(PT_EINVAL, where + "short vertex line " + std::to_string(i));
                }
                for (size_t k = 0; k < e.props.size(); ++k) {
                    float x;
                    if (rd.fmt == Fmt::ascii) {
                        char* endp = nullptr;
                        x = std::strtof(w[k].c_str(), &endp);  // the reference's stof
                        if (endp == w[k].c_str()) return pt::fail(PT_EINVAL, where + "bad number " + w[k]);
                    } else {
                        double d;
                        if (!rd.value(e.props[k].type, d)) return pt::fail(PT_EINVAL, where + "file ends inside vertex data");
                        x = (float)d;
                    }
                    val[(int)e.props[k].field] = x;
                }
                m.x.push_back(val[0]);
                m.y.push_back(val[1]);
                m.z.push_back(val[2]);
                if (m.normals) {
                    m.nx.push_back(val[3]);
                    m.ny.push_back(val[4]);
                    m.nz.push_back(val[5]);
                }
                if (m.uv) {
                    m.u.push_back(val[6]);
                    m.v.push_back(val[7]);
                }
            }
        } else {
            for (long long i = 0; i < e.count; ++i) {
                uint32_t idx[3] = {0, 0, 0};
                if (rd.fmt == Fmt::ascii) {
                    if (!rd.line(line)) return pt::fail(PT_EINVAL, where + "error reading face " + std::to_string(i));
                    const auto w = split(line);
                    if (w.empty() || std::strtol(w[0].c_str(), nullptr, 10) != 3 || w.size() < 4)
                        return pt::fail(PT_EINVAL, where + "face " + std::to_string(i) + " does not have 3 vertex indices");
                    for (int k = 0; k < 3; ++k) idx[k] = (uint32_t)std::strtol(w[1 + k].c_str(), nullptr, 10);  // stoui
                } else {
                    for (const Prop& p : e.props) {
                        double c;
                        if (!rd.value(p.count_type, c)) return pt::fail(PT_EINVAL, where + "file ends inside face data");
                        if (c != 3) return pt::fail(PT_EINVAL, where + "face " + std::to_string(i) + " does not have 3 vertex indices");
                        for (int k = 0; k < 3; ++k) {
                            double d;
                            if (!rd.value(p.item_type, d)) return pt::fail(PT_EINVAL, where + "file ends inside face data");
                            idx[k] = (uint32_t)(int64_t)d;
                        }
                    }
                }
                m.f0.push_back(idx[0]);
                m.f1.push_back(idx[1]);
                m.f2.push_back(idx[2]);
            }
        }
    }
    return PT_OK;
}

template <typename T>
T* copy_out(const std::vector<T>& v) {
    if (v.empty()) return nullptr;
    T* p = (T*)std::malloc(v.size() * sizeof(T));
    if (p) std::memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

}  // namespace

using namespace pt;

extern "C" int pt_load_ply(const char* path, pt_mesh_data* out) {
    if (!path || !out) return fail(PT_EINVAL, "path or out is NULL");
    std::memset(out, 0, sizeof(*out));
    Loaded m;
    const int rc = load(path, m);
    if (rc) return rc;
    out->num_vertices = (uint32_t)m.x.size();
    out->num_faces = (uint32_t)m.f0.size();
    out->x = copy_out(m.x);
    out->y = copy_out(m.y);
    out->z = copy_out(m.z);
    out->fv0 = copy_out(m.f0);
    out->fv1 = copy_out(m.f1);
    out->fv2 = copy_out(m.f2);
    if (m.normals) {
        out->nx = copy_out(m.nx);
        out->ny = copy_out(m.ny);
        out->nz = copy_out(m.nz);
    }
    if (m.uv) {
        out->u = copy_out(m.u);
        out->v = copy_out(m.v);
    }
    const bool ok = (out->num_vertices == 0 || (out->x && out->y && out->z)) &&
                    (out->num_faces == 0 || (out->fv0 && out->fv1 && out->fv2)) &&
                    (!m.normals || out->num_vertices == 0 || (out->nx && out->ny && out->nz)) &&
                    (!m.uv || out->num_vertices == 0 || (out->u && out->v));
    if (!ok) {
        pt_mesh_data_free(out);
        return fail(PT_ENOMEM, "host memory for the mesh");
    }
    return PT_OK;
}

extern "C" void pt_mesh_data_free(pt_mesh_data* m) {
    if (!m) return;
    for (void* p : {(void*)m->x, (void*)m->y, (void*)m->z, (void*)m->fv0, (void*)m->fv1, (void*)m->fv2, (void*)m->nx,
                    (void*)m->ny, (void*)m->nz, (void*)m->u, (void*)m->v})
        std::free(p);
    std::memset(m, 0, sizeof(*m));
}
