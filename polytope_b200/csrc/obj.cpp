// obj.cpp -- Wavefront OBJ meshes (pt_load_obj), read as the reference reads them.
//
// Reference: obj_parser::parse_file (src/common/parsers/mesh_parsers.cpp:547-598).  Per line, the
// first word decides:
//   * a word starting with '#': comment;
//   * a word starting with 'v' ("v", and also "vn", "vt", "vp"): a vertex from the next three
//     words, each read with std::stof (the leading number of the word);
//   * a word starting with 'f': a face from the next three words, each read with std::stoi (the
//     leading integer, so "7/3/2" is 7) minus 1; further corners of a polygon are ignored;
//   * anything else: ignored.
// A line with fewer words than needed reuses the last word read (the reference's `iss >> word`
// leaves the word unchanged when the line has run out).  Where the reference would throw (a word
// that is no number) or index outside its arrays later (an index 0 or past the vertices, which
// pt_scene_create rejects), this loader returns PT_EINVAL with the line number.

#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "pt_internal.h"

namespace pt {
namespace {

template <class T>
T* copy_out(const std::vector<T>& v) {
    if (v.empty()) return nullptr;
    T* p = static_cast<T*>(std::malloc(v.size() * sizeof(T)));
    if (p) std::memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

int parse(const std::string& path, pt_mesh_data& out, std::string& err) {
    std::ifstream f(path);
    if (!f) {
        err = "cannot open [" + path + "]";
        return PT_EINVAL;
    }
    std::vector<float> x, y, z;
    std::vector<uint32_t> f0, f1, f2;
    std::string line, word;
    int ln = 0;
    while (std::getline(f, line)) {
        ++ln;
        std::istringstream iss(line);
        if (!(iss >> word)) continue;
        const char first = word[0];
        if (first == '#') continue;
        if (first == 'v') {
            float v[3];
            for (float& c : v) {
                iss >> word;
                char* end = nullptr;
                c = std::strtof(word.c_str(), &end);
                if (end == word.c_str()) {
                    err = "line " + std::to_string(ln) + ": [" + word + "] is not a number";
                    return PT_EINVAL;
                }
            }
            x.push_back(v[0]);
            y.push_back(v[1]);
            z.push_back(v[2]);
        } else if (first == 'f') {
            uint32_t idx[3];
            for (uint32_t& c : idx) {
                iss >> word;
                char* end = nullptr;
                const long v = std::strtol(word.c_str(), &end, 10);
                if (end == word.c_str()) {
                    err = "line " + std::to_string(ln) + ": [" + word + "] is not an index";
                    return PT_EINVAL;
                }
                c = (uint32_t)((unsigned int)(int)v - 1u);  // stoui(word) - 1, 1-based to 0-based
            }
            f0.push_back(idx[0]);
            f1.push_back(idx[1]);
            f2.push_back(idx[2]);
        }
    }
    for (size_t k = 0; k < f0.size(); ++k) {
        if (f0[k] >= x.size() || f1[k] >= x.size() || f2[k] >= x.size()) {
            err = "face " + std::to_string(k) + " refers to a vertex that does not exist (OBJ indices start at 1)";
            return PT_EINVAL;
        }
    }
    out.num_vertices = (uint32_t)x.size();
    out.num_faces = (uint32_t)f0.size();
    out.x = copy_out(x);
    out.y = copy_out(y);
    out.z = copy_out(z);
    out.fv0 = copy_out(f0);
    out.fv1 = copy_out(f1);
    out.fv2 = copy_out(f2);
    if ((!x.empty() && (!out.x || !out.y || !out.z)) || (!f0.empty() && (!out.fv0 || !out.fv1 || !out.fv2))) {
        pt_mesh_data_free(&out);
        err = "out of host memory";
        return PT_ENOMEM;
    }
    return PT_OK;
}

}  // namespace
}  // namespace pt

extern "C" int pt_load_obj(const char* path, pt_mesh_data* out) {
    if (!path || !out) return pt::fail(PT_EINVAL, "path or out is NULL");
    std::memset(out, 0, sizeof(*out));
    std::string err;
    const int rc = pt::parse(path, *out, err);
    if (rc) return pt::fail(rc, "pt_load_obj: " + err);
    return PT_OK;
}
