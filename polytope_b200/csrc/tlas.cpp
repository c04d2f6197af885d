// tlas.cpp -- host build of the two-level scene layout (instance.h).
//
// Meshes whose descriptors share their geometry arrays (the same vertex, face and normal pointers
// and counts: what pbrt_parser.cpp:1439-1472 produces for every ObjectInstance of one object, and
// what a caller gets by reusing arrays) are instances of one geometry.  Each distinct geometry gets
// one bottom-level tree, built by the same SAH builder as the flattened scene (bvh::bound's rules)
// over its vertices in object space; the instances keep their own transform, and a top-level tree
// over the instances' world boxes (median splits on the widest centroid axis, one instance per
// leaf, in the reference node layout: low child next, high child at the node's offset) finds the
// instances a ray can reach.  Primitive ids stay the flattened scene's (mesh prim_base + face).

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "pt_internal.h"

namespace pt {
namespace {

using GeometryKey = std::tuple<const void*, const void*, const void*, const void*, const void*, const void*, uint32_t,
                               uint32_t, const void*, const void*, const void*>;

float bits_as_float(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

GeometryKey key_of(const pt_mesh_desc& d) {
    return GeometryKey{d.x, d.y, d.z, d.fv0, d.fv1, d.fv2, d.num_vertices, d.num_faces, d.nx, d.ny, d.nz};
}

// world -> object: the inverse of an affine object_to_world (last row 0 0 0 1), in double, as the
// 3x4 rows the kernels apply to ray origins (with the translation) and directions (without).
int affine_inverse(const float* m, float out[12]) {
    if (m[12] != 0.f || m[13] != 0.f || m[14] != 0.f || m[15] != 1.f) return PT_EINVAL;
    const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
    const double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
    const double det = a * A + b * B + c * C;
    if (!(std::fabs(det) > 0.0) || !std::isfinite(det)) return PT_EINVAL;
    const double inv[9] = {A / det, -(b * i - c * h) / det, (b * f - c * e) / det,
                           B / det, (a * i - c * g) / det, -(a * f - c * d) / det,
                           C / det, -(a * h - b * g) / det, (a * e - b * d) / det};
    const double t[3] = {m[3], m[7], m[11]};
    for (int r = 0; r < 3; ++r) {
        out[4 * r + 0] = (float)inv[3 * r + 0];
        out[4 * r + 1] = (float)inv[3 * r + 1];
        out[4 * r + 2] = (float)inv[3 * r + 2];
        out[4 * r + 3] = (float)-(inv[3 * r + 0] * t[0] + inv[3 * r + 1] * t[1] + inv[3 * r + 2] * t[2]);
    }
    return PT_OK;
}

struct Box {
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void add(const float* p) {
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], p[k]);
            hi[k] = std::max(hi[k], p[k]);
        }
    }
};

// Top-level tree over instance boxes, written in DFS order: node i's low child is i + 1 and its
// high child is i + offset; a leaf holds `count` consecutive entries of the leaf-ordered list.
struct TopBuilder {
    const std::vector<Box>& boxes;
    std::vector<uint32_t> order;  // instance indices in leaf order
    std::vector<pt_bvh_node> nodes;
    uint32_t depth = 0;

    explicit TopBuilder(const std::vector<Box>& b) : boxes(b) {}

    void build(std::vector<uint32_t>& items, uint32_t level) {
        depth = std::max(depth, level);
        const uint32_t me = (uint32_t)nodes.size();
        nodes.push_back(pt_bvh_node{});
        Box bb, cb;
        for (uint32_t i : items) {
            bb.add(boxes[i].lo);
            bb.add(boxes[i].hi);
            float c[3];
            for (int k = 0; k < 3; ++k) c[k] = 0.5f * (boxes[i].lo[k] + boxes[i].hi[k]);
            cb.add(c);
        }
        pt_bvh_node& n = nodes[me];
        for (int k = 0; k < 3; ++k) {
            n.bb_min[k] = bb.lo[k];
            n.bb_max[k] = bb.hi[k];
        }
        int axis = 0;
        float ext = -1.f;
        for (int k = 0; k < 3; ++k)
            if (cb.hi[k] - cb.lo[k] > ext) { ext = cb.hi[k] - cb.lo[k]; axis = k; }
        if (items.size() == 1) {
            nodes[me].offset = (uint32_t)order.size();
            nodes[me].num_faces = 1;
            nodes[me].axis = 0;
            order.push_back(items[0]);
            return;
        }
        if (ext > 0.f) {
            std::sort(items.begin(), items.end(), [&](uint32_t a, uint32_t b) {
                const float ca = boxes[a].lo[axis] + boxes[a].hi[axis], cbv = boxes[b].lo[axis] + boxes[b].hi[axis];
                return ca < cbv || (ca == cbv && a < b);
            });
        }  // else: every centroid coincides; the halves keep the instances' order
        const size_t mid = items.size() / 2;
        std::vector<uint32_t> lo(items.begin(), items.begin() + mid), hi(items.begin() + mid, items.end());
        build(lo, level + 1);
        const uint32_t high = (uint32_t)nodes.size();
        build(hi, level + 1);
        nodes[me].offset = high - me;
        nodes[me].num_faces = 0;
        nodes[me].axis = (uint16_t)axis;
    }
};

}  // namespace

int prepare_two_level_host(const pt_scene_desc* desc, HostScene& h) {
    if (!desc->meshes || desc->num_meshes == 0) return fail(PT_EINVAL, "scene has no meshes");
    if (desc->nodes) return fail(PT_EINVAL, "a two-level scene builds its own trees (nodes must be NULL)");
    for (uint32_t m = 0; m < desc->num_meshes; ++m) {
        const pt_mesh_desc& d = desc->meshes[m];
        if (d.material != PT_MAT_LAMBERT && d.material != PT_MAT_MIRROR)
            return fail(PT_EINVAL, "mesh " + std::to_string(m) + ": unknown material");
        if (d.num_faces > 65535u * 65535u) return fail(PT_EINVAL, "mesh " + std::to_string(m) + ": too many faces");
    }
    // world vertices of every instance: instance boxes, the area-light table and vertex normals,
    // bit-identical to the flattened scene's
    WorldMeshes w;
    int rc = bake_world(desc->meshes, desc->num_meshes, w);
    if (rc) return rc;
    if (w.num_prims == 0) return fail(PT_EINVAL, "scene has no faces");

    // one object-space tree per distinct geometry
    std::map<GeometryKey, uint32_t> geo_of;
    std::vector<uint32_t> geo(desc->num_meshes);
    std::vector<uint32_t> node_base, face_base;
    h.nodes.clear();
    h.tris.clear();
    h.max_depth = 0;
    for (uint32_t m = 0; m < desc->num_meshes; ++m) {
        const pt_mesh_desc& d = desc->meshes[m];
        auto it = geo_of.find(key_of(d));
        if (it != geo_of.end()) {
            geo[m] = it->second;
            continue;
        }
        if (d.num_faces == 0) return fail(PT_EINVAL, "mesh " + std::to_string(m) + " has no faces");
        const uint32_t g = (uint32_t)node_base.size();
        geo_of.emplace(key_of(d), g);
        geo[m] = g;
        pt_mesh_desc obj = d;
        for (int k = 0; k < 16; ++k) obj.object_to_world[k] = obj.world_to_object[k] = (k % 5 == 0) ? 1.f : 0.f;
        WorldMeshes wo;
        rc = bake_world(&obj, 1, wo);
        if (rc) return rc;
        BuiltTree t;
        rc = build_bvh(&obj, 1, wo, 0, t);
        if (rc) return rc;
        uint32_t depth = 0;
        rc = validate_tree(t.nodes.data(), (uint32_t)t.nodes.size(), wo.num_prims, &depth);
        if (rc) return rc;
        h.max_depth = std::max(h.max_depth, depth);
        // bottom-level node indices share the walk stack with tagged entries (bits 30 and 31)
        if ((uint64_t)h.nodes.size() + t.nodes.size() >= (1ull << 30) || (uint64_t)h.tris.size() / 12 + wo.num_prims > 0xFFFFFFF0ull)
            return fail(PT_EINVAL, "two-level scene too large");
        node_base.push_back((uint32_t)h.nodes.size());
        face_base.push_back((uint32_t)(h.tris.size() / 12));
        h.nodes.insert(h.nodes.end(), t.nodes.begin(), t.nodes.end());
        // faces in leaf order, 48 B each: {v0.xyz v1.x}{v1.yz v2.xy}{v2.z face 0 0} (object space)
        const size_t base = h.tris.size();
        h.tris.resize(base + 12 * (size_t)wo.num_prims, 0.f);
        for (size_t i = 0; i < wo.num_prims; ++i) {
            const uint32_t f = t.leaf_pairs[2 * i + 1];
            float* o = &h.tris[base + 12 * i];
            std::memcpy(o, &wo.tri[9 * (size_t)f], 9 * sizeof(float));
            o[9] = bits_as_float(f);
        }
    }
    h.num_geometries = (uint32_t)node_base.size();

    // instances and their world boxes (the baked world vertices, widened by 2^-16 of their
    // magnitude: object-space hits may land a rounding step outside the baked triangles)
    if (desc->num_meshes >= (1u << 30)) return fail(PT_EINVAL, "too many instances");
    std::vector<DeviceInstance> inst(desc->num_meshes);
    std::vector<Box> boxes(desc->num_meshes);
    for (uint32_t m = 0; m < desc->num_meshes; ++m) {
        const pt_mesh_desc& d = desc->meshes[m];
        DeviceInstance& r = inst[m];
        if (affine_inverse(d.object_to_world, r.w2o) != PT_OK)
            return fail(PT_EINVAL, "mesh " + std::to_string(m) + ": a two-level scene needs invertible affine transforms");
        std::memcpy(r.o2w, d.object_to_world, sizeof(r.o2w));
        r.node_base = node_base[geo[m]];
        r.face_base = face_base[geo[m]];
        r.prim_base = w.prim_base[m];
        r.mesh = m;
        Box& b = boxes[m];
        for (uint32_t f = 0; f < d.num_faces; ++f) {
            const float* v = &w.tri[9 * (size_t)(w.prim_base[m] + f)];
            b.add(v);
            b.add(v + 3);
            b.add(v + 6);
        }
        float mag = 0.f;
        for (int k = 0; k < 3; ++k) mag = std::max({mag, std::fabs(b.lo[k]), std::fabs(b.hi[k]), b.hi[k] - b.lo[k]});
        const float pad = std::ldexp(std::max(mag, 1e-30f), -16);
        for (int k = 0; k < 3; ++k) {
            b.lo[k] -= pad;
            b.hi[k] += pad;
        }
    }
    TopBuilder top(boxes);
    std::vector<uint32_t> all(desc->num_meshes);
    for (uint32_t m = 0; m < desc->num_meshes; ++m) all[m] = m;
    top.build(all, 0);
    h.tlas.swap(top.nodes);
    h.tlas_depth = top.depth;
    h.instances.resize(desc->num_meshes);
    for (size_t i = 0; i < top.order.size(); ++i) h.instances[i] = inst[top.order[i]];
    uint32_t tdepth = 0;
    rc = validate_tree(h.tlas.data(), (uint32_t)h.tlas.size(), (uint32_t)h.instances.size(), &tdepth);
    if (rc) return fail(rc, std::string("top-level tree: ") + pt_last_error());
    h.two_level = true;
    h.num_prims = w.num_prims;
    h.prim_base = w.prim_base;
    prepare_shading_host(desc, w, h);
    return PT_OK;
}

}  // namespace pt
