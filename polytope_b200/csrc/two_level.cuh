// two_level.cuh -- device traversal of the two-level scene layout (instance.h).
//
// The top-level tree is walked with the world ray in the reference's order (box test at pop,
// nearer child first by the sign of 1/d on the split axis); at a leaf each instance's bottom-level
// tree is walked with the ray carried into the instance's object space (origin and direction
// through the world -> object rows; the direction is not renormalised, so the ray parameter t, and
// with it MinT, is shared by both spaces).  Inside a bottom-level tree every box and face test is
// the flattened traversal's (traverse.cuh: box_hits, wald).  The closest hit over all instances
// wins; any-hit rays stop at the first accepted face.
#pragma once

#include "instance.h"
#include "traverse.cuh"

namespace pt {

constexpr int kTopStackCap = PT_TOP_STACK;

struct TwoLevelView {
    const uint4* nodes;          // every bottom-level tree, back to back
    const float4* tris;          // their leaf-ordered object-space faces {v0 v1.x}{v1.yz v2.xy}{v2.z face 0 0}
    uint32_t num_nodes;
    const uint4* top;            // top-level nodes
    uint32_t top_nodes;
    const DeviceInstance* inst;  // instances in top-level leaf order
    bool exact_tree;             // some box holds a NaN: every ray takes the exact box test
};

struct TwoLevelHit {
    TraceResult r;   // prim = global primitive id, leaf = face record index (object space)
    uint32_t inst;   // instance (top-level leaf order) of the hit
};

PT_HD void to_object(const float* m, float x, float y, float z, float w, float& ox, float& oy, float& oz) {
    // rows of the 3x4 world -> object map; w = 1 for points, 0 for directions
    ox = fadd(fadd(fadd(fmul(m[0], x), fmul(m[1], y)), fmul(m[2], z)), fmul(m[3], w));
    oy = fadd(fadd(fadd(fmul(m[4], x), fmul(m[5], y)), fmul(m[6], z)), fmul(m[7], w));
    oz = fadd(fadd(fadd(fmul(m[8], x), fmul(m[9], y)), fmul(m[10], z)), fmul(m[11], w));
}

// Transform::ApplyInPlace(Point&) (Transform.cpp:69-91) with the mesh's object_to_world: the same
// arithmetic the host uses to bake the flattened scene's world vertices, so a face's world
// vertices are bit-identical in both layouts.
PT_HD void apply_point_dev(const float* m, float& x, float& y, float& z) {
    const float nx = fadd(sum_prod(x, m[0], y, m[1]), ffma(z, m[2], m[3]));
    const float ny = fadd(sum_prod(x, m[4], y, m[5]), ffma(z, m[6], m[7]));
    const float nz = fadd(sum_prod(x, m[8], y, m[9]), ffma(z, m[10], m[11]));
    const float w = fadd(sum_prod(x, m[12], y, m[13]), ffma(z, m[14], m[15]));
    if (w == 1.0f) {
        x = nx; y = ny; z = nz;
    } else {
        const float div = fdiv(1.0f, w);
        x = fmul(nx, div); y = fmul(ny, div); z = fmul(nz, div);
    }
}

template <bool COUNT, int CAP = kStackCap>
PT_HD TwoLevelHit traverse_two_level(const TwoLevelView& v, float ox, float oy, float oz, float dx, float dy, float dz,
                                     float tmax, bool any) {
    TwoLevelHit out;
    TraceResult& res = out.r;
    res.prim = kPrimNone;
    res.leaf = kPrimNone;
    res.t = tmax;
    res.u = res.v = res.w = 0.f;
    res.nodes = res.tris = 0;
    res.overflow = false;
    out.inst = 0;
    RayState wr;
    ray_setup(wr, ox, oy, oz, dx, dy, dz);
    const bool wneg_x = wr.ix < 0, wneg_y = wr.iy < 0, wneg_z = wr.iz < 0;
    const int wmode = box_mode_for(wr, tmax, v.exact_tree);
    float min_t = tmax;
    uint32_t tstack[kTopStackCap];
    int tsp = 0;
    tstack[tsp++] = 0;
    uint32_t stack[CAP];
    while (tsp > 0) {
        const uint32_t ti = tstack[--tsp];
        if (ti >= v.top_nodes) { res.overflow = true; return out; }
        uint4 a, b;
        ldg_node(v.top + 2 * (size_t)ti, a, b);
        if (COUNT) res.nodes++;
        if (!box_test(wr, wmode, bitsf(a.x), bitsf(a.y), bitsf(a.z), bitsf(a.w), bitsf(b.x), bitsf(b.y), min_t)) continue;
        const uint32_t nf = b.w & 0xFFFFu;
        if (nf == 0) {
            if (tsp + 2 > kTopStackCap) { res.overflow = true; return out; }
            const uint32_t axis = b.w >> 16;
            const uint32_t hi = ti + b.z, lo = ti + 1;
            const bool neg = axis == 0 ? wneg_x : (axis == 1 ? wneg_y : wneg_z);
            tstack[tsp++] = neg ? lo : hi;
            tstack[tsp++] = neg ? hi : lo;
            continue;
        }
        for (uint32_t k = 0; k < nf; ++k) {
            const uint32_t ii = b.z + k;
            const DeviceInstance* in = v.inst + ii;
            float w2o[12];
#pragma unroll
            for (int q = 0; q < 12; ++q) w2o[q] = ldg(in->w2o + q);
            const uint32_t root = ldg(&in->node_base), fbase = ldg(&in->face_base), pbase = ldg(&in->prim_base);
            float lox, loy, loz, ldx, ldy, ldz;
            to_object(w2o, ox, oy, oz, 1.0f, lox, loy, loz);
            to_object(w2o, dx, dy, dz, 0.0f, ldx, ldy, ldz);
            RayState r;
            ray_setup(r, lox, loy, loz, ldx, ldy, ldz);
            const bool neg_x = r.ix < 0, neg_y = r.iy < 0, neg_z = r.iz < 0;
            const int mode = box_mode_for(r, min_t, v.exact_tree);
            int sp = 0;
            stack[sp++] = root;
            while (sp > 0) {
                const uint32_t ni = stack[--sp];
                if (ni >= v.num_nodes) { res.overflow = true; return out; }
                uint4 na, nb;
                ldg_node(v.nodes + 2 * (size_t)ni, na, nb);
                if (COUNT) res.nodes++;
                if (!box_test(r, mode, bitsf(na.x), bitsf(na.y), bitsf(na.z), bitsf(na.w), bitsf(nb.x), bitsf(nb.y), min_t))
                    continue;
                const uint32_t nfaces = nb.w & 0xFFFFu;
                if (nfaces > 0) {
                    for (uint32_t j = 0; j < nfaces; ++j) {
                        const uint32_t face = fbase + nb.z + j;
                        const size_t fi = 3 * (size_t)face;
                        const float4 q0 = ldg_face(v.tris + fi), q1 = ldg_face(v.tris + fi + 1), q2 = ldg_face(v.tris + fi + 2);
                        if (COUNT) res.tris++;
                        float t, u, vv, w;
                        if (wald(r, q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, min_t, t, u, vv, w)) {
                            min_t = t;
                            res.prim = pbase + fbits(q2.y);
                            res.leaf = face;
                            res.t = t; res.u = u; res.v = vv; res.w = w;
                            out.inst = ii;
                            if (any) return out;
                        }
                    }
                    continue;
                }
                if (sp + 2 > CAP) { res.overflow = true; return out; }
                const uint32_t axis = nb.w >> 16;
                const bool neg = axis == 0 ? neg_x : (axis == 1 ? neg_y : neg_z);
                const uint32_t hi = ni + nb.z, lo = ni + 1;
                stack[sp++] = neg ? lo : hi;
                stack[sp++] = neg ? hi : lo;
            }
        }
    }
    return out;
}

}  // namespace pt
