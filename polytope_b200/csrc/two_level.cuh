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
#include "render.h"
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

// One instance's bottom-level walk of traverse_two_level (the object-space ray `r`), with the box
// test fixed for the ray (FAST: box_hits_fast) as in traverse_walk: the two-level 6.5 M-face frame
// went from 836 to 1070 Msamples/s on a B200.  Returns 0 when the walk ends, 1 when an any-hit ray
// accepted a face, -1 on a guard failure (res.overflow set).
template <bool COUNT, int CAP, bool FAST>
PT_HD int blas_walk(const TwoLevelView& v, const RayState& r, int mode, uint32_t root, uint32_t fbase, uint32_t pbase,
                    uint32_t ii, bool any, uint32_t* stack, float& min_t, TwoLevelHit& out) {
    TraceResult& res = out.r;
    int sp = 0;
    stack[sp++] = root;
    while (sp > 0) {
        const uint32_t ni = stack[--sp];
        if (ni >= v.num_nodes) { res.overflow = true; return -1; }
        uint4 na, nb;
        ldg_node(v.nodes + 2 * (size_t)ni, na, nb);
        if (COUNT) res.nodes++;
        const bool hit = FAST ? box_hits_fast(r, bitsf(na.x), bitsf(na.y), bitsf(na.z), bitsf(na.w), bitsf(nb.x), bitsf(nb.y), min_t)
                              : box_test(r, mode, bitsf(na.x), bitsf(na.y), bitsf(na.z), bitsf(na.w), bitsf(nb.x), bitsf(nb.y), min_t);
        if (!hit) continue;
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
                    if (any) return 1;
                }
            }
            continue;
        }
        if (sp + 2 > CAP) { res.overflow = true; return -1; }
        const uint32_t axis = nb.w >> 16;
        const bool neg = neg_on(r, axis);
        const uint32_t hi = ni + nb.z, lo = ni + 1;
        stack[sp++] = neg ? lo : hi;
        stack[sp++] = neg ? hi : lo;
    }
    return 0;
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
            const bool neg = neg_on(wr, axis);
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
            const int mode = box_mode_for(r, min_t, v.exact_tree);
            const int st = mode == 0 ? blas_walk<COUNT, CAP, true>(v, r, 0, root, fbase, pbase, ii, any, stack, min_t, out)
                                     : blas_walk<COUNT, CAP, false>(v, r, mode, root, fbase, pbase, ii, any, stack, min_t, out);
            if (st != 0) return out;
        }
    }
    return out;
}

}  // namespace pt

namespace pt {

// ---- resumable two-level walk (the persistent path kernel) --------------------------------------
//
// The same walk as traverse_two_level, one node at a time, on a RayWalkT whose stack holds three
// kinds of entries: top-level nodes (kTopTag | index), instances to enter (kInstTag | index) and
// an exit marker (kExitTag) below each instance's bottom-level nodes (plain indices).  Entering an
// instance carries the world ray into its object space (k.r becomes the object ray) and pushes the
// exit marker and the instance's root; popping the marker restores the world ray.  The world ray
// itself is kept by the caller (get_world(ox, oy, oz, dx, dy, dz)).  Visit order, box and face tests
// and the per-ray counts are traverse_two_level's.
constexpr uint32_t kTopTag = 0x80000000u;
constexpr uint32_t kInstTag = 0x40000000u;
constexpr uint32_t kExitTag = 0xFFFFFFFEu;

template <int CAP, int SH>
PT_HD void walk_begin_two_level(RayWalkT<CAP, SH>& k, float ox, float oy, float oz, float dx, float dy, float dz, float tmax,
                                bool any, bool exact_tree) {
    walk_begin(k, ox, oy, oz, dx, dy, dz, tmax, any, exact_tree);
    k.stack.put(0, kTopTag);  // the top-level root
}

// A stack entry that is not a bottom-level node (bits 30 or 31 set).
PT_HD bool two_level_tagged(uint32_t e) { return e >= kInstTag; }

// Handles a tagged entry of the walk (the caller popped it): an exit marker restores the world
// ray, an instance entry carries the ray into the instance's object space and pushes the exit
// marker and the instance's root, a top-level node is tested like any node (its instances or its
// children are pushed).  `lane` keeps the walk's world ray and the current instance:
// world(ox, oy, oz, dx, dy, dz) reads the world ray, set_instance(face_base, prim_base, inst)
// records the instance entered.  Returns 0, or -1 on a guard failure.
template <bool COUNT, int CAP, int SH, class Lane>
PT_HD int two_level_transition(RayWalkT<CAP, SH>& k, uint32_t e, const RenderParams* p, const Lane& lane) {
    const bool exact = p->exact_tree != 0;
    if (e == kExitTag) {
        float ox, oy, oz, dx, dy, dz;
        lane.world(ox, oy, oz, dx, dy, dz);
        ray_setup(k.r, ox, oy, oz, dx, dy, dz);
        k.box_mode = box_mode_for(k.r, k.min_t, exact);
        return 0;
    }
    if (e & kTopTag) {
        const uint32_t ti = e & ~kTopTag;
        if (ti >= p->top_num_nodes) return -1;
        uint4 a, b;
        ldg_node((const uint4*)p->top_nodes + 2 * (size_t)ti, a, b);
        if (COUNT) k.nodes++;
        if (!box_test(k.r, k.box_mode, bitsf(a.x), bitsf(a.y), bitsf(a.z), bitsf(a.w), bitsf(b.x), bitsf(b.y), k.min_t))
            return 0;
        const uint32_t nf = b.w & 0xFFFFu;
        if (nf > 0) {  // its instances, first one on top
            if (k.sp + (int)nf > CAP) return -1;
            for (uint32_t j = nf; j-- > 0;) k.stack.put(k.sp++, kInstTag | (b.z + j));
            return 0;
        }
        if (k.sp + 2 > CAP) return -1;
        const uint32_t axis = b.w >> 16;
        const bool neg = neg_on(k.r, axis);
        const uint32_t hi = ti + b.z, lo = ti + 1;
        k.stack.put(k.sp++, kTopTag | (neg ? lo : hi));
        k.stack.put(k.sp++, kTopTag | (neg ? hi : lo));
        return 0;
    }
    // into an instance: the ray in its object space, then its root
    const uint32_t ii = e & ~kInstTag;
    const DeviceInstance* in = (const DeviceInstance*)p->instances + ii;
    float w2o[12];
#pragma unroll
    for (int q = 0; q < 12; ++q) w2o[q] = ldg(in->w2o + q);
    float ox, oy, oz, dx, dy, dz, lox, loy, loz, ldx, ldy, ldz;
    lane.world(ox, oy, oz, dx, dy, dz);
    to_object(w2o, ox, oy, oz, 1.0f, lox, loy, loz);
    to_object(w2o, dx, dy, dz, 0.0f, ldx, ldy, ldz);
    ray_setup(k.r, lox, loy, loz, ldx, ldy, ldz);
    k.box_mode = box_mode_for(k.r, k.min_t, exact);
    lane.set_instance(ldg(&in->face_base), ldg(&in->prim_base), ii);
    if (k.sp + 2 > CAP) return -1;
    k.stack.put(k.sp++, kExitTag);
    k.stack.put(k.sp++, ldg(&in->node_base));
    return 0;
}

// A bottom-level node step: walk_step's test on an untagged entry the caller popped; at a hit
// leaf the faces are leaf_off .. leaf_off + leaf_n - 1 counted from the current instance's first
// face (face_base).  Returns 1 at a hit leaf, 0 otherwise, -1 on a guard failure.
template <bool COUNT, bool FAST = false, int CAP, int SH>
PT_HD int two_level_node_step(RayWalkT<CAP, SH>& k, uint32_t ni, const uint4* __restrict__ nodes, uint32_t num_nodes,
                              uint32_t& leaf_off, uint32_t& leaf_n) {
    if (ni >= num_nodes) return -1;
    uint4 a, b;
    ldg_node(nodes + 2 * (size_t)ni, a, b);
    if (COUNT) k.nodes++;
    const bool hit = FAST ? box_hits_fast(k.r, bitsf(a.x), bitsf(a.y), bitsf(a.z), bitsf(a.w), bitsf(b.x), bitsf(b.y), k.min_t)
                          : box_test(k.r, k.box_mode, bitsf(a.x), bitsf(a.y), bitsf(a.z), bitsf(a.w), bitsf(b.x), bitsf(b.y), k.min_t);
    if (!hit) return 0;
    const uint32_t nf = b.w & 0xFFFFu;
    if (nf > 0) {
        leaf_off = b.z;
        leaf_n = nf;
        return 1;
    }
    const uint32_t axis = b.w >> 16;
    const bool neg = neg_on(k.r, axis);
    const uint32_t hi = ni + b.z, lo = ni + 1;
    if (!k.stack.put2(k.sp, neg ? lo : hi, neg ? hi : lo)) return -1;
    k.sp += 2;
    return 0;
}

// The faces of one bottom-level leaf (object space, records face_base + leaf_off + j); primitive
// ids are prim_base + local face.  Returns whether a face was accepted (the caller records the
// instance of the hit).
template <bool COUNT, int CAP, int SH>
PT_HD bool walk_leaf_two_level(RayWalkT<CAP, SH>& k, const float4* __restrict__ tris, uint32_t face_base, uint32_t leaf_off,
                               uint32_t leaf_n, uint32_t prim_base) {
    bool accepted = false;
    for (uint32_t j = 0; j < leaf_n; ++j) {
        const uint32_t face = face_base + leaf_off + j;
        const size_t ti = 3 * (size_t)face;
        const float4 q0 = ldg_face(tris + ti), q1 = ldg_face(tris + ti + 1), q2 = ldg_face(tris + ti + 2);
        if (COUNT) k.tris++;
        float tt, u, v, w;
        if (wald(k.r, q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, k.min_t, tt, u, v, w)) {
            k.min_t = tt;
            k.prim = prim_base + fbits(q2.y);
            k.leaf = face;
            k.u = u; k.v = v; k.w = w;
            accepted = true;
            if (k.any) { k.done = true; return true; }
        }
    }
    return accepted;
}

}  // namespace pt
