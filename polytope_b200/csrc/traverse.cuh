// traverse.cuh -- device traversal of the reference BVH (closest-hit and any-hit).
//
// Reference semantics reproduced exactly (paths relative to the Polytope source tree):
//   bvh::intersect_compact           src/cpu/acceleration/bvh.cpp:476-523
//     - ordered DFS; a node's own box is tested when it is popped, against the running MinT
//     - interior: if the ray's inverse direction is negative on the node's split axis the low
//       child is pushed first (so the high child pops first), else the high child first
//     - leaf: every face in leaf order goes through the Wald test
//   BoundingBox::Hits                src/cpu/structures/BoundingBox.cpp:12-85
//   Mesh::intersect Wald core        src/cpu/shapes/mesh.cpp:196-340
// Ties are "last accepted wins" because a later face with the same t passes `T > MinT*det`.
//
// Data layout in HBM (all read with 128-bit non-coherent loads):
//   nodes  32 B  {bb_min.xyz, bb_max.xyz, offset, num_faces | axis << 16}   (2 x uint4)
//   tris   48 B  {v0.xyz v1.x}{v1.yz v2.xy}{v2.z prim mesh 0} in leaf order (3 x float4)
//   rays   32 B  {org.xyz tmax}{dir.xyz flags}                              (2 x float4)
//   hits   16 B  {prim t u v}                                              (1 x uint4)
#pragma once

#include <cstdint>
#include <type_traits>

#include "config.h"
#include "exact_math.h"

namespace pt {

constexpr uint32_t kPrimNone = 0xFFFFFFFFu;
constexpr int kStackCap = PT_TRAVERSAL_STACK;

struct RayState {
    float ox, oy, oz;
    float ix, iy, iz;          // 1/d (bvh.cpp:477-481)
    int kz;                    // Wald axis permutation (mesh.cpp:196-211): kx = kz+1, ky = kx+1 (mod 3)
    float sx, sy, sz;          // shear constants (mesh.cpp:234-236)
    uint32_t neg;              // bit k: 1/d on axis k is < 0 (the child order, bvh.cpp:514-519)
};

// Whether the reference pushes the low child first at a node split on `axis` (1/d negative there).
// A shift and a mask instead of selecting the axis's 1/d and comparing it per node step: on a B200
// 1.3 M-face ray queries 2260 vs 2182 Mrays/s, the fused 6.5 M-face frame 989 vs 957 Msamples/s,
// the 256-scene batch 2324 vs 2251-2264 Mrays/s (two runs each, same box).
PT_HD bool neg_on(const RayState& r, uint32_t axis) { return (r.neg >> axis) & 1u; }

PT_HD float sel3(int k, float x, float y, float z) { return k == 0 ? x : (k == 1 ? y : z); }
PT_HD int next_axis(int k) { return k == 2 ? 0 : k + 1; }

// Only what the box and face tests read is kept, so a ray costs few registers in the persistent
// kernels; the permuted direction is needed only here, for the shear constants.
PT_HD void ray_setup(RayState& r, float ox, float oy, float oz, float dx, float dy, float dz) {
    r.ox = ox; r.oy = oy; r.oz = oz;
    r.ix = frcp(dx); r.iy = frcp(dy); r.iz = frcp(dz);
    r.neg = (r.ix < 0 ? 1u : 0u) | (r.iy < 0 ? 2u : 0u) | (r.iz < 0 ? 4u : 0u);
    const float ax = fabs_(dx), ay = fabs_(dy), az = fabs_(dz);
    int kz = 0;
    if (ay > ax && ay > az) kz = 1;
    else if (az > ax && az > ay) kz = 2;
    const int kx = next_axis(kz), ky = next_axis(kx);
    r.kz = kz;
    const float dkx = sel3(kx, dx, dy, dz), dky = sel3(ky, dx, dy, dz), dkz = sel3(kz, dx, dy, dz);
    r.sx = fdiv(-dkx, dkz);
    r.sy = fdiv(-dky, dkz);
    r.sz = frcp(dkz);
}

// Whether box_hits must evaluate the reference's "origin strictly inside" early-out.  For a ray
// whose far bound is not negative and whose 1/d has no NaN, an origin strictly inside the box
// always passes the slab test too (each axis then has one non-positive and one non-negative bound,
// or infinite ones, so near stays 0 <= far), so the early-out cannot change the result and is
// skipped.  The running MinT only ever drops to accepted t > 0, so this holds for the whole walk.
PT_HD bool needs_inside_test(const RayState& r, float tmax) {
    return !(tmax >= 0.f) || r.ix != r.ix || r.iy != r.iy || r.iz != r.iz;
}

// BoundingBox::Hits with the running MinT as the far bound.  The reference returns false as soon
// as near > far after an axis; near only grows and far only shrinks (a NaN bound leaves either
// unchanged), so testing once after the third axis gives the same answer without two branches.
PT_HD bool box_hits(const RayState& r, float b0, float b1, float b2, float b3, float b4, float b5,
                                         float min_t, bool check_inside = true) {
    if (check_inside) {
        const bool inside = r.ox > b0 && r.ox < b3 && r.oy > b1 && r.oy < b4 && r.oz > b2 && r.oz < b5;
        if (inside) return true;
    }
    const float gm = bitsf(PT_GAMMA_MUL_BITS);
    float far_t = min_t, near_t = 0.f;
    float tn = fmul(fsub(b0, r.ox), r.ix), tf = fmul(fsub(b3, r.ox), r.ix);
    float sw = tn;
    tn = tn > tf ? tf : tn;
    tf = sw > tf ? sw : tf;
    tf = fmul(tf, gm);
    near_t = (tn > near_t) ? tn : near_t;
    far_t = (tf < far_t) ? tf : far_t;
    tn = fmul(fsub(b1, r.oy), r.iy); tf = fmul(fsub(b4, r.oy), r.iy);
    sw = tn;
    tn = tn > tf ? tf : tn;
    tf = sw > tf ? sw : tf;
    tf = fmul(tf, gm);
    near_t = (tn > near_t) ? tn : near_t;
    far_t = (tf < far_t) ? tf : far_t;
    tn = fmul(fsub(b2, r.oz), r.iz); tf = fmul(fsub(b5, r.oz), r.iz);
    sw = tn;
    tn = tn > tf ? tf : tn;
    tf = sw > tf ? sw : tf;
    tf = fmul(tf, gm);
    near_t = (tn > near_t) ? tn : near_t;
    far_t = (tf < far_t) ? tf : far_t;
    return near_t <= far_t;
}

// The same test for a ray whose origin and 1/d are finite and 1/d has no zero component, on a tree
// whose boxes hold no NaN: then no (b - o) * (1/d) product is NaN (a NaN needs 0 * inf, inf - inf
// or a NaN operand), and on non-NaN operands the reference's ternaries `a > b ? b : a` / `a > b ? a
// : b` are min / max up to the sign of a zero, which the final `near <= far` comparison does not
// see.  So one min / max instruction replaces each compare-and-select, and the inside early-out is
// skipped as in box_hits (needs_inside_test is false for such rays when tmax >= 0).
#ifndef PT_PACKED_BOX
#define PT_PACKED_BOX 1
#endif
#if defined(__CUDA_ARCH__) && PT_PACKED_BOX
// sm_100 packed single-precision arithmetic: sub / mul .rn.f32x2 round each half exactly as the
// scalar __fsub_rn / __fmul_rn (no flush of subnormals), and three-input min / max.  The fast box
// test drops from 26 to 18 instructions; measured on a B200 (two runs each, same box): 1.3 M-face
// ray queries 2176 vs 2142 Mrays/s, the 6.5 M-face frame 1782 vs 1763 Msamples/s, the 256-scene
// batch 2248-2262 vs 2210-2226 Mrays/s, with the same hits and films.
__device__ __forceinline__ uint64_t pack2(float lo, float hi) {
    uint64_t v;
    asm("mov.b64 %0, {%1, %2};" : "=l"(v) : "f"(lo), "f"(hi));
    return v;
}
__device__ __forceinline__ void unpack2(uint64_t v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
#endif

PT_HD bool box_hits_fast(const RayState& r, float b0, float b1, float b2, float b3, float b4, float b5, float min_t) {
    const float gm = bitsf(PT_GAMMA_MUL_BITS);
#if defined(__CUDA_ARCH__) && PT_PACKED_BOX
    // the six slab products as three packed pairs: (x0, y0), (z0, x1), (y1, z1), the box words
    // taken in record order (b0 b1 | b2 b3 | b4 b5)
    float x0, y0, z0, x1, y1, z1;
    unpack2(mul2(sub2(pack2(b0, b1), pack2(r.ox, r.oy)), pack2(r.ix, r.iy)), x0, y0);
    unpack2(mul2(sub2(pack2(b2, b3), pack2(r.oz, r.ox)), pack2(r.iz, r.ix)), z0, x1);
    unpack2(mul2(sub2(pack2(b4, b5), pack2(r.oy, r.oz)), pack2(r.iy, r.iz)), y1, z1);
    const float near_t = fmaxf(max3f(fminf(x0, x1), fminf(y0, y1), fminf(z0, z1)), 0.f);
    const float far_t = fminf(fmul(min3f(fmaxf(x0, x1), fmaxf(y0, y1), fmaxf(z0, z1)), gm), min_t);
    return near_t <= far_t;
#else
    const float x0 = fmul(fsub(b0, r.ox), r.ix), x1 = fmul(fsub(b3, r.ox), r.ix);
    const float y0 = fmul(fsub(b1, r.oy), r.iy), y1 = fmul(fsub(b4, r.oy), r.iy);
    const float z0 = fmul(fsub(b2, r.oz), r.iz), z1 = fmul(fsub(b5, r.oz), r.iz);
    const float near_t = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), 0.f));
    // the reference scales each axis's far value by 1 + 2 gamma_3 before taking the minimum;
    // rounding is monotone and the factor positive, so scaling the minimum gives the same value
    const float far_t = fminf(fmul(fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fmaxf(z0, z1)), gm), min_t);
    return near_t <= far_t;
#endif
}

// Which box test a ray takes (walk state box_mode): 0 box_hits_fast, 1 box_hits without the inside
// early-out, 2 box_hits with it.  `exact_tree`: the tree has a NaN in some box.
PT_HD int box_mode_for(const RayState& r, float tmax, bool exact_tree) {
    if (needs_inside_test(r, tmax)) return 2;
    const float inf = bitsf(0x7F800000u);
    const bool finite = fabs_(r.ox) < inf && fabs_(r.oy) < inf && fabs_(r.oz) < inf && fabs_(r.ix) < inf &&
                        fabs_(r.iy) < inf && fabs_(r.iz) < inf && r.ix != 0.f && r.iy != 0.f && r.iz != 0.f;
    return (finite && !exact_tree) ? 0 : 1;
}

// Measured on a B200 against box_hits for every ray (two runs each, same box): 1.3 M-face ray
// queries 2150 vs 2104 Mrays/s, the 256-scene batch 2189 vs 1966 Mrays/s (wavefront pipeline) and
// 1662 vs 1631 (path pipeline), the 6.5 M-face frame's fused kernel 954 vs 922 Msamples/s.
PT_HD bool box_test(const RayState& r, int mode, float b0, float b1, float b2, float b3, float b4, float b5, float min_t) {
    return mode == 0 ? box_hits_fast(r, b0, b1, b2, b3, b4, b5, min_t) : box_hits(r, b0, b1, b2, b3, b4, b5, min_t, mode == 2);
}

PT_HD float max3abs(float x, float y, float z) {  // max_component(abs(v)), mesh.cpp:145-155
    x = fabs_(x); y = fabs_(y); z = fabs_(z);
    if (x >= y && x >= z) return x;
    if (y >= x && y >= z) return y;
    return z;
}

// One face of Mesh::intersect (mesh.cpp:196-322).  Vertices are world space.
PT_HD bool wald(const RayState& r, float v0x, float v0y, float v0z, float v1x, float v1y,
                                     float v1z, float v2x, float v2y, float v2z, float min_t, float& t_out,
                                     float& u_out, float& v_out, float& w_out) {
    // p_it = permute(v_i - O): per-component differences, then the axis permutation (a select of
    // exact differences, so the same values as permuting first)
    const int kz = r.kz, kx = next_axis(kz), ky = next_axis(kx);
    const float a0x = fsub(v0x, r.ox), a0y = fsub(v0y, r.oy), a0z = fsub(v0z, r.oz);
    const float a1x = fsub(v1x, r.ox), a1y = fsub(v1y, r.oy), a1z = fsub(v1z, r.oz);
    const float a2x = fsub(v2x, r.ox), a2y = fsub(v2y, r.oy), a2z = fsub(v2z, r.oz);
    float p0x = sel3(kx, a0x, a0y, a0z), p0y = sel3(ky, a0x, a0y, a0z), p0z = sel3(kz, a0x, a0y, a0z);
    float p1x = sel3(kx, a1x, a1y, a1z), p1y = sel3(ky, a1x, a1y, a1z), p1z = sel3(kz, a1x, a1y, a1z);
    float p2x = sel3(kx, a2x, a2y, a2z), p2y = sel3(ky, a2x, a2y, a2z), p2z = sel3(kz, a2x, a2y, a2z);
    p0x = ffma(r.sx, p0z, p0x); p0y = ffma(r.sy, p0z, p0y);
    p1x = ffma(r.sx, p1z, p1x); p1y = ffma(r.sy, p1z, p1y);
    p2x = ffma(r.sx, p2z, p2x); p2y = ffma(r.sy, p2z, p2y);
    float U = diff_prod(p1x, p2y, p1y, p2x);
    float V = diff_prod(p2x, p0y, p2y, p0x);
    float W = diff_prod(p0x, p1y, p0y, p1x);
    if (U == 0.0f || V == 0.0f || W == 0.0f) {  // mesh.cpp:252-264, without FP64 instructions
        U = f64_diff_emulated(p2y, p1x, p2x, p1y);
        V = f64_diff_emulated(p0y, p2x, p0x, p2y);
        W = f64_diff_emulated(p1y, p0x, p1x, p0y);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = fadd(fadd(U, V), W);
    if (det == 0.0f) return false;
    p0z = fmul(p0z, r.sz); p1z = fmul(p1z, r.sz); p2z = fmul(p2z, r.sz);
    const float T = ffma(U, p0z, sum_prod(V, p1z, W, p2z));
    const float md = fmul(min_t, det);
    if (det < 0.f && (T >= 0 || T < md)) return false;
    if (det > 0.f && (T <= 0 || T > md)) return false;
    const float rcp = frcp(det);
    const float t = fmul(T, rcp);
    const float g2 = bitsf(PT_GAMMA2_BITS), g3 = bitsf(PT_GAMMA3_BITS), g5 = bitsf(PT_GAMMA5_BITS);
    const float max_zt = max3abs(p0z, p1z, p2z);
    const float delta_z = fmul(g3, max_zt);
    const float max_xt = max3abs(p0x, p1x, p2x);
    const float max_yt = max3abs(p0y, p1y, p2y);
    const float delta_x = fmul(g5, fadd(max_xt, max_zt));
    const float delta_y = fmul(g5, fadd(max_yt, max_zt));
    const float delta_e = fmul(2.0f, fadd(fadd(fmul(fmul(g2, max_xt), max_yt), fmul(delta_y, max_xt)), fmul(delta_x, max_yt)));
    const float max_e = max3abs(U, V, W);
    const float delta_t = fmul(fmul(3.0f, fadd(fadd(fmul(fmul(g3, max_e), max_zt), fmul(delta_e, max_zt)), fmul(delta_z, max_e))),
                               fabs_(rcp));
    if (t <= delta_t) return false;
    t_out = t;
    u_out = fmul(U, rcp);
    v_out = fmul(V, rcp);
    w_out = fmul(W, rcp);
    return true;
}


// Traversal stack of one lane: the first SH entries live in shared memory (entry k of the lane at
// base[k * stride], so the lanes of a warp hit consecutive banks), the rest in local memory.
// SH = 0 keeps the whole stack in local memory (and is the only form the host build uses).
template <int CAP, int SH>
struct WalkStack {
    uint32_t* base;     // this lane's first shared entry (SH > 0)
    uint32_t stride;    // threads per block
    uint32_t spill[CAP - SH];
    PT_HD void put(int i, uint32_t v) {
        if constexpr (SH > 0) {
            if (i < SH) { base[i * stride] = v; return; }
        }
        spill[i - SH] = v;
    }
    PT_HD uint32_t get(int i) const {
        if constexpr (SH > 0) {
            if (i < SH) return base[i * stride];
        }
        return spill[i - SH];
    }
    // Entries i and i + 1 (an interior node's two children); false when they would pass CAP.  Both
    // in shared memory takes one test, which also rules out the overflow (measured on a B200: 1.3
    // M-face ray queries 2337 vs 2262 Mrays/s, the 256-scene batch 2406 vs 2321).
    PT_HD bool put2(int i, uint32_t first, uint32_t second) {
        if constexpr (SH >= 2) {
            if (i + 2 <= SH) {
                base[i * stride] = first;
                base[(i + 1) * stride] = second;
                return true;
            }
        }
        if (i + 2 > CAP) return false;
        put(i, first);
        put(i + 1, second);
        return true;
    }
};

// Resumable traversal state of one ray, for kernels that interleave many rays per lane.
template <int CAP = kStackCap, int SH = 0>
struct RayWalkT {
    RayState r;
    float min_t;
    uint32_t prim, leaf;
    float u, v, w;
    uint32_t nodes, tris;
    bool any, done;
    int box_mode;       // box_mode_for this ray
    int sp;
    WalkStack<CAP, SH> stack;
};
using RayWalk = RayWalkT<>;

template <int CAP, int SH>
PT_HD void walk_begin(RayWalkT<CAP, SH>& k, float ox, float oy, float oz, float dx, float dy, float dz, float tmax, bool any,
                      bool exact_tree = false) {
    ray_setup(k.r, ox, oy, oz, dx, dy, dz);
    k.box_mode = box_mode_for(k.r, tmax, exact_tree);
    k.min_t = tmax;
    k.prim = kPrimNone;
    k.leaf = kPrimNone;
    k.u = k.v = k.w = 0.f;
    k.nodes = k.tris = 0;
    k.any = any;
    k.done = false;
    k.sp = 1;
    k.stack.put(0, 0u);
}

// One step of the same walk: pops one node and tests its box.  Returns 1 when it is a leaf whose
// box is hit (its faces in leaf_off / leaf_n), 0 for any other node, -1 on a guard failure.  The
// caller checks k.sp > 0 first.  The persistent kernels step their lanes one node at a time with
// it (walk_round) instead of walking each lane to its next leaf.
template <bool COUNT, bool FAST = false, int CAP, int SH>
PT_HD int walk_step(RayWalkT<CAP, SH>& k, const uint4* __restrict__ nodes, uint32_t num_nodes, uint32_t& leaf_off,
                    uint32_t& leaf_n) {
    const uint32_t ni = k.stack.get(--k.sp);
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

// Pops nodes in the reference order until a leaf whose box is hit comes up (returned in
// leaf_off / leaf_n) or the stack runs empty.  Returns false on a guard failure.  The same
// steps as walk_step, in one loop with the direction signs hoisted.
template <bool COUNT, int CAP, int SH>
PT_HD bool walk_to_leaf(RayWalkT<CAP, SH>& k, const uint4* __restrict__ nodes, uint32_t num_nodes, uint32_t& leaf_off,
                        uint32_t& leaf_n) {
    leaf_n = 0;
    while (k.sp > 0) {
        const uint32_t ni = k.stack.get(--k.sp);
        if (ni >= num_nodes) return false;
        uint4 a, b;
        ldg_node(nodes + 2 * (size_t)ni, a, b);
        if (COUNT) k.nodes++;
        if (!box_test(k.r, k.box_mode, bitsf(a.x), bitsf(a.y), bitsf(a.z), bitsf(a.w), bitsf(b.x), bitsf(b.y), k.min_t))
            continue;
        const uint32_t nf = b.w & 0xFFFFu;
        if (nf > 0) {
            leaf_off = b.z;
            leaf_n = nf;
            return true;
        }
        const uint32_t axis = b.w >> 16;
        const bool neg = neg_on(k.r, axis);
        const uint32_t hi = ni + b.z, lo = ni + 1;
        if (!k.stack.put2(k.sp, neg ? lo : hi, neg ? hi : lo)) return false;
        k.sp += 2;
    }
    return true;
}

// Warp-level schedule of walk_step (walk_round): the lanes of a warp that are walking take node
// steps together until `batch` of them (or all, if fewer walk) have reached a leaf or ended their
// walk; then those lanes test their leaves' faces together while the rest wait, and the rest
// carry on walking in the next round.  A lane's own node and face sequence is the reference's
// whatever the batch; the batch only decides how long a lane that found a leaf waits for others,
// so that neither the node loop nor the face loop runs with a handful of lanes (stepping every
// lane to its own next leaf left about 9 of 32 lanes busy on the 1.3 M-face microbench).
// `walking` is this lane's eligibility at the start of the round; returns whether the lane walks
// on, and sets at_leaf (faces to test in leaf_off / leaf_n) or ok = false (guard failure).  STEPS
// node steps per ballot (a lane that reaches a leaf stops early): fewer votes, a little more
// waiting; which is faster depends on the kernel.
#ifdef __CUDACC__
template <bool COUNT, int STEPS, bool FAST_ROUNDS = false, int CAP, int SH>
__device__ __forceinline__ void walk_round(RayWalkT<CAP, SH>& k, bool walking, int batch, const uint4* __restrict__ nodes,
                                           uint32_t num_nodes, bool& at_leaf, bool& ok, uint32_t& leaf_off,
                                           uint32_t& leaf_n) {
    at_leaf = false;
    ok = true;
    const uint32_t cand = __ballot_sync(0xFFFFFFFFu, walking);
    const int want = __popc(cand) < batch ? __popc(cand) : batch;
    // FAST_ROUNDS: the box test is chosen once for the round when every walking lane takes the
    // min/max form (measured: the persistent path kernel's 256-scene plain frames 1562 vs 1496
    // Mrays/s; the wavefront extend kernel, at two steps per ballot, 2335 vs 2407, so it keeps the
    // per-step choice)
    auto steps = [&](auto fast) {
        constexpr bool kFast = decltype(fast)::value;
        while (true) {
            const bool w_now = walking && ok && !at_leaf && k.sp > 0;
            const uint32_t w = __ballot_sync(0xFFFFFFFFu, w_now);
            if (w == 0 || __popc(cand & ~w) >= want) break;
            if (w_now) {
                int r = walk_step<COUNT, kFast>(k, nodes, num_nodes, leaf_off, leaf_n);
#pragma unroll
                for (int extra = 1; extra < STEPS; ++extra)
                    if (r == 0 && k.sp > 0) r = walk_step<COUNT, kFast>(k, nodes, num_nodes, leaf_off, leaf_n);
                at_leaf = r > 0;
                ok = r >= 0;
            }
        }
    };
    if (FAST_ROUNDS && __all_sync(0xFFFFFFFFu, !walking || k.box_mode == 0))
        steps(std::true_type{});
    else
        steps(std::false_type{});
}
#endif

// The faces of one leaf in leaf order (Mesh::intersect per face, bvh.cpp:496-505).
template <bool COUNT, int CAP, int SH>
PT_HD void walk_leaf(RayWalkT<CAP, SH>& k, const float4* __restrict__ tris, uint32_t leaf_off, uint32_t leaf_n) {
    for (uint32_t j = 0; j < leaf_n; ++j) {
        const size_t ti = 3 * (size_t)(leaf_off + j);
        const float4 q0 = ldg_face(tris + ti), q1 = ldg_face(tris + ti + 1), q2 = ldg_face(tris + ti + 2);
        if (COUNT) k.tris++;
        float t, u, v, w;
        if (wald(k.r, q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, k.min_t, t, u, v, w)) {
            k.min_t = t;
            k.prim = fbits(q2.y);
            k.leaf = leaf_off + j;
            k.u = u; k.v = v; k.w = w;
            if (k.any) { k.done = true; return; }
        }
    }
}

struct TraceResult {
    uint32_t prim;   // global primitive id or kPrimNone
    uint32_t leaf;   // leaf-ordered index of the committed face
    float t, u, v, w;
    uint32_t nodes, tris;
    bool overflow;
};

// The walk of traverse with the box test fixed for the ray (FAST: box_hits_fast, chosen once per
// ray instead of per node).  The loop then carries neither the compare-and-select form nor the
// per-node choice: the fused 6.5 M-face frame went from 989 to 1357 Msamples/s on a B200.
template <bool COUNT, int CAP, bool FAST>
PT_HD TraceResult traverse_walk(const uint4* __restrict__ nodes, const float4* __restrict__ tris, uint32_t num_nodes,
                                const RayState& r, float tmax, bool any, int box_mode, TraceResult res) {
    uint32_t stack[CAP];
    int sp = 0;
    stack[sp++] = 0;
    float min_t = tmax;
    while (sp > 0) {
        const uint32_t ni = stack[--sp];
        if (ni >= num_nodes) { res.overflow = true; break; }  // malformed tree guard
        uint4 a, b;
        ldg_node(nodes + 2 * (size_t)ni, a, b);
        if (COUNT) res.nodes++;
        const bool hit = FAST ? box_hits_fast(r, bitsf(a.x), bitsf(a.y), bitsf(a.z), bitsf(a.w), bitsf(b.x), bitsf(b.y), min_t)
                              : box_test(r, box_mode, bitsf(a.x), bitsf(a.y), bitsf(a.z), bitsf(a.w), bitsf(b.x), bitsf(b.y), min_t);
        if (!hit) continue;
        const uint32_t nf = b.w & 0xFFFFu;
        if (nf > 0) {
            for (uint32_t k = 0; k < nf; ++k) {
                const size_t ti = 3 * (size_t)(b.z + k);
                const float4 q0 = ldg_face(tris + ti), q1 = ldg_face(tris + ti + 1), q2 = ldg_face(tris + ti + 2);
                if (COUNT) res.tris++;
                float t, u, v, w;
                if (wald(r, q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, min_t, t, u, v, w)) {
                    min_t = t;
                    res.prim = fbits(q2.y);
                    res.leaf = b.z + k;
                    res.t = t; res.u = u; res.v = v; res.w = w;
                    if (any) return res;
                }
            }
            continue;
        }
        if (sp + 2 > CAP) { res.overflow = true; break; }
        const uint32_t axis = b.w >> 16;
        const bool neg = neg_on(r, axis);
        const uint32_t hi = ni + b.z, lo = ni + 1;
        stack[sp++] = neg ? lo : hi;
        stack[sp++] = neg ? hi : lo;
    }
    return res;
}

// bvh::intersect_compact.  `any` stops at the first accepted face.  COUNT keeps the per-ray node
// and face test counts (Intersection::num_bb_hits + num_bb_misses, num_triangle_isects).  CAP is
// the stack capacity (tree depth + 2 must fit; the host checks before launching).
template <bool COUNT, int CAP = kStackCap>
PT_HD TraceResult traverse(const uint4* __restrict__ nodes, const float4* __restrict__ tris,
                                                uint32_t num_nodes, const RayState& r, float tmax, bool any,
                                                bool exact_tree = false) {
    TraceResult res;
    res.prim = kPrimNone;
    res.leaf = kPrimNone;
    res.t = tmax;
    res.u = res.v = res.w = 0.f;
    res.nodes = res.tris = 0;
    res.overflow = false;
    const int box_mode = box_mode_for(r, tmax, exact_tree);
    if (box_mode == 0) return traverse_walk<COUNT, CAP, true>(nodes, tris, num_nodes, r, tmax, any, 0, res);
    return traverse_walk<COUNT, CAP, false>(nodes, tris, num_nodes, r, tmax, any, box_mode, res);
}

}  // namespace pt
