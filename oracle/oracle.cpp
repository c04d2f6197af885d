// oracle.cpp -- CPU restatement of Polytope's ray/path-tracing hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the oracle the CUDA path is compared against; nothing in
// the product (polytope_b200/) links, loads or calls it.  It restates, function by function, the
// reference algorithm (paths relative to the Polytope source tree):
//
//   orc_apply_point      Transform::ApplyInPlace(Point&)            src/cpu/structures/Transform.cpp:69-91
//   orc_apply_normal     Transform::ApplyInPlace(Normal&)           src/cpu/structures/Transform.cpp:135-143
//   bbox_hits            BoundingBox::Hits                          src/cpu/structures/BoundingBox.cpp:12-85
//   surface_area         BoundingBox::surface_area                  src/cpu/structures/BoundingBox.cpp:146-152
//   Oracle::build        bvh::bound                                 src/cpu/acceleration/bvh.cpp:36-395
//   Oracle::compact      bvh::compact / compact_helper              src/cpu/acceleration/bvh.cpp:652-698
//   wald_test            Mesh::intersect (per-face Wald core)       src/cpu/shapes/mesh.cpp:169-355
//   Oracle::trace        bvh::intersect_compact                     src/cpu/acceleration/bvh.cpp:476-523
//   hit_frame            Mesh::intersect post-hit frame             src/cpu/shapes/mesh.cpp:366-460
//   camera_ray           PerspectiveCamera::get_ray_for_pixel       src/cpu/cameras/PerspectiveCamera.cpp:17-49
//                        + Transform::LookAt, Transform *=          Transform.cpp:322-365, Matrix4x4.cpp:244-303
//   Oracle::path_sample  PathTraceIntegrator::GetSample             src/cpu/integrators/PathTraceIntegrator.cpp:10-135
//                        (patched: counter RNG, frame from the hit mesh, area-light NEE, float film)
//   film                 BoxFilter::AddSample / Output              src/cpu/filters/BoxFilter.cpp:14-71
//
// Parity pins: the restatement is checked against the reference compiled from its own sources
// (oracle/_ref, built by oracle/Makefile) and against the golden vectors of the reference's own
// unit tests (tests/shapes/test_mesh.cpp, tests/test_bvh.cpp, tests/TestBoundingBox.cpp,
// tests/cuda/test_bvh_traversal.cpp, tests/TestIntersectionTests.cpp,
// tests/shading/test_mirror_brdf.cpp), see tests/golden/.
//
// Build flags matter: -O2 -ffp-contract=off, no -ffast-math, no -march (x86-64 baseline has no FMA
// contraction), so every + - * / sqrt is one IEEE-754 binary32 operation and std::fma is exact.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <thread>
#include <utility>
#include <vector>

namespace {

constexpr float kInf = std::numeric_limits<float>::infinity();
constexpr float kFloatMax = std::numeric_limits<float>::max();

// constants.h:62,136-148 -- gamma_n = n*eps / (1 - n*eps), eps = FLT_EPSILON / 2, evaluated in float.
constexpr float kMachEps = std::numeric_limits<float>::epsilon() * 0.5f;
constexpr float gamma_n(int n) { return (n * kMachEps) / (1 - n * kMachEps); }
constexpr float kGamma2 = gamma_n(2);
constexpr float kGamma3 = gamma_n(3);
constexpr float kGamma5 = gamma_n(5);
constexpr float kGamma7 = gamma_n(7);
// BoundingBox.cpp:27 -- 1 + 2 * Gamma(3); Gamma(n) uses 1.f - n*eps (same value for these n).
constexpr float kGammaMul = 1 + 2 * ((3 * kMachEps) / (1.f - 3 * kMachEps));
constexpr float kPi = float(3.14159265358979323846);
constexpr float kOneOverPi = 1.0f / kPi;

struct V3 { float x, y, z; };

inline float comp(const V3& v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
inline V3 sub(const V3& a, const V3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(const V3& a, const V3& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 scale(const V3& a, float t) { return {a.x * t, a.y * t, a.z * t}; }
// Vector::Dot(const Vector& v) const returns v.x*x + v.y*y + v.z*z (Vectors.cpp:44-50): `self`
// is the object the method is called on, `arg` the argument.
inline float dot(const V3& self, const V3& arg) { return arg.x * self.x + arg.y * self.y + arg.z * self.z; }
// Vector::Cross (Vectors.cpp:101-111)
inline V3 cross(const V3& s, const V3& r) {
    return {s.y * r.z - s.z * r.y, s.z * r.x - s.x * r.z, s.x * r.y - s.y * r.x};
}
// Vector::Normalize / Normal::Normalize (Vectors.cpp:11-16, 94-99)
inline V3 normalize(V3 v) {
    const float d = 1.0f / std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    v.x *= d; v.y *= d; v.z *= d;
    return v;
}

// constants.h:121-133
inline float diff_prod(float a, float b, float c, float d) {
    float cd = c * d;
    float dop = std::fma(a, b, -cd);
    float err = std::fma(-c, d, cd);
    return dop + err;
}
inline float sum_prod(float a, float b, float c, float d) {
    float cd = c * d;
    float sop = std::fma(a, b, cd);
    float err = std::fma(c, d, -cd);
    return sop + err;
}

}  // namespace

extern "C" {

// Transform::ApplyInPlace(Point&), Transform.cpp:69-91.  m is row-major Matrix[r][c].
void orc_apply_point(const float* m, float* p) {
    const float x = p[0], y = p[1], z = p[2];
    float nx = sum_prod(x, m[0], y, m[1]) + std::fma(z, m[2], m[3]);
    float ny = sum_prod(x, m[4], y, m[5]) + std::fma(z, m[6], m[7]);
    float nz = sum_prod(x, m[8], y, m[9]) + std::fma(z, m[10], m[11]);
    float w = sum_prod(x, m[12], y, m[13]) + std::fma(z, m[14], m[15]);
    if (w == 1) {
        p[0] = nx; p[1] = ny; p[2] = nz;
    } else {
        float div = 1.f / w;
        p[0] = nx * div; p[1] = ny * div; p[2] = nz * div;
    }
}

// Transform::ApplyInPlace(Normal&), Transform.cpp:135-143: transpose of the inverse.
void orc_apply_normal(const float* inv, float* n) {
    const float x = n[0], y = n[1], z = n[2];
    n[0] = x * inv[0] + y * inv[4] + z * inv[8];
    n[1] = x * inv[1] + y * inv[5] + z * inv[9];
    n[2] = x * inv[2] + y * inv[6] + z * inv[10];
}

}  // extern "C"

namespace {

struct Box { V3 p0, p1; };

// BoundingBox::surface_area, BoundingBox.cpp:146-152
inline float surface_area(const Box& b) {
    const float x = b.p1.x - b.p0.x, y = b.p1.y - b.p0.y, z = b.p1.z - b.p0.z;
    return (2 * x * y) + (2 * y * z) + (2 * z * x);
}

// BoundingBox::UnionInPlace(const BoundingBox&), BoundingBox.cpp:136-144
inline void union_in_place(Box& a, const Box& b) {
    a.p0.x = a.p0.x < b.p0.x ? a.p0.x : b.p0.x;
    a.p0.y = a.p0.y < b.p0.y ? a.p0.y : b.p0.y;
    a.p0.z = a.p0.z < b.p0.z ? a.p0.z : b.p0.z;
    a.p1.x = a.p1.x > b.p1.x ? a.p1.x : b.p1.x;
    a.p1.y = a.p1.y > b.p1.y ? a.p1.y : b.p1.y;
    a.p1.z = a.p1.z > b.p1.z ? a.p1.z : b.p1.z;
}

// BoundingBox::Hits, BoundingBox.cpp:12-85.  min_t is the running poly::Ray::MinT.
inline bool bbox_hits(const float* bb, const V3& o, const V3& inv, float min_t) {
    const bool inside = o.x > bb[0] && o.x < bb[3] && o.y > bb[1] && o.y < bb[4] && o.z > bb[2] && o.z < bb[5];
    if (inside) return true;
    float far_t = min_t;
    float near_t = 0;
    for (int a = 0; a < 3; ++a) {
        const float oa = comp(o, a), ia = comp(inv, a);
        float tn = (bb[a] - oa) * ia;
        float tf = (bb[3 + a] - oa) * ia;
        const float sw = tn;
        tn = tn > tf ? tf : tn;
        tf = sw > tf ? sw : tf;
        tf *= kGammaMul;
        near_t = (tn > near_t) ? tn : near_t;
        far_t = (tf < far_t) ? tf : far_t;
        if (a < 2) {
            if (near_t > far_t) return false;
        } else {
            return near_t <= far_t;
        }
    }
    return false;
}

// (float)((double)a*b - (double)c*d): the FP64 edge fallback of mesh.cpp:252-264.
inline float f64_diff(float a, float b, float c, float d) {
    const double ab = (double)a * (double)b;
    const double cd = (double)c * (double)d;
    return (float)(ab - cd);
}

struct Tri { V3 v0, v1, v2; };

struct WaldCommit { float t, u, v, w; };

// mesh.cpp:196-322 (one face).  Returns true and fills `c` when the face is accepted with the
// running min_t; the caller then commits (mesh.cpp:331-340).
inline bool wald_test(const Tri& tri, const V3& o, const V3& d, float min_t, WaldCommit& c) {
    const float dxa = std::fabs(d.x), dya = std::fabs(d.y), dza = std::fabs(d.z);
    int kz = 0;
    if (dya > dxa && dya > dza) kz = 1;
    else if (dza > dxa && dza > dya) kz = 2;
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    const V3 a = sub(tri.v0, o), b = sub(tri.v1, o), cc = sub(tri.v2, o);
    V3 p0 = {comp(a, kx), comp(a, ky), comp(a, kz)};
    V3 p1 = {comp(b, kx), comp(b, ky), comp(b, kz)};
    V3 p2 = {comp(cc, kx), comp(cc, ky), comp(cc, kz)};
    const V3 dp = {comp(d, kx), comp(d, ky), comp(d, kz)};
    const float sx = -dp.x / dp.z;
    const float sy = -dp.y / dp.z;
    const float sz = 1.f / dp.z;
    p0.x = std::fma(sx, p0.z, p0.x); p0.y = std::fma(sy, p0.z, p0.y);
    p1.x = std::fma(sx, p1.z, p1.x); p1.y = std::fma(sy, p1.z, p1.y);
    p2.x = std::fma(sx, p2.z, p2.x); p2.y = std::fma(sy, p2.z, p2.y);
    float U = diff_prod(p1.x, p2.y, p1.y, p2.x);
    float V = diff_prod(p2.x, p0.y, p2.y, p0.x);
    float W = diff_prod(p0.x, p1.y, p0.y, p1.x);
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = f64_diff(p2.y, p1.x, p2.x, p1.y);
        V = f64_diff(p0.y, p2.x, p0.x, p2.y);
        W = f64_diff(p1.y, p0.x, p1.x, p0.y);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = U + V + W;
    if (det == 0.0f) return false;
    p0.z *= sz; p1.z *= sz; p2.z *= sz;
    const float T = std::fma(U, p0.z, sum_prod(V, p1.z, W, p2.z));
    if (det < 0.f && (T >= 0 || T < min_t * det)) return false;
    if (det > 0.f && (T <= 0 || T > min_t * det)) return false;
    const float rcp = 1.0f / det;
    const float u = U * rcp, v = V * rcp, w = W * rcp;
    const float t = T * rcp;
    // max_component(abs(...)), mesh.cpp:145-155
    auto maxc = [](float x, float y, float z) {
        x = std::fabs(x); y = std::fabs(y); z = std::fabs(z);
        if (x >= y && x >= z) return x;
        if (y >= x && y >= z) return y;
        return z;
    };
    const float max_zt = maxc(p0.z, p1.z, p2.z);
    const float delta_z = kGamma3 * max_zt;
    const float max_xt = maxc(p0.x, p1.x, p2.x);
    const float max_yt = maxc(p0.y, p1.y, p2.y);
    const float delta_x = kGamma5 * (max_xt + max_zt);
    const float delta_y = kGamma5 * (max_yt + max_zt);
    const float delta_e = 2 * (kGamma2 * max_xt * max_yt + delta_y * max_xt + delta_x * max_yt);
    const float max_e = maxc(U, V, W);
    const float delta_t = 3 * (kGamma3 * max_e * max_zt + delta_e * max_zt + delta_z * max_e) * std::fabs(rcp);
    if (t <= delta_t) return false;
    c = {t, u, v, w};
    return true;
}

// ----------------------------------------------------------------------------------------------
// Scene: meshes with world-space vertices (ApplyInPlace of each packed vertex, as Mesh::intersect
// does per test at mesh.cpp:185-187 and bvh::bound at bvh.cpp:80-82).

struct OMesh {
    std::vector<float> x, y, z;          // packed positions (object space)
    std::vector<uint32_t> fv0, fv1, fv2;
    std::vector<float> nx, ny, nz;       // packed vertex normals (optional)
    float m[16], inv[16];
    uint32_t material;
    float albedo[3];
    int is_light;
    float emission[3];
    uint32_t prim_base;
};

struct ONode {  // byte layout of compact_bvh_node (bvh.h:24-53)
    float bb[6];
    uint32_t offset;
    uint16_t num_faces;
    uint16_t axis;
};
static_assert(sizeof(ONode) == 32, "node layout");

struct TreeNode {  // bvh_node (bvh.h:14-22)
    int low = -1, high = -1;
    uint16_t axis = 0;
    Box bb;
    std::vector<std::pair<uint32_t, uint32_t>> indices;
};

struct Camera {
    float m[16];       // CameraToWorld.Matrix
    float one_over_w, one_over_h, aspect, tan_half;
};

struct RenderDesc {
    uint32_t width, height, spp, max_depth;
    uint64_t seed;
    uint32_t flags;
};

// Counter-based RNG shared with the CUDA path: Philox4x32-10 (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11), counter = (pixel, sample, bounce, block),
// key = (seed_lo, seed_hi).  Replaces NormalizedUniformRandom (constants.h:100-104).
inline void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c[1] ^ k0;
        const uint32_t n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}
inline float u01(uint32_t x) { return (float)(x >> 8) * 5.9604644775390625e-08f; }

// sin/cos of 2*pi*u for u in [0,1): quadrant from rint(4u), Taylor polynomials of sin/cos(pi/2 r)
// for r in [-1/2, 1/2] evaluated with fma.  Replaces std::cos/std::sin(TwoPI * u1) in
// CosineSampleHemisphere (constants.h:106-115) so both sides are bit-identical.
constexpr float kS1 = 1.57079632679489661923f;
constexpr float kS3 = -0.645964097506246253655f;
constexpr float kS5 = 0.0796926262461670451206f;
constexpr float kS7 = -0.00468175413531868810256f;
constexpr float kS9 = 0.000160441184787359821833f;
constexpr float kC2 = -1.23370055013616982735f;
constexpr float kC4 = 0.253669507901048014030f;
constexpr float kC6 = -0.0208634807633529608730f;
constexpr float kC8 = 0.000919260274839426215087f;
constexpr float kC10 = -0.0000252020423730606054811f;
inline void sincos_2pi(float u, float& s, float& c) {
    const float f = 4.0f * u;
    const float q = std::nearbyint(f);  // round half to even (default rounding mode)
    const float r = f - q;
    const float r2 = r * r;
    float ps = std::fma(r2, kS9, kS7);
    ps = std::fma(r2, ps, kS5);
    ps = std::fma(r2, ps, kS3);
    ps = std::fma(r2, ps, kS1);
    const float sr = r * ps;
    float pc = std::fma(r2, kC10, kC8);
    pc = std::fma(r2, pc, kC6);
    pc = std::fma(r2, pc, kC4);
    pc = std::fma(r2, pc, kC2);
    const float cr = std::fma(r2, pc, 1.0f);
    const int quad = ((int)q) & 3;
    if (quad == 0) { s = sr; c = cr; }
    else if (quad == 1) { s = cr; c = -sr; }
    else if (quad == 2) { s = -sr; c = -cr; }
    else { s = -cr; c = sr; }
}

struct Frame {  // the fields of poly::Intersection used by the integrator
    V3 loc;       // offset spawn point (mesh.cpp:419-436)
    V3 n;         // geo_normal == bent_normal
    V3 t1, t2;
};

class Oracle {
public:
    std::vector<OMesh> meshes;
    std::vector<Tri> world;                 // world-space triangle of global prim id
    std::vector<uint32_t> prim_mesh;        // mesh of global prim id
    std::vector<ONode> nodes;
    std::vector<std::pair<uint32_t, uint32_t>> leaf;  // leaf_ordered_indices
    std::vector<uint32_t> leaf_prim;        // global prim id of leaf-ordered entry
    uint32_t num_prims = 0;
    bool has_env = false;
    float env[3] = {0, 0, 0};
    // area lights (world space)
    std::vector<uint32_t> light_prims;
    std::vector<float> light_cdf;
    float light_area = 0;

    void bake() {
        uint32_t base = 0;
        for (auto& m : meshes) { m.prim_base = base; base += (uint32_t)m.fv0.size(); }
        num_prims = base;
        world.resize(num_prims);
        prim_mesh.resize(num_prims);
        for (uint32_t mi = 0; mi < meshes.size(); ++mi) {
            const OMesh& m = meshes[mi];
            for (uint32_t f = 0; f < m.fv0.size(); ++f) {
                float v[3][3];
                const uint32_t idx[3] = {m.fv0[f], m.fv1[f], m.fv2[f]};
                for (int k = 0; k < 3; ++k) {
                    v[k][0] = m.x[idx[k]]; v[k][1] = m.y[idx[k]]; v[k][2] = m.z[idx[k]];
                    orc_apply_point(m.m, v[k]);
                }
                world[m.prim_base + f] = {{v[0][0], v[0][1], v[0][2]}, {v[1][0], v[1][1], v[1][2]},
                                          {v[2][0], v[2][1], v[2][2]}};
                prim_mesh[m.prim_base + f] = mi;
            }
        }
    }

    // bvh::bound, bvh.cpp:36-395.  Tree nodes live in `tree`; processing order is FIFO as in the
    // reference (the order does not change the tree).
    std::vector<TreeNode> tree;
    void build() {
        struct TI { Box bb; V3 c; };
        std::vector<std::vector<TI>> info(meshes.size());
        Box root_bb{{kInf, kInf, kInf}, {-kInf, -kInf, -kInf}};
        std::vector<std::pair<uint32_t, uint32_t>> master;
        master.reserve(num_prims);
        for (uint32_t mi = 0; mi < meshes.size(); ++mi) {
            const OMesh& m = meshes[mi];
            info[mi].reserve(m.fv0.size());
            for (uint32_t f = 0; f < m.fv0.size(); ++f) {
                const Tri& t = world[m.prim_base + f];
                Box b;
                b.p0.x = t.v0.x < t.v1.x ? t.v0.x : t.v1.x; b.p0.x = b.p0.x < t.v2.x ? b.p0.x : t.v2.x;
                b.p0.y = t.v0.y < t.v1.y ? t.v0.y : t.v1.y; b.p0.y = b.p0.y < t.v2.y ? b.p0.y : t.v2.y;
                b.p0.z = t.v0.z < t.v1.z ? t.v0.z : t.v1.z; b.p0.z = b.p0.z < t.v2.z ? b.p0.z : t.v2.z;
                b.p1.x = t.v0.x > t.v1.x ? t.v0.x : t.v1.x; b.p1.x = b.p1.x > t.v2.x ? b.p1.x : t.v2.x;
                b.p1.y = t.v0.y > t.v1.y ? t.v0.y : t.v1.y; b.p1.y = b.p1.y > t.v2.y ? b.p1.y : t.v2.y;
                b.p1.z = t.v0.z > t.v1.z ? t.v0.z : t.v1.z; b.p1.z = b.p1.z > t.v2.z ? b.p1.z : t.v2.z;
                root_bb.p0.x = root_bb.p0.x < b.p0.x ? root_bb.p0.x : b.p0.x;
                root_bb.p0.y = root_bb.p0.y < b.p0.y ? root_bb.p0.y : b.p0.y;
                root_bb.p0.z = root_bb.p0.z < b.p0.z ? root_bb.p0.z : b.p0.z;
                root_bb.p1.x = root_bb.p1.x > b.p1.x ? root_bb.p1.x : b.p1.x;
                root_bb.p1.y = root_bb.p1.y > b.p1.y ? root_bb.p1.y : b.p1.y;
                root_bb.p1.z = root_bb.p1.z > b.p1.z ? root_bb.p1.z : b.p1.z;
                info[mi].push_back({b, {(b.p0.x + b.p1.x) * .5f, (b.p0.y + b.p1.y) * .5f, (b.p0.z + b.p1.z) * .5f}});
                master.emplace_back(mi, f);
            }
        }
        tree.clear();
        tree.emplace_back();
        tree[0].bb = root_bb;
        tree[0].indices = master;
        size_t head = 0;  // FIFO over tree indices == BFS queue
        while (head < tree.size()) {
            const int ni = (int)head++;
            const std::vector<std::pair<uint32_t, uint32_t>> idx = tree[ni].indices;
            if (idx.size() == 1) continue;
            const float sa = surface_area(tree[ni].bb);
            if (sa == 0.f) continue;
            const float inv_sa = 1.f / sa;
            float cmin[3] = {kInf, kInf, kInf}, cmax[3] = {-kInf, -kInf, -kInf};
            for (const auto& p : idx) {
                const V3& c = info[p.first][p.second].c;
                for (int a = 0; a < 3; ++a) {
                    const float ca = comp(c, a);
                    cmin[a] = cmin[a] < ca ? cmin[a] : ca;
                    cmax[a] = cmax[a] > ca ? cmax[a] : ca;
                }
            }
            const float ext[3] = {cmax[0] - cmin[0], cmax[1] - cmin[1], cmax[2] - cmin[2]};
            if (ext[0] == ext[1] && ext[1] == ext[2] && ext[2] == 0.f) continue;
            int axis;
            if (ext[0] >= ext[1] && ext[0] >= ext[2]) axis = 0;
            else if (ext[1] >= ext[0] && ext[1] >= ext[2]) axis = 1;
            else axis = 2;
            const float width = ext[axis] / (float)12;
            std::vector<std::pair<uint32_t, uint32_t>> bucket[12];
            for (const auto& p : idx) {
                const float ca = comp(info[p.first][p.second].c, axis);
                const float raw = (ca - cmin[axis]) / (float)width;
                unsigned b = (unsigned)raw;
                if (b == 12) b--;
                bucket[b].push_back(p);
            }
            // forward scan (low side), bvh.cpp:251-287
            float fwd[12];
            Box lowbb[12];
            Box run = info[bucket[0][0].first][bucket[0][0].second].bb;
            float cnt = 0.f;
            for (int b = 0; b < 12; ++b) {
                for (const auto& p : bucket[b]) union_in_place(run, info[p.first][p.second].bb);
                lowbb[b] = run;
                cnt += bucket[b].size();
                const float cost = surface_area(run) * inv_sa * cnt * 1.f;
                fwd[b] = cost == 0 ? kInf : cost;
            }
            // backward scan (high side), bvh.cpp:289-317; bwd[k] covers buckets 11-k .. 11
            float bwd[12];
            Box highbb[12];
            run = info[bucket[11][0].first][bucket[11][0].second].bb;
            cnt = 0.f;
            for (int b = 11; b >= 0; --b) {
                for (const auto& p : bucket[b]) union_in_place(run, info[p.first][p.second].bb);
                highbb[b] = run;
                cnt += bucket[b].size();
                const float cost = surface_area(run) * inv_sa * cnt * 1.f;
                bwd[11 - b] = cost == 0 ? kInf : cost;
            }
            float total[11];
            for (int i = 0; i < 11; ++i) total[i] = 1.f + fwd[i] + bwd[11 - i - 1];
            const float leaf_cost = tree[ni].indices.size() * 1.f;
            bool make_leaf = true;
            for (int i = 0; i < 11; ++i) if (leaf_cost > total[i]) make_leaf = false;
            if (make_leaf && tree[ni].indices.size() <= 4) continue;
            int best = 0;
            float best_cost = kFloatMax;
            for (int i = 0; i < 11; ++i) if (total[i] < best_cost) { best_cost = total[i]; best = i; }
            std::vector<std::pair<uint32_t, uint32_t>> lo, hi;
            for (int b = 0; b <= best; ++b) lo.insert(lo.end(), bucket[b].begin(), bucket[b].end());
            for (int b = best + 1; b < 12; ++b) hi.insert(hi.end(), bucket[b].begin(), bucket[b].end());
            tree[ni].axis = (uint16_t)axis;
            if (lo.size() == tree[ni].indices.size() || hi.size() == tree[ni].indices.size()) continue;
            // high child is queued first, then low (bvh.cpp:371-389)
            const int h = (int)tree.size();
            tree.emplace_back();
            tree[h].indices = std::move(hi);
            tree[h].bb = highbb[best + 1];
            const int l = (int)tree.size();
            tree.emplace_back();
            tree[l].indices = std::move(lo);
            tree[l].bb = lowbb[best];
            tree[ni].high = h;
            tree[ni].low = l;
            tree[ni].indices.clear();
        }
    }

    // bvh::compact_helper, bvh.cpp:652-693 (recursion replaced by an explicit stack; same
    // pre-order, same offsets).
    void compact() {
        nodes.assign(tree.size(), ONode{});
        leaf.clear();
        leaf.reserve(num_prims);
        // returns number of descendants; iterative post-order to fill high_child_offset
        struct Item { int tn; uint32_t index; int stage; uint32_t low_count; };
        std::vector<Item> st;
        std::vector<uint32_t> ret;  // descendant counts returned by finished children
        st.push_back({0, 0, 0, 0});
        uint32_t last_ret = 0;
        while (!st.empty()) {
            Item& it = st.back();
            TreeNode& tn = tree[it.tn];
            ONode& cn = nodes[it.index];
            if (it.stage == 0) {
                for (int k = 0; k < 3; ++k) { cn.bb[k] = comp(tn.bb.p0, k); cn.bb[3 + k] = comp(tn.bb.p1, k); }
                cn.axis = tn.axis;
                if (tn.low < 0) {
                    cn.offset = (uint32_t)leaf.size();
                    // bvh.cpp:666-671: the reference comparator (kept as is, including its
                    // lhs.first < lhs.second branch) decides the in-leaf order through std::sort.
                    // It is not a strict weak order across meshes; std::sort stays in bounds with
                    // it only on 16 elements or fewer (insertion sort), so a longer leaf mixing
                    // meshes -- undefined in the reference -- is sorted by (mesh, face), the
                    // library's defined choice.
                    bool mixed = false;
                    for (const auto& p : tn.indices) mixed = mixed || p.first != tn.indices[0].first;
                    if (tn.indices.size() > 16 && mixed) {
                        std::sort(tn.indices.begin(), tn.indices.end());
                    } else {
                        std::sort(tn.indices.begin(), tn.indices.end(),
                                  [](const std::pair<uint32_t, uint32_t>& l, const std::pair<uint32_t, uint32_t>& r) {
                                      if (l.first == r.first) return l.second < r.second;
                                      return l.first < l.second;
                                  });
                    }
                    for (const auto& p : tn.indices) leaf.push_back(p);
                    cn.num_faces = (uint16_t)tn.indices.size();
                    last_ret = 0;
                    st.pop_back();
                    continue;
                }
                it.stage = 1;
                const uint32_t idx = it.index;
                st.push_back({tn.low, idx + 1, 0, 0});
                continue;
            }
            if (it.stage == 1) {
                it.low_count = 1u + last_ret;
                cn.offset = it.low_count + 1;
                cn.num_faces = 0;
                it.stage = 2;
                const uint32_t idx = it.index + 1 + it.low_count;
                const int h = tn.high;
                st.push_back({h, idx, 0, 0});
                continue;
            }
            last_ret = it.low_count + 1u + last_ret;
            st.pop_back();
        }
        leaf_prim.resize(leaf.size());
        for (size_t i = 0; i < leaf.size(); ++i) leaf_prim[i] = meshes[leaf[i].first].prim_base + leaf[i].second;
    }

    // bvh::intersect_compact, bvh.cpp:476-523 (+ Mesh::intersect commit, mesh.cpp:331-340).
    // Any-hit = the same traversal stopped at the first accepted face.
    struct HitRec { uint32_t prim; float t, u, v, w; uint32_t nodes, tris; };
    HitRec trace(const V3& o, const V3& d, float tmax, bool any) const {
        HitRec h{0xFFFFFFFFu, tmax, 0.f, 0.f, 0.f, 0, 0};
        const V3 inv = {1.f / d.x, 1.f / d.y, 1.f / d.z};
        const bool neg[3] = {inv.x < 0, inv.y < 0, inv.z < 0};
        std::vector<uint32_t> st;
        st.reserve(64);
        st.push_back(0);
        float min_t = tmax;
        while (!st.empty()) {
            const uint32_t ni = st.back();
            st.pop_back();
            const ONode& n = nodes[ni];
            h.nodes++;
            if (!bbox_hits(n.bb, o, inv, min_t)) continue;
            if (n.num_faces > 0) {
                for (uint32_t i = 0; i < n.num_faces; ++i) {
                    const uint32_t p = leaf_prim[n.offset + i];
                    WaldCommit c;
                    h.tris++;
                    if (wald_test(world[p], o, d, min_t, c)) {
                        min_t = c.t;
                        h.prim = p; h.t = c.t; h.u = c.u; h.v = c.v; h.w = c.w;
                        if (any) return h;
                    }
                }
                continue;
            }
            if (neg[n.axis]) { st.push_back(ni + 1); st.push_back(ni + n.offset); }
            else { st.push_back(ni + n.offset); st.push_back(ni + 1); }
        }
        return h;
    }

    // Mesh::intersect post-hit work, mesh.cpp:325-340 (error, Location) and 366-460 (frame),
    // computed once with the mesh that owns the committed face.
    Frame hit_frame(const HitRec& h, const V3& d) const {
        const Tri& t = world[h.prim];
        const OMesh& m = meshes[prim_mesh[h.prim]];
        const float u = h.u, v = h.v, w = h.w;
        const V3 err = scale({std::fabs(u * t.v0.x) + std::fabs(v * t.v1.x) + std::fabs(w * t.v2.x),
                              std::fabs(u * t.v0.y) + std::fabs(v * t.v1.y) + std::fabs(w * t.v2.y),
                              std::fabs(u * t.v0.z) + std::fabs(v * t.v1.z) + std::fabs(w * t.v2.z)}, kGamma7);
        const V3 loc = {std::fma(t.v0.x, u, sum_prod(t.v1.x, v, t.v2.x, w)),
                        std::fma(t.v0.y, u, sum_prod(t.v1.y, v, t.v2.y, w)),
                        std::fma(t.v0.z, u, sum_prod(t.v1.z, v, t.v2.z, w))};
        const V3 e0 = sub(t.v1, t.v0), e1 = sub(t.v2, t.v1), e2 = sub(t.v0, t.v2);
        V3 n;
        if (!m.nx.empty()) {
            const uint32_t f = h.prim - m.prim_base;
            const uint32_t id[3] = {m.fv0[f], m.fv1[f], m.fv2[f]};
            float vn[3][3];
            for (int k = 0; k < 3; ++k) {
                vn[k][0] = m.nx[id[k]]; vn[k][1] = m.ny[id[k]]; vn[k][2] = m.nz[id[k]];
                orc_apply_normal(m.inv, vn[k]);
            }
            n = {vn[0][0] * u + vn[1][0] * v + vn[2][0] * w,
                 vn[0][1] * u + vn[1][1] * v + vn[2][1] * w,
                 vn[0][2] * u + vn[1][2] * v + vn[2][2] * w};
        } else {
            n = cross(e0, e1);
        }
        const float rdn = dot(d, n);
        const float flip = rdn > 0 ? -1 : 1;
        n = scale(n, flip);
        n = normalize(n);
        const V3 an = {std::fabs(n.x), std::fabs(n.y), std::fabs(n.z)};
        const float dd = dot(err, an);
        V3 off = scale(n, dd);
        if (dot(d, n) > 0) off = {-off.x, -off.y, -off.z};
        V3 np = add(loc, off);
        float* npc[3] = {&np.x, &np.y, &np.z};
        const float oc[3] = {off.x, off.y, off.z};
        for (int i = 0; i < 3; ++i) {
            if (oc[i] > 0) *npc[i] = std::nextafter(*npc[i], kInf);
            else if (oc[i] < 0) *npc[i] = std::nextafter(*npc[i], -kInf);
        }
        const float d0 = std::fabs(dot(e0, e1)), d1 = std::fabs(dot(e1, e2)), d2 = std::fabs(dot(e2, e0));
        V3 t1;
        if (d0 > d1 && d0 > d2) t1 = e0;
        else if (d1 > d0 && d1 > d2) t1 = e1;
        else t1 = e2;
        V3 t2 = cross(t1, n);
        t1 = normalize(t1);
        t2 = normalize(t2);
        return {np, n, t1, t2};
    }

    // Area-light table for the NEE patch: every face of an emitting mesh, world-space area
    // 0.5*|e0 x e1|, CDF in mesh/face order.
    void build_lights() {
        light_prims.clear(); light_cdf.clear(); light_area = 0;
        for (uint32_t p = 0; p < num_prims; ++p) {
            if (!meshes[prim_mesh[p]].is_light) continue;
            const Tri& t = world[p];
            const V3 c = cross(sub(t.v1, t.v0), sub(t.v2, t.v0));
            const float area = 0.5f * std::sqrt(c.x * c.x + c.y * c.y + c.z * c.z);
            light_area = light_area + area;
            light_prims.push_back(p);
            light_cdf.push_back(light_area);
        }
    }

    // PathTraceIntegrator::GetSample (PathTraceIntegrator.cpp:10-135), patched:
    //  P1 counter RNG (pixel, sample, bounce); P2 frame from the hit mesh, once per hit;
    //  P3 optional area-light NEE (Lambert vertices only; BSDF-sampled emitter hits after a
    //     Lambert bounce are then not counted); radiance is accumulated and returned at every
    //     termination.  Without NEE the result equals the reference's.
    V3 path_sample(V3 o, V3 d, uint32_t pixel, uint32_t sample, const RenderDesc& rd,
                   uint32_t* primary) const {
        V3 src = {1.f, 1.f, 1.f};
        V3 L = {0.f, 0.f, 0.f};
        uint32_t bounces = 0;
        bool last_lambert = false;
        const bool nee = (rd.flags & 1u) && !light_prims.empty();
        const uint32_t k0 = (uint32_t)rd.seed, k1 = (uint32_t)(rd.seed >> 32);
        while (true) {
            if (src.x < 0.0039f && src.y < 0.0039f && src.z < 0.0039f) return L;
            const HitRec h = trace(o, d, kInf, false);
            if (bounces == 0 && primary) *primary = h.prim;
            if (h.prim == 0xFFFFFFFFu) {
                if (has_env) L = add(L, {env[0] * src.x, env[1] * src.y, env[2] * src.z});
                return L;
            }
            const OMesh& m = meshes[prim_mesh[h.prim]];
            if (m.is_light) {
                if (!(nee && last_lambert))
                    L = add(L, {m.emission[0] * src.x, m.emission[1] * src.y, m.emission[2] * src.z});
                return L;
            }
            if (bounces >= rd.max_depth) return L;
            const uint32_t bounce = bounces;
            bounces++;
            const Frame fr = hit_frame(h, d);
            uint32_t r[4] = {pixel, sample, bounce, 0u};
            philox(r, k0, k1);
            // Intersection::WorldToLocal (Intersection.cpp:10-14)
            const V3 li = normalize({dot(d, fr.t1), dot(d, fr.n), dot(d, fr.t2)});
            V3 lo;
            if (m.material == 2u) {  // MirrorBRDF::sample, mirror_brdf.h:23-35
                lo = {li.x, -li.y, li.z};
            } else {                 // LambertBRDF::sample -> CosineSampleHemisphere
                const float u0 = u01(r[0]), u1 = u01(r[1]);
                const float rr = std::sqrt(u0);
                float s, c;
                sincos_2pi(u1, s, c);
                const float one_minus = 1.0f - u0;
                lo = {rr * c, std::sqrt(0.0f < one_minus ? one_minus : 0.0f), rr * s};
                if (nee) {
                    uint32_t r2[4] = {pixel, sample, bounce, 1u};
                    philox(r2, k0, k1);
                    // light pick: first entry whose CDF exceeds u*total
                    const float target = u01(r[2]) * light_area;
                    size_t lo_i = 0, hi_i = light_cdf.size() - 1;
                    while (lo_i < hi_i) {
                        const size_t mid = (lo_i + hi_i) / 2;
                        if (target < light_cdf[mid]) hi_i = mid; else lo_i = mid + 1;
                    }
                    const Tri& lt = world[light_prims[lo_i]];
                    const OMesh& lm = meshes[prim_mesh[light_prims[lo_i]]];
                    const float su = std::sqrt(u01(r[3]));
                    const float b0 = 1.0f - su;
                    const float b1 = u01(r2[0]) * su;
                    const float b2 = (1.0f - b0) - b1;
                    const V3 y = {b0 * lt.v0.x + b1 * lt.v1.x + b2 * lt.v2.x,
                                  b0 * lt.v0.y + b1 * lt.v1.y + b2 * lt.v2.y,
                                  b0 * lt.v0.z + b1 * lt.v1.z + b2 * lt.v2.z};
                    const V3 dv = sub(y, fr.loc);
                    const float dist2 = dot(dv, dv);
                    const float dist = std::sqrt(dist2);
                    const V3 wi = scale(dv, 1.0f / dist);
                    const float cos_x = dot(wi, fr.n);
                    const V3 ln = normalize(cross(sub(lt.v1, lt.v0), sub(lt.v2, lt.v0)));
                    const float cos_l = std::fabs(dot(wi, ln));
                    if (cos_x > 0.f && cos_l > 0.f && dist2 > 0.f) {
                        const HitRec sh = trace(fr.loc, wi, dist * 0.999f, true);
                        if (sh.prim == 0xFFFFFFFFu) {
                            const float g = (cos_x * cos_l) / dist2;
                            const float wgt = g * light_area * kOneOverPi;
                            L = add(L, {src.x * m.albedo[0] * lm.emission[0] * wgt,
                                        src.y * m.albedo[1] * lm.emission[1] * wgt,
                                        src.z * m.albedo[2] * lm.emission[2] * wgt});
                        }
                    }
                }
            }
            // Intersection::LocalToWorld (Intersection.cpp:16-23)
            const V3 wo = normalize({fr.t1.x * lo.x + fr.n.x * lo.y + fr.t2.x * lo.z,
                                     fr.t1.y * lo.x + fr.n.y * lo.y + fr.t2.y * lo.z,
                                     fr.t1.z * lo.x + fr.n.z * lo.y + fr.t2.z * lo.z});
            o = fr.loc;
            d = wo;
            src = {src.x * m.albedo[0], src.y * m.albedo[1], src.z * m.albedo[2]};
            last_lambert = (m.material != 2u);
        }
    }
};

// Transform::LookAt(eye, lookAt, up, right_handed=false) (Transform.cpp:322-365) applied to an
// identity Transform with operator*= (Matrix4x4.cpp:244-303), as pbrt_parser.cpp:1099-1119 does;
// then the PerspectiveCamera constants (PerspectiveCamera.cpp:17-25).
Camera make_camera(const float* eye, const float* look, const float* up_in, float fov, uint32_t w, uint32_t h) {
    float m[16];
    m[3] = eye[0]; m[7] = eye[1]; m[11] = eye[2]; m[15] = 1;
    V3 dir = normalize(sub({look[0], look[1], look[2]}, {eye[0], eye[1], eye[2]}));
    V3 up = normalize({up_in[0], up_in[1], up_in[2]});
    V3 left = cross(up, dir);
    Camera c{};
    const float llen = std::sqrt(left.x * left.x + left.y * left.y + left.z * left.z);
    if (llen == 0) {
        for (int i = 0; i < 16; ++i) m[i] = (i % 5 == 0) ? 1.f : 0.f;
    } else {
        left = normalize(left);
        const V3 nup = cross(dir, left);
        m[0] = left.x; m[4] = left.y; m[8] = left.z; m[12] = 0;
        m[1] = nup.x; m[5] = nup.y; m[9] = nup.z; m[13] = 0;
        m[2] = dir.x; m[6] = dir.y; m[10] = dir.z; m[14] = 0;
    }
    // identity *= m  (row r of identity dotted with column c of m, left to right)
    float id[16];
    for (int i = 0; i < 16; ++i) id[i] = (i % 5 == 0) ? 1.f : 0.f;
    for (int r = 0; r < 4; ++r)
        for (int cc = 0; cc < 4; ++cc)
            c.m[r * 4 + cc] = id[r * 4 + 0] * m[0 * 4 + cc] + id[r * 4 + 1] * m[1 * 4 + cc] +
                              id[r * 4 + 2] * m[2 * 4 + cc] + id[r * 4 + 3] * m[3 * 4 + cc];
    c.one_over_w = 1.0f / (float)w;
    c.one_over_h = 1.0f / (float)h;
    c.aspect = (float)w * c.one_over_h;
    constexpr float pi_over_180 = 3.14159265358979323846 / 180.0f;
    c.tan_half = (float)std::tan(fov * pi_over_180 * .5f);
    return c;
}

// PerspectiveCamera::get_ray_for_pixel (PerspectiveCamera.cpp:27-49) with LeftHanded = true,
// Transform::Apply(Ray) (Transform.cpp:93-133,163-175).
void camera_ray(const Camera& c, float px, float py, V3& o, V3& d) {
    const float ndc_x = px * c.one_over_w;
    const float ndc_y = py * c.one_over_h;
    const float cx = (2 * ndc_x - 1) * c.aspect * c.tan_half;
    const float cy = (1 - 2 * ndc_y) * c.tan_half;
    V3 dir = normalize({cx, cy, 1.f});
    const float* m = c.m;
    o = {0.f * m[0] + 0.f * m[1] + 0.f * m[2] + m[3], 0.f * m[4] + 0.f * m[5] + 0.f * m[6] + m[7],
         0.f * m[8] + 0.f * m[9] + 0.f * m[10] + m[11]};
    const float ow = 0.f * m[12] + 0.f * m[13] + 0.f * m[14] + m[15];
    if (ow != 1) {
        const float div = 1.f / ow;
        o = scale(o, div);
    }
    V3 wd = {dir.x * m[0] + dir.y * m[1] + dir.z * m[2], dir.x * m[4] + dir.y * m[5] + dir.z * m[6],
             dir.x * m[8] + dir.y * m[9] + dir.z * m[10]};
    d = normalize(wd);
}

template <class F>
void parallel_for(uint64_t n, int threads, F f) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    if (n < 4096 || threads == 1) { f(0, n); return; }
    std::vector<std::thread> ts;
    const uint64_t chunk = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        const uint64_t b = t * chunk, e = std::min<uint64_t>(n, b + chunk);
        if (b >= e) break;
        ts.emplace_back([=]() { f(b, e); });
    }
    for (auto& t : ts) t.join();
}

}  // namespace

// ------------------------------------------------------------------------------------------------
// C interface used by tests/ (ctypes) and by bench.py's CPU-baseline leg.

extern "C" {

typedef struct orc_mesh {
    const float *x, *y, *z;
    uint32_t num_vertices;
    const uint32_t *fv0, *fv1, *fv2;
    uint32_t num_faces;
    const float *nx, *ny, *nz;
    float object_to_world[16];
    float world_to_object[16];
    uint32_t material;
    float albedo[3];
    int32_t is_light;
    float emission[3];
} orc_mesh;

typedef struct orc_ray { float org[3]; float tmax; float dir[3]; uint32_t flags; } orc_ray;
typedef struct orc_hit { uint32_t prim; float t; float u; float v; } orc_hit;

void* orc_scene_create(const orc_mesh* ms, uint32_t n, int has_env, const float* env) {
    Oracle* o = new Oracle();
    o->meshes.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        OMesh& m = o->meshes[i];
        const orc_mesh& s = ms[i];
        m.x.assign(s.x, s.x + s.num_vertices);
        m.y.assign(s.y, s.y + s.num_vertices);
        m.z.assign(s.z, s.z + s.num_vertices);
        m.fv0.assign(s.fv0, s.fv0 + s.num_faces);
        m.fv1.assign(s.fv1, s.fv1 + s.num_faces);
        m.fv2.assign(s.fv2, s.fv2 + s.num_faces);
        if (s.nx) {
            m.nx.assign(s.nx, s.nx + s.num_vertices);
            m.ny.assign(s.ny, s.ny + s.num_vertices);
            m.nz.assign(s.nz, s.nz + s.num_vertices);
        }
        std::memcpy(m.m, s.object_to_world, sizeof(m.m));
        std::memcpy(m.inv, s.world_to_object, sizeof(m.inv));
        m.material = s.material;
        std::memcpy(m.albedo, s.albedo, sizeof(m.albedo));
        m.is_light = s.is_light;
        std::memcpy(m.emission, s.emission, sizeof(m.emission));
    }
    o->has_env = has_env != 0;
    if (env) std::memcpy(o->env, env, sizeof(o->env));
    o->bake();
    o->build();
    o->compact();
    o->build_lights();
    return o;
}

void orc_scene_destroy(void* s) { delete static_cast<Oracle*>(s); }

uint32_t orc_num_nodes(void* s) { return (uint32_t)static_cast<Oracle*>(s)->nodes.size(); }
uint32_t orc_num_prims(void* s) { return static_cast<Oracle*>(s)->num_prims; }

void orc_get_tree(void* s, void* nodes_out, uint32_t* pairs_out) {
    Oracle* o = static_cast<Oracle*>(s);
    std::memcpy(nodes_out, o->nodes.data(), o->nodes.size() * sizeof(ONode));
    for (size_t i = 0; i < o->leaf.size(); ++i) {
        pairs_out[2 * i] = o->leaf[i].first;
        pairs_out[2 * i + 1] = o->leaf[i].second;
    }
}

// World-space triangles (9 floats per global prim id).
void orc_get_world(void* s, float* out) {
    Oracle* o = static_cast<Oracle*>(s);
    std::memcpy(out, o->world.data(), o->world.size() * sizeof(Tri));
}

void orc_trace(void* s, const orc_ray* rays, uint64_t n, orc_hit* hits, uint32_t* node_tests,
               uint32_t* tri_tests, int threads) {
    const Oracle* o = static_cast<Oracle*>(s);
    parallel_for(n, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; ++i) {
            const orc_ray& r = rays[i];
            const Oracle::HitRec h = o->trace({r.org[0], r.org[1], r.org[2]}, {r.dir[0], r.dir[1], r.dir[2]},
                                              r.tmax, (r.flags & 1u) != 0);
            hits[i] = {h.prim, h.t, h.u, h.v};
            if (node_tests) node_tests[i] = h.nodes;
            if (tri_tests) tri_tests[i] = h.tris;
        }
    });
}

// Post-hit frame for closest hits (loc, n, t1, t2: 12 floats per ray; zeros on a miss).
void orc_hit_frames(void* s, const orc_ray* rays, uint64_t n, float* out) {
    const Oracle* o = static_cast<Oracle*>(s);
    for (uint64_t i = 0; i < n; ++i) {
        const orc_ray& r = rays[i];
        const V3 d = {r.dir[0], r.dir[1], r.dir[2]};
        const Oracle::HitRec h = o->trace({r.org[0], r.org[1], r.org[2]}, d, r.tmax, false);
        float* f = out + 12 * i;
        if (h.prim == 0xFFFFFFFFu) { std::memset(f, 0, 12 * sizeof(float)); continue; }
        const Frame fr = o->hit_frame(h, d);
        const float v[12] = {fr.loc.x, fr.loc.y, fr.loc.z, fr.n.x, fr.n.y, fr.n.z,
                             fr.t1.x, fr.t1.y, fr.t1.z, fr.t2.x, fr.t2.y, fr.t2.z};
        std::memcpy(f, v, sizeof(v));
    }
}

// Camera rays for pixel centres (CenterSampler: x+0.5, y+0.5), row-major.
void orc_camera_rays(const float* eye, const float* look, const float* up, float fov, uint32_t w, uint32_t h,
                     orc_ray* out) {
    const Camera c = make_camera(eye, look, up, fov, w, h);
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) {
            V3 o, d;
            camera_ray(c, x + 0.5f, y + 0.5f, o, d);
            out[y * w + x] = {{o.x, o.y, o.z}, kInf, {d.x, d.y, d.z}, 0u};
        }
}

typedef struct orc_render_desc {
    uint32_t width, height, spp, max_depth;
    uint64_t seed;
    uint32_t flags;  // 1 = NEE, 2 = jittered samples
    float eye[3], look_at[3], up[3], fov;
} orc_render_desc;

// The patched render call: for each pixel, samples in order, film = sum of per-sample clamped
// radiance times 1/spp (BoxFilter.cpp:14-71).  Rows [row_begin, row_end) only (bounded CPU
// baseline samples); rgb/prim are full-frame arrays.
void orc_render_rows(void* s, const orc_render_desc* rd, uint32_t row_begin, uint32_t row_end, float* rgb,
                     uint32_t* prim, int threads) {
    const Oracle* o = static_cast<Oracle*>(s);
    const Camera cam = make_camera(rd->eye, rd->look_at, rd->up, rd->fov, rd->width, rd->height);
    const RenderDesc d{rd->width, rd->height, rd->spp, rd->max_depth, rd->seed, rd->flags};
    const uint32_t k0 = (uint32_t)rd->seed, k1 = (uint32_t)(rd->seed >> 32);
    const uint64_t first = (uint64_t)row_begin * rd->width;
    const uint64_t count = (uint64_t)(row_end - row_begin) * rd->width;
    parallel_for(count, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; ++i) {
            const uint32_t pix = (uint32_t)(first + i);
            const uint32_t x = pix % rd->width, y = pix / rd->width;
            V3 sum = {0.f, 0.f, 0.f};
            for (uint32_t smp = 0; smp < rd->spp; ++smp) {
                float px = x + 0.5f, py = y + 0.5f;
                if (rd->flags & 2u) {
                    uint32_t r[4] = {pix, smp, 0xFFFFu, 0u};
                    philox(r, k0, k1);
                    px = (float)x + u01(r[0]);
                    py = (float)y + u01(r[1]);
                }
                V3 ro, rdir;
                camera_ray(cam, px, py, ro, rdir);
                uint32_t p0 = 0xFFFFFFFFu;
                V3 L = o->path_sample(ro, rdir, pix, smp, d, smp == 0 ? &p0 : nullptr);
                if (smp == 0 && prim) prim[pix] = p0;
                if (L.x > 255) L.x = 255;
                if (L.y > 255) L.y = 255;
                if (L.z > 255) L.z = 255;
                sum = add(sum, L);
            }
            const float div = 1.0f / rd->spp;
            rgb[3 * pix + 0] = sum.x * div;
            rgb[3 * pix + 1] = sum.y * div;
            rgb[3 * pix + 2] = sum.z * div;
        }
    });
}


// Compaction of a hand-made tree shape (tests/test_bvh.cpp compact*): low[i], high[i] child
// indices (-1 for a leaf), node 0 the root.  Writes the compacted offset of each node in DFS
// order (high_child_offset for interior nodes).
void orc_compact_shape(const int* low, const int* high, uint32_t n, uint32_t* offsets_out) {
    Oracle o;
    o.tree.assign(n, TreeNode{});
    for (uint32_t i = 0; i < n; ++i) {
        o.tree[i].low = low[i];
        o.tree[i].high = high[i];
        o.tree[i].bb.p1.x = (float)i;  // tag: the tests identify nodes by bb.p1.x
    }
    o.num_prims = 0;
    o.compact();
    for (uint32_t i = 0; i < n; ++i) offsets_out[2 * i] = (uint32_t)o.nodes[i].bb[3], offsets_out[2 * i + 1] = o.nodes[i].offset;
}

// Intersection::WorldToLocal / LocalToWorld (Intersection.cpp:10-23); MirrorBRDF::sample
// (mirror_brdf.h:23-35).
void orc_world_to_local(const float* t1, const float* n, const float* t2, const float* w, float* out) {
    const V3 W = {w[0], w[1], w[2]};
    const V3 l = normalize({dot(W, {t1[0], t1[1], t1[2]}), dot(W, {n[0], n[1], n[2]}), dot(W, {t2[0], t2[1], t2[2]})});
    out[0] = l.x; out[1] = l.y; out[2] = l.z;
}
void orc_mirror_sample(const float* in, float* out) { out[0] = in[0]; out[1] = -in[1]; out[2] = in[2]; }
void orc_normalize(float* v) {
    const V3 r = normalize({v[0], v[1], v[2]});
    v[0] = r.x; v[1] = r.y; v[2] = r.z;
}

// Exposed pieces for unit tests.
float orc_f64_diff(float a, float b, float c, float d) { return f64_diff(a, b, c, d); }
void orc_sincos_2pi(float u, float* s, float* c) { sincos_2pi(u, *s, *c); }
void orc_philox(uint32_t* ctr, uint64_t seed) { philox(ctr, (uint32_t)seed, (uint32_t)(seed >> 32)); }
int orc_bbox_hits(const float* bb, const float* o, const float* d, float min_t) {
    const V3 inv = {1.f / d[0], 1.f / d[1], 1.f / d[2]};
    return bbox_hits(bb, {o[0], o[1], o[2]}, inv, min_t) ? 1 : 0;
}
// Single-face Wald test with the committed values, for fixtures (returns 1 on accept).
int orc_wald(const float* tri9, const float* o, const float* d, float min_t, float* tuvw) {
    Tri t{{tri9[0], tri9[1], tri9[2]}, {tri9[3], tri9[4], tri9[5]}, {tri9[6], tri9[7], tri9[8]}};
    WaldCommit c;
    if (!wald_test(t, {o[0], o[1], o[2]}, {d[0], d[1], d[2]}, min_t, c)) return 0;
    tuvw[0] = c.t; tuvw[1] = c.u; tuvw[2] = c.v; tuvw[3] = c.w;
    return 1;
}
// PNGFilm::Output (src/cpu/films/PNGFilm.cpp:27-44): RGBA8, each channel
// static_cast<unsigned char>(v > 255 ? 255 : v), alpha 255, index 4 * (y * width + x).
void orc_film_to_rgba8(const float* rgb, uint32_t npix, uint8_t* out) {
    for (uint32_t i = 0; i < npix; ++i) {
        const float r = rgb[3 * (size_t)i], g = rgb[3 * (size_t)i + 1], b = rgb[3 * (size_t)i + 2];
        out[4 * (size_t)i + 0] = static_cast<unsigned char>(r > 255 ? 255 : r);
        out[4 * (size_t)i + 1] = static_cast<unsigned char>(g > 255 ? 255 : g);
        out[4 * (size_t)i + 2] = static_cast<unsigned char>(b > 255 ? 255 : b);
        out[4 * (size_t)i + 3] = static_cast<unsigned char>(255);
    }
}
float orc_gamma(int n) {
    switch (n) { case 2: return kGamma2; case 3: return kGamma3; case 5: return kGamma5; case 7: return kGamma7; default: return kGammaMul; }
}

}  // extern "C"
