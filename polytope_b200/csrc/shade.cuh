// shade.cuh -- device shading for the path tracer: camera rays, the post-hit frame, BSDF
// sampling and area-light next-event estimation.
//
// Reference (paths relative to the Polytope source tree):
//   PerspectiveCamera::get_ray_for_pixel      src/cpu/cameras/PerspectiveCamera.cpp:27-49
//   Mesh::intersect post-hit frame            src/cpu/shapes/mesh.cpp:325-340, 366-460
//   Intersection::WorldToLocal/LocalToWorld   src/cpu/structures/Intersection.cpp:10-23
//   LambertBRDF / CosineSampleHemisphere      src/cpu/shading/brdf/lambert_brdf.h:48-57, constants.h:106-115
//   MirrorBRDF::sample                        src/cpu/shading/brdf/mirror_brdf.h:23-35
//   PathTraceIntegrator::GetSample            src/cpu/integrators/PathTraceIntegrator.cpp:10-135
// with the render-loop definitions the CPU oracle shares: Philox4x32-10 keyed (pixel, sample,
// bounce, block) for every random number, sin/cos(2 pi u) from exact_math.h, the frame computed
// once from the mesh owning the hit face, and optional area-light NEE.  Every float operation is
// the oracle's, in its order, so images agree bit for bit.
#pragma once

#include "render.h"
#include "traverse.cuh"

namespace pt {

struct F3 { float x, y, z; };

PT_HD F3 f3(float x, float y, float z) { return {x, y, z}; }
PT_HD F3 vsub(F3 a, F3 b) { return {fsub(a.x, b.x), fsub(a.y, b.y), fsub(a.z, b.z)}; }
PT_HD F3 vadd(F3 a, F3 b) { return {fadd(a.x, b.x), fadd(a.y, b.y), fadd(a.z, b.z)}; }
PT_HD F3 vscale(F3 a, float t) { return {fmul(a.x, t), fmul(a.y, t), fmul(a.z, t)}; }
// Vector::Dot: arg.x*self.x + arg.y*self.y + arg.z*self.z (summed left to right)
PT_HD float vdot(F3 s, F3 a) { return fadd(fadd(fmul(a.x, s.x), fmul(a.y, s.y)), fmul(a.z, s.z)); }
PT_HD F3 vcross(F3 s, F3 r) {
    return {fsub(fmul(s.y, r.z), fmul(s.z, r.y)), fsub(fmul(s.z, r.x), fmul(s.x, r.z)),
            fsub(fmul(s.x, r.y), fmul(s.y, r.x))};
}
PT_HD F3 vnorm(F3 v) {
    const float d = frcp(fsqrt(fadd(fadd(fmul(v.x, v.x), fmul(v.y, v.y)), fmul(v.z, v.z))));
    return {fmul(v.x, d), fmul(v.y, d), fmul(v.z, d)};
}

// Camera ray through film position (px, py), LeftHanded = true.
PT_HD void camera_ray(const CameraConst& c, float px, float py, F3& o, F3& d) {
    const float ndc_x = fmul(px, c.one_over_w);
    const float ndc_y = fmul(py, c.one_over_h);
    const float cx = fmul(fmul(fsub(fmul(2.0f, ndc_x), 1.0f), c.aspect), c.tan_half);
    const float cy = fmul(fsub(1.0f, fmul(2.0f, ndc_y)), c.tan_half);
    const F3 dir = vnorm(f3(cx, cy, 1.0f));
    const float* m = c.m;
    const F3 wd = {fadd(fadd(fmul(dir.x, m[0]), fmul(dir.y, m[1])), fmul(dir.z, m[2])),
                   fadd(fadd(fmul(dir.x, m[4]), fmul(dir.y, m[5])), fmul(dir.z, m[6])),
                   fadd(fadd(fmul(dir.x, m[8]), fmul(dir.y, m[9])), fmul(dir.z, m[10]))};
    o = f3(c.org[0], c.org[1], c.org[2]);
    d = vnorm(wd);
}

struct HitFrame {
    F3 loc;   // spawn point after the robust offset
    F3 n;     // geo_normal == bent_normal, facing the incoming ray
    F3 t1, t2;
    uint32_t mesh;
};

// Post-hit frame of the committed face (v0, v1, v2 world space).
PT_HD HitFrame hit_frame(F3 v0, F3 v1, F3 v2, float u, float v, float w, F3 d,
                                              const float* __restrict__ vnormals) {
    const float g7 = bitsf(PT_GAMMA7_BITS);
    const F3 err = vscale(f3(fadd(fadd(fabs_(fmul(u, v0.x)), fabs_(fmul(v, v1.x))), fabs_(fmul(w, v2.x))),
                             fadd(fadd(fabs_(fmul(u, v0.y)), fabs_(fmul(v, v1.y))), fabs_(fmul(w, v2.y))),
                             fadd(fadd(fabs_(fmul(u, v0.z)), fabs_(fmul(v, v1.z))), fabs_(fmul(w, v2.z)))),
                          g7);
    const F3 loc = {ffma(v0.x, u, sum_prod(v1.x, v, v2.x, w)), ffma(v0.y, u, sum_prod(v1.y, v, v2.y, w)),
                    ffma(v0.z, u, sum_prod(v1.z, v, v2.z, w))};
    const F3 e0 = vsub(v1, v0), e1 = vsub(v2, v1), e2 = vsub(v0, v2);
    F3 n;
    if (vnormals) {
        const float* q = vnormals;
        n = {fadd(fadd(fmul(q[0], u), fmul(q[3], v)), fmul(q[6], w)),
             fadd(fadd(fmul(q[1], u), fmul(q[4], v)), fmul(q[7], w)),
             fadd(fadd(fmul(q[2], u), fmul(q[5], v)), fmul(q[8], w))};
    } else {
        n = vcross(e0, e1);
    }
    const float rdn = vdot(d, n);
    const float flip = rdn > 0 ? -1.0f : 1.0f;
    n = vnorm(vscale(n, flip));
    const F3 an = {fabs_(n.x), fabs_(n.y), fabs_(n.z)};
    const float dd = vdot(err, an);
    F3 off = vscale(n, dd);
    if (vdot(d, n) > 0) off = {-off.x, -off.y, -off.z};
    F3 np = vadd(loc, off);
    if (off.x > 0) np.x = next_up(np.x); else if (off.x < 0) np.x = next_down(np.x);
    if (off.y > 0) np.y = next_up(np.y); else if (off.y < 0) np.y = next_down(np.y);
    if (off.z > 0) np.z = next_up(np.z); else if (off.z < 0) np.z = next_down(np.z);
    const float d0 = fabs_(vdot(e0, e1)), d1 = fabs_(vdot(e1, e2)), d2 = fabs_(vdot(e2, e0));
    F3 t1;
    if (d0 > d1 && d0 > d2) t1 = e0;
    else if (d1 > d0 && d1 > d2) t1 = e1;
    else t1 = e2;
    F3 t2 = vcross(t1, n);
    HitFrame f;
    f.loc = np;
    f.n = n;
    f.t1 = vnorm(t1);
    f.t2 = vnorm(t2);
    return f;
}

PT_HD void load_face(const float4* __restrict__ tris, uint32_t leaf, F3& v0, F3& v1, F3& v2,
                                          uint32_t& mesh) {
    const float4 q0 = ldg(tris + 3 * (size_t)leaf), q1 = ldg(tris + 3 * (size_t)leaf + 1),
                 q2 = ldg(tris + 3 * (size_t)leaf + 2);
    v0 = f3(q0.x, q0.y, q0.z);
    v1 = f3(q0.w, q1.x, q1.y);
    v2 = f3(q1.z, q1.w, q2.x);
    mesh = fbits(q2.z);
}

struct MeshRec {  // DeviceMesh, as the kernels read it
    uint32_t material;
    int32_t is_light;
    float albedo[3];
    float emission[3];
    int32_t has_normals;
};

// Area-light sample for NEE at a Lambert vertex: returns true with the (unoccluded) contribution
// weight components when the light point faces the vertex.
struct LightSample {
    F3 wi;
    float dist;
    F3 le;
    float wgt;
    bool valid;
};

PT_HD LightSample sample_light(const RenderParams& p, const HitFrame& f, float u_pick, float u_a,
                                                    float u_b) {
    LightSample ls;
    ls.valid = false;
    const float target = fmul(u_pick, p.light_area);
    uint32_t lo = 0, hi = p.num_lights - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2;
        if (target < ldg(p.light_cdf + mid)) hi = mid; else lo = mid + 1;
    }
    const float* L = p.light_tris + 12 * (size_t)lo;
    const F3 a = f3(ldg(L + 0), ldg(L + 1), ldg(L + 2));
    const F3 b = f3(ldg(L + 3), ldg(L + 4), ldg(L + 5));
    const F3 c = f3(ldg(L + 6), ldg(L + 7), ldg(L + 8));
    const uint32_t lmesh = fbits(ldg(L + 10));
    const float su = fsqrt(u_a);
    const float b0 = fsub(1.0f, su);
    const float b1 = fmul(u_b, su);
    const float b2 = fsub(fsub(1.0f, b0), b1);
    const F3 y = {fadd(fadd(fmul(b0, a.x), fmul(b1, b.x)), fmul(b2, c.x)),
                  fadd(fadd(fmul(b0, a.y), fmul(b1, b.y)), fmul(b2, c.y)),
                  fadd(fadd(fmul(b0, a.z), fmul(b1, b.z)), fmul(b2, c.z))};
    const F3 dv = vsub(y, f.loc);
    const float dist2 = vdot(dv, dv);
    const float dist = fsqrt(dist2);
    const F3 wi = vscale(dv, frcp(dist));
    const float cos_x = vdot(wi, f.n);
    const F3 ln = vnorm(vcross(vsub(b, a), vsub(c, a)));
    const float cos_l = fabs_(vdot(wi, ln));
    if (cos_x > 0.f && cos_l > 0.f && dist2 > 0.f) {
        const MeshRec* mr = (const MeshRec*)p.meshes + lmesh;
        const float g = fdiv(fmul(cos_x, cos_l), dist2);
        ls.wgt = fmul(fmul(g, p.light_area), frcp(3.14159265358979323846f));
        ls.le = f3(mr->emission[0], mr->emission[1], mr->emission[2]);
        ls.wi = wi;
        ls.dist = dist;
        ls.valid = true;
    }
    return ls;
}

}  // namespace pt
