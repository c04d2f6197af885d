// path.cuh -- one path of the patched PathTraceIntegrator::GetSample
// (src/cpu/integrators/PathTraceIntegrator.cpp:10-135) as host/device code: the per-hit shading
// step shared by the fused and the wavefront kernels, the camera ray of a path and the fused path
// loop.  The kernels in render.cu are the only callers in the library; the functions are also
// host-compilable so that an off-line harness can run the exact kernel arithmetic on a CPU.
#pragma once

#include "shade.cuh"
#include "two_level.cuh"

namespace pt {

struct PathState {
    F3 o, d;
    F3 src;        // throughput (ReflectanceSpectrum src)
    F3 L;          // accumulated radiance
    uint32_t bounces;
    uint32_t last_lambert;
};

struct ShadowReq {
    F3 o, wi;
    float tmax;
    F3 contrib;
    bool valid;
};

PT_HD bool throughput_is_zero(const F3& s) {  // ReflectanceSpectrum::is_zero
    return s.x < 0.0039f && s.y < 0.0039f && s.z < 0.0039f;
}

// One loop iteration of PathTraceIntegrator::GetSample after the intersection (lines 46-132 of
// PathTraceIntegrator.cpp, patched as described in shade.cuh), given the hit face's world vertices
// and mesh.  Returns true when the path goes on with the new ray in s.o / s.d; fills `sh` when a
// shadow ray must be traced.
PT_HD bool shade_face(const RenderParams& p, PathState& s, uint32_t prim, F3 v0, F3 v1, F3 v2, uint32_t mesh,
                      float u, float v, float w, uint32_t pixel, uint32_t sample, ShadowReq& sh) {
    const bool nee = (p.flags & PT_RENDER_NEE) && p.num_lights > 0;
    const MeshRec mr = ((const MeshRec*)p.meshes)[mesh];
    if (mr.is_light) {
        if (!(nee && s.last_lambert))
            s.L = vadd(s.L, f3(fmul(mr.emission[0], s.src.x), fmul(mr.emission[1], s.src.y), fmul(mr.emission[2], s.src.z)));
        return false;
    }
    if (s.bounces >= p.max_depth) return false;
    const uint32_t bounce = s.bounces++;
    // interpolated vertex normals only for meshes that have them (Mesh::intersect, mesh.cpp:385-410:
    // per mesh, so a scene can mix meshes with and without normals)
    const HitFrame fr = hit_frame(v0, v1, v2, u, v, w, s.d,
                                  (p.prim_normals && mr.has_normals) ? p.prim_normals + 9 * (size_t)prim : nullptr);
    uint32_t r[4] = {pixel, sample, bounce, 0u};
    philox4x32(r, p.seed_lo, p.seed_hi);
    const F3 d = s.d;
    const F3 li = vnorm(f3(vdot(d, fr.t1), vdot(d, fr.n), vdot(d, fr.t2)));
    F3 lo;
    const bool mirror = mr.material == PT_MAT_MIRROR;
    if (mirror) {
        lo = f3(li.x, -li.y, li.z);
    } else {
        const float u0 = u01(r[0]), u1 = u01(r[1]);
        const float rr = fsqrt(u0);
        float sn, cs;
        sincos_2pi(u1, sn, cs);
        const float one_minus = fsub(1.0f, u0);
        lo = f3(fmul(rr, cs), fsqrt(0.0f < one_minus ? one_minus : 0.0f), fmul(rr, sn));
        if (nee) {
            uint32_t r2[4] = {pixel, sample, bounce, 1u};
            philox4x32(r2, p.seed_lo, p.seed_hi);
            const LightSample ls = sample_light(p, fr, u01(r[2]), u01(r[3]), u01(r2[0]));
            if (ls.valid) {
                sh.valid = true;
                sh.o = fr.loc;
                sh.wi = ls.wi;
                sh.tmax = fmul(ls.dist, 0.999f);
                sh.contrib = f3(fmul(fmul(fmul(s.src.x, mr.albedo[0]), ls.le.x), ls.wgt),
                                fmul(fmul(fmul(s.src.y, mr.albedo[1]), ls.le.y), ls.wgt),
                                fmul(fmul(fmul(s.src.z, mr.albedo[2]), ls.le.z), ls.wgt));
            }
        }
    }
    s.d = vnorm(f3(fadd(fadd(fmul(fr.t1.x, lo.x), fmul(fr.n.x, lo.y)), fmul(fr.t2.x, lo.z)),
                   fadd(fadd(fmul(fr.t1.y, lo.x), fmul(fr.n.y, lo.y)), fmul(fr.t2.y, lo.z)),
                   fadd(fadd(fmul(fr.t1.z, lo.x), fmul(fr.n.z, lo.y)), fmul(fr.t2.z, lo.z))));
    s.o = fr.loc;
    s.src = f3(fmul(s.src.x, mr.albedo[0]), fmul(s.src.y, mr.albedo[1]), fmul(s.src.z, mr.albedo[2]));
    s.last_lambert = mirror ? 0u : 1u;
    return true;
}

PT_HD bool shade_miss(const RenderParams& p, PathState& s) {
    if (p.has_env) s.L = vadd(s.L, f3(fmul(p.env[0], s.src.x), fmul(p.env[1], s.src.y), fmul(p.env[2], s.src.z)));
    return false;
}

// The shading step of a flattened scene: the hit face's world vertices from the leaf-ordered
// face records.
PT_HD bool shade_hit(const RenderParams& p, PathState& s, uint32_t prim, uint32_t leaf, float u,
                                          float v, float w, uint32_t pixel, uint32_t sample, ShadowReq& sh) {
    sh.valid = false;
    if (prim == kPrimNone) return shade_miss(p, s);
    F3 v0, v1, v2;
    uint32_t mesh;
    load_face((const float4*)p.tris, leaf, v0, v1, v2, mesh);
    return shade_face(p, s, prim, v0, v1, v2, mesh, u, v, w, pixel, sample, sh);
}

// The shading step of a two-level scene: the object-space face record carried to world space
// with its instance's object_to_world, as the flattened scene's vertices were baked.
PT_HD bool shade_hit_two_level(const RenderParams& p, PathState& s, uint32_t prim, uint32_t face, uint32_t inst,
                               float u, float v, float w, uint32_t pixel, uint32_t sample, ShadowReq& sh) {
    sh.valid = false;
    if (prim == kPrimNone) return shade_miss(p, s);
    const float4* tris = (const float4*)p.tris;
    const float4 q0 = ldg(tris + 3 * (size_t)face), q1 = ldg(tris + 3 * (size_t)face + 1), q2 = ldg(tris + 3 * (size_t)face + 2);
    const DeviceInstance* in = (const DeviceInstance*)p.instances + inst;
    float m[16];
    for (int k = 0; k < 16; ++k) m[k] = ldg(in->o2w + k);
    F3 v0 = f3(q0.x, q0.y, q0.z), v1 = f3(q0.w, q1.x, q1.y), v2 = f3(q1.z, q1.w, q2.x);
    apply_point_dev(m, v0.x, v0.y, v0.z);
    apply_point_dev(m, v1.x, v1.y, v1.z);
    apply_point_dev(m, v2.x, v2.y, v2.z);
    return shade_face(p, s, prim, v0, v1, v2, ldg(&in->mesh), u, v, w, pixel, sample, sh);
}

PT_HD TwoLevelView two_level_view(const RenderParams& p) {
    return TwoLevelView{(const uint4*)p.nodes, (const float4*)p.tris, p.num_nodes, (const uint4*)p.top_nodes,
                        p.top_num_nodes, (const DeviceInstance*)p.instances, p.exact_tree != 0};
}

// Camera ray of a path (pixel centre, or jittered with the (pixel, sample, 0xFFFF) RNG block).
PT_HD void path_camera(const RenderParams& p, uint64_t path, uint32_t& pixel, uint32_t& sample,
                                            F3& o, F3& d) {
    const uint32_t npix = p.width * p.height;
    sample = (uint32_t)(path / npix);
    pixel = (uint32_t)(path % npix);
    const uint32_t x = pixel % p.width, y = pixel / p.width;
    float px = (float)x + 0.5f, py = (float)y + 0.5f;
    if (p.flags & PT_RENDER_JITTER) {
        uint32_t r[4] = {pixel, sample, 0xFFFFu, 0u};
        philox4x32(r, p.seed_lo, p.seed_hi);
        px = fadd((float)x, u01(r[0]));
        py = fadd((float)y, u01(r[1]));
    }
    camera_ray(p.cam, px, py, o, d);
}

PT_HD void clamp_store(float* out, const F3& L) {  // BoxFilter::AddSample clamp
    out[0] = L.x > 255 ? 255.f : L.x;
    out[1] = L.y > 255 ? 255.f : L.y;
    out[2] = L.z > 255 ? 255.f : L.z;
}

// ---- fused pipeline -------------------------------------------------------------------------

// The fused path loop on a two-level scene (same steps as path_fused).
template <int CAP>
PT_HD uint32_t path_fused_two_level(const RenderParams& p, uint64_t path, float* out, uint32_t* primary) {
    const TwoLevelView view = two_level_view(p);
    const float inf = bitsf(0x7F800000u);
    uint32_t pixel, sample;
    PathState s;
    path_camera(p, path, pixel, sample, s.o, s.d);
    s.src = f3(1.f, 1.f, 1.f);
    s.L = f3(0.f, 0.f, 0.f);
    s.bounces = 0;
    s.last_lambert = 0;
    uint32_t rays = 0;
    while (!throughput_is_zero(s.src)) {
        const TwoLevelHit h = traverse_two_level<false, CAP>(view, s.o.x, s.o.y, s.o.z, s.d.x, s.d.y, s.d.z, inf, false);
        ++rays;
        if (h.r.overflow) { raise_flag(p.err); break; }
        if (s.bounces == 0 && sample == 0 && primary) primary[pixel] = h.r.prim;
        ShadowReq sh;
        const bool more = shade_hit_two_level(p, s, h.r.prim, h.r.leaf, h.inst, h.r.u, h.r.v, h.r.w, pixel, sample, sh);
        if (sh.valid) {
            const TwoLevelHit t = traverse_two_level<false, CAP>(view, sh.o.x, sh.o.y, sh.o.z, sh.wi.x, sh.wi.y, sh.wi.z,
                                                                 sh.tmax, true);
            ++rays;
            if (t.r.overflow) { raise_flag(p.err); break; }
            if (t.r.prim == kPrimNone) s.L = vadd(s.L, sh.contrib);
        }
        if (!more) break;
    }
    clamp_store(out, s.L);
    return rays;
}

// Returns the number of rays traced (camera + bounce + shadow).  TWO_LEVEL: the scene may be a
// two-level one (p.instances), traced with traverse_two_level.
template <int CAP = kStackCap, bool TWO_LEVEL = false>
PT_HD uint32_t path_fused(const RenderParams& p, uint64_t path, float* out, uint32_t* primary) {
    if (TWO_LEVEL && p.instances) return path_fused_two_level<CAP>(p, path, out, primary);
    const uint4* nodes = (const uint4*)p.nodes;
    const float4* tris = (const float4*)p.tris;
    const float inf = bitsf(0x7F800000u);
    uint32_t pixel, sample;
    PathState s;
    path_camera(p, path, pixel, sample, s.o, s.d);
    s.src = f3(1.f, 1.f, 1.f);
    s.L = f3(0.f, 0.f, 0.f);
    s.bounces = 0;
    s.last_lambert = 0;
    uint32_t rays = 0;
    while (!throughput_is_zero(s.src)) {
        RayState rs;
        ray_setup(rs, s.o.x, s.o.y, s.o.z, s.d.x, s.d.y, s.d.z);
        const TraceResult h = traverse<false, CAP>(nodes, tris, p.num_nodes, rs, inf, false, p.exact_tree != 0);
        ++rays;
        if (h.overflow) { raise_flag(p.err); break; }
        if (s.bounces == 0 && sample == 0 && primary) primary[pixel] = h.prim;
        ShadowReq sh;
        const bool more = shade_hit(p, s, h.prim, h.leaf, h.u, h.v, h.w, pixel, sample, sh);
        if (sh.valid) {
            RayState sr;
            ray_setup(sr, sh.o.x, sh.o.y, sh.o.z, sh.wi.x, sh.wi.y, sh.wi.z);
            const TraceResult t = traverse<false, CAP>(nodes, tris, p.num_nodes, sr, sh.tmax, true, p.exact_tree != 0);
            ++rays;
            if (t.overflow) { raise_flag(p.err); break; }
            if (t.prim == kPrimNone) s.L = vadd(s.L, sh.contrib);
        }
        if (!more) break;
    }
    clamp_store(out, s.L);
    return rays;
}

}  // namespace pt
