// ref_driver.cpp -- a C interface over the reference's own compiled sources.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with the Polytope sources
// (bvh.cpp, mesh.cpp, the structures, PerspectiveCamera.cpp, Logger.cpp; read in place from the
// reference tree, never copied) into oracle/_ref/libpolyref.so.  It is used to pin the CPU
// restatement in oracle/oracle.cpp, to generate golden fixtures, and as the timed CPU baseline.
//
// What runs here is the reference's code: poly::bvh::bound / compact / intersect_compact,
// poly::Mesh::intersect, poly::BoundingBox::Hits, poly::Transform, poly::PerspectiveCamera,
// poly::Intersection::WorldToLocal / LocalToWorld, poly::MirrorBRDF::sample, the spectrum types,
// the PLY / OBJ / PBRT parsers, and PNGFilm::Output with BoxFilter and lodepng.  The only code of
// this file's own is the glue and the render-loop patches that the reference cannot run as shipped
// (its RNG is seeded from std::random_device, constants.h:86-104):
//   P1 counter-based RNG (Philox4x32-10) keyed (pixel, sample, bounce); portable sin/cos of 2*pi*u
//   P2 the post-hit frame comes from the mesh that owns the hit face: the hit face is re-tested
//      alone on its own mesh (poly::Mesh::intersect with MinT = +inf), which recomputes the commit
//      and the frame exactly once (mesh.cpp:331-460)
//   P3 area-light next-event estimation with a shadow ray (closest-hit predicate with MinT = tmax)
//   P4 float film (per-sample clamp at 255, mean) and the primary-hit id
// The integrator loop mirrors PathTraceIntegrator::GetSample (PathTraceIntegrator.cpp:10-135).

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common/parsers/mesh_parsers.h"
#include "common/parsers/pbrt_parser.h"
#include "cpu/acceleration/bvh.h"
#include "cpu/runners/AbstractRunner.h"
#include "cpu/scenes/skyboxes/ColorSkybox.h"
#include "cpu/shading/brdf/lambert_brdf.h"
#include "cpu/cameras/PerspectiveCamera.h"
#include "cpu/shading/brdf/mirror_brdf.h"
#include "cpu/structures/stats.h"
#include "cpu/films/PNGFilm.h"
#include "cpu/filters/BoxFilter.h"
#include "../lib/lodepng.h"  // lodepng, beside the reference sources (REF/lib)

// Globals the reference translation units expect (defined by src/cpu/main.cpp in the reference).
poly::Logger Log;

// poly::Logger (src/common/utilities/Logger.h:18-44) only carries debug chatter on this path; its
// members are defined here as quiet glue instead of linking Logger.cpp (which writes coloured
// timestamps to stdout from inside the hot loop).  Errors still go to stderr.
namespace poly {
void Logger::debug(const char*, ...) {}
void Logger::info(const char*, ...) {}
void Logger::warning(const char*, ...) {}
void Logger::error(const char* format, ...) {
    va_list args;
    va_start(args, format);
    std::vfprintf(stderr, format, args);
    va_end(args);
    std::fputc('\n', stderr);
}
void Logger::debug(const std::string&) {}
void Logger::info(const std::string&) {}
void Logger::warning(const std::string&) {}
void Logger::error(const std::string& text) { std::fprintf(stderr, "%s\n", text.c_str()); }
}  // namespace poly
// The path globals of src/common/utilities/GlobalDefines.h come from PNGFilm.cpp, which includes
// that header; the parsers below only see absolute paths.
thread_local poly::stats thread_stats;
poly::stats main_stats;

// The ISPC brute-force intersector (src/cpu/shapes/mesh_intersect.ispc) is only reachable from
// Mesh::intersect(Ray&, Intersection&) (mesh.cpp:469-557), which the BVH path never calls; ispc is
// not installed, so the symbol is a stub that reports no hit.
namespace ispc {
extern "C" void soa_linear_intersect(const float*, const float*, const float*, float, float, float, float, float,
                                     float, float& t, uint32_t& face, bool& hits, uint32_t) {
    t = poly::FloatMax;
    face = 0;
    hits = false;
}
}  // namespace ispc

namespace {

struct RefScene {
    std::vector<std::shared_ptr<poly::mesh_geometry>> geoms;
    std::vector<std::unique_ptr<poly::Mesh>> meshes;
    std::vector<poly::Mesh*> mesh_ptrs;
    std::unordered_map<const poly::Mesh*, uint32_t> mesh_index;
    std::vector<uint32_t> prim_base;
    std::vector<uint32_t> material;
    std::vector<poly::ReflectanceSpectrum> albedo;
    poly::bvh bvh;
    bool has_env = false;
    poly::SpectralPowerDistribution env;
    // area-light table (world space)
    std::vector<uint32_t> light_mesh, light_face;
    std::vector<float> light_cdf;
    float light_area = 0;
};

struct ref_mesh {  // same layout as pt_mesh_desc / orc_mesh
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
};

poly::Matrix4x4 to_matrix(const float* m) {
    return poly::Matrix4x4(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8], m[9], m[10], m[11], m[12], m[13],
                           m[14], m[15]);
}

poly::Point world_vertex(const poly::Mesh* m, uint32_t face, int k) {
    const auto& g = *m->mesh_geometry;
    const uint32_t vi = k == 0 ? g.fv0[face] : (k == 1 ? g.fv1[face] : g.fv2[face]);
    poly::Point p(g.x_packed[vi], g.y_packed[vi], g.z_packed[vi]);
    m->object_to_world->ApplyInPlace(p);
    return p;
}

// Philox4x32-10 (Salmon et al., SC'11); the same generator the CUDA path and the restatement use.
void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[1] = (uint32_t)p1;
        c[3] = (uint32_t)p0;
        c[0] = n0;
        c[2] = n2;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}
float u01(uint32_t x) { return (float)(x >> 8) * 5.9604644775390625e-08f; }

// Portable sin/cos(2*pi*u): quadrant rint(4u) plus Taylor polynomials of sin/cos(pi/2 * r).
void sincos_2pi(float u, float& s, float& c) {
    const float f = 4.0f * u;
    const float q = std::nearbyint(f);
    const float r = f - q;
    const float r2 = r * r;
    float ps = std::fma(r2, 0.000160441184787359821833f, -0.00468175413531868810256f);
    ps = std::fma(r2, ps, 0.0796926262461670451206f);
    ps = std::fma(r2, ps, -0.645964097506246253655f);
    ps = std::fma(r2, ps, 1.57079632679489661923f);
    const float sr = r * ps;
    float pc = std::fma(r2, -0.0000252020423730606054811f, 0.000919260274839426215087f);
    pc = std::fma(r2, pc, -0.0208634807633529608730f);
    pc = std::fma(r2, pc, 0.253669507901048014030f);
    pc = std::fma(r2, pc, -1.23370055013616982735f);
    const float cr = std::fma(r2, pc, 1.0f);
    switch (((int)q) & 3) {
        case 0: s = sr; c = cr; break;
        case 1: s = cr; c = -sr; break;
        case 2: s = -sr; c = -cr; break;
        default: s = -cr; c = sr; break;
    }
}

template <class F>
void parallel_for(uint64_t n, int threads, F f) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    if (n < 1024 || threads == 1) { f(0, n); return; }
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

extern "C" {

typedef struct ref_ray { float org[3]; float tmax; float dir[3]; uint32_t flags; } ref_ray;
typedef struct ref_hit { uint32_t prim; float t; float u; float v; } ref_hit;

void* ref_scene_create(const ref_mesh* ms, uint32_t n, int has_env, const float* env) {
    RefScene* s = new RefScene();
    uint32_t base = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const ref_mesh& d = ms[i];
        auto g = std::make_shared<poly::mesh_geometry>();
        for (uint32_t v = 0; v < d.num_vertices; ++v) {
            if (d.nx) {
                poly::Point p(d.x[v], d.y[v], d.z[v]);
                poly::Normal nn(d.nx[v], d.ny[v], d.nz[v]);
                g->add_vertex(p, nn);
            } else {
                g->add_vertex(d.x[v], d.y[v], d.z[v]);
            }
        }
        g->has_vertex_normals = d.nx != nullptr;
        for (uint32_t f = 0; f < d.num_faces; ++f) g->add_packed_face(d.fv0[f], d.fv1[f], d.fv2[f]);
        g->unpack_faces();
        auto o2w = std::make_shared<poly::Transform>(to_matrix(d.object_to_world), to_matrix(d.world_to_object));
        auto w2o = std::make_shared<poly::Transform>(to_matrix(d.world_to_object), to_matrix(d.object_to_world));
        std::shared_ptr<poly::Material> mat;
        if (d.material == 2u)
            mat = std::make_shared<poly::Material>(std::make_shared<poly::MirrorBRDF>(
                poly::ReflectanceSpectrum(d.albedo[0], d.albedo[1], d.albedo[2])));
        auto mesh = std::unique_ptr<poly::Mesh>(new poly::Mesh(o2w, w2o, mat, g));
        if (d.is_light) mesh->spd = std::make_shared<poly::SpectralPowerDistribution>(d.emission[0], d.emission[1], d.emission[2]);
        s->mesh_index[mesh.get()] = i;
        s->mesh_ptrs.push_back(mesh.get());
        s->meshes.push_back(std::move(mesh));
        s->geoms.push_back(g);
        s->prim_base.push_back(base);
        s->material.push_back(d.material);
        s->albedo.emplace_back(d.albedo[0], d.albedo[1], d.albedo[2]);
        base += d.num_faces;
    }
    s->has_env = has_env != 0;
    if (env) s->env = poly::SpectralPowerDistribution(env[0], env[1], env[2]);
    s->bvh.num_nodes = 0;
    s->bvh.bound(s->mesh_ptrs);
    s->bvh.compact();
    // area lights: every face of an emitting mesh, in mesh/face order
    for (uint32_t i = 0; i < n; ++i) {
        const poly::Mesh* m = s->mesh_ptrs[i];
        if (!m->is_light()) continue;
        for (uint32_t f = 0; f < m->mesh_geometry->num_faces; ++f) {
            const poly::Point v0 = world_vertex(m, f, 0), v1 = world_vertex(m, f, 1), v2 = world_vertex(m, f, 2);
            const poly::Vector c = (v1 - v0).Cross(v2 - v0);
            const float area = 0.5f * c.Length();
            s->light_area = s->light_area + area;
            s->light_mesh.push_back(i);
            s->light_face.push_back(f);
            s->light_cdf.push_back(s->light_area);
        }
    }
    return s;
}

void ref_scene_destroy(void* p) { delete static_cast<RefScene*>(p); }
uint32_t ref_num_nodes(void* p) { return static_cast<RefScene*>(p)->bvh.compact_root->num_nodes; }

// The compacted nodes (32 bytes each, poly::compact_bvh_node) and leaf_ordered_indices pairs.
void ref_get_tree(void* p, void* nodes_out, uint32_t* pairs_out) {
    RefScene* s = static_cast<RefScene*>(p);
    const poly::compact_bvh* c = s->bvh.compact_root;
    static_assert(sizeof(poly::compact_bvh_node) == 32, "node size");
    std::memcpy(nodes_out, c->nodes, sizeof(poly::compact_bvh_node) * c->num_nodes);
    for (size_t i = 0; i < c->leaf_ordered_indices.size(); ++i) {
        pairs_out[2 * i] = c->leaf_ordered_indices[i].first;
        pairs_out[2 * i + 1] = c->leaf_ordered_indices[i].second;
    }
}

// Closest-hit queries through poly::bvh::intersect_compact (any-hit rays: the same query with
// MinT = tmax; only the hit/miss outcome is meaningful for them).
void ref_trace(void* p, const ref_ray* rays, uint64_t n, ref_hit* hits, uint32_t* node_tests, uint32_t* tri_tests,
               int threads) {
    const RefScene* s = static_cast<RefScene*>(p);
    parallel_for(n, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; ++i) {
            const ref_ray& r = rays[i];
            poly::Ray ray(r.org[0], r.org[1], r.org[2], r.dir[0], r.dir[1], r.dir[2]);
            ray.MinT = r.tmax;
            poly::Intersection isect;
            isect.x = -1;
            isect.y = -1;
            s->bvh.intersect_compact(ray, isect);
            if (isect.Hits) {
                const uint32_t mi = s->mesh_index.at(isect.Shape);
                hits[i] = {s->prim_base[mi] + isect.faceIndex, ray.MinT, isect.u, isect.v};
            } else {
                hits[i] = {0xFFFFFFFFu, ray.MinT, 0.f, 0.f};
            }
            if (node_tests) node_tests[i] = isect.num_bb_hits + isect.num_bb_misses;
            if (tri_tests) tri_tests[i] = isect.num_triangle_isects;
        }
    });
}

// poly::BoundingBox::Hits on one box (golden cases of tests/cuda/test_bvh_traversal.cpp).
int ref_bbox_hits(const float* bb, const float* o, const float* d, float min_t) {
    poly::BoundingBox box(poly::Point(bb[0], bb[1], bb[2]), poly::Point(bb[3], bb[4], bb[5]));
    poly::Ray ray(o[0], o[1], o[2], d[0], d[1], d[2]);
    ray.MinT = min_t;
    const poly::Vector inv(1.f / d[0], 1.f / d[1], 1.f / d[2]);
    return box.Hits(ray, inv) ? 1 : 0;
}

}  // extern "C"

namespace {

struct RefFrame {
    bool hit;
    uint32_t mesh, face;
    poly::Intersection isect;  // frame recomputed on the owning mesh
};

// Scene::intersect (Scene.cpp:12-31) + P2 (re-test the hit face alone on its own mesh).
RefFrame intersect_with_frame(const RefScene* s, const poly::Point& o, const poly::Vector& d) {
    RefFrame f{};
    poly::Ray ray(o, d);
    poly::Intersection isect;
    isect.x = -1;
    isect.y = -1;
    s->bvh.intersect_compact(ray, isect);
    f.hit = isect.Hits;
    if (!f.hit) return f;
    f.mesh = s->mesh_index.at(isect.Shape);
    f.face = isect.faceIndex;
    poly::Ray again(o, d);
    again.MinT = poly::Infinity;
    f.isect = poly::Intersection();
    f.isect.x = -1;
    f.isect.y = -1;
    const unsigned int face = f.face;
    s->mesh_ptrs[f.mesh]->intersect(again, f.isect, &face, 1);
    return f;
}

poly::SpectralPowerDistribution path_sample(const RefScene* s, poly::Ray ray, uint32_t pixel, uint32_t sample,
                                            uint32_t max_depth, uint64_t seed, uint32_t flags, uint32_t* primary) {
    poly::Ray current_ray = ray;
    unsigned num_bounces = 0;
    poly::ReflectanceSpectrum src(1.f, 1.f, 1.f);
    poly::SpectralPowerDistribution L;
    bool last_lambert = false;
    const bool nee = (flags & 1u) && !s->light_cdf.empty();
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    while (true) {
        if (src.is_zero()) return L;
        const RefFrame hf = intersect_with_frame(s, current_ray.Origin, current_ray.Direction);
        if (num_bounces == 0 && primary) *primary = hf.hit ? s->prim_base[hf.mesh] + hf.face : 0xFFFFFFFFu;
        if (!hf.hit) {
            if (s->has_env) {
                poly::SpectralPowerDistribution e = s->env;
                L += e * src;
            }
            return L;
        }
        const poly::Mesh* mesh = s->mesh_ptrs[hf.mesh];
        if (mesh->is_light()) {
            if (!(nee && last_lambert)) {
                poly::SpectralPowerDistribution e = *mesh->spd;
                L += e * src;
            }
            return L;
        }
        if (num_bounces >= max_depth) return L;
        const uint32_t bounce = num_bounces;
        num_bounces++;
        const poly::Intersection& isect = hf.isect;
        uint32_t r[4] = {pixel, sample, bounce, 0u};
        philox(r, k0, k1);
        const poly::Vector local_in = isect.WorldToLocal(current_ray.Direction);
        poly::Vector local_out;
        poly::ReflectanceSpectrum refl;
        const bool mirror = s->material[hf.mesh] == 2u;
        if (mirror) {
            float pdf;
            local_out = mesh->material->BRDF->sample(local_in, 0.f, 0.f, refl, pdf);
        } else {
            refl = s->albedo[hf.mesh];
            const float u0 = u01(r[0]), u1 = u01(r[1]);
            const float rr = std::sqrt(u0);
            float sn, cs;
            sincos_2pi(u1, sn, cs);
            local_out = poly::Vector(rr * cs, std::sqrt(std::max(0.0f, 1.0f - u0)), rr * sn);
            if (nee) {
                uint32_t r2[4] = {pixel, sample, bounce, 1u};
                philox(r2, k0, k1);
                const float target = u01(r[2]) * s->light_area;
                size_t lo = 0, hi = s->light_cdf.size() - 1;
                while (lo < hi) {
                    const size_t mid = (lo + hi) / 2;
                    if (target < s->light_cdf[mid]) hi = mid; else lo = mid + 1;
                }
                const poly::Mesh* lm = s->mesh_ptrs[s->light_mesh[lo]];
                const uint32_t lf = s->light_face[lo];
                const poly::Point v0 = world_vertex(lm, lf, 0), v1 = world_vertex(lm, lf, 1), v2 = world_vertex(lm, lf, 2);
                const float su = std::sqrt(u01(r[3]));
                const float b0 = 1.0f - su;
                const float b1 = u01(r2[0]) * su;
                const float b2 = (1.0f - b0) - b1;
                const poly::Point y(b0 * v0.x + b1 * v1.x + b2 * v2.x, b0 * v0.y + b1 * v1.y + b2 * v2.y,
                                    b0 * v0.z + b1 * v1.z + b2 * v2.z);
                const poly::Vector dv = y - isect.Location;
                const float dist2 = dv.Dot(dv);
                const float dist = std::sqrt(dist2);
                const poly::Vector wi = dv * (1.0f / dist);
                const float cos_x = wi.Dot(isect.bent_normal);
                poly::Vector ln = (v1 - v0).Cross(v2 - v0);
                ln.Normalize();
                const float cos_l = std::fabs(wi.Dot(ln));
                if (cos_x > 0.f && cos_l > 0.f && dist2 > 0.f) {
                    poly::Ray shadow(isect.Location, wi);
                    shadow.MinT = dist * 0.999f;
                    poly::Intersection si;
                    si.x = -1;
                    si.y = -1;
                    s->bvh.intersect_compact(shadow, si);
                    if (!si.Hits) {
                        const float g = (cos_x * cos_l) / dist2;
                        const float wgt = g * s->light_area * poly::OneOverPi;
                        const poly::SpectralPowerDistribution& le = *lm->spd;
                        L += poly::SpectralPowerDistribution(src.r * refl.r * le.r * wgt, src.g * refl.g * le.g * wgt,
                                                             src.b * refl.b * le.b * wgt);
                    }
                }
            }
        }
        const poly::Vector world_out = isect.LocalToWorld(local_out);
        current_ray = poly::Ray(isect.Location, world_out);
        src = src * refl;
        last_lambert = !mirror;
    }
}

}  // namespace

extern "C" {

typedef struct ref_render_desc {
    uint32_t width, height, spp, max_depth;
    uint64_t seed;
    uint32_t flags;
    float eye[3], look_at[3], up[3], fov;
} ref_render_desc;

// Camera rays for pixel centres through poly::PerspectiveCamera (LookAt as the PBRT parser builds it).
static std::unique_ptr<poly::PerspectiveCamera> make_camera(const ref_render_desc* rd) {
    poly::Point eye(rd->eye[0], rd->eye[1], rd->eye[2]);
    poly::Point look(rd->look_at[0], rd->look_at[1], rd->look_at[2]);
    poly::Vector up(rd->up[0], rd->up[1], rd->up[2]);
    poly::Transform current;
    poly::Transform t = poly::Transform::LookAt(eye, look, up, false);
    current *= t;
    poly::CameraSettings settings(poly::Bounds(rd->width, rd->height), rd->fov);
    return std::unique_ptr<poly::PerspectiveCamera>(new poly::PerspectiveCamera(settings, current, true));
}

void ref_camera_rays(const ref_render_desc* rd, ref_ray* out) {
    auto cam = make_camera(rd);
    for (uint32_t y = 0; y < rd->height; ++y)
        for (uint32_t x = 0; x < rd->width; ++x) {
            const poly::Ray r = cam->get_ray_for_pixel(poly::Point2f(x + 0.5f, y + 0.5f));
            out[y * rd->width + x] = {{r.Origin.x, r.Origin.y, r.Origin.z}, poly::Infinity,
                                      {r.Direction.x, r.Direction.y, r.Direction.z}, 0u};
        }
}

// Post-hit frames (Location, normal, Tangent1, Tangent2) of closest hits, 12 floats per ray.
void ref_hit_frames(void* p, const ref_ray* rays, uint64_t n, float* out) {
    const RefScene* s = static_cast<RefScene*>(p);
    for (uint64_t i = 0; i < n; ++i) {
        const ref_ray& r = rays[i];
        const RefFrame f = intersect_with_frame(s, poly::Point(r.org[0], r.org[1], r.org[2]),
                                                poly::Vector(r.dir[0], r.dir[1], r.dir[2]));
        float* o = out + 12 * i;
        if (!f.hit) { std::memset(o, 0, 12 * sizeof(float)); continue; }
        const poly::Intersection& x = f.isect;
        const float v[12] = {x.Location.x, x.Location.y, x.Location.z, x.bent_normal.x, x.bent_normal.y,
                             x.bent_normal.z, x.Tangent1.x, x.Tangent1.y, x.Tangent1.z, x.Tangent2.x,
                             x.Tangent2.y, x.Tangent2.z};
        std::memcpy(o, v, sizeof(v));
    }
}

// The patched render call over rows [row_begin, row_end): for each pixel the samples in order,
// film = (sum of per-sample radiance clamped at 255) * (1/spp) as BoxFilter::AddSample/Output.
void ref_render_rows(void* p, const ref_render_desc* rd, uint32_t row_begin, uint32_t row_end, float* rgb,
                     uint32_t* prim, int threads) {
    const RefScene* s = static_cast<RefScene*>(p);
    auto cam = make_camera(rd);
    const uint32_t k0 = (uint32_t)rd->seed, k1 = (uint32_t)(rd->seed >> 32);
    const uint64_t first = (uint64_t)row_begin * rd->width;
    const uint64_t count = (uint64_t)(row_end - row_begin) * rd->width;
    parallel_for(count, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; ++i) {
            const uint32_t pix = (uint32_t)(first + i);
            const uint32_t x = pix % rd->width, y = pix / rd->width;
            poly::SpectralPowerDistribution accum;
            for (uint32_t smp = 0; smp < rd->spp; ++smp) {
                poly::Point2f loc(x + 0.5f, y + 0.5f);
                if (rd->flags & 2u) {
                    uint32_t r[4] = {pix, smp, 0xFFFFu, 0u};
                    philox(r, k0, k1);
                    loc = poly::Point2f((float)x + u01(r[0]), (float)y + u01(r[1]));
                }
                poly::Ray ray = cam->get_ray_for_pixel(loc);
                uint32_t p0 = 0xFFFFFFFFu;
                poly::SpectralPowerDistribution L =
                    path_sample(s, ray, pix, smp, rd->max_depth, rd->seed, rd->flags, smp == 0 ? &p0 : nullptr);
                if (smp == 0 && prim) prim[pix] = p0;
                if (L.r > 255) L.r = 255;
                if (L.g > 255) L.g = 255;
                if (L.b > 255) L.b = 255;
                accum += L;
            }
            const float divisor = 1.0f / rd->spp;
            accum *= divisor;
            rgb[3 * pix + 0] = accum.r;
            rgb[3 * pix + 1] = accum.g;
            rgb[3 * pix + 2] = accum.b;
        }
    });
}

// ply_parser::parse_file on one file (the reference's own PLY reader).  Counts are returned
// first (pass NULL arrays); a second call copies the packed arrays out.
int ref_load_ply(const char* path, uint32_t* num_vertices, uint32_t* num_faces, int* has_normals, float* x, float* y,
                 float* z, float* nx, float* ny, float* nz, uint32_t* fv0, uint32_t* fv1, uint32_t* fv2) {
    auto g = std::make_shared<poly::mesh_geometry>();
    const poly::ply_parser parser;
    parser.parse_file(g, path);
    *num_vertices = (uint32_t)g->x_packed.size();
    *num_faces = (uint32_t)g->fv0.size();
    *has_normals = g->has_vertex_normals ? 1 : 0;
    if (x) {
        std::memcpy(x, g->x_packed.data(), 4 * g->x_packed.size());
        std::memcpy(y, g->y_packed.data(), 4 * g->y_packed.size());
        std::memcpy(z, g->z_packed.data(), 4 * g->z_packed.size());
        std::memcpy(fv0, g->fv0.data(), 4 * g->fv0.size());
        std::memcpy(fv1, g->fv1.data(), 4 * g->fv1.size());
        std::memcpy(fv2, g->fv2.data(), 4 * g->fv2.size());
        if (g->has_vertex_normals && nx) {
            std::memcpy(nx, g->nx_packed.data(), 4 * g->nx_packed.size());
            std::memcpy(ny, g->ny_packed.data(), 4 * g->ny_packed.size());
            std::memcpy(nz, g->nz_packed.data(), 4 * g->nz_packed.size());
        }
    }
    return 0;
}

int ref_load_obj(const char* path, uint32_t* num_vertices, uint32_t* num_faces, float* x, float* y, float* z,
                 uint32_t* fv0, uint32_t* fv1, uint32_t* fv2) {
    auto g = std::make_shared<poly::mesh_geometry>();
    const poly::obj_parser parser;
    parser.parse_file(g, path);
    *num_vertices = (uint32_t)g->x_packed.size();
    *num_faces = (uint32_t)g->fv0.size();
    if (x) {
        std::memcpy(x, g->x_packed.data(), 4 * g->x_packed.size());
        std::memcpy(y, g->y_packed.data(), 4 * g->y_packed.size());
        std::memcpy(z, g->z_packed.data(), 4 * g->z_packed.size());
        std::memcpy(fv0, g->fv0.data(), 4 * g->fv0.size());
        std::memcpy(fv1, g->fv1.data(), 4 * g->fv1.size());
        std::memcpy(fv2, g->fv2.data(), 4 * g->fv2.size());
    }
    return 0;
}

// ---- the reference's PBRT scene parser (pbrt_parser.cpp), for the pt_load_pbrt parity tests ----
// ref_pbrt_load parses a file with poly::pbrt_parser::parse_file and keeps the runner it returns;
// the accessors copy out what the renderer would use.  A file the reference cannot parse ends the
// process (its ERROR macro exits), so the tests give it only well-formed files.

struct RefPbrt {
    std::unique_ptr<poly::AbstractRunner> runner;
};

void* ref_pbrt_load(const char* path) {
    poly::pbrt_parser parser;
    auto* r = new RefPbrt();
    r->runner = parser.parse_file(path);
    return r;
}

void ref_pbrt_free(void* h) { delete static_cast<RefPbrt*>(h); }

// u[0..5] = width, height, spp, max_depth, number of shapes, has_env; f[0..2] = env;
// f[3..12] = eye, look-at, up, fov; f[13..28] = camera-to-world matrix (row-major)
void ref_pbrt_info(void* h, uint32_t* u, float* f) {
    const poly::AbstractRunner& run = *static_cast<RefPbrt*>(h)->runner;
    const poly::Scene& sc = *run.Scene;
    u[0] = run.Bounds.x;
    u[1] = run.Bounds.y;
    u[2] = run.NumSamples;
    u[3] = (uint32_t)run.Integrator->MaxDepth;
    u[4] = (uint32_t)sc.Shapes.size();
    const auto* sky = dynamic_cast<const poly::ColorSkybox*>(sc.Skybox.get());
    u[5] = sky ? 1 : 0;
    const poly::SpectralPowerDistribution env = sky ? sky->GetSpd(poly::Vector(0, 0, 1)) : poly::SpectralPowerDistribution();
    f[0] = sky ? env.r : 0.f;
    f[1] = sky ? env.g : 0.f;
    f[2] = sky ? env.b : 0.f;
    const poly::AbstractCamera& cam = *sc.Camera;
    const float v[10] = {cam.eye.x, cam.eye.y, cam.eye.z, cam.lookAt.x, cam.lookAt.y, cam.lookAt.z,
                         cam.up.x, cam.up.y, cam.up.z, cam.Settings.FieldOfView};
    std::memcpy(f + 3, v, sizeof(v));
    for (int k = 0; k < 16; ++k) f[13 + k] = cam.CameraToWorld.Matrix.Matrix[k / 4][k % 4];
}

// u[0..4] = vertices, faces, has normals, material type (0 = none), is light;
// f[0..15] object-to-world, f[16..31] the inverse stored in the object-to-world transform (what
// Mesh::intersect transforms vertex normals with), f[32..34] reflectance, f[35..37] radiance.
// Arrays are copied when x is non-null.
void ref_pbrt_mesh(void* h, uint32_t i, uint32_t* u, float* f, float* x, float* y, float* z, float* nx, float* ny,
                   float* nz, uint32_t* fv0, uint32_t* fv1, uint32_t* fv2) {
    const poly::Mesh& m = *static_cast<RefPbrt*>(h)->runner->Scene->Shapes[i];
    const poly::mesh_geometry& g = *m.mesh_geometry;
    u[0] = (uint32_t)g.x_packed.size();
    u[1] = (uint32_t)g.fv0.size();
    u[2] = g.has_vertex_normals ? 1 : 0;
    u[3] = 0;
    u[4] = m.is_light() ? 1 : 0;
    for (int k = 0; k < 16; ++k) {
        f[k] = m.object_to_world->Matrix.Matrix[k / 4][k % 4];
        f[16 + k] = m.object_to_world->Inverse.Matrix[k / 4][k % 4];
    }
    f[32] = f[33] = f[34] = 0.f;
    if (m.material && m.material->BRDF) {
        u[3] = (uint32_t)m.material->BRDF->brdf_type;
        if (const auto* l = dynamic_cast<const poly::LambertBRDF*>(m.material->BRDF.get())) {
            f[32] = l->refl.r; f[33] = l->refl.g; f[34] = l->refl.b;
        } else if (const auto* r = dynamic_cast<const poly::MirrorBRDF*>(m.material->BRDF.get())) {
            f[32] = r->refl.r; f[33] = r->refl.g; f[34] = r->refl.b;
        }
    }
    f[35] = m.spd ? m.spd->r : 0.f;
    f[36] = m.spd ? m.spd->g : 0.f;
    f[37] = m.spd ? m.spd->b : 0.f;
    if (!x) return;
    std::memcpy(x, g.x_packed.data(), 4 * g.x_packed.size());
    std::memcpy(y, g.y_packed.data(), 4 * g.y_packed.size());
    std::memcpy(z, g.z_packed.data(), 4 * g.z_packed.size());
    std::memcpy(fv0, g.fv0.data(), 4 * g.fv0.size());
    std::memcpy(fv1, g.fv1.data(), 4 * g.fv1.size());
    std::memcpy(fv2, g.fv2.data(), 4 * g.fv2.size());
    if (g.has_vertex_normals && nx) {
        std::memcpy(nx, g.nx_packed.data(), 4 * g.nx_packed.size());
        std::memcpy(ny, g.ny_packed.data(), 4 * g.ny_packed.size());
        std::memcpy(nz, g.nz_packed.data(), 4 * g.nz_packed.size());
    }
}


// ---- the reference's film output (PNGFilm.cpp:20-58) and its PNG library, for the output tests ----
// ref_png_film writes a float film (width*height*3, row-major) the way the reference's render call
// ends: each pixel enters a BoxFilter as one sample at its centre, then PNGFilm::Output quantises
// and encodes with lodepng.  A film the reference cannot encode ends the process (ERROR exits).
void ref_png_film(const float* rgb, uint32_t width, uint32_t height, const char* path) {
    const poly::Bounds bounds(width, height);
    auto filter = std::make_unique<poly::BoxFilter>(bounds);
    filter->SetSamples(1);
    poly::PNGFilm film(bounds, path, std::move(filter));
    for (uint32_t y = 0; y < height; ++y)
        for (uint32_t x = 0; x < width; ++x) {
            const float* p = rgb + 3 * ((size_t)y * width + x);
            film.AddSample(poly::Point2f((float)x + 0.5f, (float)y + 0.5f),
                           poly::Sample(poly::SpectralPowerDistribution(p[0], p[1], p[2])));
        }
    film.Output();
}

// lodepng's decoder: a PNG file as RGBA8.  Returns lodepng's error code (0 = ok); *w and *h are
// set on success, and rgba receives min(cap, w*h*4) bytes.
unsigned ref_png_decode(const char* path, uint32_t* w, uint32_t* h, uint8_t* rgba, size_t cap) {
    std::vector<unsigned char> out;
    unsigned ww = 0, hh = 0;
    const unsigned err = lodepng::decode(out, ww, hh, std::string(path));
    if (err) return err;
    *w = ww;
    *h = hh;
    std::memcpy(rgba, out.data(), std::min(cap, out.size()));
    return 0;
}

}  // extern "C"
