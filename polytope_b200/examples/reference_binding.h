// reference_binding.h -- the binding a Polytope maintainer adds on the reference's side to render
// through libpolytope_b200: a poly::Scene converted to a pt_scene_desc, the device scene made from
// it, and a GpuRunner that takes the place of TileRunner in the render call.
//
// It is compiled inside Polytope's source tree (include path = Polytope's src/, plus this
// library's include/), against the reference's own classes:
//   poly::Scene (src/cpu/scenes/Scene.h:19-37), poly::Mesh / poly::mesh_geometry
//   (src/cpu/shapes/mesh.h:17-113), poly::compact_bvh (src/cpu/acceleration/bvh.h:24-77),
//   poly::LambertBRDF / poly::MirrorBRDF (src/cpu/shading/brdf/), poly::ColorSkybox
//   (src/cpu/scenes/skyboxes/ColorSkybox.h), poly::AbstractRunner (src/cpu/runners/AbstractRunner.h:17-55).
// The render call it serves is main.cpp:187-220: spawn runner threads, join, Output().
//
// Everything here is plain C++14 over the C ABI; nothing of the library's internals is visible.

#ifndef POLYTOPE_B200_REFERENCE_BINDING_H
#define POLYTOPE_B200_REFERENCE_BINDING_H

#include <cstring>
#include <memory>
#include <vector>

#include "polytope_b200.h"

#include "cpu/acceleration/bvh.h"
#include "cpu/cameras/AbstractCamera.h"
#include "cpu/films/AbstractFilm.h"
#include "cpu/films/PNGFilm.h"
#include "cpu/runners/AbstractRunner.h"
#include "cpu/scenes/Scene.h"
#include "cpu/scenes/skyboxes/ColorSkybox.h"
#include "cpu/shading/brdf/lambert_brdf.h"
#include "cpu/shading/brdf/mirror_brdf.h"
#include "cpu/structures/Sample.h"

namespace poly_b200 {

// A pt_scene_desc together with the arrays it points into.  The mesh descriptors point straight
// into the reference's mesh_geometry vectors (no copy); `pairs` holds the leaf-ordered (mesh, face)
// list re-packed from std::pair<unsigned, unsigned> into the flat uint32 pairs the ABI takes.
struct scene_desc {
   std::vector<pt_mesh_desc> meshes;
   std::vector<uint32_t> pairs;
   pt_scene_desc desc{};
};

// poly::Scene -> pt_scene_desc.  Meshes keep Scene::Shapes order, which defines the global
// primitive ids (prim_base[m] + face) and the (mesh, face) pairs of the tree.  With keep_tree the
// caller's own compacted tree (Scene::bvh_root after bound() + compact(), main.cpp:153-160) is
// passed through -- poly::compact_bvh_node and pt_bvh_node have the same 32-byte layout -- and
// otherwise pt_scene_create runs its own identical SAH build.  Returns PT_EINVAL for a shape that
// is neither an emitter nor carries a Lambert or mirror BRDF (glossy and textured materials have
// no counterpart on the device).
inline int describe_scene(poly::Scene &scene, scene_desc &out, bool keep_tree) {
   out.meshes.assign(scene.Shapes.size(), pt_mesh_desc{});
   for (size_t i = 0; i < scene.Shapes.size(); ++i) {
      const poly::Mesh *m = scene.Shapes[i];
      const poly::mesh_geometry &g = *m->mesh_geometry;
      pt_mesh_desc &o = out.meshes[i];
      o.x = g.x_packed.data();
      o.y = g.y_packed.data();
      o.z = g.z_packed.data();
      o.num_vertices = (uint32_t) g.x_packed.size();
      o.fv0 = g.fv0.data();
      o.fv1 = g.fv1.data();
      o.fv2 = g.fv2.data();
      o.num_faces = (uint32_t) g.fv0.size();
      if (g.has_vertex_normals) {
         o.nx = g.nx_packed.data();
         o.ny = g.ny_packed.data();
         o.nz = g.nz_packed.data();
      }
      // Row-major poly::Transform::Matrix, and the inverse stored beside it: Mesh::intersect turns
      // vertex normals to world space with object_to_world->ApplyInPlace(Normal&), which reads
      // that stored Inverse (Transform.cpp:135-143).
      std::memcpy(o.object_to_world, m->object_to_world->Matrix.Matrix, sizeof(o.object_to_world));
      std::memcpy(o.world_to_object, m->object_to_world->Inverse.Matrix, sizeof(o.world_to_object));
      o.is_light = m->is_light() ? 1 : 0;
      if (o.is_light) {
         o.emission[0] = m->spd->r;
         o.emission[1] = m->spd->g;
         o.emission[2] = m->spd->b;
      }
      const poly::AbstractBRDF *brdf = (m->material && m->material->BRDF) ? m->material->BRDF.get() : nullptr;
      if (const auto *l = dynamic_cast<const poly::LambertBRDF *>(brdf)) {
         if (l->texture) return PT_EINVAL;
         o.material = PT_MAT_LAMBERT;
         o.albedo[0] = l->refl.r;
         o.albedo[1] = l->refl.g;
         o.albedo[2] = l->refl.b;
      } else if (const auto *r = dynamic_cast<const poly::MirrorBRDF *>(brdf)) {
         o.material = PT_MAT_MIRROR;
         o.albedo[0] = r->refl.r;
         o.albedo[1] = r->refl.g;
         o.albedo[2] = r->refl.b;
      } else if (o.is_light) {
         o.material = PT_MAT_LAMBERT;  // an emitter's material is never sampled (the path ends there)
      } else {
         return PT_EINVAL;
      }
   }
   out.desc = pt_scene_desc{};
   out.desc.meshes = out.meshes.data();
   out.desc.num_meshes = (uint32_t) out.meshes.size();
   out.pairs.clear();
   const poly::compact_bvh *c = scene.bvh_root.compact_root;
   if (keep_tree && c != nullptr) {
      out.pairs.reserve(2 * c->leaf_ordered_indices.size());
      for (const auto &p : c->leaf_ordered_indices) {
         out.pairs.push_back(p.first);
         out.pairs.push_back(p.second);
      }
      out.desc.nodes = reinterpret_cast<const pt_bvh_node *>(c->nodes);
      out.desc.num_nodes = (uint32_t) c->num_nodes;
      out.desc.leaf_pairs = out.pairs.data();
   }
   if (const auto *sky = dynamic_cast<const poly::ColorSkybox *>(scene.Skybox.get())) {
      const poly::SpectralPowerDistribution spd = sky->GetSpd(poly::Vector(0, 0, 1));
      out.desc.has_env = 1;
      out.desc.env[0] = spd.r;
      out.desc.env[1] = spd.g;
      out.desc.env[2] = spd.b;
   }
   return PT_OK;
}

// The device copy of the scene.  Returns nullptr on failure with the reason in pt_last_error();
// the descriptor's arrays are copied, so the host scene may change or go away afterwards.
inline pt_scene *make_gpu_scene(poly::Scene &scene, bool keep_tree = true) {
   scene_desc d;
   if (describe_scene(scene, d, keep_tree) != PT_OK) return nullptr;
   pt_scene *out = nullptr;
   if (pt_scene_create(&d.desc, &out) != PT_OK) return nullptr;
   return out;
}

// The render description of one frame as the runner's pieces define it: Bounds, NumSamples,
// the integrator's MaxDepth and the camera's LookAt and field of view (AbstractCamera.h:25-30,
// set by pbrt_parser.cpp:1171-1173).  `seed` keys the counter RNG; `flags` are PT_RENDER_*.
inline pt_render_desc describe_render(const poly::AbstractRunner &runner, uint64_t seed, uint32_t flags) {
   const poly::AbstractCamera &cam = *runner.Scene->Camera;
   pt_render_desc rd{};
   rd.width = (uint32_t) runner.Bounds.x;
   rd.height = (uint32_t) runner.Bounds.y;
   rd.spp = runner.NumSamples;
   rd.max_depth = (uint32_t) runner.Integrator->MaxDepth;
   rd.seed = seed;
   rd.flags = flags;
   float eye[3] = {cam.eye.x, cam.eye.y, cam.eye.z};
   float look[3] = {cam.lookAt.x, cam.lookAt.y, cam.lookAt.z};
   float up[3] = {cam.up.x, cam.up.y, cam.up.z};
   if (eye[0] == look[0] && eye[1] == look[1] && eye[2] == look[2]) {
      // No LookAt in the file: the camera-to-world transform is the identity and the members keep
      // their zero defaults.  LookAt (0,0,0) (0,0,1) (0,1,0) gives the same matrix.
      const float e[3] = {0, 0, 0}, l[3] = {0, 0, 1}, u[3] = {0, 1, 0};
      std::memcpy(eye, e, sizeof(e));
      std::memcpy(look, l, sizeof(l));
      std::memcpy(up, u, sizeof(u));
   }
   std::memcpy(rd.camera.eye, eye, sizeof(eye));
   std::memcpy(rd.camera.look_at, look, sizeof(look));
   std::memcpy(rd.camera.up, up, sizeof(up));
   rd.camera.fov_deg = cam.Settings.FieldOfView;
   return rd;
}

// A PNG film whose bytes were quantised on the device (pt_render_rgba8): Output() writes them to
// the same file PNGFilm would (PNGFilm::Output, src/cpu/films/PNGFilm.cpp:20-58: clamp at 255,
// truncation, alpha 255, then the PNG) through pt_write_png.  The film takes no samples.
class DevicePNGFilm : public poly::AbstractFilm {
public:
   const std::string Filename;
   std::vector<uint8_t> rgba;           // width * height * 4, filled by GpuRunner::Run
   int status = PT_OK;

   DevicePNGFilm(const poly::Bounds bounds, std::string filename)
      : AbstractFilm(bounds, nullptr), Filename(std::move(filename)) {}

   void AddSample(const poly::Point2f &, const poly::Sample &) override {}
   void Output() override {
      if (rgba.size() != 4 * (size_t) Bounds.x * Bounds.y) {
         status = PT_EINVAL;
         Log.error("DevicePNGFilm::Output: no rendered frame");
         return;
      }
      status = pt_write_png(Filename.c_str(), rgba.data(), (uint32_t) Bounds.x, (uint32_t) Bounds.y);
      if (status != PT_OK) Log.error(std::string("pt_write_png: ") + pt_last_error());
   }
};

// Stands in for TileRunner in the render call (main.cpp:187-220): thread 0 renders the whole
// frame with one library call, the other threads return at once, and Output() then writes the
// film.  With a DevicePNGFilm (use_device_png) the frame is quantised on the device and only its
// bytes come back; Output() writes them.  With any other film each pixel's float value enters the
// film as one sample at the pixel centre; BoxFilter::Output divides by the number of samples it
// holds (one), so the PNG gets the rendered values unchanged.  A failed call leaves `status` at the
// PT_E* code and the reason in Log.error; the film then stays empty.
class GpuRunner : public poly::AbstractRunner {
public:
   GpuRunner(std::unique_ptr<poly::AbstractSampler> sampler, poly::Scene *scene,
             std::unique_ptr<poly::AbstractIntegrator> integrator, std::unique_ptr<poly::AbstractFilm> film,
             unsigned int num_samples, poly::Bounds bounds, pt_scene *gpu_scene)
      : AbstractRunner(std::move(sampler), scene, std::move(integrator), std::move(film), num_samples, bounds),
        gpu(gpu_scene) {}

   pt_scene *gpu;                       // from make_gpu_scene; owned by the caller
   uint64_t seed = 1;                   // counter-RNG key
   uint32_t flags = PT_RENDER_NEE;      // PT_RENDER_*
   int status = PT_OK;
   std::vector<float> rgb;              // the float film, width * height * 3 (float-film mode)

   // Replaces the runner's PNGFilm with a DevicePNGFilm writing the same file.  Returns false (and
   // keeps the film) when the film is not a PNGFilm.
   bool use_device_png() {
      const auto *png = dynamic_cast<const poly::PNGFilm *>(Film.get());
      if (png == nullptr) return false;
      Film.reset(new DevicePNGFilm(Film->Bounds, png->Filename));
      return true;
   }

   void Run(int threadId) override {
      if (threadId != 0) return;
      const pt_render_desc rd = describe_render(*this, seed, flags);
      if (auto *dev = dynamic_cast<DevicePNGFilm *>(Film.get())) {
         dev->rgba.assign(4 * (size_t) rd.width * rd.height, 0);
         status = pt_render_rgba8(gpu, &rd, dev->rgba.data(), nullptr, 0, nullptr);
         if (status != PT_OK) {
            dev->rgba.clear();
            Log.error(std::string("pt_render_rgba8: ") + pt_last_error());
         }
         return;
      }
      rgb.assign(3 * (size_t) rd.width * rd.height, 0.f);
      status = pt_render(gpu, &rd, rgb.data(), nullptr, 0, nullptr);
      if (status != PT_OK) {
         Log.error(std::string("pt_render: ") + pt_last_error());
         return;
      }
      for (uint32_t y = 0; y < rd.height; ++y) {
         for (uint32_t x = 0; x < rd.width; ++x) {
            const float *p = &rgb[3 * ((size_t) y * rd.width + x)];
            Film->AddSample(poly::Point2f((float) x + 0.5f, (float) y + 0.5f),
                            poly::Sample(poly::SpectralPowerDistribution(p[0], p[1], p[2])));
         }
      }
   }
};

}  // namespace poly_b200

#endif  // POLYTOPE_B200_REFERENCE_BINDING_H
