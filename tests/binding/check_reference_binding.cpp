// check_reference_binding.cpp -- test driver for polytope_b200/examples/reference_binding.h.
//
// Built by tests/test_reference_binding_cpu.py against the reference's own headers and its
// compiled classes (oracle/_ref/libpolyref.so) plus libpolytope_b200.so, where the reference tree
// is present.  For one PBRT file it runs the reference's parse and BVH build as main.cpp does
// (pbrt_parser::parse_file, bvh::bound, bvh::compact), converts the scene with the binding, and
// checks, bit for bit:
//   1. the library's own SAH build (pt_bvh_build) of the converted meshes reproduces the tree the
//      reference built -- nodes and leaf-ordered (mesh, face) pairs;
//   2. the converted descriptors equal what the library's reader (pt_load_pbrt) makes of the same
//      file: geometry, matrices, materials, radiances, environment, and the render description;
//   3. without a CUDA device, make_gpu_scene returns nullptr with the library's message and
//      GpuRunner::Run records the failure instead of ending the process.
// With `--render DIR THREADS` (needs a device) it then runs the render call of main.cpp:187-220
// with GpuRunner in place of TileRunner -- Spawn(i) for each thread, join, Output() -- twice, on
// fresh parses of the file: once into the reference's own PNGFilm (float film through BoxFilter
// and lodepng) and once with DevicePNGFilm (quantised on the device, written by pt_write_png).  It
// leaves DIR/film.bin (the float film), DIR/float_film.png and DIR/device_film.png for the test.
// Prints one summary line and exits 0 when every check holds, 1 otherwise.
//
// Built by oracle/Makefile as oracle/_ref/check_reference_binding where the reference tree is
// present (it needs the reference's headers), and by tests/test_reference_binding_cpu.py.

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <thread>
#include <vector>

#include "common/parsers/pbrt_parser.h"
#include "reference_binding.h"

static int failures = 0;

static void check(bool ok, const std::string &what) {
   if (!ok) {
      std::fprintf(stderr, "MISMATCH: %s\n", what.c_str());
      ++failures;
   }
}

// bitwise equality of float arrays (so -0.0 vs 0.0 and NaN payloads count)
static bool same_bits(const void *a, const void *b, size_t bytes) {
   if (bytes == 0) return true;
   if (a == nullptr || b == nullptr) return false;
   return std::memcmp(a, b, bytes) == 0;
}

// The render call as main.cpp:187-220 makes it, on a fresh parse of `path`, with GpuRunner in
// place of the parsed TileRunner; `device_png` swaps the PNGFilm for a DevicePNGFilm.  The PNG the
// film writes is moved to `dest`.  Returns the runner's float film (empty in device-PNG mode).
static std::vector<float> render_once(const std::string &path, pt_scene *gpu, int threads, bool device_png,
                                      const std::string &dest) {
   poly::pbrt_parser parser;
   std::unique_ptr<poly::AbstractRunner> parsed = parser.parse_file(path);
   const auto *png = dynamic_cast<const poly::PNGFilm *>(parsed->Film.get());
   check(png != nullptr, "the parsed film is a PNGFilm");
   if (png == nullptr) return {};
   const std::string written = png->Filename;
   poly_b200::GpuRunner runner(std::move(parsed->Sampler), parsed->Scene, std::move(parsed->Integrator),
                               std::move(parsed->Film), parsed->NumSamples, parsed->Bounds, gpu);
   if (device_png) check(runner.use_device_png(), "use_device_png");
   std::vector<std::thread> pool;
   for (int i = 0; i < threads; ++i) pool.emplace_back(runner.Spawn(i));
   for (auto &t : pool) t.join();
   check(runner.status == PT_OK, std::string("GpuRunner::Run: ") + pt_last_error());
   runner.Output();
   if (device_png) {
      const auto *dev = dynamic_cast<const poly_b200::DevicePNGFilm *>(runner.Film.get());
      check(dev != nullptr && dev->status == PT_OK, "DevicePNGFilm::Output");
   }
   check(std::rename(written.c_str(), dest.c_str()) == 0, "the film wrote " + written);
   return runner.rgb;
}

static void render_call(const std::string &path, pt_scene *gpu, const std::string &dir, int threads) {
   const std::vector<float> film = render_once(path, gpu, threads, false, dir + "/float_film.png");
   std::ofstream out(dir + "/film.bin", std::ios::binary);
   out.write(reinterpret_cast<const char *>(film.data()), (std::streamsize) (film.size() * sizeof(float)));
   check(out.good() && !film.empty(), "film.bin");
   render_once(path, gpu, threads, true, dir + "/device_film.png");
}

int main(int argc, char **argv) {
   if (argc < 2) {
      std::fprintf(stderr, "usage: %s scene.pbrt\n", argv[0]);
      return 2;
   }
   const std::string path = argv[1];
   poly::pbrt_parser parser;
   std::unique_ptr<poly::AbstractRunner> runner = parser.parse_file(path);
   poly::Scene &scene = *runner->Scene;
   // The reference's bvh::bound dereferences a root that an empty world never creates (main.cpp
   // would crash there); the library refuses such a scene with PT_EINVAL instead.
   const bool empty = scene.Shapes.empty();
   if (!empty) {
      scene.bvh_root.bound(scene.Shapes);
      scene.bvh_root.compact();
   }

   poly_b200::scene_desc d;
   check(poly_b200::describe_scene(scene, d, true) == PT_OK, "describe_scene");
   const uint32_t nm = d.desc.num_meshes;
   uint64_t faces = 0;
   for (const auto &m : d.meshes) faces += m.num_faces;

   // 1. the library's SAH build against the reference's tree
   uint32_t nn = 0;
   const int counted = pt_bvh_build(d.meshes.data(), nm, 0, nullptr, &nn, nullptr);
   if (empty) {
      check(counted == PT_EINVAL, "an empty world is refused");
   } else {
      check(counted == PT_OK, std::string("pt_bvh_build count: ") + pt_last_error());
      std::vector<pt_bvh_node> nodes(nn);
      std::vector<uint32_t> pairs(2 * faces);
      check(pt_bvh_build(d.meshes.data(), nm, 0, nodes.data(), &nn, pairs.data()) == PT_OK,
            std::string("pt_bvh_build: ") + pt_last_error());
      check(nn == d.desc.num_nodes, "node count " + std::to_string(nn) + " vs " + std::to_string(d.desc.num_nodes));
      check(nn == d.desc.num_nodes && same_bits(nodes.data(), d.desc.nodes, sizeof(pt_bvh_node) * nn), "tree nodes");
      check(pairs.size() == d.pairs.size() && same_bits(pairs.data(), d.pairs.data(), 4 * pairs.size()),
            "leaf pairs");
   }

   // 2. the binding's descriptors against the library's reader
   pt_pbrt_scene *file = nullptr;
   check(pt_load_pbrt(path.c_str(), &file) == PT_OK, std::string("pt_load_pbrt: ") + pt_last_error());
   if (file != nullptr) {
      pt_pbrt_info info{};
      const pt_mesh_desc *mine = nullptr;
      pt_pbrt_get_info(file, &info);
      pt_pbrt_get_meshes(file, &mine);
      check(info.num_meshes == nm, "mesh count");
      for (uint32_t i = 0; i < nm && i < info.num_meshes; ++i) {
         const pt_mesh_desc &a = d.meshes[i], &b = mine[i];
         const std::string at = " of mesh " + std::to_string(i);
         check(a.num_vertices == b.num_vertices && a.num_faces == b.num_faces, "sizes" + at);
         if (a.num_vertices != b.num_vertices || a.num_faces != b.num_faces) continue;
         const size_t vb = 4 * (size_t) a.num_vertices, fb = 4 * (size_t) a.num_faces;
         check(same_bits(a.x, b.x, vb) && same_bits(a.y, b.y, vb) && same_bits(a.z, b.z, vb), "vertices" + at);
         check(same_bits(a.fv0, b.fv0, fb) && same_bits(a.fv1, b.fv1, fb) && same_bits(a.fv2, b.fv2, fb), "faces" + at);
         check((a.nx == nullptr) == (b.nx == nullptr), "has normals" + at);
         if (a.nx && b.nx)
            check(same_bits(a.nx, b.nx, vb) && same_bits(a.ny, b.ny, vb) && same_bits(a.nz, b.nz, vb), "normals" + at);
         check(same_bits(a.object_to_world, b.object_to_world, 64), "object_to_world" + at);
         check(same_bits(a.world_to_object, b.world_to_object, 64), "world_to_object" + at);
         check(a.is_light == b.is_light, "is_light" + at);
         check(same_bits(a.emission, b.emission, 12), "emission" + at);
         if (!a.is_light) check(a.material == b.material && same_bits(a.albedo, b.albedo, 12), "material" + at);
      }
      check(info.has_env == d.desc.has_env && (!info.has_env || same_bits(info.env, d.desc.env, 12)), "environment");
      const pt_render_desc rd = poly_b200::describe_render(*runner, 1, PT_RENDER_NEE);
      check(rd.width == info.width && rd.height == info.height && rd.spp == info.spp && rd.max_depth == info.max_depth,
            "render settings");
      check(same_bits(&rd.camera, &info.camera, sizeof(pt_camera)), "camera");
      pt_pbrt_free(file);
   }

   // 3. the device calls: on a machine without a device both fail cleanly
   pt_scene *gpu = poly_b200::make_gpu_scene(scene);
   const std::string why = gpu ? "" : pt_last_error();
   poly_b200::GpuRunner g(std::move(runner->Sampler), runner->Scene, std::move(runner->Integrator),
                          std::move(runner->Film), runner->NumSamples, runner->Bounds, gpu);
   if (gpu == nullptr) {
      g.Run(0);
      check(g.status != PT_OK, "GpuRunner::Run without a device scene");
   }
   if (argc >= 5 && std::string(argv[2]) == "--render") {
      check(gpu != nullptr, "--render needs a device scene: " + why);
      if (gpu != nullptr) render_call(path, gpu, argv[3], std::atoi(argv[4]));
   }
   std::printf("meshes %u faces %llu nodes %u device %s\n", nm, (unsigned long long) faces, nn,
               gpu ? "yes" : ("no (" + why + ")").c_str());
   if (gpu) pt_scene_destroy(gpu);
   return failures == 0 ? 0 : 1;
}
