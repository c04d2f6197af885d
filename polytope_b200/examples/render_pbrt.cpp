// render_pbrt.cpp -- the reference's command-line render (src/cpu/main.cpp: parse the scene file,
// build the BVH, render, write the PNG) through the library's C ABI.
//
//   render_pbrt scene.pbrt out.png [--persistent] [--seed N]
//
// Build (from the repository root, next to the library), as one command:
//   g++ -O2 -std=c++17 -I include polytope_b200/examples/render_pbrt.cpp -o render_pbrt
//       -L polytope_b200/lib -lpolytope_b200 -Wl,-rpath,polytope_b200/lib
// Exit status 0 on success; otherwise the library's message is printed (without a CUDA device
// every launching call returns PT_ECUDA: there is no CPU fallback).

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "polytope_b200.h"

static int fail(const char* what) {
    std::fprintf(stderr, "%s: %s\n", what, pt_last_error());
    return 1;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s scene.pbrt out.png [--persistent] [--seed N]\n", argv[0]);
        return 2;
    }
    uint32_t flags = PT_RENDER_NEE;
    uint64_t seed = 1;
    for (int i = 3; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--persistent")) flags |= PT_RENDER_PERSISTENT;
        else if (!std::strcmp(argv[i], "--seed") && i + 1 < argc) seed = std::strtoull(argv[++i], nullptr, 10);
    }
    const auto t0 = std::chrono::steady_clock::now();
    pt_pbrt_scene* file = nullptr;
    if (pt_load_pbrt(argv[1], &file) != PT_OK) return fail("pt_load_pbrt");
    pt_pbrt_info info{};
    const pt_mesh_desc* meshes = nullptr;
    pt_pbrt_get_info(file, &info);
    pt_pbrt_get_meshes(file, &meshes);
    pt_scene_desc sd{};
    sd.meshes = meshes;
    sd.num_meshes = info.num_meshes;
    sd.has_env = info.has_env;
    std::memcpy(sd.env, info.env, sizeof(sd.env));
    pt_scene* scene = nullptr;
    const int rc = pt_scene_create(&sd, &scene);  // the SAH build (identical to the reference's) + upload
    pt_pbrt_free(file);
    if (rc != PT_OK) return fail("pt_scene_create");
    const auto t1 = std::chrono::steady_clock::now();

    pt_render_desc rd{};
    rd.width = info.width;
    rd.height = info.height;
    rd.spp = info.spp;
    rd.max_depth = info.max_depth;
    rd.seed = seed;
    rd.flags = flags;
    rd.camera = info.camera;
    std::vector<float> rgb(3 * (size_t)rd.width * rd.height);
    if (pt_render(scene, &rd, rgb.data(), nullptr, 0, nullptr) != PT_OK) return fail("pt_render");
    const auto t2 = std::chrono::steady_clock::now();

    // PNGFilm::Output's bytes, then the file
    std::vector<uint8_t> rgba(4 * (size_t)rd.width * rd.height);
    for (size_t p = 0; p < (size_t)rd.width * rd.height; ++p) {
        for (int c = 0; c < 3; ++c) {
            const float v = rgb[3 * p + c];
            rgba[4 * p + c] = (uint8_t)(v > 255.f ? 255.f : (v > 0.f ? v : 0.f));
        }
        rgba[4 * p + 3] = 255;
    }
    if (pt_write_png(argv[2], rgba.data(), rd.width, rd.height) != PT_OK) return fail("pt_write_png");
    pt_scene_destroy(scene);
    const double load_s = std::chrono::duration<double>(t1 - t0).count();
    const double render_s = std::chrono::duration<double>(t2 - t1).count();
    std::printf("%u meshes, %ux%u, %u spp, depth %u: scene %.3f s, render %.3f s -> %s\n", info.num_meshes, rd.width,
                rd.height, rd.spp, rd.max_depth, load_s, render_s, argv[2]);
    return 0;
}
