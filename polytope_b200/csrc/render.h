// render.h -- path-tracer structures shared by the host orchestration and the kernels.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/polytope_b200.h"

namespace pt {

struct CameraConst {
    float m[16];          // CameraToWorld.Matrix (row-major)
    float one_over_w, one_over_h, aspect, tan_half;
    float org[3];         // world-space ray origin
};

CameraConst make_camera(const pt_camera& c, uint32_t width, uint32_t height);

// Everything a path needs, by value in kernel parameter space.
struct RenderParams {
    const void* nodes;        // uint4 x 2 per node
    const void* tris;         // float4 x 3 per leaf-ordered face
    uint32_t num_nodes;
    const void* meshes;       // DeviceMesh per mesh
    const float* prim_normals;  // 9 floats per prim or null
    const float* light_tris;  // 12 floats per light face
    const float* light_cdf;
    uint32_t num_lights;
    float light_area;
    int has_env;
    float env[3];
    CameraConst cam;
    uint32_t width, height, spp, max_depth;
    uint32_t seed_lo, seed_hi;
    uint32_t flags;
    int* err;
    unsigned long long* rays_traced;  // optional: counts camera + bounce + shadow rays
    // two-level scenes (pt_scene_create_two_level): instances (DeviceInstance, top-level leaf
    // order) and the top-level tree; null for a flattened scene, whose nodes / tris are world space
    const void* instances;
    const void* top_nodes;
    uint32_t top_num_nodes;
    uint32_t exact_tree;  // some tree box holds a NaN: every ray takes the exact box test
};

// Paths [first, first + count) in sample-major order (path p = sample * W*H + pixel).
cudaError_t launch_path_wave(const RenderParams& p, uint64_t first, uint32_t count, float* radiance,
                             uint32_t* primary, cudaStream_t s);
// film_sum[pixel] += radiance of that pixel's samples inside the wave, in sample order.
cudaError_t launch_resolve_wave(uint64_t first, uint32_t count, uint32_t num_pixels, const float* radiance,
                                float* film_sum, cudaStream_t s);
cudaError_t launch_finish_film(const float* film_sum, uint32_t num_pixels, uint32_t spp, float* rgb, cudaStream_t s);
// rgb (3 floats per pixel) -> RGBA8 as PNGFilm::Output stores it (output.cu).
cudaError_t launch_film_to_rgba8(const float* rgb, uint32_t num_pixels, uint8_t* rgba, cudaStream_t s);

}  // namespace pt

struct pt_scene;
namespace pt {
RenderParams render_params(const pt_scene* s, const pt_render_desc* desc);
int check_render_desc(const pt_scene* s, const pt_render_desc* desc);

}  // namespace pt
