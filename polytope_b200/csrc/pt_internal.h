// pt_internal.h -- host-side internals shared by the C++ and CUDA translation units.
#pragma once

#include <cstdint>
#include <cstddef>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/polytope_b200.h"
#include "config.h"
#include "instance.h"

#define PT_RAY_COUNTERS 256

namespace pt {

// ---- error state ------------------------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);  // sets the message, returns code

// ---- host BVH build (identical to the reference) ------------------------------------------------
// Runs f(begin, end) over [0, n) split into contiguous ranges, one per thread (threads <= 0: one
// per hardware thread), on the calling thread alone when the work is small.  Host-side helper for
// per-element loops whose elements are independent.
template <class F>
void parallel_ranges(size_t n, int threads, F f) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    if (threads == 1 || n < 65536) {
        f((size_t)0, n);
        return;
    }
    const size_t chunk = (n + (size_t)threads - 1) / (size_t)threads;
    std::vector<std::thread> pool;
    for (size_t b = 0; b < n; b += chunk) pool.emplace_back(f, b, std::min(n, b + chunk));
    for (std::thread& t : pool) t.join();
}

struct WorldMeshes {
    // world-space triangle of each global primitive id (9 floats), owning mesh and face
    std::vector<float> tri;        // 9 * num_prims
    std::vector<uint32_t> prim_mesh;
    std::vector<uint32_t> prim_base;  // per mesh
    uint32_t num_prims = 0;
};

// Applies each mesh's object_to_world to its packed vertices exactly as
// Transform::ApplyInPlace(Point&) does (Transform.cpp:69-91).
void apply_point(const float* m, float p[3]);
void apply_normal(const float* inv, float n[3]);
int bake_world(const pt_mesh_desc* meshes, uint32_t num_meshes, WorldMeshes& out);

struct BuiltTree {
    std::vector<pt_bvh_node> nodes;
    std::vector<uint32_t> leaf_pairs;  // 2 per leaf-ordered entry: (mesh, face)
    uint32_t max_depth = 0;
};
int build_bvh(const pt_mesh_desc* meshes, uint32_t num_meshes, const WorldMeshes& w, int threads, BuiltTree& out);

// Ray queries behind pt_trace / pt_trace_counted (abi.cpp).
int scene_trace(pt_scene* s, const pt_ray* rays, uint64_t n, pt_hit* hits, uint32_t* node_tests,
                uint32_t* tri_tests, uint32_t mem_flags, void* stream);

// Checks that every child / leaf range stays inside the arrays and computes the deepest level.
int validate_tree(const pt_bvh_node* nodes, uint32_t num_nodes, uint32_t num_leaf_entries, uint32_t* max_depth);

// ---- device scene -------------------------------------------------------------------------------
struct DeviceMesh {  // per-mesh shading record (device)
    uint32_t material;
    int32_t is_light;
    float albedo[3];
    float emission[3];
    int32_t has_normals;  // the mesh has vertex normals (mesh_geometry::has_vertex_normals)
};

struct HostScene {  // host copy of everything a scene handle uploads
    std::vector<pt_bvh_node> nodes;
    std::vector<float> tris;          // 12 floats per leaf-ordered face
    std::vector<DeviceMesh> meshes;
    std::vector<float> normals;       // 9 floats per prim, empty without vertex normals
    std::vector<float> light_tris;    // 12 floats per light face
    std::vector<float> light_cdf;
    float light_area = 0.f;
    uint32_t num_prims = 0;
    uint32_t max_depth = 0;
    std::vector<uint32_t> prim_base;
    // two-level layout (pt_scene_create_two_level): `nodes` / `tris` then hold every distinct
    // geometry's object-space tree and faces back to back, and these the instances and the top
    // level over their world boxes
    bool two_level = false;
    std::vector<DeviceInstance> instances;
    std::vector<pt_bvh_node> tlas;
    uint32_t tlas_depth = 0;
    uint32_t num_geometries = 0;
};
int prepare_scene_host(const pt_scene_desc* desc, HostScene& out);
// The two-level layout of a scene description (tlas.cpp); shading data as prepare_scene_host.
int prepare_two_level_host(const pt_scene_desc* desc, HostScene& out);
// Shading records, world vertex normals and the area-light table of a scene (abi.cpp), shared by
// both layouts.
void prepare_shading_host(const pt_scene_desc* desc, const WorldMeshes& w, HostScene& h);

struct SceneDev {
    // traversal data
    void* nodes = nullptr;        // num_nodes * 32 B  (pt_bvh_node)
    void* tris = nullptr;         // num_prims * 48 B  (3 x float4 per leaf-ordered entry)
    // shading data
    void* meshes = nullptr;       // num_meshes * DeviceMesh
    void* prim_normals = nullptr; // num_prims * 9 floats (world vertex normals by prim id) or null
    void* prim_tri = nullptr;     // num_prims * 9 floats world triangle by prim id
    void* light_tris = nullptr;   // num_lights * 12 floats: v0, v1, v2, then (prim, mesh, 0, 0)
    void* light_cdf = nullptr;    // num_lights floats
    uint32_t num_lights = 0;
    float light_area = 0.f;
    // two-level scenes only
    void* instances = nullptr;    // num_instances * DeviceInstance, in top-level leaf order
    void* tlas_nodes = nullptr;   // tlas_num_nodes * 32 B
    uint32_t num_instances = 0;
    uint32_t tlas_num_nodes = 0;
};

}  // namespace pt

struct pt_scene {
    pt::SceneDev dev;
    uint32_t num_nodes = 0;
    uint32_t num_prims = 0;
    uint32_t num_meshes = 0;
    uint32_t max_depth = 0;
    uint64_t device_bytes = 0;
    int device = 0;
    int has_env = 0;
    float env[3] = {0.f, 0.f, 0.f};
    bool has_normals = false;
    std::vector<uint32_t> prim_base;
    // staging for host-pointer calls (lazily allocated, guarded by staging_mu)
    std::mutex staging_mu;
    void* pin_in = nullptr;
    void* pin_out = nullptr;
    void* dev_in = nullptr;
    void* dev_out = nullptr;
    size_t staging_rays = 0;
    void* streams[4] = {};  // host-pointer traces: copies in, two kernel streams, copies out
    void* events[16] = {};
    // device ints set when a kernel hits a guard: err_flag by the asynchronous (device-memory)
    // calls, cleared when pt_scene_status reports it; trace_err by the host-memory pt_trace call
    // that holds staging_mu
    void* err_flag = nullptr;
    void* trace_err = nullptr;
    bool two_level = false;  // made by pt_scene_create_two_level
    bool nan_boxes = false;  // some tree box holds a NaN (every ray then takes the exact box test)
    // ray counters of the persistent trace kernel: one per launch in flight, taken round-robin
    void* ray_counters = nullptr;
    std::atomic<uint32_t> counter_next{0};
    pt_trace_tuning trace_tuning{16, 64};
};
