// abi.cpp -- the C ABI (include/polytope_b200.h): scene upload, ray queries, error reporting.

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "exact_math.h"
#include "launch.h"
#include "pt_internal.h"

namespace pt {

namespace {
thread_local std::string g_last_error;

struct DeviceGuard {  // makes `dev` current for the scope and restores the caller's device
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int cuda_fail(cudaError_t e, const char* what) {
    return fail(PT_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define PT_CUDA(call)                                     \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

template <class T>
int upload(void** dst, const T* src, size_t count, uint64_t& bytes) {
    const size_t nb = sizeof(T) * count;
    if (nb == 0) { *dst = nullptr; return PT_OK; }
    cudaError_t e = cudaMalloc(dst, nb);
    if (e != cudaSuccess) return fail(PT_ENOMEM, std::string("cudaMalloc scene buffer: ") + cudaGetErrorString(e));
    bytes += nb;
    e = cudaMemcpy(*dst, src, nb, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy scene buffer");
    return PT_OK;
}

void free_scene(pt_scene* s) {
    if (!s) return;
    DeviceGuard g(s->device);
    void* bufs[] = {s->dev.nodes, s->dev.tris, s->dev.meshes, s->dev.prim_normals, s->dev.prim_tri,
                    s->dev.light_tris, s->dev.light_cdf, s->dev.instances, s->dev.tlas_nodes, s->dev_in, s->dev_out,
                    s->err_flag, s->trace_err, s->ray_counters};
    for (void* b : bufs)
        if (b) cudaFree(b);
    if (s->pin_in) cudaFreeHost(s->pin_in);
    if (s->pin_out) cudaFreeHost(s->pin_out);
    for (void*& st : s->streams)
        if (st) cudaStreamDestroy((cudaStream_t)st);
    for (void*& ev : s->events)
        if (ev) cudaEventDestroy((cudaEvent_t)ev);
    delete s;
}

bool is_pinned(const void* p) {
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeHost;
}

// Rays per chunk of the host-pointer pipeline.  Measured on the 16.7 M-ray microbench end to end:
// 1 M-ray chunks 1436 Mrays/s, 512 K 1413, 2 M 1339 (longer fill and drain), 256 K 1030.
constexpr size_t kChunkRays = size_t(1) << 20;
constexpr int kSlots = 4;  // chunks in flight: one being copied in, one or two in kernels, one copied out

int ensure_staging(pt_scene* s) {
    if (s->staging_rays) return PT_OK;
    for (int i = 0; i < 4; ++i) {
        PT_CUDA(cudaStreamCreateWithFlags((cudaStream_t*)&s->streams[i], cudaStreamNonBlocking));
    }
    for (int i = 0; i < 3 * kSlots + 1; ++i)
        PT_CUDA(cudaEventCreateWithFlags((cudaEvent_t*)&s->events[i], cudaEventDisableTiming));
    const size_t in_b = kSlots * kChunkRays * sizeof(pt_ray), out_b = kSlots * kChunkRays * sizeof(pt_hit);
    if (cudaMalloc(&s->dev_in, in_b) != cudaSuccess || cudaMalloc(&s->dev_out, out_b) != cudaSuccess ||
        cudaMalloc(&s->trace_err, sizeof(int)) != cudaSuccess)
        return fail(PT_ENOMEM, "cudaMalloc staging buffers");
    if (cudaMallocHost(&s->pin_in, in_b) != cudaSuccess || cudaMallocHost(&s->pin_out, out_b) != cudaSuccess)
        return fail(PT_ENOMEM, "cudaMallocHost staging buffers");
    s->staging_rays = kChunkRays;
    return PT_OK;
}

}  // namespace

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int scene_trace(pt_scene* s, const pt_ray* rays, uint64_t n, pt_hit* hits, uint32_t* node_tests, uint32_t* tri_tests,
                uint32_t mem_flags, void* stream) {
    if (!s) return fail(PT_EINVAL, "scene is NULL");
    if (n == 0) return PT_OK;
    if (!rays || !hits) return fail(PT_EINVAL, "rays or hits is NULL");
    if ((int)s->max_depth + 2 > PT_TRAVERSAL_STACK)
        return fail(PT_ESTACK, "tree depth " + std::to_string(s->max_depth) + " exceeds the traversal stack");
    DeviceGuard g(s->device);
    TraceArgs a{};
    a.nodes = s->dev.nodes;
    a.tris = s->dev.tris;
    a.num_nodes = s->num_nodes;
    a.err = (int*)s->err_flag;
    a.shared_stack = (int)s->trace_tuning.shared_stack;
    a.chunk = s->trace_tuning.queue_chunk;
    a.instances = s->dev.instances;
    a.top_nodes = s->dev.tlas_nodes;
    a.top_num_nodes = s->dev.tlas_num_nodes;
    a.exact_tree = s->nan_boxes;
    auto next_counter = [s]() {
        return (void*)((unsigned long long*)s->ray_counters + (s->counter_next.fetch_add(1) % PT_RAY_COUNTERS));
    };
    if (mem_flags & PT_MEM_DEVICE) {
        a.counter = next_counter();
        a.rays = rays;
        a.hits = hits;
        a.n = n;
        a.node_tests = node_tests;
        a.tri_tests = tri_tests;
        cudaError_t e = launch_trace(a, (cudaStream_t)stream);
        if (e != cudaSuccess) return cuda_fail(e, "trace kernel launch");
        return PT_OK;
    }
    // Host pointers: 1 M-ray chunks through kSlots staging slots and three engines at once -- a
    // stream of host->device copies, two kernel streams (so one chunk's kernel tail overlaps the
    // next), and a stream of device->host copies -- ordered per slot by events.  Pageable arrays
    // go through the pinned staging of their slot.
    std::lock_guard<std::mutex> lock(s->staging_mu);
    int rc = ensure_staging(s);
    if (rc) return rc;
    cudaStream_t h2d = (cudaStream_t)s->streams[0], d2h = (cudaStream_t)s->streams[3];
    cudaStream_t kst[2] = {(cudaStream_t)s->streams[1], (cudaStream_t)s->streams[2]};
    cudaEvent_t* ev = (cudaEvent_t*)s->events;
    cudaEvent_t *ev_in = ev, *ev_k = ev + kSlots, *ev_out = ev + 2 * kSlots, dep = ev[3 * kSlots];
    PT_CUDA(cudaEventRecord(dep, (cudaStream_t)stream));
    for (int i = 0; i < 4; ++i) PT_CUDA(cudaStreamWaitEvent((cudaStream_t)s->streams[i], dep, 0));
    a.err = (int*)s->trace_err;  // this call's own flag: the asynchronous calls raise err_flag
    PT_CUDA(cudaMemsetAsync(s->trace_err, 0, sizeof(int), h2d));  // before every copy-in, so before every kernel
    const bool pin_rays = is_pinned(rays), pin_hits = is_pinned(hits);
    const bool counted = node_tests || tri_tests;
    uint32_t* dcounts = nullptr;
    if (counted && cudaMalloc(&dcounts, 2 * sizeof(uint32_t) * n) != cudaSuccess)
        return fail(PT_ENOMEM, "cudaMalloc count buffers");
    struct Free { uint32_t* p; ~Free() { if (p) cudaFree(p); } } free_counts{dcounts};
    // Chunks: full slots in the middle, and a quarter then a half slot at both ends on long calls.
    // The kernels wait for the first chunk's copy-in, and the last chunk's kernel and copy-out are
    // all that runs after the final copy-in: short end chunks shorten both waits.
    std::vector<std::pair<uint64_t, uint64_t>> chunks;  // (first ray, count)
    if (n >= 4 * (uint64_t)kChunkRays) {
        const uint64_t q = kChunkRays / 4, h = kChunkRays / 2;
        chunks.push_back({0, q});
        chunks.push_back({q, h});
        uint64_t off = q + h;
        while (n - off > h + q) {
            const uint64_t cnt = std::min<uint64_t>(kChunkRays, n - off - (h + q));
            chunks.push_back({off, cnt});
            off += cnt;
        }
        chunks.push_back({off, h});
        chunks.push_back({off + h, q});
    } else {
        for (uint64_t off = 0; off < n; off += kChunkRays) chunks.push_back({off, std::min<uint64_t>(kChunkRays, n - off)});
    }
    const uint64_t nchunks = chunks.size();
    uint64_t in_slot[kSlots];
    for (int k = 0; k < kSlots; ++k) in_slot[k] = ~0ull;  // chunk whose data occupies each slot
    auto drain = [&](int slot) -> int {  // pageable hits: move the slot's results out
        if (in_slot[slot] == ~0ull) return PT_OK;
        PT_CUDA(cudaEventSynchronize(ev_out[slot]));
        if (!pin_hits) {
            const uint64_t off = chunks[in_slot[slot]].first, cnt = chunks[in_slot[slot]].second;
            std::memcpy(hits + off, (pt_hit*)s->pin_out + slot * kChunkRays, cnt * sizeof(pt_hit));
        }
        in_slot[slot] = ~0ull;
        return PT_OK;
    };
    for (uint64_t c = 0; c < nchunks; ++c) {
        const int slot = (int)(c % kSlots);
        const bool reused = in_slot[slot] != ~0ull;
        if (reused && !pin_hits) {
            rc = drain(slot);
            if (rc) return rc;
        }
        const uint64_t off = chunks[c].first, cnt = chunks[c].second;
        pt_ray* din = (pt_ray*)s->dev_in + slot * kChunkRays;
        pt_hit* dout = (pt_hit*)s->dev_out + slot * kChunkRays;
        const void* src = rays + off;
        if (!pin_rays) {
            if (reused) PT_CUDA(cudaEventSynchronize(ev_in[slot]));  // the slot's previous copy-in has read it
            std::memcpy((pt_ray*)s->pin_in + slot * kChunkRays, rays + off, cnt * sizeof(pt_ray));
            src = (pt_ray*)s->pin_in + slot * kChunkRays;
        }
        if (reused) PT_CUDA(cudaStreamWaitEvent(h2d, ev_k[slot], 0));  // din is free once its kernel ran
        PT_CUDA(cudaMemcpyAsync(din, src, cnt * sizeof(pt_ray), cudaMemcpyHostToDevice, h2d));
        PT_CUDA(cudaEventRecord(ev_in[slot], h2d));
        cudaStream_t k = kst[c & 1];
        PT_CUDA(cudaStreamWaitEvent(k, ev_in[slot], 0));
        if (reused) PT_CUDA(cudaStreamWaitEvent(k, ev_out[slot], 0));  // dout is free once copied out
        a.rays = din;
        a.hits = dout;
        a.n = cnt;
        a.counter = next_counter();
        a.node_tests = counted ? dcounts + off : nullptr;
        a.tri_tests = counted ? dcounts + n + off : nullptr;
        cudaError_t e = launch_trace(a, k);
        if (e != cudaSuccess) return cuda_fail(e, "trace kernel launch");
        PT_CUDA(cudaEventRecord(ev_k[slot], k));
        PT_CUDA(cudaStreamWaitEvent(d2h, ev_k[slot], 0));
        void* dst = pin_hits ? (void*)(hits + off) : (void*)((pt_hit*)s->pin_out + slot * kChunkRays);
        PT_CUDA(cudaMemcpyAsync(dst, dout, cnt * sizeof(pt_hit), cudaMemcpyDeviceToHost, d2h));
        PT_CUDA(cudaEventRecord(ev_out[slot], d2h));
        in_slot[slot] = c;
    }
    for (uint64_t c = nchunks > kSlots ? nchunks - kSlots : 0; c < nchunks; ++c) {
        rc = drain((int)(c % kSlots));
        if (rc) return rc;
    }
    PT_CUDA(cudaStreamSynchronize(d2h));
    if (counted) {
        std::vector<uint32_t> tmp(2 * n);
        PT_CUDA(cudaMemcpy(tmp.data(), dcounts, 2 * n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        if (node_tests) std::memcpy(node_tests, tmp.data(), n * sizeof(uint32_t));
        if (tri_tests) std::memcpy(tri_tests, tmp.data() + n, n * sizeof(uint32_t));
    }
    int err = 0;
    PT_CUDA(cudaMemcpy(&err, s->trace_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return fail(PT_ESTACK, "a ray exceeded the traversal stack (malformed or too deep tree)");
    return PT_OK;
}


// Host-side layout of a scene (everything pt_scene_create uploads).
int prepare_scene_host(const pt_scene_desc* desc, HostScene& h) {
    if (!desc->meshes || desc->num_meshes == 0) return fail(PT_EINVAL, "scene has no meshes");
    for (uint32_t m = 0; m < desc->num_meshes; ++m) {
        const pt_mesh_desc& d = desc->meshes[m];
        if (d.material != PT_MAT_LAMBERT && d.material != PT_MAT_MIRROR)
            return fail(PT_EINVAL, "mesh " + std::to_string(m) + ": unknown material");
    }
    WorldMeshes w;
    int rc = bake_world(desc->meshes, desc->num_meshes, w);
    if (rc) return rc;
    BuiltTree t;
    if (desc->nodes) {
        if (!desc->leaf_pairs) return fail(PT_EINVAL, "nodes given without leaf_pairs");
        t.nodes.assign(desc->nodes, desc->nodes + desc->num_nodes);
        t.leaf_pairs.assign(desc->leaf_pairs, desc->leaf_pairs + 2 * (size_t)w.num_prims);
        for (size_t i = 0; i < w.num_prims; ++i) {
            const uint32_t m = t.leaf_pairs[2 * i], f = t.leaf_pairs[2 * i + 1];
            if (m >= desc->num_meshes || f >= desc->meshes[m].num_faces)
                return fail(PT_EINVAL, "leaf pair " + std::to_string(i) + " out of range");
        }
    } else {
        rc = build_bvh(desc->meshes, desc->num_meshes, w, 0, t);
        if (rc) return rc;
    }
    rc = validate_tree(t.nodes.data(), (uint32_t)t.nodes.size(), w.num_prims, &h.max_depth);
    if (rc) return rc;
    h.num_prims = w.num_prims;
    h.prim_base = w.prim_base;
    h.nodes.swap(t.nodes);
    // faces in leaf order, 48 B each: {v0.xyz v1.x}{v1.yz v2.xy}{v2.z prim mesh 0}
    h.tris.assign(12 * (size_t)w.num_prims, 0.f);
    for (size_t i = 0; i < w.num_prims; ++i) {
        const uint32_t m = t.leaf_pairs[2 * i], f = t.leaf_pairs[2 * i + 1];
        const uint32_t p = w.prim_base[m] + f;
        float* o = &h.tris[12 * i];
        std::memcpy(o, &w.tri[9 * (size_t)p], 9 * sizeof(float));
        o[9] = bitsf(p);
        o[10] = bitsf(m);
    }
    prepare_shading_host(desc, w, h);
    return PT_OK;
}

void prepare_shading_host(const pt_scene_desc* desc, const WorldMeshes& w, HostScene& h) {
    h.meshes.resize(desc->num_meshes);
    bool any_normals = false;
    for (uint32_t m = 0; m < desc->num_meshes; ++m) {
        const pt_mesh_desc& d = desc->meshes[m];
        h.meshes[m].material = d.material;
        h.meshes[m].is_light = d.is_light ? 1 : 0;
        std::memcpy(h.meshes[m].albedo, d.albedo, sizeof(d.albedo));
        std::memcpy(h.meshes[m].emission, d.emission, sizeof(d.emission));
        h.meshes[m].has_normals = (d.nx && d.ny && d.nz) ? 1 : 0;
        if (h.meshes[m].has_normals) any_normals = true;
    }
    if (any_normals) {  // world vertex normals per prim (Transform::ApplyInPlace(Normal&), mesh.cpp:388-400)
        h.normals.assign(9 * (size_t)w.num_prims, 0.f);
        for (uint32_t m = 0; m < desc->num_meshes; ++m) {
            const pt_mesh_desc& d = desc->meshes[m];
            if (!(d.nx && d.ny && d.nz)) continue;
            for (uint32_t f = 0; f < d.num_faces; ++f) {
                const uint32_t vi[3] = {d.fv0[f], d.fv1[f], d.fv2[f]};
                float* o = &h.normals[9 * (size_t)(w.prim_base[m] + f)];
                for (int k = 0; k < 3; ++k) {
                    o[3 * k] = d.nx[vi[k]];
                    o[3 * k + 1] = d.ny[vi[k]];
                    o[3 * k + 2] = d.nz[vi[k]];
                    apply_normal(d.world_to_object, &o[3 * k]);
                }
            }
        }
    }
    // area lights (every face of an emitting mesh, mesh/face order): world triangle, then the
    // running sum of 0.5 * |(v1 - v0) x (v2 - v0)| as the CDF
    h.light_area = 0.f;
    for (uint32_t p = 0; p < w.num_prims; ++p) {
        const uint32_t m = w.prim_mesh[p];
        if (!desc->meshes[m].is_light) continue;
        const float* v = &w.tri[9 * (size_t)p];
        const float e0[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]};
        const float e1[3] = {v[6] - v[0], v[7] - v[1], v[8] - v[2]};
        const float c[3] = {e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0]};
        const float area = 0.5f * std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        h.light_area = h.light_area + area;
        for (int k = 0; k < 9; ++k) h.light_tris.push_back(v[k]);
        h.light_tris.push_back(bitsf(p));  // 12 floats per record: v0 v1 v2, prim, mesh, pad
        h.light_tris.push_back(bitsf(m));
        h.light_tris.push_back(0.f);
        h.light_cdf.push_back(h.light_area);
    }
}

}  // namespace pt

using namespace pt;

extern "C" {

const char* pt_last_error(void) { return g_last_error.c_str(); }
const char* pt_version(void) { return "polytope_b200 0.1 (sm_100a)"; }

int pt_bvh_build(const pt_mesh_desc* meshes, uint32_t num_meshes, int threads, pt_bvh_node* nodes_out,
                 uint32_t* num_nodes_out, uint32_t* leaf_pairs_out) {
    if (!meshes || num_meshes == 0) return fail(PT_EINVAL, "no meshes");
    if (!num_nodes_out) return fail(PT_EINVAL, "num_nodes_out is NULL");
    WorldMeshes w;
    int rc = bake_world(meshes, num_meshes, w);
    if (rc) return rc;
    BuiltTree t;
    rc = build_bvh(meshes, num_meshes, w, threads, t);
    if (rc) return rc;
    if (!nodes_out) {
        *num_nodes_out = (uint32_t)t.nodes.size();
        return PT_OK;
    }
    if (*num_nodes_out < t.nodes.size()) return fail(PT_EINVAL, "nodes_out too small");
    std::memcpy(nodes_out, t.nodes.data(), t.nodes.size() * sizeof(pt_bvh_node));
    *num_nodes_out = (uint32_t)t.nodes.size();
    if (leaf_pairs_out) std::memcpy(leaf_pairs_out, t.leaf_pairs.data(), t.leaf_pairs.size() * sizeof(uint32_t));
    return PT_OK;
}

}  // extern "C"

namespace {
int device_count_ok() {
    int ndev = 0;
    cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(PT_ECUDA, "no CUDA device available (there is no CPU fallback)");
    }
    return PT_OK;
}

// Uploads a prepared scene (either layout) into a new handle.
int create_from_host(const pt_scene_desc* desc, HostScene& h, pt_scene** out) {
    int rc = PT_OK;
    std::unique_ptr<pt_scene> s(new pt_scene());
    cudaGetDevice(&s->device);
    s->num_nodes = (uint32_t)h.nodes.size();
    s->num_prims = h.num_prims;
    s->num_meshes = desc->num_meshes;
    s->max_depth = h.max_depth;
    s->prim_base = h.prim_base;
    s->has_env = desc->has_env;
    std::memcpy(s->env, desc->env, sizeof(s->env));
    s->has_normals = !h.normals.empty();
    s->dev.num_lights = (uint32_t)h.light_cdf.size();
    s->dev.light_area = h.light_area;

    DeviceGuard g(s->device);
    uint64_t bytes = 0;
    if ((rc = upload(&s->dev.nodes, h.nodes.data(), h.nodes.size(), bytes))) { free_scene(s.release()); return rc; }
    if ((rc = upload(&s->dev.tris, h.tris.data(), h.tris.size(), bytes))) { free_scene(s.release()); return rc; }
    if ((rc = upload(&s->dev.meshes, h.meshes.data(), h.meshes.size(), bytes))) { free_scene(s.release()); return rc; }
    if ((rc = upload(&s->dev.prim_normals, h.normals.data(), h.normals.size(), bytes))) { free_scene(s.release()); return rc; }
    if ((rc = upload(&s->dev.light_tris, h.light_tris.data(), h.light_tris.size(), bytes))) { free_scene(s.release()); return rc; }
    if ((rc = upload(&s->dev.light_cdf, h.light_cdf.data(), h.light_cdf.size(), bytes))) { free_scene(s.release()); return rc; }
    if (cudaMalloc(&s->err_flag, sizeof(int)) != cudaSuccess) { free_scene(s.release()); return fail(PT_ENOMEM, "cudaMalloc error flag"); }
    cudaMemset(s->err_flag, 0, sizeof(int));
    if (cudaMalloc(&s->ray_counters, 8 * PT_RAY_COUNTERS) != cudaSuccess) { free_scene(s.release()); return fail(PT_ENOMEM, "cudaMalloc ray counters"); }
    auto has_nan = [](const std::vector<pt_bvh_node>& nodes) {
        for (const pt_bvh_node& n : nodes)
            for (int k = 0; k < 3; ++k)
                if (n.bb_min[k] != n.bb_min[k] || n.bb_max[k] != n.bb_max[k]) return true;
        return false;
    };
    s->nan_boxes = has_nan(h.nodes) || has_nan(h.tlas);
    if (h.two_level) {
        s->two_level = true;
        s->dev.num_instances = (uint32_t)h.instances.size();
        s->dev.tlas_num_nodes = (uint32_t)h.tlas.size();
        if ((rc = upload(&s->dev.instances, h.instances.data(), h.instances.size(), bytes))) { free_scene(s.release()); return rc; }
        if ((rc = upload(&s->dev.tlas_nodes, h.tlas.data(), h.tlas.size(), bytes))) { free_scene(s.release()); return rc; }
    }
    s->device_bytes = bytes;
    *out = s.release();
    return PT_OK;
}
}  // namespace

extern "C" {

int pt_scene_create(const pt_scene_desc* desc, pt_scene** out) {
    if (!desc || !out) return fail(PT_EINVAL, "desc or out is NULL");
    *out = nullptr;
    int rc = device_count_ok();
    if (rc) return rc;
    HostScene h;
    rc = prepare_scene_host(desc, h);
    if (rc) return rc;
    return create_from_host(desc, h, out);
}

int pt_scene_create_two_level(const pt_scene_desc* desc, pt_scene** out) {
    if (!desc || !out) return fail(PT_EINVAL, "desc or out is NULL");
    *out = nullptr;
    int rc = device_count_ok();
    if (rc) return rc;
    HostScene h;
    rc = prepare_two_level_host(desc, h);
    if (rc) return rc;
    if (h.tlas_depth + 2 > (uint32_t)PT_TOP_STACK) return fail(PT_ESTACK, "top-level tree too deep");
    // the persistent path kernel keeps both levels and the instance-exit marker on one stack
    if (h.tlas_depth + h.max_depth + 4 > (uint32_t)PT_TRAVERSAL_STACK)
        return fail(PT_ESTACK, "top-level plus bottom-level tree depth exceeds the traversal stack");
    return create_from_host(desc, h, out);
}

int pt_two_level_plan(const pt_scene_desc* desc, pt_two_level_info* info) {
    if (!desc || !info) return fail(PT_EINVAL, "desc or info is NULL");
    HostScene h;
    int rc = prepare_two_level_host(desc, h);
    if (rc) return rc;
    info->num_instances = (uint32_t)h.instances.size();
    info->num_geometries = h.num_geometries;
    info->blas_nodes = (uint32_t)h.nodes.size();
    info->blas_faces = (uint32_t)(h.tris.size() / 12);
    info->tlas_nodes = (uint32_t)h.tlas.size();
    info->max_depth = h.max_depth;
    info->tlas_depth = h.tlas_depth;
    info->num_prims = h.num_prims;
    info->device_bytes = sizeof(pt_bvh_node) * (uint64_t)h.nodes.size() + 4ull * h.tris.size() +
                         sizeof(DeviceMesh) * (uint64_t)h.meshes.size() + 4ull * h.normals.size() +
                         4ull * h.light_tris.size() + 4ull * h.light_cdf.size() +
                         sizeof(DeviceInstance) * (uint64_t)h.instances.size() + sizeof(pt_bvh_node) * (uint64_t)h.tlas.size();
    return PT_OK;
}

int pt_scene_destroy(pt_scene* scene) {
    if (!scene) return PT_OK;
    free_scene(scene);
    return PT_OK;
}

int pt_scene_get_info(const pt_scene* s, pt_scene_info* info) {
    if (!s || !info) return fail(PT_EINVAL, "scene or info is NULL");
    info->num_nodes = s->num_nodes;
    info->num_prims = s->num_prims;
    info->num_meshes = s->num_meshes;
    info->max_depth = s->max_depth;
    info->device_bytes = s->device_bytes;
    return PT_OK;
}

int pt_trace(pt_scene* scene, const pt_ray* rays, uint64_t n, pt_hit* hits, uint32_t mem_flags, void* stream) {
    return scene_trace(scene, rays, n, hits, nullptr, nullptr, mem_flags, stream);
}

int pt_trace_counted(pt_scene* scene, const pt_ray* rays, uint64_t n, pt_hit* hits, uint32_t* node_tests,
                     uint32_t* tri_tests, uint32_t mem_flags, void* stream) {
    if (!node_tests && !tri_tests) return fail(PT_EINVAL, "no count outputs");
    return scene_trace(scene, rays, n, hits, node_tests, tri_tests, mem_flags, stream);
}

int pt_scene_set_trace_tuning(pt_scene* scene, const pt_trace_tuning* t) {
    if (!scene || !t) return fail(PT_EINVAL, "scene or tuning is NULL");
    if (t->shared_stack > 32 || (t->shared_stack & 7u))
        return fail(PT_EINVAL, "shared_stack must be 0, 8, 16, 24 or 32");
    if (t->queue_chunk < 32 || t->queue_chunk > 4096 || (t->queue_chunk & 31u))
        return fail(PT_EINVAL, "queue_chunk must be a multiple of 32 in [32, 4096]");
    scene->trace_tuning = *t;
    return PT_OK;
}

int pt_scene_get_trace_tuning(const pt_scene* scene, pt_trace_tuning* t) {
    if (!scene || !t) return fail(PT_EINVAL, "scene or tuning is NULL");
    *t = scene->trace_tuning;
    return PT_OK;
}

int pt_trace_autotune(pt_scene* scene, const pt_ray* rays_dev, uint64_t n, pt_hit* hits_dev, pt_trace_tuning* best,
                      float* best_ms) {
    if (!scene || !rays_dev || !hits_dev || !n) return fail(PT_EINVAL, "scene, rays or hits is NULL");
    const pt_trace_tuning saved = scene->trace_tuning;
    pt_trace_tuning cur = saved;
    float cur_ms = 1e30f;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto time_it = [&](const pt_trace_tuning& t, float& ms) -> int {
        scene->trace_tuning = t;
        int rc = pt_trace(scene, rays_dev, n, hits_dev, PT_MEM_DEVICE, nullptr);  // warm-up
        if (rc) return rc;
        ms = 1e30f;
        for (int r = 0; r < 5; ++r) {  // fastest of five single launches: robust to a noisy neighbour
            cudaEventRecord(e0, 0);
            if ((rc = pt_trace(scene, rays_dev, n, hits_dev, PT_MEM_DEVICE, nullptr))) return rc;
            cudaEventRecord(e1, 0);
            cudaEventSynchronize(e1);
            float one = 0.f;
            cudaEventElapsedTime(&one, e0, e1);
            ms = std::min(ms, one);
        }
        return PT_OK;
    };
    int rc = PT_OK;
    for (uint32_t sh : {0u, 8u, 16u, 24u, 32u}) {
        pt_trace_tuning t = cur;
        t.shared_stack = sh;
        float ms = 0.f;
        if ((rc = time_it(t, ms))) break;
        if (ms < cur_ms) { cur_ms = ms; cur = t; }
    }
    for (uint32_t ch : {32u, 64u, 128u, 256u}) {
        if (rc) break;
        pt_trace_tuning t = cur;
        t.queue_chunk = ch;
        float ms = 0.f;
        if ((rc = time_it(t, ms))) break;
        if (ms < cur_ms) { cur_ms = ms; cur = t; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    scene->trace_tuning = rc ? saved : cur;
    if (rc) return rc;
    if (best) *best = cur;
    if (best_ms) *best_ms = cur_ms;
    return PT_OK;
}

// ---- exact-arithmetic hooks for the parity tests ------------------------------------------------

float pt_host_f64_diff_emulated(float a, float b, float c, float d) { return f64_diff_emulated(a, b, c, d); }

int pt_selftest_device(int which, const void* in, void* out, uint32_t n, uint64_t seed) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(PT_ECUDA, "no CUDA device available");
    }
    if (which < 0 || which > 3) return fail(PT_EINVAL, "unknown selftest");
    const size_t in_b = which == 1 ? 4 * (size_t)n : (which == 3 ? 64 * (size_t)n : 16 * (size_t)n);
    const size_t out_b = (which == 0 || which == 3) ? 4 * (size_t)n : (which == 1 ? 8 * (size_t)n : 16 * (size_t)n);
    void *din = nullptr, *dout = nullptr;
    if (cudaMalloc(&din, in_b) != cudaSuccess || cudaMalloc(&dout, out_b) != cudaSuccess) {
        if (din) cudaFree(din);
        return fail(PT_ENOMEM, "cudaMalloc selftest");
    }
    cudaMemcpy(din, in, in_b, cudaMemcpyHostToDevice);
    cudaError_t e;
    if (which == 0) e = launch_selftest_f64((const float*)din, (float*)dout, n, 0);
    else if (which == 1) e = launch_selftest_sincos((const float*)din, (float*)dout, n, 0);
    else if (which == 2) e = launch_selftest_philox((const uint32_t*)din, (uint32_t*)dout, n, seed, 0);
    else e = launch_selftest_box((const float*)din, (uint32_t*)dout, n, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, out_b, cudaMemcpyDeviceToHost);
    cudaFree(din);
    cudaFree(dout);
    if (e != cudaSuccess) return cuda_fail(e, "selftest");
    return PT_OK;
}

}  // extern "C"
