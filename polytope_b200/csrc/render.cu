// render.cu -- the render call (TileRunner::Run + AbstractRunner::Trace + PathTraceIntegrator)
// as sm_100a kernels.  Paths are numbered sample-major (path = sample * W*H + pixel) and rendered
// in waves.  Two pipelines compute identical results:
//   * fused:     one thread runs a whole path (camera ray, bounces, shadow rays);
//   * wavefront: per bounce an extend kernel (closest hit) over a compacted queue, a shade kernel
//                that appends the next rays and the shadow rays to queues with warp-vote
//                compaction and one atomic per warp, and a shadow kernel (any hit).
// Either way a resolve kernel then adds each pixel's samples to the film in sample order (the
// order of BoxFilter::Output's sum, BoxFilter.cpp:54-71), so the film is deterministic and equal
// to the CPU oracle's bit for bit.

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "batch.h"
#include "launch.h"
#include "pt_internal.h"
#include "render.h"
#include "path.cuh"
#include "wavefront.h"

static_assert(sizeof(pt::MeshRec) == sizeof(pt::DeviceMesh) && alignof(pt::MeshRec) == alignof(pt::DeviceMesh),
              "the kernels' mesh record must match the uploaded one");

namespace pt {

__global__ void __launch_bounds__(128) path_kernel(const RenderParams p, uint64_t first, uint32_t count,
                                                   float* __restrict__ radiance, uint32_t* __restrict__ primary) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t rays = 0;
    if (i < count) rays = path_fused(p, first + i, radiance + 3 * (size_t)i, primary);
    if (p.rays_traced) {
        const uint32_t sum = __reduce_add_sync(0xFFFFFFFFu, rays);
        if ((threadIdx.x & 31u) == 0 && sum) atomicAdd(p.rays_traced, (unsigned long long)sum);
    }
}

// ---- resolve ----------------------------------------------------------------------------------

__global__ void resolve_kernel(uint64_t first, uint32_t count, uint32_t npix, const float* __restrict__ radiance,
                               float* __restrict__ film) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= npix) return;
    // samples s with first <= s*npix + x < first + count, in increasing s
    const uint64_t end = first + count;
    uint64_t s = first / npix;
    if (s * npix + x < first) ++s;
    float r = film[3 * (size_t)x], g = film[3 * (size_t)x + 1], b = film[3 * (size_t)x + 2];
    for (uint64_t pth = s * npix + x; pth < end; pth += npix) {
        const size_t k = 3 * (size_t)(pth - first);
        r = fadd(r, radiance[k]);
        g = fadd(g, radiance[k + 1]);
        b = fadd(b, radiance[k + 2]);
    }
    film[3 * (size_t)x] = r;
    film[3 * (size_t)x + 1] = g;
    film[3 * (size_t)x + 2] = b;
}

__global__ void finish_kernel(const float* __restrict__ film, uint32_t npix, uint32_t spp, float* __restrict__ rgb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * npix) return;
    rgb[i] = fmul(film[i], frcp((float)spp));  // accum *= 1.0f / numSamples (BoxFilter.cpp:65-67)
}

// ---- launchers ----------------------------------------------------------------------------------

cudaError_t launch_path_wave(const RenderParams& p, uint64_t first, uint32_t count, float* radiance, uint32_t* primary,
                             cudaStream_t s) {
    if (!count) return cudaSuccess;
    path_kernel<<<(count + 127) / 128, 128, 0, s>>>(p, first, count, radiance, primary);
    return cudaGetLastError();
}

cudaError_t launch_resolve_wave(uint64_t first, uint32_t count, uint32_t npix, const float* radiance, float* film,
                                cudaStream_t s) {
    resolve_kernel<<<(npix + 255) / 256, 256, 0, s>>>(first, count, npix, radiance, film);
    return cudaGetLastError();
}
cudaError_t launch_finish_film(const float* film, uint32_t npix, uint32_t spp, float* rgb, cudaStream_t s) {
    finish_kernel<<<(3 * npix + 255) / 256, 256, 0, s>>>(film, npix, spp, rgb);
    return cudaGetLastError();
}

}  // namespace pt

using namespace pt;

namespace {
// Temporaries of a render come from a stream-ordered pool per device, owned by the library, that
// keeps up to 2 GiB cached between calls.  A cudaMalloc / cudaFree pair per frame synchronises
// the whole device on every call, and on a device holding tens of GB of resident scenes single
// frees were seen to stall for 0.1-1 s.
cudaMemPool_t render_pool(int device) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    if (device < 0 || device >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[device]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = 2ull << 30;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[device] = p;
    }
    return pools[device];
}

struct DevBuf {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    bool pooled = false;
    // Stream-ordered on `st` from `pool` (plain cudaMalloc if the pool could not be made).
    bool alloc(size_t n, cudaMemPool_t pool, cudaStream_t st) {
        s = st;
        pooled = pool != nullptr;
        const cudaError_t e = pooled ? cudaMallocFromPoolAsync(&p, n, pool, st) : cudaMalloc(&p, n);
        if (e != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return p != nullptr;
    }
    ~DevBuf() {
        if (!p) return;
        if (pooled) cudaFreeAsync(p, s); else cudaFree(p);
    }
};
}  // namespace

namespace pt {
RenderParams render_params(const pt_scene* s, const pt_render_desc* desc) {
    RenderParams p{};
    p.nodes = s->dev.nodes;
    p.tris = s->dev.tris;
    p.num_nodes = s->num_nodes;
    p.meshes = s->dev.meshes;
    p.prim_normals = (const float*)s->dev.prim_normals;
    p.light_tris = (const float*)s->dev.light_tris;
    p.light_cdf = (const float*)s->dev.light_cdf;
    p.num_lights = s->dev.num_lights;
    p.light_area = s->dev.light_area;
    p.has_env = s->has_env;
    std::memcpy(p.env, s->env, sizeof(p.env));
    p.cam = make_camera(desc->camera, desc->width, desc->height);
    p.width = desc->width;
    p.height = desc->height;
    p.spp = desc->spp;
    p.max_depth = desc->max_depth;
    p.seed_lo = (uint32_t)desc->seed;
    p.seed_hi = (uint32_t)(desc->seed >> 32);
    p.flags = desc->flags;
    p.err = (int*)s->err_flag;
    return p;
}

int check_render_desc(const pt_scene* s, const pt_render_desc* desc) {
    if (!s || !desc) return fail(PT_EINVAL, "scene or desc is NULL");
    if (desc->width == 0 || desc->height == 0 || desc->spp == 0) return fail(PT_EINVAL, "empty frame");
    if ((uint64_t)desc->width * desc->height > (1u << 30)) return fail(PT_EINVAL, "frame too large");
    if ((uint64_t)desc->width * desc->height * desc->spp > (1ull << 40)) return fail(PT_EINVAL, "too many samples");
    if (desc->max_depth > 1024) return fail(PT_EINVAL, "max_depth above 1024");
    if (desc->flags & ~(uint32_t)(PT_RENDER_NEE | PT_RENDER_JITTER | PT_RENDER_WAVEFRONT | PT_RENDER_PERSISTENT | PT_RENDER_FUSED))
        return fail(PT_EINVAL, "unknown render flags");
    const uint32_t pipes = desc->flags & (PT_RENDER_WAVEFRONT | PT_RENDER_PERSISTENT | PT_RENDER_FUSED);
    if (pipes & (pipes - 1))
        return fail(PT_EINVAL, "PT_RENDER_WAVEFRONT, PT_RENDER_PERSISTENT and PT_RENDER_FUSED exclude each other");
    if ((int)s->max_depth + 2 > PT_TRAVERSAL_STACK) return fail(PT_ESTACK, "tree too deep for the traversal stack");
    return PT_OK;
}
}  // namespace pt

extern "C" int pt_render(pt_scene* s, const pt_render_desc* desc, float* rgb_out, uint32_t* primary_out,
                         uint32_t mem_flags, void* stream) {
    int rc = check_render_desc(s, desc);
    if (rc) return rc;
    if (!rgb_out) return fail(PT_EINVAL, "rgb_out is NULL");
    const uint64_t npix64 = (uint64_t)desc->width * desc->height;
    const uint32_t npix = (uint32_t)npix64;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != s->device) cudaSetDevice(s->device);
    struct Restore { int d; ~Restore() { if (d >= 0) cudaSetDevice(d); } } restore{prev != s->device ? prev : -1};

    const bool dev_out = (mem_flags & PT_MEM_DEVICE) != 0;
    RenderParams p = render_params(s, desc);
    // Pipelines: the persistent path kernel unless PT_RENDER_FUSED or PT_RENDER_WAVEFRONT is given
    // (the wave engine runs both the queue-based kernels and the persistent path kernel).
    const bool fused = (desc->flags & PT_RENDER_FUSED) != 0;
    const bool persistent = !fused && (desc->flags & PT_RENDER_WAVEFRONT) == 0;
    const bool wavefront = !fused;
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t total = npix64 * desc->spp;
    // Default wave: 4 M paths for the fused and queue-based kernels (the queues cost ~140 B per
    // path), 32 M for the persistent path kernel (12 B per path; longer waves shorten its tail).
    uint64_t wave = desc->wave_paths ? desc->wave_paths : (persistent ? (1ull << 25) : (1ull << 22));
    if (wave > total) wave = total;
    cudaMemPool_t pool = render_pool(s->device);
    DevBuf rad, film, rgb_dev, prim_dev, wsbuf, tables;
    // the film sums, then (host-memory calls) this call's own error flag
    const size_t film_bytes = (12 * (size_t)npix + 15) & ~(size_t)15;
    if ((!wavefront && !rad.alloc(12 * (size_t)wave, pool, st)) || !film.alloc(film_bytes + 16, pool, st))
        return fail(PT_ENOMEM, "device memory for the render buffers");
    // A host-memory call waits for its frame and reports a guard failure of its own kernels; a
    // device-memory call returns once the work is queued, and its kernels raise the scene's flag,
    // which pt_scene_status reads.
    int* call_err = (int*)((char*)film.p + film_bytes);
    p.err = dev_out ? (int*)s->err_flag : call_err;
    WfState ws{};
    WfPlan plan;
    if (wavefront) {
        if (!wsbuf.alloc(wf_state_bytes((uint32_t)wave, persistent), pool, st))
            return fail(PT_ENOMEM, "device memory for the wavefront queues");
        wf_state_carve(wsbuf.p, (uint32_t)wave, ws, persistent);
        wf_plan_all(plan, {npix}, {desc->spp}, {desc->max_depth}, wave);
    }
    float* rgb_d = rgb_out;
    uint32_t* prim_d = primary_out;
    if (!dev_out) {
        if (!rgb_dev.alloc(12 * (size_t)npix, pool, st)) return fail(PT_ENOMEM, "device memory for the film");
        rgb_d = (float*)rgb_dev.p;
        if (primary_out) {
            if (!prim_dev.alloc(4 * (size_t)npix, pool, st)) return fail(PT_ENOMEM, "device memory for the primary ids");
            prim_d = (uint32_t*)prim_dev.p;
        }
    }
    cudaError_t e = cudaMemsetAsync(film.p, 0, film_bytes + 16, st);
    if (wavefront) {
        // one item: device copies of its parameters and of the plan's tables, staged in one
        // host block and copied with one call
        const size_t pbytes = (sizeof(RenderParams) + 255) & ~(size_t)255;
        const size_t ibytes = (sizeof(WfItem) + 255) & ~(size_t)255;
        const size_t sbytes = ((sizeof(WfSegment) * plan.segments.size()) + 255) & ~(size_t)255;
        const size_t rbytes = ((sizeof(WfPixels) * plan.resolve.size()) + 255) & ~(size_t)255;
        const size_t fbytes = sizeof(WfPixels) * plan.finish.size();
        const size_t tbytes = pbytes + ibytes + sbytes + rbytes + fbytes;
        if (!tables.alloc(tbytes, pool, st)) return fail(PT_ENOMEM, "device memory for the wavefront tables");
        char* tb = (char*)tables.p;
        RenderParams* d_params = (RenderParams*)tb;
        WfItem* d_item = (WfItem*)(tb + pbytes);
        WfSegment* d_segs = (WfSegment*)(tb + pbytes + ibytes);
        WfPixels* d_res = (WfPixels*)(tb + pbytes + ibytes + sbytes);
        WfPixels* d_fin = (WfPixels*)(tb + pbytes + ibytes + sbytes + rbytes);
        const WfItem item{d_params, (float*)film.p, rgb_d, prim_d, npix, desc->spp};
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_params, &p, sizeof(p), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_item, &item, sizeof(item), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_segs, plan.segments.data(), sizeof(WfSegment) * plan.segments.size(), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_res, plan.resolve.data(), sizeof(WfPixels) * plan.resolve.size(), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_fin, plan.finish.data(), sizeof(WfPixels) * plan.finish.size(), cudaMemcpyHostToDevice, st);
        WfTuning t;
        t.stack_cap = stack_cap_for(s->max_depth, 0);
        t.paths = persistent;
        for (size_t k = 0; e == cudaSuccess && k < plan.waves.size(); ++k)
            e = wf_launch_wave(d_item, d_segs, d_res, d_fin, plan.waves[k], ws, t, nullptr, st);
    } else {
        for (uint64_t first = 0; e == cudaSuccess && first < total; first += wave) {
            const uint32_t cnt = (uint32_t)std::min<uint64_t>(wave, total - first);
            e = launch_path_wave(p, first, cnt, (float*)rad.p, prim_d, st);
            if (e == cudaSuccess) e = launch_resolve_wave(first, cnt, npix, (const float*)rad.p, (float*)film.p, st);
        }
        if (e == cudaSuccess) e = launch_finish_film((const float*)film.p, npix, desc->spp, rgb_d, st);
    }
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("render launch: ") + cudaGetErrorString(e));
    // Device-memory output: the temporaries go back to the pool in stream order, so nothing here
    // waits for the frame.
    if (dev_out) return PT_OK;
    int err = 0;
    e = cudaMemcpyAsync(rgb_out, rgb_d, 12 * (size_t)npix, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && primary_out)
        e = cudaMemcpyAsync(primary_out, prim_d, 4 * (size_t)npix, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, call_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("render: ") + cudaGetErrorString(e));
    if (err) return fail(PT_ESTACK, "a path exceeded the traversal stack");
    return PT_OK;
}

extern "C" int pt_scene_status(pt_scene* s, void* stream) {
    if (!s) return fail(PT_EINVAL, "scene is NULL");
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != s->device) cudaSetDevice(s->device);
    struct Restore { int d; ~Restore() { if (d >= 0) cudaSetDevice(d); } } restore{prev != s->device ? prev : -1};
    cudaStream_t st = (cudaStream_t)stream;
    int err = 0;
    cudaError_t e = cudaMemcpyAsync(&err, s->err_flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && err) e = cudaMemsetAsync(s->err_flag, 0, sizeof(int), st);
    if (e == cudaSuccess && err) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("scene status: ") + cudaGetErrorString(e));
    if (err) return fail(PT_ESTACK, "a kernel on this scene exceeded the traversal stack or met a malformed tree");
    return PT_OK;
}
