// render.cu -- the render call (TileRunner::Run + AbstractRunner::Trace + PathTraceIntegrator)
// as sm_100a kernels.  Paths are numbered sample-major (path = sample * W*H + pixel) and rendered
// in waves.  Three pipelines compute identical results:
//   * persistent (the default): one persistent path kernel per wave (wavefront.cu wf_path_kernel)
//                whose lanes take the next path as soon as theirs ends;
//   * fused:     one thread runs a whole path (camera ray, bounces, shadow rays), one launch per
//                wave (path_kernel below; the default for two-level scenes);
//   * wavefront: per bounce an extend kernel (closest hit) over a compacted queue, a shade kernel
//                that appends the next rays and the shadow rays to queues with warp-vote
//                compaction and one atomic per warp, and a shadow kernel (any hit).
// Each way a resolve kernel then adds each pixel's samples to the film in sample order (the
// order of BoxFilter::Output's sum, BoxFilter.cpp:54-71), so the film is deterministic and equal
// to the CPU oracle's bit for bit.

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "batch.h"
#include "launch.h"
#include "pt_internal.h"
#include "render.h"
#include "path.cuh"
#include "wavefront.h"

static_assert(sizeof(pt::MeshRec) == sizeof(pt::DeviceMesh) && alignof(pt::MeshRec) == alignof(pt::DeviceMesh),
              "the kernels' mesh record must match the uploaded one");

namespace pt {

// 8 resident blocks of 128 per SM (64 registers, some spilled) instead of the 96 registers the
// compiler picks unbounded: on a B200 the 6.55 M-face frame 1362 -> 1691 Msamples/s (flattened)
// and 1073 -> 1256 (two-level); 6, 7, 9, 10 and 12 blocks measured 1491, 1600, 1576, 1532, 1532.
template <bool TWO_LEVEL>
__global__ void __launch_bounds__(128, 8) path_kernel(const RenderParams p, uint64_t first, uint32_t count,
                                                   float* __restrict__ radiance, uint32_t* __restrict__ primary) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t rays = 0;
    if (i < count) rays = path_fused<kStackCap, TWO_LEVEL>(p, first + i, radiance + 3 * (size_t)i, primary);
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

// ---- small host -> device uploads without a stream sync --------------------------------------------
//
// cudaMemcpyAsync from pageable host memory waits for the work already queued on the stream before
// it copies, so a frame's parameter tables copied that way would hold the caller until the previous
// frame on the stream has finished.  Kernel parameters are captured at launch instead: the tables
// travel as by-value blocks of a copy kernel, queued behind the earlier work like any launch.
struct UploadBlock {
    uint32_t words[960];  // 3840 bytes per launch, inside the 4 KB kernel-parameter space
};

__global__ void __launch_bounds__(256) upload_kernel(const UploadBlock blk, uint32_t nwords, uint32_t* __restrict__ dst) {
    for (uint32_t i = threadIdx.x; i < nwords; i += blockDim.x) dst[i] = blk.words[i];
}

cudaError_t upload_async(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if ((bytes & 3u) || ((uintptr_t)dst & 3u)) return cudaErrorInvalidValue;
    const size_t per = sizeof(UploadBlock::words);
    for (size_t off = 0; off < bytes; off += per) {
        const size_t n = bytes - off < per ? bytes - off : per;
        UploadBlock blk;
        std::memcpy(blk.words, (const char*)src + off, n);
        upload_kernel<<<1, 256, 0, s>>>(blk, (uint32_t)(n / 4), (uint32_t*)((char*)dst + off));
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// ---- launchers ----------------------------------------------------------------------------------

cudaError_t launch_path_wave(const RenderParams& p, uint64_t first, uint32_t count, float* radiance, uint32_t* primary,
                             cudaStream_t s) {
    if (!count) return cudaSuccess;
    if (p.instances)
        path_kernel<true><<<(count + 127) / 128, 128, 0, s>>>(p, first, count, radiance, primary);
    else
        path_kernel<false><<<(count + 127) / 128, 128, 0, s>>>(p, first, count, radiance, primary);
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
    p.instances = s->dev.instances;
    p.top_nodes = s->dev.tlas_nodes;
    p.top_num_nodes = s->dev.tlas_num_nodes;
    p.exact_tree = s->nan_boxes ? 1u : 0u;
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
    if (s->two_level && (desc->flags & PT_RENDER_WAVEFRONT))
        return fail(PT_EINVAL, "a two-level scene renders with the persistent or the fused pipeline "
                               "(PT_RENDER_WAVEFRONT walks flattened trees only)");
    return PT_OK;
}
}  // namespace pt

namespace {
// Queue chunk of the persistent path kernel for a frame of `total` paths (see enqueue_frame).
uint32_t path_chunk_for(uint64_t total, int device) {
    static std::atomic<int> sms_of[64] = {};
    int sms = (device >= 0 && device < 64) ? sms_of[device].load(std::memory_order_relaxed) : 0;
    if (sms == 0) {
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0) {
            cudaGetLastError();
            sms = 148;
        }
        if (device >= 0 && device < 64) sms_of[device].store(sms, std::memory_order_relaxed);
    }
    const uint64_t warps = (uint64_t)sms * PT_PATH_MIN_BLOCKS * 4;  // resident warps: blocks of 128 threads
    return total / (warps * 16) >= 128 ? 128u : 64u;
}

// Queues one frame on `st`: every wave, the film sums and the finished film into rgb_d (device),
// sample 0's primary ids into prim_d (device, optional).  Guard failures raise `err`.  The
// temporaries come from the render pool and go back to it in stream order, so nothing here waits
// for the device.
int enqueue_frame(pt_scene* s, const pt_render_desc* desc, float* rgb_d, uint32_t* prim_d, int* err, cudaStream_t st) {
    const uint64_t npix64 = (uint64_t)desc->width * desc->height;
    const uint32_t npix = (uint32_t)npix64;
    RenderParams p = render_params(s, desc);
    p.err = err;
    // Pipelines: the persistent path kernel unless PT_RENDER_FUSED or PT_RENDER_WAVEFRONT is given
    // (the wave engine runs both the queue-based kernels and the persistent path kernel).
    // two-level scenes default to the fused kernel: their persistent walk measured slower (599
    // against 819 Msamples/s on the 6.5 M-face instanced frame), the top-level steps and instance
    // entries interrupting the warp-voted node steps; PT_RENDER_PERSISTENT still selects it
    const bool fused = (desc->flags & PT_RENDER_FUSED) != 0 || (s->two_level && !(desc->flags & PT_RENDER_PERSISTENT));
    const bool persistent = !fused && (desc->flags & PT_RENDER_WAVEFRONT) == 0;
    const bool wavefront = !fused;
    const uint64_t total = npix64 * desc->spp;
    // Default wave: 4 M paths for the fused and queue-based kernels (the queues cost ~140 B per
    // path), 32 M for the persistent path kernel (12 B per path; longer waves shorten its tail).
    uint64_t wave = desc->wave_paths ? desc->wave_paths : (persistent ? (1ull << 25) : (1ull << 22));
    if (wave > total) wave = total;
    cudaMemPool_t pool = render_pool(s->device);
    DevBuf rad, film, wsbuf, tables;
    if ((!wavefront && !rad.alloc(12 * (size_t)wave, pool, st)) || !film.alloc(12 * (size_t)npix, pool, st))
        return fail(PT_ENOMEM, "device memory for the render buffers");
    WfState ws{};
    WfPlan plan;
    if (wavefront) {
        if (!wsbuf.alloc(wf_state_bytes((uint32_t)wave, persistent), pool, st))
            return fail(PT_ENOMEM, "device memory for the wavefront queues");
        wf_state_carve(wsbuf.p, (uint32_t)wave, ws, persistent);
        wf_plan_all(plan, {npix}, {desc->spp}, {desc->max_depth}, wave);
    }
    cudaError_t e = cudaMemsetAsync(film.p, 0, 12 * (size_t)npix, st);
    if (wavefront) {
        // one item: device copies of its parameters and of the plan's tables
        const size_t pbytes = (sizeof(RenderParams) + 255) & ~(size_t)255;
        const size_t ibytes = (sizeof(WfItem) + 255) & ~(size_t)255;
        const size_t sbytes = ((sizeof(WfSegment) * plan.segments.size()) + 255) & ~(size_t)255;
        const size_t rbytes = ((sizeof(WfPixels) * plan.resolve.size()) + 255) & ~(size_t)255;
        const size_t fbytes = sizeof(WfPixels) * plan.finish.size();
        if (!tables.alloc(((pbytes + ibytes + sbytes + rbytes + fbytes) + 3) & ~(size_t)3, pool, st))
            return fail(PT_ENOMEM, "device memory for the wavefront tables");
        char* tb = (char*)tables.p;
        RenderParams* d_params = (RenderParams*)tb;
        WfItem* d_item = (WfItem*)(tb + pbytes);
        WfSegment* d_segs = (WfSegment*)(tb + pbytes + ibytes);
        WfPixels* d_res = (WfPixels*)(tb + pbytes + ibytes + sbytes);
        WfPixels* d_fin = (WfPixels*)(tb + pbytes + ibytes + sbytes + rbytes);
        const WfItem item{d_params, (float*)film.p, rgb_d, prim_d, npix, desc->spp};
        // the tables in one host block, uploaded without waiting for the stream's earlier work
        std::vector<char> host(((pbytes + ibytes + sbytes + rbytes + fbytes) + 3) & ~(size_t)3, 0);
        std::memcpy(host.data(), &p, sizeof(p));
        std::memcpy(host.data() + pbytes, &item, sizeof(item));
        std::memcpy(host.data() + pbytes + ibytes, plan.segments.data(), sizeof(WfSegment) * plan.segments.size());
        std::memcpy(host.data() + pbytes + ibytes + sbytes, plan.resolve.data(), sizeof(WfPixels) * plan.resolve.size());
        std::memcpy(host.data() + pbytes + ibytes + sbytes + rbytes, plan.finish.data(), sizeof(WfPixels) * plan.finish.size());
        if (e == cudaSuccess) e = upload_async(tb, host.data(), host.size(), st);
        WfTuning t;
        t.stack_cap = stack_cap_for(s->max_depth, 0);
        t.paths = persistent;
        t.two_level = s->two_level;
        // paths a warp takes per fetch: large chunks cost fewer fetches on a large frame (128
        // measured best on the 6.5 M-face 1920x1080x64 frame: 1771 Msamples/s against 1721 at 64,
        // 1751 at 256, 1660 at 512), while a frame too small to give every resident warp 16
        // fetches of 128 paths keeps 64 (the 256-scene batch's frames rendered one by one slowed
        // from 1437 to 1365 Mrays/s with 128 everywhere)
        if (persistent) t.queue_chunk = path_chunk_for(total, s->device);
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
    return PT_OK;
}

struct DeviceScope {  // makes the scene's device current for the call, restores the caller's
    int prev = -1;
    explicit DeviceScope(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev); else prev = -1;
    }
    ~DeviceScope() { if (prev >= 0) cudaSetDevice(prev); }
};
}  // namespace

extern "C" int pt_render(pt_scene* s, const pt_render_desc* desc, float* rgb_out, uint32_t* primary_out,
                         uint32_t mem_flags, void* stream) {
    int rc = check_render_desc(s, desc);
    if (rc) return rc;
    if (!rgb_out) return fail(PT_EINVAL, "rgb_out is NULL");
    DeviceScope scope(s->device);
    cudaStream_t st = (cudaStream_t)stream;
    // Device-memory output: the frame is only queued, and a guard failure raises the scene's flag
    // (pt_scene_status).
    if (mem_flags & PT_MEM_DEVICE) return enqueue_frame(s, desc, rgb_out, primary_out, (int*)s->err_flag, st);
    // Host-memory output: device film, primary ids and this call's own error flag, then copies out
    // and a wait for the frame.
    const size_t npix = (size_t)desc->width * desc->height;
    cudaMemPool_t pool = render_pool(s->device);
    DevBuf out;
    const size_t rgb_bytes = 12 * npix, prim_bytes = primary_out ? 4 * npix : 0;
    if (!out.alloc(rgb_bytes + prim_bytes + 16, pool, st)) return fail(PT_ENOMEM, "device memory for the film");
    float* rgb_d = (float*)out.p;
    uint32_t* prim_d = primary_out ? (uint32_t*)((char*)out.p + rgb_bytes) : nullptr;
    int* call_err = (int*)((char*)out.p + ((rgb_bytes + prim_bytes + 15) & ~(size_t)15));
    cudaError_t e = cudaMemsetAsync(call_err, 0, sizeof(int), st);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("render: ") + cudaGetErrorString(e));
    rc = enqueue_frame(s, desc, rgb_d, prim_d, call_err, st);
    if (rc) return rc;
    int err = 0;
    e = cudaMemcpyAsync(rgb_out, rgb_d, rgb_bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && primary_out) e = cudaMemcpyAsync(primary_out, prim_d, prim_bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, call_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("render: ") + cudaGetErrorString(e));
    if (err) return fail(PT_ESTACK, "a path exceeded the traversal stack");
    return PT_OK;
}

extern "C" int pt_render_rgba8(pt_scene* s, const pt_render_desc* desc, uint8_t* rgba_out, uint32_t* primary_out,
                               uint32_t mem_flags, void* stream) {
    int rc = check_render_desc(s, desc);
    if (rc) return rc;
    if (!rgba_out) return fail(PT_EINVAL, "rgba_out is NULL");
    DeviceScope scope(s->device);
    cudaStream_t st = (cudaStream_t)stream;
    const bool dev_out = (mem_flags & PT_MEM_DEVICE) != 0;
    const size_t npix = (size_t)desc->width * desc->height;
    cudaMemPool_t pool = render_pool(s->device);
    // the float film stays on the device; host-memory calls also stage the bytes, the primary ids
    // and their own error flag there
    const size_t rgb_bytes = 12 * npix, byte_bytes = dev_out ? 0 : 4 * npix;
    const size_t prim_bytes = (!dev_out && primary_out) ? 4 * npix : 0;
    DevBuf tmp;
    if (!tmp.alloc(rgb_bytes + byte_bytes + prim_bytes + 16, pool, st)) return fail(PT_ENOMEM, "device memory for the film");
    float* rgb_d = (float*)tmp.p;
    uint8_t* bytes_d = dev_out ? rgba_out : (uint8_t*)tmp.p + rgb_bytes;
    uint32_t* prim_d = dev_out ? primary_out : (primary_out ? (uint32_t*)((char*)tmp.p + rgb_bytes + byte_bytes) : nullptr);
    int* call_err = dev_out ? (int*)s->err_flag
                            : (int*)((char*)tmp.p + ((rgb_bytes + byte_bytes + prim_bytes + 15) & ~(size_t)15));
    cudaError_t e = dev_out ? cudaSuccess : cudaMemsetAsync(call_err, 0, sizeof(int), st);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("render: ") + cudaGetErrorString(e));
    rc = enqueue_frame(s, desc, rgb_d, prim_d, call_err, st);
    if (rc) return rc;
    e = launch_film_to_rgba8(rgb_d, (uint32_t)npix, bytes_d, st);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("film to RGBA8: ") + cudaGetErrorString(e));
    if (dev_out) return PT_OK;
    int err = 0;
    e = cudaMemcpyAsync(rgba_out, bytes_d, 4 * npix, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && primary_out) e = cudaMemcpyAsync(primary_out, prim_d, prim_bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, call_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("render: ") + cudaGetErrorString(e));
    if (err) return fail(PT_ESTACK, "a path exceeded the traversal stack");
    return PT_OK;
}

extern "C" int pt_scene_status(pt_scene* s, void* stream) {
    if (!s) return fail(PT_EINVAL, "scene is NULL");
    DeviceScope scope(s->device);
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
