// render.cu -- the render call (TileRunner::Run + AbstractRunner::Trace + PathTraceIntegrator)
// as sm_100a kernels.  Paths are numbered sample-major (path = sample * W*H + pixel) and rendered
// in waves.  Two pipelines compute identical results:
//   * fused:     one thread runs a whole path (camera ray, bounces, shadow rays);
//   * wavefront: per bounce an extend kernel (closest hit) over a compacted queue, a shade kernel
//                that appends the next rays and the shadow rays to queues with warp-vote
//                compaction and one atomic per warp, and a shadow kernel (any hit).
// Either way a resolve kernel then adds each pixel's samples to the film in sample order (the
// order of BoxFilter::Output's sum, BoxFilter.cpp:54-71), so the film is deterministic and equal
// to the CPU checker's bit for bit.

#include <algorithm>
#include <cstring>
#include <string>

#include "launch.h"
#include "pt_internal.h"
#include "render.h"
#include "path.cuh"

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

// ---- wavefront pipeline -----------------------------------------------------------------------

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Appends one entry per lane with pred == true: one atomicAdd per warp, slots in lane order.
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool pred) {
    const uint32_t active = __activemask();
    const uint32_t mask = __ballot_sync(active, pred);
    if (mask == 0) return 0xFFFFFFFFu;
    const uint32_t leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(active, base, leader);
    return pred ? base + __popc(mask & ((1u << lane_id()) - 1u)) : 0xFFFFFFFFu;
}

__global__ void __launch_bounds__(128) wf_init_kernel(const RenderParams p, uint64_t first, uint32_t count, WaveState ws,
                                                      uint32_t* __restrict__ queue) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        ws.counters[0] = count;  // current extend queue
        ws.counters[1] = 0;      // next extend queue
        ws.counters[2] = 0;      // shadow queue
    }
    if (i >= count) return;
    uint32_t pixel, sample;
    F3 o, d;
    path_camera(p, first + i, pixel, sample, o, d);
    ws.ray_o[i] = make_float4(o.x, o.y, o.z, 0.f);
    ws.ray_d[i] = make_float4(d.x, d.y, d.z, 0.f);
    ws.thr[i] = make_float4(1.f, 1.f, 1.f, 0.f);
    ws.rad[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    ws.bounces[i] = 0;
    queue[i] = i;
}

__global__ void __launch_bounds__(128) wf_extend_kernel(const RenderParams p, WaveState ws, const uint32_t* __restrict__ queue,
                                                        const uint32_t* __restrict__ count_ptr) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *count_ptr) return;
    const uint32_t slot = queue[i];
    const float4 o = ws.ray_o[slot], d = ws.ray_d[slot];
    RayState rs;
    ray_setup(rs, o.x, o.y, o.z, d.x, d.y, d.z);
    const TraceResult h = traverse<false>((const uint4*)p.nodes, (const float4*)p.tris, p.num_nodes, rs,
                                          __int_as_float(0x7F800000), false);
    if (h.overflow) atomicExch(p.err, 1);
    ws.hit0[slot] = make_uint4(h.overflow ? kPrimNone : h.prim, h.leaf, __float_as_uint(h.u), __float_as_uint(h.v));
    ws.hit1[slot] = h.w;
}

__global__ void __launch_bounds__(128) wf_shade_kernel(const RenderParams p, uint64_t first, WaveState ws,
                                                       const uint32_t* __restrict__ queue, const uint32_t* __restrict__ count_ptr,
                                                       uint32_t* __restrict__ next_queue, uint32_t* next_count,
                                                       uint32_t* __restrict__ primary) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < *count_ptr;
    bool more = false, shadow = false;
    uint32_t slot = 0;
    ShadowReq sh;
    sh.valid = false;
    PathState s;
    if (live) {
        slot = queue[i];
        const uint32_t npix = p.width * p.height;
        const uint64_t path = first + slot;
        const uint32_t sample = (uint32_t)(path / npix), pixel = (uint32_t)(path % npix);
        const float4 o = ws.ray_o[slot], d = ws.ray_d[slot], t = ws.thr[slot], l = ws.rad[slot];
        s.o = f3(o.x, o.y, o.z);
        s.d = f3(d.x, d.y, d.z);
        s.src = f3(t.x, t.y, t.z);
        s.L = f3(l.x, l.y, l.z);
        s.last_lambert = __float_as_uint(t.w);
        s.bounces = ws.bounces[slot];
        const uint4 h0 = ws.hit0[slot];
        if (s.bounces == 0 && sample == 0 && primary) primary[pixel] = h0.x;
        more = shade_hit(p, s, h0.x, h0.y, __uint_as_float(h0.z), __uint_as_float(h0.w), ws.hit1[slot], pixel, sample, sh);
        more = more && !throughput_is_zero(s.src);  // the loop head's is_zero test for the next bounce
        shadow = sh.valid;
        ws.rad[slot] = make_float4(s.L.x, s.L.y, s.L.z, 0.f);
        if (more) {
            ws.ray_o[slot] = make_float4(s.o.x, s.o.y, s.o.z, 0.f);
            ws.ray_d[slot] = make_float4(s.d.x, s.d.y, s.d.z, 0.f);
            ws.thr[slot] = make_float4(s.src.x, s.src.y, s.src.z, __uint_as_float(s.last_lambert));
            ws.bounces[slot] = s.bounces;
        }
    }
    const uint32_t qn = warp_append(next_count, more);
    if (more) next_queue[qn] = slot;
    const uint32_t qs = warp_append(ws.counters + 2, shadow);
    if (shadow) {
        ws.sh_o[qs] = make_float4(sh.o.x, sh.o.y, sh.o.z, sh.tmax);
        ws.sh_d[qs] = make_float4(sh.wi.x, sh.wi.y, sh.wi.z, __uint_as_float(slot));
        ws.sh_c[qs] = make_float4(sh.contrib.x, sh.contrib.y, sh.contrib.z, 0.f);
    }
}

__global__ void __launch_bounds__(128) wf_shadow_kernel(const RenderParams p, WaveState ws) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ws.counters[2]) return;
    const float4 o = ws.sh_o[i], d = ws.sh_d[i];
    RayState rs;
    ray_setup(rs, o.x, o.y, o.z, d.x, d.y, d.z);
    const TraceResult h = traverse<false>((const uint4*)p.nodes, (const float4*)p.tris, p.num_nodes, rs, o.w, true);
    if (h.overflow) { atomicExch(p.err, 1); return; }
    if (h.prim != kPrimNone) return;
    const uint32_t slot = __float_as_uint(d.w);
    const float4 c = ws.sh_c[i];
    float4 l = ws.rad[slot];  // one shadow ray per path per bounce: no other writer
    l.x = fadd(l.x, c.x);
    l.y = fadd(l.y, c.y);
    l.z = fadd(l.z, c.z);
    ws.rad[slot] = l;
}

// Next bounce: the queue just filled becomes current (its count stays), the consumed queue and
// the shadow queue empty.
__global__ void wf_advance_kernel(uint32_t* counters, uint32_t consumed) {
    counters[consumed] = 0;
    counters[2] = 0;
}

__global__ void __launch_bounds__(256) wf_store_kernel(WaveState ws, uint32_t count, float* __restrict__ radiance) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float4 l = ws.rad[i];
    clamp_store(radiance + 3 * (size_t)i, f3(l.x, l.y, l.z));
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

cudaError_t launch_wavefront_wave(const RenderParams& p, uint64_t first, uint32_t count, const WaveState& ws,
                                  float* radiance, uint32_t* primary, cudaStream_t s) {
    if (!count) return cudaSuccess;
    const uint32_t blocks = (count + 127) / 128;
    wf_init_kernel<<<blocks, 128, 0, s>>>(p, first, count, ws, ws.queue[0]);
    uint32_t cur = 0;
    for (uint32_t b = 0; b <= p.max_depth; ++b) {
        const uint32_t nxt = cur ^ 1u;
        wf_extend_kernel<<<blocks, 128, 0, s>>>(p, ws, ws.queue[cur], ws.counters + cur);
        wf_shade_kernel<<<blocks, 128, 0, s>>>(p, first, ws, ws.queue[cur], ws.counters + cur, ws.queue[nxt],
                                               ws.counters + nxt, primary);
        wf_shadow_kernel<<<blocks, 128, 0, s>>>(p, ws);
        wf_advance_kernel<<<1, 1, 0, s>>>(ws.counters, cur);
        cur = nxt;
    }
    wf_store_kernel<<<(count + 255) / 256, 256, 0, s>>>(ws, count, radiance);
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

void wave_state_carve(void* base, uint32_t count, WaveState& ws) {
    char* q = (char*)base;
    auto take = [&](size_t n) { char* r = q; q += (n + 255) & ~(size_t)255; return r; };
    ws.ray_o = (float4*)take(16 * (size_t)count);
    ws.ray_d = (float4*)take(16 * (size_t)count);
    ws.thr = (float4*)take(16 * (size_t)count);
    ws.rad = (float4*)take(16 * (size_t)count);
    ws.bounces = (uint32_t*)take(4 * (size_t)count);
    ws.hit0 = (uint4*)take(16 * (size_t)count);
    ws.hit1 = (float*)take(4 * (size_t)count);
    ws.queue[0] = (uint32_t*)take(4 * (size_t)count);
    ws.queue[1] = (uint32_t*)take(4 * (size_t)count);
    ws.sh_o = (float4*)take(16 * (size_t)count);
    ws.sh_d = (float4*)take(16 * (size_t)count);
    ws.sh_c = (float4*)take(16 * (size_t)count);
    ws.counters = (uint32_t*)take(64);
}

size_t wave_state_alloc_bytes(uint32_t count) {
    size_t n = 0;
    auto take = [&](size_t b) { n += (b + 255) & ~(size_t)255; };
    for (int k = 0; k < 4; ++k) take(16 * (size_t)count);
    take(4 * (size_t)count);
    take(16 * (size_t)count);
    take(4 * (size_t)count);
    take(4 * (size_t)count);
    take(4 * (size_t)count);
    for (int k = 0; k < 3; ++k) take(16 * (size_t)count);
    take(64);
    return n;
}

}  // namespace pt

using namespace pt;

namespace {
struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
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
    if (desc->flags & ~(uint32_t)(PT_RENDER_NEE | PT_RENDER_JITTER | PT_RENDER_WAVEFRONT))
        return fail(PT_EINVAL, "unknown render flags");
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

    const RenderParams p = render_params(s, desc);
    const bool wavefront = (desc->flags & PT_RENDER_WAVEFRONT) != 0;
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t total = npix64 * desc->spp;
    uint32_t wave = desc->wave_paths ? desc->wave_paths : (wavefront ? (1u << 21) : (1u << 22));
    if (wave > total) wave = (uint32_t)total;
    DevBuf rad, film, rgb_dev, prim_dev, wsbuf;
    if (cudaMalloc(&rad.p, 12 * (size_t)wave) != cudaSuccess || cudaMalloc(&film.p, 12 * (size_t)npix) != cudaSuccess)
        return fail(PT_ENOMEM, "cudaMalloc render buffers");
    WaveState ws{};
    if (wavefront) {
        if (cudaMalloc(&wsbuf.p, wave_state_alloc_bytes(wave)) != cudaSuccess)
            return fail(PT_ENOMEM, "cudaMalloc wavefront queues");
        wave_state_carve(wsbuf.p, wave, ws);
    }
    const bool dev_out = (mem_flags & PT_MEM_DEVICE) != 0;
    float* rgb_d = rgb_out;
    uint32_t* prim_d = primary_out;
    if (!dev_out) {
        if (cudaMalloc(&rgb_dev.p, 12 * (size_t)npix) != cudaSuccess) return fail(PT_ENOMEM, "cudaMalloc film");
        rgb_d = (float*)rgb_dev.p;
        if (primary_out) {
            if (cudaMalloc(&prim_dev.p, 4 * (size_t)npix) != cudaSuccess) return fail(PT_ENOMEM, "cudaMalloc prim");
            prim_d = (uint32_t*)prim_dev.p;
        }
    }
    cudaError_t e = cudaMemsetAsync(film.p, 0, 12 * (size_t)npix, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->err_flag, 0, sizeof(int), st);
    for (uint64_t first = 0; e == cudaSuccess && first < total; first += wave) {
        const uint32_t cnt = (uint32_t)std::min<uint64_t>(wave, total - first);
        e = wavefront ? launch_wavefront_wave(p, first, cnt, ws, (float*)rad.p, prim_d, st)
                      : launch_path_wave(p, first, cnt, (float*)rad.p, prim_d, st);
        if (e == cudaSuccess) e = launch_resolve_wave(first, cnt, npix, (const float*)rad.p, (float*)film.p, st);
    }
    if (e == cudaSuccess) e = launch_finish_film((const float*)film.p, npix, desc->spp, rgb_d, st);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("render launch: ") + cudaGetErrorString(e));
    if (!dev_out) {
        e = cudaMemcpyAsync(rgb_out, rgb_d, 12 * (size_t)npix, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && primary_out)
            e = cudaMemcpyAsync(primary_out, prim_d, 4 * (size_t)npix, cudaMemcpyDeviceToHost, st);
    }
    // the temporaries are freed at scope exit: the stream must be done with them
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("render: ") + cudaGetErrorString(e));
    int err = 0;
    cudaMemcpy(&err, s->err_flag, sizeof(int), cudaMemcpyDeviceToHost);
    if (err) return fail(PT_ESTACK, "a path exceeded the traversal stack");
    return PT_OK;
}
