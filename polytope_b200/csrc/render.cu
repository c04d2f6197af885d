// render.cu -- the render call (TileRunner::Run + AbstractRunner::Trace + PathTraceIntegrator)
// as sm_100a kernels: one fused path kernel per wave of (pixel, sample) paths in sample-major
// order, then a resolve kernel that adds each pixel's samples to the film in sample order (the
// order of BoxFilter::Output's sum, BoxFilter.cpp:54-71), so the film is deterministic and equal
// to the CPU checker's bit for bit.

#include <algorithm>
#include <cstring>
#include <string>

#include "launch.h"
#include "pt_internal.h"
#include "render.h"
#include "shade.cuh"

namespace pt {

__device__ __forceinline__ void path_radiance(const RenderParams& p, uint32_t pixel, uint32_t sample, F3 o, F3 d,
                                              uint32_t* primary, float out[3]) {
    const uint4* nodes = (const uint4*)p.nodes;
    const float4* tris = (const float4*)p.tris;
    const MeshRec* meshes = (const MeshRec*)p.meshes;
    const bool nee = (p.flags & PT_RENDER_NEE) && p.num_lights > 0;
    const float inf = __int_as_float(0x7F800000);
    F3 src = f3(1.f, 1.f, 1.f);
    F3 L = f3(0.f, 0.f, 0.f);
    uint32_t bounces = 0;
    bool last_lambert = false;
    while (true) {
        if (src.x < 0.0039f && src.y < 0.0039f && src.z < 0.0039f) break;  // ReflectanceSpectrum::is_zero
        RayState rs;
        ray_setup(rs, o.x, o.y, o.z, d.x, d.y, d.z);
        const TraceResult h = traverse<false>(nodes, tris, p.num_nodes, rs, inf, false);
        if (h.overflow) { atomicExch(p.err, 1); break; }
        if (bounces == 0 && primary) primary[pixel] = h.prim;
        if (h.prim == kPrimNone) {
            if (p.has_env) L = vadd(L, f3(fmul(p.env[0], src.x), fmul(p.env[1], src.y), fmul(p.env[2], src.z)));
            break;
        }
        F3 v0, v1, v2;
        uint32_t mesh;
        load_face(tris, h.leaf, v0, v1, v2, mesh);
        const MeshRec mr = meshes[mesh];
        if (mr.is_light) {
            if (!(nee && last_lambert))
                L = vadd(L, f3(fmul(mr.emission[0], src.x), fmul(mr.emission[1], src.y), fmul(mr.emission[2], src.z)));
            break;
        }
        if (bounces >= p.max_depth) break;
        const uint32_t bounce = bounces++;
        const HitFrame fr = hit_frame(v0, v1, v2, h.u, h.v, h.w, d, p.prim_normals ? p.prim_normals + 9 * (size_t)h.prim : nullptr);
        uint32_t r[4] = {pixel, sample, bounce, 0u};
        philox4x32(r, p.seed_lo, p.seed_hi);
        const F3 li = vnorm(f3(vdot(d, fr.t1), vdot(d, fr.n), vdot(d, fr.t2)));
        F3 lo;
        const bool mirror = mr.material == PT_MAT_MIRROR;
        if (mirror) {
            lo = f3(li.x, -li.y, li.z);
        } else {
            const float u0 = u01(r[0]), u1 = u01(r[1]);
            const float rr = fsqrt(u0);
            float s, c;
            sincos_2pi(u1, s, c);
            const float one_minus = fsub(1.0f, u0);
            lo = f3(fmul(rr, c), fsqrt(0.0f < one_minus ? one_minus : 0.0f), fmul(rr, s));
            if (nee) {
                uint32_t r2[4] = {pixel, sample, bounce, 1u};
                philox4x32(r2, p.seed_lo, p.seed_hi);
                const LightSample ls = sample_light(p, fr, u01(r[2]), u01(r[3]), u01(r2[0]));
                if (ls.valid) {
                    RayState sr;
                    ray_setup(sr, fr.loc.x, fr.loc.y, fr.loc.z, ls.wi.x, ls.wi.y, ls.wi.z);
                    const TraceResult sh = traverse<false>(nodes, tris, p.num_nodes, sr, fmul(ls.dist, 0.999f), true);
                    if (sh.overflow) { atomicExch(p.err, 1); break; }
                    if (sh.prim == kPrimNone) {
                        L = vadd(L, f3(fmul(fmul(fmul(src.x, mr.albedo[0]), ls.le.x), ls.wgt),
                                       fmul(fmul(fmul(src.y, mr.albedo[1]), ls.le.y), ls.wgt),
                                       fmul(fmul(fmul(src.z, mr.albedo[2]), ls.le.z), ls.wgt)));
                    }
                }
            }
        }
        const F3 wo = vnorm(f3(fadd(fadd(fmul(fr.t1.x, lo.x), fmul(fr.n.x, lo.y)), fmul(fr.t2.x, lo.z)),
                               fadd(fadd(fmul(fr.t1.y, lo.x), fmul(fr.n.y, lo.y)), fmul(fr.t2.y, lo.z)),
                               fadd(fadd(fmul(fr.t1.z, lo.x), fmul(fr.n.z, lo.y)), fmul(fr.t2.z, lo.z))));
        o = fr.loc;
        d = wo;
        src = f3(fmul(src.x, mr.albedo[0]), fmul(src.y, mr.albedo[1]), fmul(src.z, mr.albedo[2]));
        last_lambert = !mirror;
    }
    // BoxFilter::AddSample clamp (BoxFilter.cpp:30-33)
    out[0] = L.x > 255 ? 255.f : L.x;
    out[1] = L.y > 255 ? 255.f : L.y;
    out[2] = L.z > 255 ? 255.f : L.z;
}

__global__ void __launch_bounds__(128) path_kernel(const RenderParams p, uint64_t first, uint32_t count,
                                                   float* __restrict__ radiance, uint32_t* __restrict__ primary) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint64_t path = first + i;
    const uint32_t npix = p.width * p.height;
    const uint32_t sample = (uint32_t)(path / npix);
    const uint32_t pixel = (uint32_t)(path % npix);
    const uint32_t x = pixel % p.width, y = pixel / p.width;
    float px = (float)x + 0.5f, py = (float)y + 0.5f;
    if (p.flags & PT_RENDER_JITTER) {
        uint32_t r[4] = {pixel, sample, 0xFFFFu, 0u};
        philox4x32(r, p.seed_lo, p.seed_hi);
        px = fadd((float)x, u01(r[0]));
        py = fadd((float)y, u01(r[1]));
    }
    F3 o, d;
    camera_ray(p.cam, px, py, o, d);
    float L[3];
    path_radiance(p, pixel, sample, o, d, sample == 0 ? primary : nullptr, L);
    radiance[3 * (size_t)i + 0] = L[0];
    radiance[3 * (size_t)i + 1] = L[1];
    radiance[3 * (size_t)i + 2] = L[2];
}

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
struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};
}  // namespace

extern "C" int pt_render(pt_scene* s, const pt_render_desc* desc, float* rgb_out, uint32_t* primary_out,
                         uint32_t mem_flags, void* stream) {
    if (!s || !desc || !rgb_out) return fail(PT_EINVAL, "scene, desc or rgb_out is NULL");
    if (desc->width == 0 || desc->height == 0 || desc->spp == 0) return fail(PT_EINVAL, "empty frame");
    const uint64_t npix64 = (uint64_t)desc->width * desc->height;
    if (npix64 > (1u << 30)) return fail(PT_EINVAL, "frame too large");
    if (desc->flags & ~(uint32_t)(PT_RENDER_NEE | PT_RENDER_JITTER | PT_RENDER_WAVEFRONT))
        return fail(PT_EINVAL, "unknown render flags");
    if ((int)s->max_depth + 2 > PT_TRAVERSAL_STACK) return fail(PT_ESTACK, "tree too deep for the traversal stack");
    const uint32_t npix = (uint32_t)npix64;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != s->device) cudaSetDevice(s->device);
    struct Restore { int d; ~Restore() { if (d >= 0) cudaSetDevice(d); } } restore{prev != s->device ? prev : -1};

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

    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t total = npix64 * desc->spp;
    uint32_t wave = desc->wave_paths ? desc->wave_paths : (1u << 22);
    if (wave > total) wave = (uint32_t)total;
    DevBuf rad, film, rgb_dev, prim_dev;
    if (cudaMalloc(&rad.p, 12 * (size_t)wave) != cudaSuccess || cudaMalloc(&film.p, 12 * (size_t)npix) != cudaSuccess)
        return fail(PT_ENOMEM, "cudaMalloc render buffers");
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
        e = launch_path_wave(p, first, cnt, (float*)rad.p, prim_d, st);
        if (e == cudaSuccess) e = launch_resolve_wave(first, cnt, npix, (const float*)rad.p, (float*)film.p, st);
    }
    if (e == cudaSuccess) e = launch_finish_film((const float*)film.p, npix, desc->spp, rgb_d, st);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("render launch: ") + cudaGetErrorString(e));
    if (dev_out) {
        // buffers freed at scope exit: make the stream finish with them first
        e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(PT_ECUDA, std::string("render: ") + cudaGetErrorString(e));
    } else {
        e = cudaMemcpyAsync(rgb_out, rgb_d, 12 * (size_t)npix, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && primary_out)
            e = cudaMemcpyAsync(primary_out, prim_d, 4 * (size_t)npix, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(PT_ECUDA, std::string("render copy-out: ") + cudaGetErrorString(e));
    }
    int err = 0;
    cudaMemcpy(&err, s->err_flag, sizeof(int), cudaMemcpyDeviceToHost);
    if (err) return fail(PT_ESTACK, "a path exceeded the traversal stack");
    return PT_OK;
}
