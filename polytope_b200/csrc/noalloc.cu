// noalloc.cu -- pt_render_noalloc: the fused render with its scratch memory in a fixed device array.
//
// pt_render allocates its scratch (the per-wave radiance buffer and the film sums) with
// cudaMalloc and releases it with cudaFree on every call.  Some callers cannot do that: an
// application that owns the whole device-memory budget and forbids allocations once it has
// started, or a per-frame loop that cannot afford cudaFree's implicit device-wide synchronisation.
// This entry point runs the same kernels with the scratch taken from a file-scope device array
// instead, so the call itself allocates nothing.  Limits: at most kMaxPixels pixels per frame and
// at most kMaxWavePaths paths per wave (6 MiB in total, held by every device that loads the
// library until the process exits).  Like every asynchronous call it leaves guard failures of its
// kernels in the scene's device flag, which pt_scene_status reports once the frame is done.

#include <mutex>
#include <string>

#include "pt_internal.h"
#include "render.h"

namespace pt {
namespace {

constexpr uint32_t kMaxPixels = 512u * 512u;      // film sums: 3 floats per pixel
constexpr uint32_t kMaxWavePaths = 512u * 512u;   // wave radiance: 3 floats per path
constexpr size_t kFilmFloats = 3 * (size_t)kMaxPixels;
constexpr size_t kWaveFloats = 3 * (size_t)kMaxWavePaths;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float g_render_scratch[kFilmFloats + kWaveFloats];

std::mutex g_scratch_mu;
float* g_scratch_addr[kMaxDevices] = {};

// The device address of g_render_scratch on `device` (which must be current).  In host code the
// array's name only stands for the symbol; the address has to be looked up once per device.
int scratch_for_device(int device, float** out) {
    if (device < 0 || device >= kMaxDevices) return fail(PT_EINVAL, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_render_scratch);
        if (e != cudaSuccess) return fail(PT_ECUDA, std::string("cudaGetSymbolAddress(render scratch): ") + cudaGetErrorString(e));
        g_scratch_addr[device] = (float*)p;
    }
    *out = g_scratch_addr[device];
    return PT_OK;
}

}  // namespace
}  // namespace pt

using namespace pt;

extern "C" int pt_render_noalloc(pt_scene* s, const pt_render_desc* desc, float* rgb_dev, uint32_t* primary_dev,
                                 void* stream) {
    int rc = check_render_desc(s, desc);
    if (rc) return rc;
    if (!rgb_dev) return fail(PT_EINVAL, "rgb_dev is NULL");
    if (desc->flags & (PT_RENDER_WAVEFRONT | PT_RENDER_PERSISTENT))
        return fail(PT_EINVAL, "pt_render_noalloc runs the fused path kernel only (PT_RENDER_WAVEFRONT and "
                               "PT_RENDER_PERSISTENT are not accepted)");
    const uint64_t npix64 = (uint64_t)desc->width * desc->height;
    if (npix64 > kMaxPixels)
        return fail(PT_EINVAL, "frame of " + std::to_string(npix64) + " pixels exceeds the pt_render_noalloc limit of " +
                                   std::to_string(kMaxPixels) + " pixels (use pt_render)");
    const uint32_t npix = (uint32_t)npix64;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return fail(PT_ECUDA, "cudaGetDevice failed");
    if (prev != s->device && cudaSetDevice(s->device) != cudaSuccess) return fail(PT_ECUDA, "cudaSetDevice failed");
    struct Restore { int d; ~Restore() { if (d >= 0) cudaSetDevice(d); } } restore{prev != s->device ? prev : -1};

    float* scratch = nullptr;
    rc = scratch_for_device(s->device, &scratch);
    if (rc) return rc;
    float* film = scratch;                 // kFilmFloats
    float* radiance = scratch + kFilmFloats;  // kWaveFloats

    const RenderParams p = render_params(s, desc);
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t total = npix64 * desc->spp;
    uint64_t wave = desc->wave_paths ? desc->wave_paths : kMaxWavePaths;
    if (wave > kMaxWavePaths) wave = kMaxWavePaths;
    if (wave > total) wave = total;
    // The array keeps the previous call's contents: the film sums must start at zero.
    cudaError_t e = cudaMemsetAsync(film, 0, 12 * (size_t)npix, st);
    for (uint64_t first = 0; e == cudaSuccess && first < total; first += wave) {
        const uint32_t cnt = (uint32_t)(total - first < wave ? total - first : wave);
        e = launch_path_wave(p, first, cnt, radiance, primary_dev, st);
        if (e == cudaSuccess) e = launch_resolve_wave(first, cnt, npix, radiance, film, st);
    }
    if (e == cudaSuccess) e = launch_finish_film(film, npix, desc->spp, rgb_dev, st);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("pt_render_noalloc launch: ") + cudaGetErrorString(e));
    return PT_OK;
}
