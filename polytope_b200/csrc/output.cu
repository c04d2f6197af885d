// output.cu -- the film in the reference's PNG byte format, computed on the device.
//
// PNGFilm::Output (src/cpu/films/PNGFilm.cpp:20-45) stores each channel as
// static_cast<unsigned char>(v > 255 ? 255 : v) with alpha 255, row-major RGBA8.  The kernel below
// does the same per pixel, so only 4 bytes per pixel leave the device instead of 12.

#include <string>

#include "pt_internal.h"
#include "render.h"

namespace pt {

__device__ __forceinline__ unsigned char quantize_channel(float v) {
    const float c = v > 255.f ? 255.f : v;  // the reference's clamp; NaN stays NaN
    // float -> unsigned char truncates toward zero on [0, 256); non-negative films only, NaN -> 0
    return (unsigned char)__float2uint_rz(c);
}

__global__ void __launch_bounds__(256) rgba8_kernel(const float* __restrict__ rgb, uint32_t npix,
                                                   uchar4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const float r = rgb[3 * (size_t)i], g = rgb[3 * (size_t)i + 1], b = rgb[3 * (size_t)i + 2];
    out[i] = make_uchar4(quantize_channel(r), quantize_channel(g), quantize_channel(b), 255);
}

cudaError_t launch_film_to_rgba8(const float* rgb, uint32_t npix, uint8_t* rgba, cudaStream_t s) {
    if (npix == 0) return cudaSuccess;
    rgba8_kernel<<<(npix + 255) / 256, 256, 0, s>>>(rgb, npix, (uchar4*)rgba);
    return cudaGetLastError();
}

}  // namespace pt

using namespace pt;

extern "C" int pt_film_to_rgba8(const float* rgb_dev, uint32_t width, uint32_t height, uint8_t* rgba_out,
                                uint32_t mem_flags, void* stream) {
    if (!rgb_dev || !rgba_out) return fail(PT_EINVAL, "rgb_dev or rgba_out is NULL");
    const uint64_t npix = (uint64_t)width * height;
    if (npix == 0) return PT_OK;
    if (npix > (1u << 30)) return fail(PT_EINVAL, "film too large");
    cudaStream_t st = (cudaStream_t)stream;
    const bool dev_out = (mem_flags & PT_MEM_DEVICE) != 0;
    void* out = rgba_out;
    if (!dev_out && cudaMallocAsync(&out, 4 * npix, st) != cudaSuccess) {
        cudaGetLastError();
        return fail(PT_ENOMEM, "device memory for the RGBA8 film");
    }
    cudaError_t e = launch_film_to_rgba8(rgb_dev, (uint32_t)npix, (uint8_t*)out, st);
    if (!dev_out) {
        if (e == cudaSuccess) e = cudaMemcpyAsync(rgba_out, out, 4 * npix, cudaMemcpyDeviceToHost, st);
        cudaFreeAsync(out, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("film to RGBA8: ") + cudaGetErrorString(e));
    return PT_OK;
}
