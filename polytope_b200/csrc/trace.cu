// trace.cu -- ray-query kernels (Scene::intersect replacement) for sm_100a.
//
// One thread per ray, reference-order traversal (traverse.cuh).  Rays and hits stream through
// HBM once (32 B in, 16 B out per ray); nodes and faces are read with 128-bit read-only loads and
// stay resident in the 126 MB L2 for scenes up to a few million faces.

#include "launch.h"
#include "traverse.cuh"

namespace pt {

template <bool COUNT>
__global__ void __launch_bounds__(128) trace_kernel(const uint4* __restrict__ nodes, const float4* __restrict__ tris,
                                                    uint32_t num_nodes, const float4* __restrict__ rays,
                                                    uint4* __restrict__ hits, uint64_t n, uint32_t* node_tests,
                                                    uint32_t* tri_tests, int* err) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 r0 = __ldg(rays + 2 * i);
    const float4 r1 = __ldg(rays + 2 * i + 1);
    RayState rs;
    ray_setup(rs, r0.x, r0.y, r0.z, r1.x, r1.y, r1.z);
    const bool any = (__float_as_uint(r1.w) & 1u) != 0;
    const TraceResult tr = traverse<COUNT>(nodes, tris, num_nodes, rs, r0.w, any);
    uint4 h;
    h.x = tr.prim;
    h.y = __float_as_uint(tr.t);
    h.z = __float_as_uint(tr.u);
    h.w = __float_as_uint(tr.v);
    if (tr.overflow) {
        h.x = 0xFFFFFFFEu;
        atomicExch(err, 1);
    }
    hits[i] = h;
    if (COUNT) {
        if (node_tests) node_tests[i] = tr.nodes;
        if (tri_tests) tri_tests[i] = tr.tris;
    }
}

cudaError_t launch_trace(const TraceArgs& a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    const uint32_t block = 128;
    const uint64_t grid = (a.n + block - 1) / block;
    if (grid > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    if (a.node_tests || a.tri_tests)
        trace_kernel<true><<<(unsigned)grid, block, 0, s>>>(
            (const uint4*)a.nodes, (const float4*)a.tris, a.num_nodes, (const float4*)a.rays, (uint4*)a.hits, a.n,
            a.node_tests, a.tri_tests, a.err);
    else
        trace_kernel<false><<<(unsigned)grid, block, 0, s>>>(
            (const uint4*)a.nodes, (const float4*)a.tris, a.num_nodes, (const float4*)a.rays, (uint4*)a.hits, a.n,
            nullptr, nullptr, a.err);
    return cudaGetLastError();
}

// ---- self-tests of the exact helpers ------------------------------------------------------------

__global__ void selftest_f64_kernel(const float4* in, float* out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = in[i];
    out[i] = f64_diff_emulated(v.x, v.y, v.z, v.w);
}

__global__ void selftest_sincos_kernel(const float* u, float2* out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s, c;
    sincos_2pi(u[i], s, c);
    out[i] = make_float2(s, c);
}

__global__ void selftest_philox_kernel(const uint4* in, uint4* out, uint32_t n, uint32_t k0, uint32_t k1) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 v = in[i];
    uint32_t c[4] = {v.x, v.y, v.z, v.w};
    philox4x32(c, k0, k1);
    out[i] = make_uint4(c[0], c[1], c[2], c[3]);
}

cudaError_t launch_selftest_f64(const float* in4, float* out, uint32_t n, cudaStream_t s) {
    if (!n) return cudaSuccess;
    selftest_f64_kernel<<<(n + 127) / 128, 128, 0, s>>>((const float4*)in4, out, n);
    return cudaGetLastError();
}
cudaError_t launch_selftest_sincos(const float* u, float* out2, uint32_t n, cudaStream_t s) {
    if (!n) return cudaSuccess;
    selftest_sincos_kernel<<<(n + 127) / 128, 128, 0, s>>>(u, (float2*)out2, n);
    return cudaGetLastError();
}
cudaError_t launch_selftest_philox(const uint32_t* in4, uint32_t* out4, uint32_t n, uint64_t seed, cudaStream_t s) {
    if (!n) return cudaSuccess;
    selftest_philox_kernel<<<(n + 127) / 128, 128, 0, s>>>((const uint4*)in4, (uint4*)out4, n, (uint32_t)seed,
                                                          (uint32_t)(seed >> 32));
    return cudaGetLastError();
}

}  // namespace pt
