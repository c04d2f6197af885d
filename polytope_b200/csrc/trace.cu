// trace.cu -- ray-query kernels (Scene::intersect replacement) for sm_100a.
//
// One thread per ray, reference-order traversal (traverse.cuh).  Rays and hits stream through
// HBM once (32 B in, 16 B out per ray); nodes and faces are read with 128-bit read-only loads and
// stay resident in the 126 MB L2 for scenes up to a few million faces.

#include <type_traits>

#include "launch.h"
#include "traverse.cuh"
#include "two_level.cuh"

namespace pt {

template <bool COUNT>
__global__ void __launch_bounds__(128) trace_kernel(const uint4* __restrict__ nodes, const float4* __restrict__ tris,
                                                    uint32_t num_nodes, const float4* __restrict__ rays,
                                                    uint4* __restrict__ hits, uint64_t n, uint32_t* node_tests,
                                                    uint32_t* tri_tests, int* err, bool exact_tree) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 r0 = ld_stream(rays + 2 * i);
    const float4 r1 = ld_stream(rays + 2 * i + 1);
    RayState rs;
    ray_setup(rs, r0.x, r0.y, r0.z, r1.x, r1.y, r1.z);
    const bool any = (__float_as_uint(r1.w) & 1u) != 0;
    const TraceResult tr = traverse<COUNT>(nodes, tris, num_nodes, rs, r0.w, any, exact_tree);
    uint4 h;
    h.x = tr.prim;
    h.y = __float_as_uint(tr.t);
    h.z = __float_as_uint(tr.u);
    h.w = __float_as_uint(tr.v);
    if (tr.overflow) {
        h.x = 0xFFFFFFFEu;
        atomicExch(err, 1);
    }
    st_stream(hits + i, h);
    if (COUNT) {
        if (node_tests) node_tests[i] = tr.nodes;
        if (tri_tests) tri_tests[i] = tr.tris;
    }
}

// Persistent variant: a grid sized to the SMs; each warp takes chunks of kChunk rays from a global
// counter and refills a lane as soon as its ray finishes, so lanes stay busy despite rays of very
// different cost (any-hit rays stop early, closest-hit rays run long).  Each pass of the outer loop
// steps the walking lanes node by node until PT_LEAF_BATCH_TRACE of them hold a leaf or have
// ended, then tests those leaves' faces together (walk_round, traverse.cuh).  A ray's own node and face order is exactly
// the reference's; only which rays share a warp, and when a lane waits, changes.
// 8 blocks of 128 per SM (64 registers, almost no spills) measured 2.6 % faster than 9 blocks at
// 56 registers, where the warp vote's live state spilled.
// Node steps a walking lane takes between ballots (a lane that reaches a leaf stops early).
// Measured on a B200 (16.7 M microbench rays, two runs each, same box): 1 step 2142 -> 2 steps
// (before the node-step changes); with them 2 steps 2428, 3 steps 2470, 4 steps 2067 Mrays/s.
#ifndef PT_TRACE_STEPS
#define PT_TRACE_STEPS 3
#endif
template <bool COUNT, int SH>
__global__ void __launch_bounds__(128, 8) trace_persistent_kernel(const uint4* __restrict__ nodes,
                                                               const float4* __restrict__ tris, uint32_t num_nodes,
                                                               const float4* __restrict__ rays, uint4* __restrict__ hits,
                                                               uint64_t n, uint32_t* node_tests, uint32_t* tri_tests,
                                                               int* err, unsigned long long* counter, uint32_t kChunk,
                                                               bool exact_tree) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint64_t pool_next = 0, pool_end = 0;
    bool exhausted = false, active = false;
    uint64_t idx = 0;
    __shared__ uint32_t sstack[SH > 0 ? SH * 128 : 1];
    RayWalkT<kStackCap, SH> k;
    k.stack.base = sstack + threadIdx.x;
    k.stack.stride = 128;
    while (true) {
        // refill idle lanes from the warp's chunk
        const uint32_t need = __ballot_sync(0xFFFFFFFFu, !active);
        if (need && !exhausted && pool_next >= pool_end) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(counter, (unsigned long long)kChunk);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base >= n) {
                exhausted = true;
            } else {
                pool_next = base;
                pool_end = base + kChunk < n ? base + kChunk : n;
            }
        }
        if (need) {
            const uint64_t avail = pool_end - pool_next;
            const uint32_t rank = __popc(need & lt_mask);
            if (!active && rank < avail) {
                idx = pool_next + rank;
                const float4 r0 = ld_stream(rays + 2 * idx);
                const float4 r1 = ld_stream(rays + 2 * idx + 1);
                walk_begin(k, r0.x, r0.y, r0.z, r1.x, r1.y, r1.z, r0.w, (__float_as_uint(r1.w) & 1u) != 0, exact_tree);
                active = true;
            }
            const uint64_t took = (uint64_t)__popc(need) < avail ? (uint64_t)__popc(need) : avail;
            pool_next += took;
        }
        if (!__any_sync(0xFFFFFFFFu, active)) {
            if (exhausted || pool_next >= pool_end) {
                if (exhausted) break;
            }
            continue;
        }
        uint32_t leaf_off = 0, leaf_n = 0;
        bool ok, at_leaf;
        if constexpr (PT_LEAF_BATCH_TRACE > 0) {
            // walk_round (traverse.cuh), written out here: the compiler allocates this form with
            // fewer spills, which measured 9 % faster on the 1.3 M-face microbench; each lane takes
            // up to PT_TRACE_STEPS node steps per ballot (fewer votes; a lane that reaches a leaf
            // skips the rest)
            ok = true;
            at_leaf = false;
            const uint32_t cand = __ballot_sync(0xFFFFFFFFu, active && k.sp > 0);
            const int want = __popc(cand) < PT_LEAF_BATCH_TRACE ? __popc(cand) : PT_LEAF_BATCH_TRACE;
            // the round's node steps, with the box test chosen once for the warp when every ray in
            // it takes the min/max form (box_mode 0) instead of per step: 2437 vs 2337 Mrays/s on a
            // B200 (1.3 M faces, 16.7 M rays)
            auto round = [&](auto fast) {
                constexpr bool kFast = decltype(fast)::value;
                while (true) {
                    const bool walking = active && ok && !at_leaf && k.sp > 0;
                    const uint32_t w = __ballot_sync(0xFFFFFFFFu, walking);
                    if (w == 0 || __popc(cand & ~w) >= want) break;
                    if (walking) {
                        int r = walk_step<COUNT, kFast>(k, nodes, num_nodes, leaf_off, leaf_n);
#pragma unroll
                        for (int extra = 1; extra < PT_TRACE_STEPS; ++extra)
                            if (r == 0 && k.sp > 0) r = walk_step<COUNT, kFast>(k, nodes, num_nodes, leaf_off, leaf_n);
                        at_leaf = r > 0;
                        ok = r >= 0;
                    }
                }
            };
            if (__all_sync(0xFFFFFFFFu, !active || k.box_mode == 0))
                round(std::true_type{});
            else
                round(std::false_type{});
        } else {
            ok = !active || walk_to_leaf<COUNT>(k, nodes, num_nodes, leaf_off, leaf_n);
            at_leaf = active && ok && leaf_n > 0;
        }
        if (at_leaf) walk_leaf<COUNT>(k, tris, leaf_off, leaf_n);
        if (active) {
            if (!ok || k.done || k.sp == 0) {
                uint4 h;
                h.x = ok ? k.prim : 0xFFFFFFFEu;
                h.y = __float_as_uint(k.min_t);
                h.z = __float_as_uint(k.u);
                h.w = __float_as_uint(k.v);
                if (!ok) atomicExch(err, 1);
                st_stream(hits + idx, h);
                if (COUNT) {
                    if (node_tests) node_tests[idx] = k.nodes;
                    if (tri_tests) tri_tests[idx] = k.tris;
                }
                active = false;
            }
        }
    }
}

// Ray queries on a two-level scene: one thread per ray, traverse_two_level.
template <bool COUNT>
__global__ void __launch_bounds__(128) trace_two_level_kernel(const TwoLevelView v, const float4* __restrict__ rays,
                                                              uint4* __restrict__ hits, uint64_t n, uint32_t* node_tests,
                                                              uint32_t* tri_tests, int* err) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 r0 = ld_stream(rays + 2 * i);
    const float4 r1 = ld_stream(rays + 2 * i + 1);
    const bool any = (__float_as_uint(r1.w) & 1u) != 0;
    const TwoLevelHit th = traverse_two_level<COUNT>(v, r0.x, r0.y, r0.z, r1.x, r1.y, r1.z, r0.w, any);
    uint4 h;
    h.x = th.r.prim;
    h.y = __float_as_uint(th.r.t);
    h.z = __float_as_uint(th.r.u);
    h.w = __float_as_uint(th.r.v);
    if (th.r.overflow) {
        h.x = 0xFFFFFFFEu;
        atomicExch(err, 1);
    }
    st_stream(hits + i, h);
    if (COUNT) {
        if (node_tests) node_tests[i] = th.r.nodes;
        if (tri_tests) tri_tests[i] = th.r.tris;
    }
}

cudaError_t launch_trace(const TraceArgs& a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    if (a.instances) {
        const TwoLevelView v{(const uint4*)a.nodes, (const float4*)a.tris, a.num_nodes, (const uint4*)a.top_nodes,
                             a.top_num_nodes, (const DeviceInstance*)a.instances, a.exact_tree};
        const uint64_t grid = (a.n + 127) / 128;
        if (grid > 0x7FFFFFFFull) return cudaErrorInvalidValue;
        if (a.node_tests || a.tri_tests)
            trace_two_level_kernel<true><<<(unsigned)grid, 128, 0, s>>>(v, (const float4*)a.rays, (uint4*)a.hits, a.n,
                                                                        a.node_tests, a.tri_tests, a.err);
        else
            trace_two_level_kernel<false><<<(unsigned)grid, 128, 0, s>>>(v, (const float4*)a.rays, (uint4*)a.hits, a.n,
                                                                         nullptr, nullptr, a.err);
        return cudaGetLastError();
    }
    if (a.counter) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const bool counted = a.node_tests || a.tri_tests;
        const int sh = a.shared_stack;
        auto pick = [sh](auto k0, auto k8, auto k16, auto k24, auto k32) {
            return sh >= 32 ? k32 : sh >= 24 ? k24 : sh >= 16 ? k16 : sh >= 8 ? k8 : k0;
        };
        auto kern_f = pick(trace_persistent_kernel<false, 0>, trace_persistent_kernel<false, 8>, trace_persistent_kernel<false, 16>,
                           trace_persistent_kernel<false, 24>, trace_persistent_kernel<false, 32>);
        auto kern_t = pick(trace_persistent_kernel<true, 0>, trace_persistent_kernel<true, 8>, trace_persistent_kernel<true, 16>,
                           trace_persistent_kernel<true, 24>, trace_persistent_kernel<true, 32>);
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, counted ? kern_t : kern_f, 128, 0);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) per_sm = 1;
        uint64_t grid = (uint64_t)sms * per_sm;
        const uint32_t ch = a.chunk ? a.chunk : 64u;
        const uint64_t need = ((a.n + ch - 1) / ch * 32 + 127) / 128;
        if (grid > need) grid = need;
        e = cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), s);
        if (e != cudaSuccess) return e;
        if (counted)
            kern_t<<<(unsigned)grid, 128, 0, s>>>((const uint4*)a.nodes, (const float4*)a.tris, a.num_nodes,
                                                  (const float4*)a.rays, (uint4*)a.hits, a.n, a.node_tests, a.tri_tests,
                                                  a.err, (unsigned long long*)a.counter, a.chunk ? a.chunk : 64u, a.exact_tree);
        else
            kern_f<<<(unsigned)grid, 128, 0, s>>>((const uint4*)a.nodes, (const float4*)a.tris, a.num_nodes,
                                                  (const float4*)a.rays, (uint4*)a.hits, a.n, nullptr, nullptr, a.err,
                                                  (unsigned long long*)a.counter, a.chunk ? a.chunk : 64u, a.exact_tree);
        return cudaGetLastError();
    }
    const uint32_t block = 128;
    const uint64_t grid = (a.n + block - 1) / block;
    if (grid > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    if (a.node_tests || a.tri_tests)
        trace_kernel<true><<<(unsigned)grid, block, 0, s>>>(
            (const uint4*)a.nodes, (const float4*)a.tris, a.num_nodes, (const float4*)a.rays, (uint4*)a.hits, a.n,
            a.node_tests, a.tri_tests, a.err, a.exact_tree);
    else
        trace_kernel<false><<<(unsigned)grid, block, 0, s>>>(
            (const uint4*)a.nodes, (const float4*)a.tris, a.num_nodes, (const float4*)a.rays, (uint4*)a.hits, a.n,
            nullptr, nullptr, a.err, a.exact_tree);
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

__global__ void selftest_box_kernel(const float* in, uint32_t* out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* c = in + 16 * (size_t)i;
    RayState r;
    ray_setup(r, c[6], c[7], c[8], c[9], c[10], c[11]);
    // as a traversal runs it: the scene-level NaN flag set when this box holds a NaN, then the
    // ray's own box mode (the min/max test for finite rays)
    bool nan_box = false;
    for (int k = 0; k < 6; ++k) nan_box = nan_box || c[k] != c[k];
    out[i] = box_test(r, box_mode_for(r, c[12], nan_box), c[0], c[1], c[2], c[3], c[4], c[5], c[12]) ? 1u : 0u;
}

cudaError_t launch_selftest_box(const float* in16, uint32_t* hit, uint32_t n, cudaStream_t s) {
    if (!n) return cudaSuccess;
    selftest_box_kernel<<<(n + 127) / 128, 128, 0, s>>>(in16, hit, n);
    return cudaGetLastError();
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
