// launch.h -- host-callable launchers implemented in the .cu translation units.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace pt {

struct TraceArgs {
    const void* nodes;     // uint4 x 2 per node
    const void* tris;      // float4 x 3 per leaf-ordered face
    uint32_t num_nodes;
    const void* rays;      // float4 x 2 per ray
    void* hits;            // uint4 per ray
    uint64_t n;
    uint32_t* node_tests;  // optional
    uint32_t* tri_tests;   // optional
    int* err;              // device flag, set to 1 when a ray overflowed its stack
    void* counter;         // device 64-bit ray counter for the persistent kernel (null: one thread per ray)
    int shared_stack;      // stack entries per lane kept in shared memory (0, 8 or 16)
    uint32_t chunk;        // rays a warp takes per fetch (0 = 64)
    // two-level scenes: instances and the top-level tree (null for a flattened scene)
    const void* instances = nullptr;
    const void* top_nodes = nullptr;
    uint32_t top_num_nodes = 0;
    bool exact_tree = false;  // some box holds a NaN: every ray takes the exact box test
};

cudaError_t launch_trace(const TraceArgs& a, cudaStream_t s);

// Device self-tests of the exact-arithmetic helpers (used by the GPU parity tests).
cudaError_t launch_selftest_f64(const float* in4, float* out, uint32_t n, cudaStream_t s);
cudaError_t launch_selftest_sincos(const float* u, float* out2, uint32_t n, cudaStream_t s);
cudaError_t launch_selftest_philox(const uint32_t* in4, uint32_t* out4, uint32_t n, uint64_t seed, cudaStream_t s);
// Box test as the traversal kernels run it: in16 = {bb[6], org[3], dir[3], tmax, 0, 0, 0}.
cudaError_t launch_selftest_box(const float* in16, uint32_t* hit, uint32_t n, cudaStream_t s);

}  // namespace pt
