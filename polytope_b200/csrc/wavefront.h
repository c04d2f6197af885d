// wavefront.h -- the multi-render wavefront engine, shared by pt_render's wavefront mode,
// pt_batch and pt_server.
//
// A wave is a set of path slots.  Each slot runs one path of one render (item); the slots of a
// wave are grouped in segments, each a run of consecutive paths of one item (paths of a render
// are numbered sample-major: path = sample * npix + pixel).  Per bounce an extend kernel traces
// the queued slots' rays (closest hit), a shade kernel runs the integrator step and appends the
// next rays and the shadow rays to queues (warp-vote compaction, one atomic per warp), and a
// shadow kernel traces the shadow rays (any hit).  The extend and shadow kernels are persistent:
// warps fetch chunks of queue entries and refill lanes as rays finish.  After the last bounce the
// clamped radiance of each slot is added to its item's film sums in sample order (resolve), and
// items whose last path ran in this wave get their film (finish).
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "render.h"

namespace pt {

struct WfItem {
    const RenderParams* params;  // device copy of the render's parameters
    float* film;                 // device film sums (3 floats per pixel), zero before the first wave
    float* rgb;                  // device film output (3 floats per pixel)
    uint32_t* primary;           // device primary ids (or null)
    uint32_t npix, spp;
};

// Slots [slot_base, slot_base + count) of a wave run paths [local_begin, local_begin + count) of
// item `item`.
struct WfSegment {
    uint32_t item;
    uint32_t pad;
    uint64_t local_begin;
    uint64_t slot_base;
    uint64_t count;
};

// Resolve / finish work: pixels [pix_begin, pix_begin + pix_count) of the item of segment `seg`;
// `base` is the prefix of pix_count over the wave's entries.
struct WfPixels {
    uint32_t seg;
    uint32_t pix_begin, pix_count;
    uint32_t item;
    uint64_t base;
};

struct WfState {
    float4* ray_o;       // origin.xyz, w = item (bits)
    float4* ray_d;       // direction.xyz, w = bounces (bits)
    float4* thr;         // throughput rgb, w = last bounce was Lambert (bits)
    float4* rad;         // accumulated radiance rgb
    uint64_t* path;      // local path index within the item
    uint4* hit;          // prim, leaf, u, v
    float* hit_w;        // w barycentric
    uint32_t* queue[2];  // extend queues (ping-pong)
    float4* sh_o;        // shadow rays: origin, tmax
    float4* sh_d;        // direction, slot (bits)
    float4* sh_c;        // contribution rgb
    float* radiance;     // clamped path radiance, 3 floats per slot (resolve input)
    uint32_t* counters;  // [0], [1] extend queue lengths, [2] shadow queue length; u64 fetch counters at [4], [6]
    uint32_t capacity;
};

// Device bytes of the state of `capacity` slots, and its layout in one buffer.  paths_only keeps
// just the radiance and the counters (all the persistent path kernel uses).
size_t wf_state_bytes(uint32_t capacity, bool paths_only = false);
void wf_state_carve(void* base, uint32_t capacity, WfState& ws, bool paths_only = false);

struct WfTuning {
    uint32_t threads_per_block = 128;  // extend / shadow kernels
    uint32_t queue_chunk = 64;         // rays a warp takes per fetch in the persistent kernels
    int stack_cap = 64;                // traversal stack entries
    bool paths = false;                // one thread per whole path instead of per-bounce kernels
    bool two_level = false;            // (paths only) some item is a two-level scene
};

// One wave: `count` slots, `bounces` extend/shade/shadow iterations, and its ranges in the plan's
// segment / resolve / finish tables.
struct WfWave {
    uint32_t count;
    uint32_t bounces;
    uint32_t seg_begin, seg_count;
    uint32_t res_begin, res_count;
    uint64_t res_pixels;
    uint32_t fin_begin, fin_count;
    uint64_t fin_pixels;
};

struct WfPlan {
    std::vector<WfWave> waves;
    std::vector<WfSegment> segments;
    std::vector<WfPixels> resolve;
    std::vector<WfPixels> finish;
};

// Appends one wave made of the given segments (each a path range of an item).  `npix`, `spp` and
// `max_depth` are per item; an item is finished in this wave when a segment reaches its last path.
void wf_add_wave(WfPlan& plan, const std::vector<WfSegment>& segs, const std::vector<uint32_t>& npix,
                 const std::vector<uint32_t>& spp, const std::vector<uint32_t>& max_depth);

// Plans waves of at most wave_paths slots over the items' paths concatenated in item order.
void wf_plan_all(WfPlan& plan, const std::vector<uint32_t>& npix, const std::vector<uint32_t>& spp,
                 const std::vector<uint32_t>& max_depth, uint64_t wave_paths);

// Enqueues one wave on `s` (per-bounce kernels, or with t.paths one kernel running whole paths).  d_items / d_segments / d_resolve / d_finish are device copies of the
// plan's tables (the wave's ranges index into them).
cudaError_t wf_launch_wave(const WfItem* d_items, const WfSegment* d_segments, const WfPixels* d_resolve,
                           const WfPixels* d_finish, const WfWave& w, const WfState& ws, const WfTuning& t,
                           unsigned long long* rays_traced, cudaStream_t s);

}  // namespace pt
