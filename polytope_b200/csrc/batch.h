// batch.h -- the multi-render kernel shared by pt_batch_* and the serving loop.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "render.h"

namespace pt {

// A pixel range of one render inside a launch: the launch's pixels are numbered
// base .. base + px_count - 1 for this item, which covers pixels px_begin .. px_begin + px_count - 1
// of its frame.  Items are sorted by base.
struct BatchItem {
    const RenderParams* params;  // device copy of the render's parameters
    float* rgb;                  // device film of the whole frame (3 floats per pixel)
    uint32_t* primary;           // device primary ids of the whole frame
    uint32_t px_begin;
    uint32_t px_count;
    uint64_t base;
};

// Smallest supported stack capacity >= max(tree depth + 2, requested); 0 if none fits.
int stack_cap_for(uint32_t max_tree_depth, uint32_t requested);
int check_tuning(const pt_batch_tuning& t);
// two_level: some item is a two-level scene (the kernel then handles both layouts).
cudaError_t launch_batch(const BatchItem* items, uint32_t n_items, uint64_t first, uint64_t count,
                         unsigned long long* counter, const pt_batch_tuning& t, int cap, unsigned long long* rays,
                         cudaStream_t s, bool two_level = false);

}  // namespace pt
