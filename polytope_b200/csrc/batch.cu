// batch.cu -- many renders in one persistent launch (batched uneven scenes), shared with the
// serving loop.
//
// Work is pixel-major: a lane takes one pixel of one render and traces that pixel's samples in
// sample order, summing the clamped radiance as BoxFilter::Output does (BoxFilter.cpp:54-71), so
// every film is bit-identical to pt_render's whatever the mix.  A grid sized to the SMs runs until
// the launch's pixel range is exhausted: warps take chunks of pixels from a global counter and a
// lane starts its next pixel as soon as its current one has all its samples, so renders of very
// different resolution, spp, depth and scene size share the GPU without idle lanes.  The launch
// sequence of a batch (counter resets + waves) is captured once in a CUDA graph and replayed.

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "batch.h"
#include "path.cuh"
#include "pt_internal.h"
#include "wavefront.h"

namespace pt {

// At most 64 registers (4 blocks of 256, 8 of 128 per SM), as the fused path kernel: the 6.55
// M-face frame as a one-item batch 1816 -> 1865 Msamples/s on a B200.
template <int CAP, bool TWO_LEVEL>
__global__ void __launch_bounds__(256, 4) batch_kernel(const BatchItem* __restrict__ items, uint32_t n_items, uint64_t first,
                                                    uint64_t count, unsigned long long* counter, uint32_t chunk,
                                                    unsigned long long* rays_traced) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint64_t pool_next = 0, pool_end = 0;
    bool exhausted = false, active = false;
    const RenderParams* p = nullptr;
    const BatchItem* it = nullptr;
    uint32_t px = 0, npix = 0, sample = 0, spp = 0;
    float sum[3] = {0.f, 0.f, 0.f};
    uint32_t rays = 0;
    while (true) {
        const uint32_t need = __ballot_sync(0xFFFFFFFFu, !active);
        if (need && !exhausted && pool_next >= pool_end) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(counter, (unsigned long long)chunk);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base >= count) {
                exhausted = true;
            } else {
                pool_next = base;
                pool_end = base + chunk < count ? base + chunk : count;
            }
        }
        if (need) {
            const uint64_t avail = pool_end - pool_next;
            const uint32_t rank = __popc(need & lt_mask);
            if (!active && rank < avail) {
                const uint64_t g = first + pool_next + rank;
                uint32_t lo = 0, hi = n_items - 1;  // last item whose base <= g
                while (lo < hi) {
                    const uint32_t mid = (lo + hi + 1) / 2;
                    if (items[mid].base <= g) lo = mid; else hi = mid - 1;
                }
                it = items + lo;
                p = it->params;
                px = it->px_begin + (uint32_t)(g - it->base);
                npix = p->width * p->height;
                spp = p->spp;
                sample = 0;
                sum[0] = sum[1] = sum[2] = 0.f;
                active = true;
            }
            const uint64_t took = (uint64_t)__popc(need) < avail ? (uint64_t)__popc(need) : avail;
            pool_next += took;
        }
        if (!__any_sync(0xFFFFFFFFu, active)) {
            if (exhausted) break;
            continue;
        }
        if (active) {
            float L[3];
            rays += path_fused<CAP, TWO_LEVEL>(*p, (uint64_t)sample * npix + px, L, sample == 0 ? it->primary : nullptr);
            sum[0] = fadd(sum[0], L[0]);
            sum[1] = fadd(sum[1], L[1]);
            sum[2] = fadd(sum[2], L[2]);
            if (++sample == spp) {
                const float inv = frcp((float)spp);
                it->rgb[3 * (size_t)px + 0] = fmul(sum[0], inv);
                it->rgb[3 * (size_t)px + 1] = fmul(sum[1], inv);
                it->rgb[3 * (size_t)px + 2] = fmul(sum[2], inv);
                active = false;
            }
        }
    }
    if (rays_traced) {
        const uint32_t s = __reduce_add_sync(0xFFFFFFFFu, rays);
        if (lane == 0 && s) atomicAdd(rays_traced, (unsigned long long)s);
    }
}

namespace {
template <int CAP, bool TWO_LEVEL>
cudaError_t launch_cap(const BatchItem* items, uint32_t n_items, uint64_t first, uint64_t count, unsigned long long* counter,
                       const pt_batch_tuning& t, unsigned long long* rays, cudaStream_t s) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<CAP, TWO_LEVEL>, (int)t.threads_per_block, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const uint64_t warps_needed = (count + t.queue_chunk - 1) / t.queue_chunk;
    uint64_t grid = (uint64_t)sms * per_sm;
    const uint64_t grid_needed = (warps_needed * 32 + t.threads_per_block - 1) / t.threads_per_block;
    if (grid > grid_needed) grid = grid_needed ? grid_needed : 1;
    e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    batch_kernel<CAP, TWO_LEVEL><<<(unsigned)grid, t.threads_per_block, 0, s>>>(items, n_items, first, count, counter,
                                                                              t.queue_chunk, rays);
    return cudaGetLastError();
}
}  // namespace

int stack_cap_for(uint32_t max_tree_depth, uint32_t requested) {
    const uint32_t need = max_tree_depth + 2;
    const int caps[] = {24, 32, 48, 64};
    for (int c : caps)
        if ((uint32_t)c >= need && (uint32_t)c >= requested) return c;
    return 0;
}

cudaError_t launch_batch(const BatchItem* items, uint32_t n_items, uint64_t first, uint64_t count, unsigned long long* counter,
                         const pt_batch_tuning& t, int cap, unsigned long long* rays, cudaStream_t s, bool two_level) {
    if (count == 0) return cudaSuccess;
    if (two_level) {  // some item is a two-level scene: the kernel that handles both layouts
        switch (cap) {
            case 24: return launch_cap<24, true>(items, n_items, first, count, counter, t, rays, s);
            case 32: return launch_cap<32, true>(items, n_items, first, count, counter, t, rays, s);
            case 48: return launch_cap<48, true>(items, n_items, first, count, counter, t, rays, s);
            default: return launch_cap<64, true>(items, n_items, first, count, counter, t, rays, s);
        }
    }
    switch (cap) {
        case 24: return launch_cap<24, false>(items, n_items, first, count, counter, t, rays, s);
        case 32: return launch_cap<32, false>(items, n_items, first, count, counter, t, rays, s);
        case 48: return launch_cap<48, false>(items, n_items, first, count, counter, t, rays, s);
        default: return launch_cap<64, false>(items, n_items, first, count, counter, t, rays, s);
    }
}

int check_tuning(const pt_batch_tuning& t) {
    if (t.threads_per_block != 64 && t.threads_per_block != 128 && t.threads_per_block != 256)
        return fail(PT_EINVAL, "threads_per_block must be 64, 128 or 256");
    if (t.queue_chunk < 32 || t.queue_chunk > 4096 || (t.queue_chunk & 31u))
        return fail(PT_EINVAL, "queue_chunk must be a multiple of 32 in [32, 4096]");
    if (t.stack_depth > PT_TRAVERSAL_STACK) return fail(PT_EINVAL, "stack_depth above the traversal stack limit");
    if (t.pipeline != PT_PIPELINE_FUSED && t.pipeline != PT_PIPELINE_WAVEFRONT && t.pipeline != PT_PIPELINE_PATHS)
        return fail(PT_EINVAL, "unknown pipeline");
    return PT_OK;
}

}  // namespace pt

using namespace pt;

struct pt_batch {
    std::vector<pt_scene*> scenes;
    std::vector<uint32_t> npix;
    uint32_t n = 0;
    uint64_t total_pixels = 0;
    pt_batch_tuning tuning{};
    int cap = 64;
    int device = 0;
    bool two_level = false;   // some item is a two-level scene (fused or path pipeline)
    void* params = nullptr;   // RenderParams[n]
    void* items = nullptr;    // BatchItem[n]
    void* films = nullptr;    // all rgb outputs
    void* prims = nullptr;    // all primary ids
    std::vector<size_t> film_off, prim_off;
    void* counters = nullptr; // 2 x u64: ray counter, rays traced
    void* wf = nullptr;       // wavefront: film sums, items, plan tables, wave state
    void* wf_films = nullptr;
    size_t wf_film_bytes = 0;
    WfPlan plan;
    WfState ws{};
    WfTuning wt;
    WfItem* d_items = nullptr;
    WfSegment* d_segs = nullptr;
    WfPixels* d_res = nullptr;
    WfPixels* d_fin = nullptr;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~pt_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (stream) cudaStreamDestroy(stream);
        for (void* b : {params, items, films, prims, counters, wf})
            if (b) cudaFree(b);
    }
};

namespace {
// Wavefront pipeline of a batch, before capture: plan the waves over all items' paths, allocate
// the film sums, the device tables and the wave state in one buffer, and upload the tables.
int wf_build(pt_batch* b, const pt_batch_item* items, const pt_batch_tuning& t) {
    std::vector<uint32_t> npix(b->n), spp(b->n), depth(b->n);
    uint64_t total_paths = 0;
    for (uint32_t i = 0; i < b->n; ++i) {
        npix[i] = b->npix[i];
        spp[i] = items[i].desc.spp;
        depth[i] = items[i].desc.max_depth;
        total_paths += (uint64_t)npix[i] * spp[i];
    }
    uint64_t wave = t.wave_pixels ? t.wave_pixels : (1ull << 22);
    if (wave > total_paths) wave = total_paths;
    if (wave > (1ull << 30)) return fail(PT_EINVAL, "wave above 2^30 paths");
    wf_plan_all(b->plan, npix, spp, depth, wave);
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    std::vector<size_t> film_off(b->n);
    size_t film_bytes = 0;
    for (uint32_t i = 0; i < b->n; ++i) { film_off[i] = film_bytes; film_bytes += up(12 * (size_t)npix[i]); }
    const WfPlan& plan = b->plan;
    const size_t item_bytes = up(sizeof(WfItem) * b->n), seg_bytes = up(sizeof(WfSegment) * plan.segments.size());
    const size_t res_bytes = up(sizeof(WfPixels) * plan.resolve.size());
    const size_t fin_bytes = up(sizeof(WfPixels) * std::max<size_t>(1, plan.finish.size()));
    const size_t tables = item_bytes + seg_bytes + res_bytes + fin_bytes;
    const bool paths = t.pipeline == PT_PIPELINE_PATHS;
    if (cudaMalloc(&b->wf, film_bytes + tables + wf_state_bytes((uint32_t)wave, paths)) != cudaSuccess)
        return fail(PT_ENOMEM, "cudaMalloc wavefront batch buffers");
    char* base = (char*)b->wf;
    b->wf_films = base;
    b->wf_film_bytes = film_bytes;
    b->d_items = (WfItem*)(base + film_bytes);
    b->d_segs = (WfSegment*)(base + film_bytes + item_bytes);
    b->d_res = (WfPixels*)(base + film_bytes + item_bytes + seg_bytes);
    b->d_fin = (WfPixels*)(base + film_bytes + item_bytes + seg_bytes + res_bytes);
    wf_state_carve(base + film_bytes + tables, (uint32_t)wave, b->ws, paths);
    std::vector<char> host(tables, 0);
    std::vector<WfItem> hi(b->n);
    for (uint32_t i = 0; i < b->n; ++i)
        hi[i] = WfItem{(const RenderParams*)b->params + i, (float*)(base + film_off[i]),
                       (float*)((char*)b->films + b->film_off[i]), (uint32_t*)((char*)b->prims + b->prim_off[i]), npix[i], spp[i]};
    std::memcpy(host.data(), hi.data(), sizeof(WfItem) * b->n);
    std::memcpy(host.data() + item_bytes, plan.segments.data(), sizeof(WfSegment) * plan.segments.size());
    std::memcpy(host.data() + item_bytes + seg_bytes, plan.resolve.data(), sizeof(WfPixels) * plan.resolve.size());
    std::memcpy(host.data() + item_bytes + seg_bytes + res_bytes, plan.finish.data(), sizeof(WfPixels) * plan.finish.size());
    const cudaError_t e = cudaMemcpy(base + film_bytes, host.data(), tables, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("wavefront tables: ") + cudaGetErrorString(e));
    b->wt.threads_per_block = t.threads_per_block;
    b->wt.queue_chunk = t.queue_chunk;
    b->wt.stack_cap = b->cap;
    b->wt.paths = t.pipeline == PT_PIPELINE_PATHS;
    b->wt.two_level = b->two_level;
    return PT_OK;
}

// During capture: clear the film sums, then every wave.
cudaError_t wf_enqueue(pt_batch* b, unsigned long long* rays) {
    cudaError_t e = cudaMemsetAsync(b->wf_films, 0, b->wf_film_bytes, b->stream);
    for (size_t k = 0; e == cudaSuccess && k < b->plan.waves.size(); ++k)
        e = wf_launch_wave(b->d_items, b->d_segs, b->d_res, b->d_fin, b->plan.waves[k], b->ws, b->wt, rays, b->stream);
    return e;
}
}  // namespace

extern "C" int pt_batch_default_tuning(pt_batch_tuning* t) {
    if (!t) return fail(PT_EINVAL, "tuning is NULL");
    t->wave_pixels = 0;
    t->threads_per_block = 128;
    t->stack_depth = 0;
    t->queue_chunk = 64;
    t->pipeline = PT_PIPELINE_WAVEFRONT;
    return PT_OK;
}

extern "C" int pt_batch_create(const pt_batch_item* items, uint32_t n, const pt_batch_tuning* tuning, pt_batch** out) {
    if (!items || !out || n == 0) return fail(PT_EINVAL, "items or out is NULL, or no items");
    *out = nullptr;
    pt_batch_tuning t;
    if (tuning) t = *tuning; else pt_batch_default_tuning(&t);
    int rc = check_tuning(t);
    if (rc) return rc;
    std::unique_ptr<pt_batch> b(new pt_batch());
    b->n = n;
    b->tuning = t;
    uint32_t max_depth = 0;
    std::vector<RenderParams> hp(n);
    for (uint32_t i = 0; i < n; ++i) {
        rc = check_render_desc(items[i].scene, &items[i].desc);
        if (rc) return fail(rc, "batch item " + std::to_string(i) + ": " + pt_last_error());
        if (items[i].desc.flags & (PT_RENDER_WAVEFRONT | PT_RENDER_PERSISTENT | PT_RENDER_FUSED))
            return fail(PT_EINVAL, "batch items take the batch's pipeline (no PT_RENDER_WAVEFRONT / PERSISTENT / FUSED)");
        if (i && items[i].scene->device != items[0].scene->device) return fail(PT_EINVAL, "batch items on different devices");
        if (items[i].scene->two_level) {
            if (t.pipeline == PT_PIPELINE_WAVEFRONT)
                return fail(PT_EINVAL, "batch item " + std::to_string(i) +
                                           ": a two-level scene needs PT_PIPELINE_PATHS or PT_PIPELINE_FUSED");
            b->two_level = true;
        }
        max_depth = std::max(max_depth, items[i].scene->max_depth);
        b->scenes.push_back(items[i].scene);
        hp[i] = render_params(items[i].scene, &items[i].desc);
        b->npix.push_back(items[i].desc.width * items[i].desc.height);
    }
    b->cap = stack_cap_for(max_depth, t.stack_depth);
    if (!b->cap) return fail(PT_ESTACK, "tree depth exceeds the traversal stack");
    b->device = items[0].scene->device;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != b->device) cudaSetDevice(b->device);
    struct Restore { int d; ~Restore() { if (d >= 0) cudaSetDevice(d); } } restore{prev != b->device ? prev : -1};
    size_t fbytes = 0, pbytes = 0;
    for (uint32_t i = 0; i < n; ++i) {
        b->film_off.push_back(fbytes);
        b->prim_off.push_back(pbytes);
        fbytes += ((12 * (size_t)b->npix[i]) + 255) & ~(size_t)255;
        pbytes += ((4 * (size_t)b->npix[i]) + 255) & ~(size_t)255;
    }
    if (cudaMalloc(&b->params, sizeof(RenderParams) * n) != cudaSuccess || cudaMalloc(&b->items, sizeof(BatchItem) * n) != cudaSuccess ||
        cudaMalloc(&b->films, fbytes) != cudaSuccess || cudaMalloc(&b->prims, pbytes) != cudaSuccess ||
        cudaMalloc(&b->counters, 16) != cudaSuccess)
        return fail(PT_ENOMEM, "cudaMalloc batch buffers");
    std::vector<BatchItem> hi(n);
    uint64_t base = 0;
    for (uint32_t i = 0; i < n; ++i) {
        hp[i].rays_traced = nullptr;
        hi[i].params = (const RenderParams*)b->params + i;
        hi[i].rgb = (float*)((char*)b->films + b->film_off[i]);
        hi[i].primary = (uint32_t*)((char*)b->prims + b->prim_off[i]);
        hi[i].px_begin = 0;
        hi[i].px_count = b->npix[i];
        hi[i].base = base;
        base += b->npix[i];
    }
    b->total_pixels = base;
    cudaError_t e = cudaMemcpy(b->params, hp.data(), sizeof(RenderParams) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->items, hi.data(), sizeof(BatchItem) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("batch setup: ") + cudaGetErrorString(e));
    if (t.pipeline != PT_PIPELINE_FUSED) {
        rc = wf_build(b.get(), items, t);
        if (rc) return rc;
    }
    // capture: reset the rays-traced counter, then the launches
    unsigned long long* ctr = (unsigned long long*)b->counters;
    e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctr + 1, 0, sizeof(unsigned long long), b->stream);
    if (t.pipeline == PT_PIPELINE_FUSED) {
        const uint64_t wave = t.wave_pixels ? t.wave_pixels : b->total_pixels;
        for (uint64_t first = 0; e == cudaSuccess && first < b->total_pixels; first += wave) {
            const uint64_t cnt = std::min<uint64_t>(wave, b->total_pixels - first);
            e = launch_batch((const BatchItem*)b->items, n, first, cnt, ctr, t, b->cap, ctr + 1, b->stream, b->two_level);
        }
    } else if (e == cudaSuccess) {
        e = wf_enqueue(b.get(), ctr + 1);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
    if (e == cudaSuccess) e = e2;
    b->graph = g;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("batch graph: ") + cudaGetErrorString(e));
    *out = b.release();
    return PT_OK;
}

extern "C" int pt_batch_run(pt_batch* b, void* stream) {
    if (!b) return fail(PT_EINVAL, "batch is NULL");
    const cudaError_t e = cudaGraphLaunch(b->exec, stream ? (cudaStream_t)stream : b->stream);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
    if (!stream) {
        const cudaError_t e2 = cudaStreamSynchronize(b->stream);
        if (e2 != cudaSuccess) return fail(PT_ECUDA, std::string("batch run: ") + cudaGetErrorString(e2));
    }
    return PT_OK;
}

extern "C" int pt_batch_output(pt_batch* b, uint32_t i, float* rgb_out, uint32_t* primary_out, uint64_t* rays_traced) {
    if (!b || i >= b->n) return fail(PT_EINVAL, "bad batch or item index");
    cudaError_t e = cudaSuccess;
    if (rgb_out) e = cudaMemcpy(rgb_out, (char*)b->films + b->film_off[i], 12 * (size_t)b->npix[i], cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && primary_out)
        e = cudaMemcpy(primary_out, (char*)b->prims + b->prim_off[i], 4 * (size_t)b->npix[i], cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && rays_traced)
        e = cudaMemcpy(rays_traced, (unsigned long long*)b->counters + 1, 8, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(PT_ECUDA, std::string("batch output: ") + cudaGetErrorString(e));
    return PT_OK;
}

extern "C" int pt_batch_destroy(pt_batch* b) {
    delete b;
    return PT_OK;
}

namespace {
// One timed run of a candidate: build the batch, one warm-up replay, then the mean of two replays.
int time_candidate(const pt_batch_item* items, uint32_t n, const pt_batch_tuning& c, float& ms) {
    pt_batch* b = nullptr;
    int rc = pt_batch_create(items, n, &c, &b);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    rc = pt_batch_run(b, nullptr);
    ms = 0.f;
    if (!rc) {
        cudaEventRecord(e0, b->stream);
        for (int r = 0; r < 2; ++r) cudaGraphLaunch(b->exec, b->stream);
        cudaEventRecord(e1, b->stream);
        const cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) rc = fail(PT_ECUDA, std::string("autotune run: ") + cudaGetErrorString(e));
        cudaEventElapsedTime(&ms, e0, e1);
        ms *= 0.5f;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    pt_batch_destroy(b);
    return rc;
}
}  // namespace

// Coordinate descent over the four knobs (threads per block, queue chunk, stack depth, wave size),
// each swept with the others held at the best so far.
extern "C" int pt_batch_autotune(const pt_batch_item* items, uint32_t n, pt_batch_tuning* best, double* best_ms,
                                 pt_batch_tune_result* results, uint32_t* num_results) {
    if (!items || !n || !best) return fail(PT_EINVAL, "items or best is NULL");
    uint32_t max_depth = 0;
    uint64_t total = 0, total_paths = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (!items[i].scene) return fail(PT_EINVAL, "NULL scene");
        max_depth = std::max(max_depth, items[i].scene->max_depth);
        total += (uint64_t)items[i].desc.width * items[i].desc.height;
        total_paths += (uint64_t)items[i].desc.width * items[i].desc.height * items[i].desc.spp;
    }
    const uint32_t cap_results = num_results ? *num_results : 0;
    uint32_t written = 0;
    pt_batch_tuning cur;
    pt_batch_default_tuning(&cur);
    cur.stack_depth = (uint32_t)stack_cap_for(max_depth, 0);
    if (!cur.stack_depth) return fail(PT_ESTACK, "tree depth exceeds the traversal stack");
    float cur_ms = 0.f;
    int rc = time_candidate(items, n, cur, cur_ms);
    if (rc) return rc;
    if (results && written < cap_results) results[written++] = pt_batch_tune_result{cur, cur_ms};
    // knob order: pipeline, wave size, threads per block, queue chunk, stack depth -- the wave size
    // comes early because the best chunk depends on it (measured on the 6.5 M-face frame: chunk 32
    // wins with the default 4 M-path waves, 128 with 32 M-path waves)
    for (int knob : {0, 4, 1, 2, 3}) {
        std::vector<pt_batch_tuning> cands;
        if (knob == 0)
            for (uint32_t v : {PT_PIPELINE_FUSED, PT_PIPELINE_WAVEFRONT, PT_PIPELINE_PATHS}) { auto c = cur; c.pipeline = v; cands.push_back(c); }
        if (knob == 1) for (uint32_t v : {64u, 128u, 256u}) { auto c = cur; c.threads_per_block = v; cands.push_back(c); }
        if (knob == 2) for (uint32_t v : {32u, 64u, 128u, 256u}) { auto c = cur; c.queue_chunk = v; cands.push_back(c); }
        if (knob == 3) for (uint32_t v : {24u, 32u, 48u, 64u}) { if (v < max_depth + 2) continue; auto c = cur; c.stack_depth = v; cands.push_back(c); }
        if (knob == 4) {
            const uint64_t limit = cur.pipeline == PT_PIPELINE_FUSED ? total : total_paths;
            const uint64_t opts_f[] = {0ull, 1ull << 20, 1ull << 22, 1ull << 24};
            const uint64_t opts_w[] = {1ull << 22, 1ull << 23, 1ull << 24, 1ull << 25};  // larger waves: shorter tails
            for (int k = 0; k < 4; ++k) {
                const uint64_t v = cur.pipeline == PT_PIPELINE_FUSED ? opts_f[k] : opts_w[k];
                if (v && v >= limit) continue;
                auto c = cur;
                c.wave_pixels = v;
                cands.push_back(c);
            }
        }
        for (const auto& c : cands) {
            if (std::memcmp(&c, &cur, sizeof(c)) == 0) continue;
            float ms = 0.f;
            rc = time_candidate(items, n, c, ms);
            if (rc) return rc;
            if (results && written < cap_results) results[written++] = pt_batch_tune_result{c, ms};
            if (ms < cur_ms) { cur_ms = ms; cur = c; }
        }
    }
    *best = cur;
    if (best_ms) *best_ms = cur_ms;
    if (num_results) *num_results = written;
    return PT_OK;
}
