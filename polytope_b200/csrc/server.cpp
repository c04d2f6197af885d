// server.cpp -- the serving loop: continuous batching of render requests over resident scenes.
//
// Scenes stay resident in HBM (pt_scene handles).  Requests (scene, resolution, spp, depth) are
// queued by pt_server_submit; a scheduler thread admits them while the in-flight limit, the
// device-memory budget (parameters, film, primary ids and film sums of each request) and the
// pinned host arena for finished films allow, and plans waves: a wave takes work (paths for the
// wave pipelines, pixels for the fused one) from the admitted requests, oldest first
// (PT_SERVE_OLDEST_FIRST) or a fair share from each (PT_SERVE_FAIR_SHARE), and traces it in one
// multi-render launch sequence, so requests that arrive while others run join the next wave and
// their work overlaps on the device.
//
// Two waves are kept queued on the stream: while the GPU runs wave k the host plans and enqueues
// wave k+1, then retires wave k.  The films of the requests a wave finishes are copied by DMA into
// the pinned host arena on a second stream right behind the wave's kernels, so the copies overlap
// the next wave and no host thread copies or page-faults on the completion path; retiring waits
// for those copies and returns the requests' device memory to a stream-ordered pool owned by the
// server, so no call here synchronises the whole device.  pt_server_fetch copies a film out of the
// arena and frees its space.  Pixels are independent and each pixel's samples are summed in sample
// order, so a request's film is bit-identical whether it ran alone or in any mix.

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "batch.h"
#include "pt_internal.h"
#include "serve_sched.h"
#include "wavefront.h"

using Clock = std::chrono::steady_clock;

namespace {

#ifndef PT_SERVE_WAVES_QUEUED
#define PT_SERVE_WAVES_QUEUED 2
#endif
constexpr int kWavesQueued = PT_SERVE_WAVES_QUEUED;  // waves enqueued on the stream at once (host planning overlaps the GPU)

// A request; its scheduling state (state, cancel, total and planned work units -- pixels for the
// fused pipeline, sample-major paths for the wave pipelines) is the serve::Work base.
struct Request : pt::serve::Work {
    uint64_t ticket = 0;
    pt_scene* scene = nullptr;
    pt_render_desc desc{};
    pt::RenderParams params{};
    uint32_t npix = 0;
    size_t bytes = 0;             // device bytes
    void* dev = nullptr;          // RenderParams, rgb (3 floats/px), primary ids, film sums (wave pipelines)
    size_t host_off = ~(size_t)0; // finished film in the host arena: rgb then primary ids
    uint32_t param_slot = ~0u;    // pinned staging slot of its parameters while admitted
    bool launched = false, retired = false;
    uint32_t waves_queued = 0;    // queued waves that hold work of this request
    Clock::time_point submitted, admitted, first_wave, last_wave, done;
};

static_assert(sizeof(pt::RenderParams) <= 256, "request layout reserves 256 bytes for the parameters");

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }
size_t request_bytes(uint32_t npix, bool wave_engine) {
    return 256 + up256(12 * (size_t)npix) + up256(4 * (size_t)npix) + (wave_engine ? 12 * (size_t)npix : 0);
}
size_t host_bytes(uint32_t npix) { return up256(16 * (size_t)npix); }
float* req_rgb(const Request* r) { return (float*)((char*)r->dev + 256); }
uint32_t* req_prim(const Request* r) { return (uint32_t*)((char*)r->dev + 256 + up256(12 * (size_t)r->npix)); }
float* req_film(const Request* r) { return (float*)((char*)r->dev + 256 + up256(12 * (size_t)r->npix) + up256(4 * (size_t)r->npix)); }

// First-fit allocator over the pinned host arena (offsets; adjacent free blocks merge).
class ArenaAllocator {
  public:
    void reset(size_t size) {
        free_.clear();
        if (size) free_[0] = size;
    }
    bool alloc(size_t n, size_t& off) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            off = it->first;
            const size_t left = it->second - n;
            free_.erase(it);
            if (left) free_[off + n] = left;
            return true;
        }
        return false;
    }
    void release(size_t off, size_t n) {
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + n == next->first) {
            n += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += n;
                return;
            }
        }
        free_[off] = n;
    }

  private:
    std::map<size_t, size_t> free_;
};

// A wave enqueued on the stream and not yet retired.
struct WaveInFlight {
    int slot = 0;                      // staging / event slot
    cudaError_t launch = cudaSuccess;  // error from enqueueing it
    std::vector<Request*> members;     // requests with work in this wave
    std::vector<Request*> finishing;   // requests whose last work unit is in this wave
};

}  // namespace

struct pt_server {
    pt_server_config cfg{};
    int device = 0;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv;       // new work, freed memory, or stop
    std::condition_variable done_cv;  // a request finished
    std::deque<Request*> pending;
    std::vector<Request*> active;     // admission order
    std::unordered_map<uint64_t, std::unique_ptr<Request>> all;
    std::vector<std::unique_ptr<Request>> failed;  // fetched failures, freed at destroy
    bool stop = false;
    bool blocked = false;             // admission waits for device or host memory to free up
    uint64_t next_ticket = 1;
    size_t mem_in_use = 0;
    std::string worker_error;
    // device / pinned resources of the scheduler
    cudaStream_t stream = nullptr;       // waves
    cudaStream_t copy_stream = nullptr;  // finished films -> host arena
    cudaMemPool_t pool = nullptr;        // request memory (stream-ordered)
    cudaEvent_t ev_start[kWavesQueued] = {}, ev_end[kWavesQueued] = {}, ev_copied[kWavesQueued] = {};
    // Pinned staging of each admitted request's parameters: a copy from pageable memory would
    // first wait for everything already queued on the stream, stalling the scheduler behind the
    // running waves.  One 256-byte slot per in-flight request.
    char* h_params = nullptr;
    std::vector<uint32_t> free_param_slots;
    char* arena = nullptr;               // pinned host memory for finished films
    size_t arena_size = 0;
    ArenaAllocator arena_alloc;          // guarded by mu
    void* d_items = nullptr;
    pt::BatchItem* h_items = nullptr;    // pinned, kWavesQueued * max_items
    void* d_counters = nullptr;          // [0] fetch counter of the fused launch, [1] rays traced (cumulative)
    unsigned long long* h_rays = nullptr;  // pinned, one per slot
    uint32_t max_items = 0;
    // wave pipelines: wave state and per-wave tables (device + pinned staging per slot)
    bool wave_engine = false;            // PT_PIPELINE_WAVEFRONT or PT_PIPELINE_PATHS: work in paths
    void* d_wave = nullptr;
    pt::WfState ws{};
    void* d_tables = nullptr;
    char* h_tables = nullptr;
    size_t table_bytes = 0;
    // statistics
    uint64_t waves = 0, completed = 0, rays_traced = 0, cancelled = 0;
    double busy_ms = 0.0, blocked_ms = 0.0, plan_ms = 0.0, retire_wait_ms = 0.0;
    uint64_t waves_launched = 0;
    size_t host_in_use = 0;

    void run();
    void admit();
    void plan(WaveInFlight& w, std::vector<uint32_t>& take, std::vector<uint64_t>& first);
    cudaError_t enqueue(WaveInFlight& w, const std::vector<uint32_t>& take, const std::vector<uint64_t>& first);
    void retire(WaveInFlight& w);
    void release_device(Request* r);  // with mu held
    void finish_cancel(Request* r);   // with mu held
    bool has_unplanned() const {
        for (const Request* r : active)
            if (pt::serve::open(*r)) return true;
        return false;
    }
};

// Admits queued requests in arrival order while the in-flight limit, the device-memory budget and
// the host arena allow (mu held).  With nothing admitted, one request is always tried against the
// device, so a request larger than the budget still runs alone.
void pt_server::admit() {
    if (pending.empty()) return;
    const size_t budget = cfg.memory_budget;  // fixed at creation: a driver query per admission cost milliseconds
    blocked = false;
    while (!pending.empty() && active.size() < cfg.max_inflight) {
        Request* r = pending.front();
        const size_t need = request_bytes(r->npix, wave_engine);
        if (!pt::serve::fits(mem_in_use, need, budget, active.empty())) {
            blocked = true;
            break;
        }
        size_t off = 0;
        if (!arena_alloc.alloc(host_bytes(r->npix), off)) {
            blocked = true;  // finished films not fetched yet hold the arena
            break;
        }
        if (cudaMallocFromPoolAsync(&r->dev, need, pool, stream) != cudaSuccess) {
            cudaGetLastError();
            r->dev = nullptr;
            arena_alloc.release(off, host_bytes(r->npix));
            if (!active.empty()) {
                blocked = true;
                break;
            }
            r->state = PT_ENOMEM;
            pending.pop_front();
            done_cv.notify_all();
            continue;
        }
        r->host_off = off;
        host_in_use += host_bytes(r->npix);
        r->bytes = need;
        mem_in_use += need;
        r->params.rays_traced = nullptr;
        r->param_slot = free_param_slots.back();  // active.size() < max_inflight, so one is free
        free_param_slots.pop_back();
        char* hp = h_params + 256 * (size_t)r->param_slot;
        std::memcpy(hp, &r->params, sizeof(r->params));
        cudaMemcpyAsync(r->dev, hp, sizeof(r->params), cudaMemcpyHostToDevice, stream);
        if (wave_engine) cudaMemsetAsync(req_film(r), 0, 12 * (size_t)r->npix, stream);
        r->state = 1;
        r->admitted = Clock::now();
        pending.pop_front();
        active.push_back(r);
    }
}

// Picks the next wave's work (mu held) by the configured policy (serve::plan_wave).
void pt_server::plan(WaveInFlight& w, std::vector<uint32_t>& take, std::vector<uint64_t>& first) {
    const uint64_t room = wave_engine ? std::min<uint64_t>(cfg.wave_pixels, ws.capacity) : cfg.wave_pixels;
    std::vector<pt::serve::Work*> view(active.begin(), active.end());
    std::vector<pt::serve::Take> takes;
    pt::serve::plan_wave(view, room, cfg.policy, max_items, takes);
    for (const pt::serve::Take& t : takes) {
        Request* r = active[t.index];
        if (!r->launched) {
            r->launched = true;
            r->first_wave = Clock::now();
        }
        w.members.push_back(r);
        ++r->waves_queued;
        take.push_back((uint32_t)t.count);
        first.push_back(t.first);
        if (r->planned == r->total) w.finishing.push_back(r);
    }
}

// Enqueues the wave's tables and kernels on the stream, the rays-traced read-back and the wave's
// end event; then, on the copy stream behind that event, the DMA of every film the wave finishes
// into the host arena, and the wave's copied event.
cudaError_t pt_server::enqueue(WaveInFlight& w, const std::vector<uint32_t>& take, const std::vector<uint64_t>& first) {
    uint32_t max_depth = 0;
    for (Request* r : w.members) max_depth = std::max(max_depth, r->scene->max_depth);
    const int cap = pt::stack_cap_for(max_depth, cfg.tuning.stack_depth);
    unsigned long long* rays = (unsigned long long*)d_counters + 1;
    cudaError_t e = cudaEventRecord(ev_start[w.slot], stream);
    if (!wave_engine) {
        pt::BatchItem* hi = h_items + (size_t)w.slot * max_items;
        uint64_t base = 0;
        for (size_t i = 0; i < w.members.size(); ++i) {
            Request* r = w.members[i];
            pt::BatchItem& it = hi[i];
            it.params = (const pt::RenderParams*)r->dev;
            it.rgb = req_rgb(r);
            it.primary = req_prim(r);
            it.px_begin = (uint32_t)first[i];
            it.px_count = take[i];
            it.base = base;
            base += take[i];
        }
        // d_items is shared by the queued waves: this copy is stream-ordered after the previous
        // wave's kernel, its last reader.
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_items, hi, sizeof(pt::BatchItem) * w.members.size(), cudaMemcpyHostToDevice, stream);
        bool two_level = false;
        for (Request* r : w.members) two_level = two_level || r->scene->two_level;
        if (e == cudaSuccess)
            e = pt::launch_batch((const pt::BatchItem*)d_items, (uint32_t)w.members.size(), 0, base,
                                 (unsigned long long*)d_counters, cfg.tuning, cap, rays, stream, two_level);
    } else {
        // one segment of consecutive paths per request; tables through this slot's pinned staging
        pt::WfPlan plan;
        std::vector<pt::WfSegment> segs;
        std::vector<uint32_t> npix, spp, depth;
        std::vector<pt::WfItem> witems;
        uint64_t slot = 0;
        for (size_t i = 0; i < w.members.size(); ++i) {
            Request* r = w.members[i];
            witems.push_back(pt::WfItem{(const pt::RenderParams*)r->dev, req_film(r), req_rgb(r), req_prim(r), r->npix, r->desc.spp});
            npix.push_back(r->npix);
            spp.push_back(r->desc.spp);
            depth.push_back(r->desc.max_depth);
            segs.push_back(pt::WfSegment{(uint32_t)i, 0, first[i], slot, take[i]});
            slot += take[i];
        }
        pt::wf_add_wave(plan, segs, npix, spp, depth);
        const size_t ib = up256(sizeof(pt::WfItem) * witems.size()), sb = up256(sizeof(pt::WfSegment) * plan.segments.size());
        const size_t rb = up256(sizeof(pt::WfPixels) * plan.resolve.size());
        char* ht = h_tables + (size_t)w.slot * table_bytes;
        std::memcpy(ht, witems.data(), sizeof(pt::WfItem) * witems.size());
        std::memcpy(ht + ib, plan.segments.data(), sizeof(pt::WfSegment) * plan.segments.size());
        std::memcpy(ht + ib + sb, plan.resolve.data(), sizeof(pt::WfPixels) * plan.resolve.size());
        std::memcpy(ht + ib + sb + rb, plan.finish.data(), sizeof(pt::WfPixels) * plan.finish.size());
        const size_t used = ib + sb + rb + sizeof(pt::WfPixels) * plan.finish.size();
        // the device tables are shared by the queued waves, like d_items above
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_tables, ht, used, cudaMemcpyHostToDevice, stream);
        pt::WfTuning wt;
        wt.threads_per_block = cfg.tuning.threads_per_block;
        wt.queue_chunk = cfg.tuning.queue_chunk;
        wt.stack_cap = cap;
        wt.paths = cfg.tuning.pipeline == PT_PIPELINE_PATHS;
        for (Request* r : w.members) wt.two_level = wt.two_level || r->scene->two_level;
        char* dt = (char*)d_tables;
        if (e == cudaSuccess)
            e = pt::wf_launch_wave((const pt::WfItem*)dt, (const pt::WfSegment*)(dt + ib), (const pt::WfPixels*)(dt + ib + sb),
                                   (const pt::WfPixels*)(dt + ib + sb + rb), plan.waves[0], ws, wt, rays, stream);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_rays + w.slot, rays, 8, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev_end[w.slot], stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(copy_stream, ev_end[w.slot], 0);
    for (Request* r : w.finishing) {
        if (e != cudaSuccess) break;
        char* h = arena + r->host_off;
        const size_t n = r->npix;
        e = cudaMemcpyAsync(h, req_rgb(r), 12 * n, cudaMemcpyDeviceToHost, copy_stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h + 12 * n, req_prim(r), 4 * n, cudaMemcpyDeviceToHost, copy_stream);
    }
    if (e == cudaSuccess) e = cudaEventRecord(ev_copied[w.slot], copy_stream);
    return e;
}

// Returns a request's device memory to the pool, stream-ordered after its film copies, and drops
// it from the active set (mu held).  Its film stays in the host arena until fetched.
void pt_server::release_device(Request* r) {
    if (r->param_slot != ~0u) {  // its copy ran long before the request's waves finished
        free_param_slots.push_back(r->param_slot);
        r->param_slot = ~0u;
    }
    if (r->dev) {
        cudaFreeAsync(r->dev, copy_stream);
        r->dev = nullptr;
        mem_in_use -= r->bytes;
    }
    r->done = Clock::now();
    active.erase(std::remove(active.begin(), active.end(), r), active.end());
    ++completed;
    blocked = false;
}

// Ends a cancelled request (mu held): its device memory goes back to the pool and its host arena
// space is freed; the ticket stays until fetched.  No queued wave holds its work any more, and
// every film copy of a wave that finished it has been waited for, so the only device work that
// can still touch its memory is the parameter upload and film clear of its admission, queued on
// the wave stream: the memory is freed in that stream's order.
void pt_server::finish_cancel(Request* r) {
    r->state = 3;
    r->cancel = false;
    if (r->param_slot != ~0u) {
        free_param_slots.push_back(r->param_slot);
        r->param_slot = ~0u;
    }
    if (r->dev) {
        cudaFreeAsync(r->dev, stream);
        r->dev = nullptr;
        mem_in_use -= r->bytes;
    }
    r->done = Clock::now();
    active.erase(std::remove(active.begin(), active.end(), r), active.end());
    if (r->host_off != ~(size_t)0) {
        arena_alloc.release(r->host_off, host_bytes(r->npix));
        host_in_use -= host_bytes(r->npix);
        r->host_off = ~(size_t)0;
    }
    ++cancelled;
    blocked = false;
}

// Waits for a wave and the copies of the films it finished; those requests are done.
void pt_server::retire(WaveInFlight& w) {
    cudaError_t e = w.launch;
    if (e == cudaSuccess) e = cudaEventSynchronize(ev_end[w.slot]);
    const auto kernels_done = Clock::now();
    if (e == cudaSuccess) e = cudaEventSynchronize(ev_copied[w.slot]);
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, ev_start[w.slot], ev_end[w.slot]);
    {
        std::lock_guard<std::mutex> lock(mu);
        busy_ms += ms;
        ++waves;
        for (Request* r : w.members) --r->waves_queued;
        if (e == cudaSuccess) {
            rays_traced = h_rays[w.slot];
            for (Request* r : w.finishing) {
                r->retired = true;
                r->last_wave = kernels_done;
                if (r->state != 1 || r->cancel) continue;
                r->state = 2;
                release_device(r);
            }
            // cancelled requests whose last queued wave this was
            for (Request* r : w.members)
                if (pt::serve::cancel_ends_on_retire(r->state, r->cancel, r->waves_queued)) finish_cancel(r);
        } else {
            worker_error = std::string("serving wave: ") + cudaGetErrorString(e);
            for (Request* r : w.members) {
                if (r->state == 1) r->state = PT_ECUDA;
                if (r->dev || std::find(active.begin(), active.end(), r) != active.end()) release_device(r);
            }
        }
    }
    done_cv.notify_all();
}

void pt_server::run() {
    cudaSetDevice(device);
    std::deque<WaveInFlight> queued;
    int next_slot = 0;
    std::vector<uint32_t> take;
    std::vector<uint64_t> first;
    while (true) {
        WaveInFlight w;
        take.clear();
        first.clear();
        bool stopping;
        {
            std::unique_lock<std::mutex> lock(mu);
            if (queued.empty()) {
                const bool waiting_for_room = !pending.empty() && blocked;
                const auto t0 = Clock::now();
                cv.wait(lock, [&] { return stop || (!pending.empty() && !blocked) || has_unplanned(); });
                if (waiting_for_room) blocked_ms += std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
            }
            stopping = stop;
            if (!stopping) {
                const auto t0 = Clock::now();
                admit();
                plan(w, take, first);
                plan_ms += std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
            }
        }
        if (stopping && queued.empty()) return;
        const bool launched = !w.members.empty();
        if (launched) {
            const auto t0 = Clock::now();
            w.slot = next_slot;
            next_slot = (next_slot + 1) % kWavesQueued;
            w.launch = enqueue(w, take, first);
            queued.push_back(std::move(w));
            std::lock_guard<std::mutex> lock(mu);
            plan_ms += std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
            ++waves_launched;
        }
        // Retire the oldest wave when the queue is full, or when there was nothing to launch
        // (its completion frees memory and in-flight slots for the next admissions).
        if (!queued.empty() && (queued.size() >= (size_t)kWavesQueued || !launched)) {
            const auto t0 = Clock::now();
            retire(queued.front());
            queued.pop_front();
            std::lock_guard<std::mutex> lock(mu);
            retire_wait_ms += std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
        }
    }
}

using namespace pt;

namespace {
void destroy_resources(pt_server* s) {
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
    for (int i = 0; i < kWavesQueued; ++i) {
        if (s->ev_start[i]) cudaEventDestroy(s->ev_start[i]);
        if (s->ev_end[i]) cudaEventDestroy(s->ev_end[i]);
        if (s->ev_copied[i]) cudaEventDestroy(s->ev_copied[i]);
    }
    if (s->d_items) cudaFree(s->d_items);
    if (s->d_counters) cudaFree(s->d_counters);
    if (s->h_items) cudaFreeHost(s->h_items);
    if (s->h_rays) cudaFreeHost(s->h_rays);
    if (s->h_params) cudaFreeHost(s->h_params);
    if (s->arena) cudaFreeHost(s->arena);
    if (s->d_wave) cudaFree(s->d_wave);
    if (s->d_tables) cudaFree(s->d_tables);
    if (s->h_tables) cudaFreeHost(s->h_tables);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->stream) cudaStreamDestroy(s->stream);
}
}  // namespace

extern "C" int pt_server_create(const pt_server_config* cfg, pt_server** out) {
    if (!cfg || !out) return fail(PT_EINVAL, "cfg or out is NULL");
    *out = nullptr;
    if (cfg->max_inflight == 0 || cfg->max_inflight > 65536) return fail(PT_EINVAL, "max_inflight must be in [1, 65536]");
    if (cfg->policy != PT_SERVE_OLDEST_FIRST && cfg->policy != PT_SERVE_FAIR_SHARE) return fail(PT_EINVAL, "unknown policy");
    int rc = check_tuning(cfg->tuning);
    if (rc) return rc;
    std::unique_ptr<pt_server> s(new pt_server());
    s->cfg = *cfg;
    if (!s->cfg.wave_pixels) s->cfg.wave_pixels = 1u << 20;
    s->arena_size = cfg->host_budget ? (size_t)up256(cfg->host_budget) : ((size_t)1 << 30);
    if (cudaGetDevice(&s->device) != cudaSuccess) return fail(PT_ECUDA, "no CUDA device available");
    if (!s->cfg.memory_budget) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return fail(PT_ECUDA, "cudaMemGetInfo failed");
        s->cfg.memory_budget = (uint64_t)(0.8 * (double)free_b);
    }
    s->max_items = std::min<uint32_t>(cfg->max_inflight, 4096);
    s->wave_engine = cfg->tuning.pipeline != PT_PIPELINE_FUSED;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = s->device;
    bool ok = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMemPoolCreate(&s->pool, &props) == cudaSuccess &&
              cudaMalloc(&s->d_items, sizeof(BatchItem) * s->max_items) == cudaSuccess &&
              cudaMallocHost((void**)&s->h_items, sizeof(BatchItem) * s->max_items * kWavesQueued) == cudaSuccess &&
              cudaMallocHost((void**)&s->h_rays, sizeof(unsigned long long) * kWavesQueued) == cudaSuccess &&
              cudaMallocHost((void**)&s->arena, s->arena_size) == cudaSuccess &&
              cudaMallocHost((void**)&s->h_params, 256 * (size_t)cfg->max_inflight) == cudaSuccess &&
              cudaMalloc(&s->d_counters, 16) == cudaSuccess && cudaMemset(s->d_counters, 0, 16) == cudaSuccess;
    for (int i = 0; ok && i < kWavesQueued; ++i)
        ok = cudaEventCreate(&s->ev_start[i]) == cudaSuccess && cudaEventCreate(&s->ev_end[i]) == cudaSuccess &&
             cudaEventCreateWithFlags(&s->ev_copied[i], cudaEventDisableTiming) == cudaSuccess;
    if (ok) {
        s->arena_alloc.reset(s->arena_size);
        for (uint32_t i = cfg->max_inflight; i-- > 0;) s->free_param_slots.push_back(i);
        // keep freed request memory in the pool for the next admissions instead of returning it
        // to the driver at every synchronisation
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        // and map the first min(budget, 4 GiB) now (64 in-flight 1024^2 requests hold about
        // 1.8 GiB), so that admissions take memory the pool already has instead of growing it on
        // the scheduler thread while the queued waves run dry
        const size_t prime = (size_t)std::min<uint64_t>(s->cfg.memory_budget, 4ull << 30);
        void* block = nullptr;
        if (prime && cudaMallocFromPoolAsync(&block, prime, s->pool, s->stream) == cudaSuccess) {
            cudaFreeAsync(block, s->stream);
            cudaStreamSynchronize(s->stream);
        } else {
            cudaGetLastError();  // the pool then grows on demand, as before
        }
    }
    if (ok && s->wave_engine) {
        const uint64_t cap_paths = std::min<uint64_t>(s->cfg.wave_pixels, 1ull << 26);
        const uint32_t n = s->max_items;
        s->table_bytes = up256(up256(sizeof(WfItem) * n) + up256(sizeof(WfSegment) * n) + up256(sizeof(WfPixels) * 2 * n) +
                               sizeof(WfPixels) * n);
        const bool paths = cfg->tuning.pipeline == PT_PIPELINE_PATHS;
        ok = cudaMalloc(&s->d_wave, wf_state_bytes((uint32_t)cap_paths, paths)) == cudaSuccess &&
             cudaMalloc(&s->d_tables, s->table_bytes) == cudaSuccess &&
             cudaMallocHost((void**)&s->h_tables, s->table_bytes * kWavesQueued) == cudaSuccess;
        if (ok) wf_state_carve(s->d_wave, (uint32_t)cap_paths, s->ws, paths);
    }
    if (!ok) {
        cudaGetLastError();
        destroy_resources(s.get());
        return fail(PT_ENOMEM, "server buffers");
    }
    pt_server* raw = s.get();
    s->worker = std::thread([raw] { raw->run(); });
    *out = s.release();
    return PT_OK;
}

extern "C" int pt_server_submit(pt_server* s, pt_scene* scene, const pt_render_desc* desc, uint64_t* ticket) {
    if (!s || !ticket) return fail(PT_EINVAL, "server or ticket is NULL");
    int rc = check_render_desc(scene, desc);
    if (rc) return rc;
    if (desc->flags & (PT_RENDER_WAVEFRONT | PT_RENDER_PERSISTENT | PT_RENDER_FUSED))
        return fail(PT_EINVAL, "served requests take the server's pipeline (no PT_RENDER_WAVEFRONT / PERSISTENT / FUSED)");
    if (scene->device != s->device) return fail(PT_EINVAL, "scene lives on another device");
    if (scene->two_level && s->cfg.tuning.pipeline == PT_PIPELINE_WAVEFRONT)
        return fail(PT_EINVAL, "a two-level scene is served by PT_PIPELINE_PATHS or PT_PIPELINE_FUSED");
    if (!stack_cap_for(scene->max_depth, s->cfg.tuning.stack_depth)) return fail(PT_ESTACK, "tree too deep");
    std::unique_ptr<Request> r(new Request());
    r->scene = scene;
    r->desc = *desc;
    r->params = render_params(scene, desc);
    r->npix = desc->width * desc->height;
    if (host_bytes(r->npix) > s->arena_size) return fail(PT_EINVAL, "film larger than the server's host budget");
    r->total = s->wave_engine ? (uint64_t)r->npix * desc->spp : r->npix;
    r->submitted = Clock::now();
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stop) return fail(PT_EINVAL, "server is shutting down");
    r->ticket = s->next_ticket++;
    *ticket = r->ticket;
    s->pending.push_back(r.get());
    s->all.emplace(r->ticket, std::move(r));
    s->cv.notify_one();
    return PT_OK;
}

extern "C" int pt_server_poll(pt_server* s, uint64_t ticket, int* state, double* latency_ms) {
    if (!s || !state) return fail(PT_EINVAL, "server or state is NULL");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return fail(PT_EINVAL, "unknown ticket");
    *state = it->second->state;
    if (latency_ms)
        *latency_ms = it->second->state == 2
                          ? std::chrono::duration<double, std::milli>(it->second->done - it->second->submitted).count()
                          : -1.0;
    return PT_OK;
}

extern "C" int pt_server_timing(pt_server* s, uint64_t ticket, pt_request_timing* t) {
    if (!s || !t) return fail(PT_EINVAL, "server or timing is NULL");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return fail(PT_EINVAL, "unknown ticket");
    const Request* r = it->second.get();
    auto ms = [&](bool reached, Clock::time_point p) {
        return reached ? std::chrono::duration<double, std::milli>(p - r->submitted).count() : -1.0;
    };
    t->admitted_ms = ms(r->state != 0, r->admitted);
    t->first_wave_ms = ms(r->launched, r->first_wave);
    t->last_wave_ms = ms(r->retired, r->last_wave);
    t->done_ms = ms(r->state == 2, r->done);
    return PT_OK;
}

extern "C" int pt_server_wait(pt_server* s, uint64_t ticket, uint32_t timeout_ms, int* state) {
    if (!s || !state) return fail(PT_EINVAL, "server or state is NULL");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return fail(PT_EINVAL, "unknown ticket");
    Request* r = it->second.get();
    const bool ok = s->done_cv.wait_for(lock, std::chrono::milliseconds(timeout_ms),
                                        [&] { return r->state == 2 || r->state == 3 || r->state < 0; });
    *state = r->state;
    if (!ok) return fail(PT_ETIMEOUT, "request not finished within the timeout");
    return PT_OK;
}

extern "C" int pt_server_fetch(pt_server* s, uint64_t ticket, float* rgb_out, uint32_t* primary_out) {
    if (!s) return fail(PT_EINVAL, "server is NULL");
    std::unique_ptr<Request> r;
    std::string err;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        auto it = s->all.find(ticket);
        if (it == s->all.end()) return fail(PT_EINVAL, "unknown ticket");
        if (it->second->state != 2 && it->second->state != 3 && it->second->state >= 0)
            return fail(PT_EINVAL, "request not finished");
        r = std::move(it->second);  // the ticket is gone; its arena block stays taken until released below
        s->all.erase(it);
        err = s->worker_error;
    }
    // copy out without the server lock, so the scheduler keeps planning while a large film is copied
    const size_t n = r->npix;
    if (r->state == 2) {
        const char* h = s->arena + r->host_off;
        if (rgb_out) std::memcpy(rgb_out, h, 12 * n);
        if (primary_out) std::memcpy(primary_out, h + 12 * n, 4 * n);
    }
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (r->host_off != ~(size_t)0) {
            s->arena_alloc.release(r->host_off, host_bytes(r->npix));
            s->host_in_use -= host_bytes(r->npix);
            s->blocked = false;
        }
        if (r->state < 0 || r->state == 3) {
            const int st = r->state == 3 ? PT_ECANCELED : r->state;
            // a failed request may still be named by a queued wave: keep it alive until destroy
            s->failed.push_back(std::move(r));
            s->cv.notify_one();
            return st == PT_ECANCELED ? fail(st, "request was cancelled") : fail(st, "request failed: " + err);
        }
    }
    s->cv.notify_one();  // admission may have waited for arena space
    return PT_OK;
}

extern "C" int pt_server_cancel(pt_server* s, uint64_t ticket) {
    if (!s) return fail(PT_EINVAL, "server is NULL");
    {
        std::lock_guard<std::mutex> lock(s->mu);
        auto it = s->all.find(ticket);
        if (it == s->all.end()) return fail(PT_EINVAL, "unknown ticket");
        Request* r = it->second.get();
        switch (pt::serve::on_cancel(r->state, r->cancel, r->waves_queued)) {
            case pt::serve::CancelAction::EndNow:
                if (r->state == pt::serve::kQueued) {  // nothing of it is on the device
                    s->pending.erase(std::remove(s->pending.begin(), s->pending.end(), r), s->pending.end());
                    r->state = pt::serve::kCancelled;
                    ++s->cancelled;
                } else {  // admitted, and no queued wave holds its work
                    r->cancel = true;
                    s->finish_cancel(r);
                }
                break;
            case pt::serve::CancelAction::EndAfterWaves:  // the scheduler ends it when its last queued wave retires
                r->cancel = true;
                break;
            case pt::serve::CancelAction::AlreadyCancelling:
                return PT_OK;
            case pt::serve::CancelAction::Refuse:
                return fail(PT_EINVAL, "request already finished");
        }
    }
    s->done_cv.notify_all();
    s->cv.notify_one();  // admission may have waited for the memory it held
    return PT_OK;
}

extern "C" int pt_server_get_stats(pt_server* s, pt_server_stats* st) {
    if (!s || !st) return fail(PT_EINVAL, "server or stats is NULL");
    std::lock_guard<std::mutex> lock(s->mu);
    st->waves = s->waves;
    st->completed = s->completed;
    st->rays_traced = s->rays_traced;
    st->busy_ms = s->busy_ms;
    st->pending = s->pending.size();
    st->active = s->active.size();
    st->device_bytes_in_use = s->mem_in_use;
    st->blocked_ms = s->blocked_ms;
    st->host_bytes_in_use = s->host_in_use;
    st->plan_ms = s->plan_ms;
    st->retire_wait_ms = s->retire_wait_ms;
    st->waves_launched = s->waves_launched;
    st->cancelled = s->cancelled;
    return PT_OK;
}

extern "C" int pt_server_destroy(pt_server* s) {
    if (!s) return PT_OK;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();  // the worker retires its queued waves first
    for (auto& kv : s->all)
        if (kv.second->dev) cudaFreeAsync(kv.second->dev, s->stream);
    destroy_resources(s);
    delete s;
    return PT_OK;
}
