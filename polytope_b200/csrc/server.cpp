// server.cpp -- the serving loop: continuous batching of render requests over resident scenes.
//
// Scenes stay resident in HBM (pt_scene handles).  Requests (scene, resolution, spp, depth) are
// queued by pt_server_submit; a scheduler thread admits them while the in-flight limit and the
// device-memory budget (film + primary ids of each admitted request) allow, and runs waves: each
// wave takes a fair share of pixels from every admitted request and traces them in one persistent
// launch of the multi-render kernel (batch.cu), so requests that arrive while others run join the
// next wave and their work overlaps on the device.  A request completes when its last pixel is
// done; its film is copied to host memory and its device memory is released for the next
// admissions.  Pixels are independent and each pixel's samples are summed in sample order, so a
// request's film is bit-identical whether it ran alone or in any mix.

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "batch.h"
#include "pt_internal.h"
#include "wavefront.h"

using Clock = std::chrono::steady_clock;

namespace {

struct Request {
    uint64_t ticket = 0;
    pt_scene* scene = nullptr;
    pt_render_desc desc{};
    pt::RenderParams params{};
    uint32_t npix = 0;
    uint32_t next_px = 0;         // fused pipeline: pixels done
    uint64_t next_path = 0;       // wavefront pipeline: paths done (sample-major)
    uint64_t total_paths = 0;
    size_t bytes = 0;
    void* dev = nullptr;          // RenderParams, rgb (3 floats/px), primary ids, film sums (wavefront)
    int state = 0;                // 0 queued, 1 admitted, 2 done, < 0 error
    Clock::time_point submitted, done;
    std::vector<float> rgb;
    std::vector<uint32_t> prim;
};

static_assert(sizeof(pt::RenderParams) <= 256, "request layout reserves 256 bytes for the parameters");

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }
size_t request_bytes(uint32_t npix, bool wavefront) {
    return 256 + up256(12 * (size_t)npix) + up256(4 * (size_t)npix) + (wavefront ? 12 * (size_t)npix : 0);
}
float* req_rgb(const Request* r) { return (float*)((char*)r->dev + 256); }
uint32_t* req_prim(const Request* r) { return (uint32_t*)((char*)r->dev + 256 + up256(12 * (size_t)r->npix)); }
float* req_film(const Request* r) { return (float*)((char*)r->dev + 256 + up256(12 * (size_t)r->npix) + up256(4 * (size_t)r->npix)); }

}  // namespace

struct pt_server {
    pt_server_config cfg{};
    int device = 0;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv;       // new work or stop
    std::condition_variable done_cv;  // a request finished
    std::deque<Request*> pending;
    std::vector<Request*> active;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> all;
    bool stop = false;
    uint64_t next_ticket = 1;
    size_t mem_in_use = 0;
    std::string worker_error;
    // device / pinned resources of the scheduler
    cudaStream_t stream = nullptr;
    void* d_items = nullptr;
    pt::BatchItem* h_items = nullptr;  // pinned
    void* d_counters = nullptr;        // ray counter, rays traced
    uint32_t max_items = 0;
    // wavefront pipeline: wave state and per-wave tables (device + pinned staging)
    bool wavefront = false;
    void* d_wave = nullptr;
    pt::WfState ws{};
    void* d_tables = nullptr;
    char* h_tables = nullptr;
    size_t table_bytes = 0;
    // statistics
    uint64_t waves = 0, completed = 0, rays_traced = 0;
    double busy_ms = 0.0;

    void run();
};

void pt_server::run() {
    cudaSetDevice(device);
    std::vector<Request*> wave_reqs;
    std::vector<uint32_t> wave_take;
    while (true) {
        {
            std::unique_lock<std::mutex> lock(mu);
            cv.wait(lock, [&] { return stop || !pending.empty() || !active.empty(); });
            if (stop) return;
            // admission: in-flight limit and device-memory budget
            size_t free_b = 0, total_b = 0;
            cudaMemGetInfo(&free_b, &total_b);
            while (!pending.empty() && active.size() < cfg.max_inflight) {
                Request* r = pending.front();
                const size_t need = request_bytes(r->npix, wavefront);
                const size_t budget = cfg.memory_budget ? cfg.memory_budget : (size_t)(0.8 * (double)free_b) + mem_in_use;
                if (mem_in_use + need > budget && !active.empty()) break;
                if (cudaMalloc(&r->dev, need) != cudaSuccess) {
                    cudaGetLastError();
                    if (!active.empty()) break;  // wait for memory to free up
                    r->state = PT_ENOMEM;
                    pending.pop_front();
                    done_cv.notify_all();
                    continue;
                }
                r->bytes = need;
                mem_in_use += need;
                r->params.rays_traced = nullptr;
                cudaMemcpyAsync(r->dev, &r->params, sizeof(r->params), cudaMemcpyHostToDevice, stream);
                if (wavefront) cudaMemsetAsync(req_film(r), 0, 12 * (size_t)r->npix, stream);
                r->state = 1;
                pending.pop_front();
                active.push_back(r);
            }
            // one wave: a fair share of pixels from every admitted request
            wave_reqs.clear();
            wave_take.clear();
            if (!active.empty()) {
                const uint64_t share = std::max<uint64_t>(1024, cfg.wave_pixels / active.size());
                uint64_t room = wavefront ? ws.capacity : ~0ull;
                for (Request* r : active) {
                    if (wave_reqs.size() >= max_items || room == 0) break;
                    const uint64_t left = wavefront ? r->total_paths - r->next_path : (uint64_t)(r->npix - r->next_px);
                    const uint32_t take = (uint32_t)std::min<uint64_t>(std::min<uint64_t>(share, left), room);
                    if (!take) continue;
                    if (wavefront) room -= take;
                    wave_reqs.push_back(r);
                    wave_take.push_back(take);
                }
            }
        }
        if (wave_reqs.empty()) continue;
        uint32_t max_depth = 0;
        for (Request* r : wave_reqs) max_depth = std::max(max_depth, r->scene->max_depth);
        const auto t0 = Clock::now();
        const int cap = pt::stack_cap_for(max_depth, cfg.tuning.stack_depth);
        cudaError_t e = cudaMemsetAsync((unsigned long long*)d_counters + 1, 0, 8, stream);
        if (!wavefront) {
            uint64_t base = 0;
            for (size_t i = 0; i < wave_reqs.size(); ++i) {
                Request* r = wave_reqs[i];
                pt::BatchItem& it = h_items[i];
                it.params = (const pt::RenderParams*)r->dev;
                it.rgb = req_rgb(r);
                it.primary = req_prim(r);
                it.px_begin = r->next_px;
                it.px_count = wave_take[i];
                it.base = base;
                base += wave_take[i];
            }
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(d_items, h_items, sizeof(pt::BatchItem) * wave_reqs.size(), cudaMemcpyHostToDevice, stream);
            if (e == cudaSuccess)
                e = pt::launch_batch((const pt::BatchItem*)d_items, (uint32_t)wave_reqs.size(), 0, base,
                                     (unsigned long long*)d_counters, cfg.tuning, cap, (unsigned long long*)d_counters + 1, stream);
        } else {
            // one wave: a segment of consecutive paths per request, tables through pinned staging
            pt::WfPlan plan;
            std::vector<pt::WfSegment> segs;
            std::vector<uint32_t> npix, spp, depth;
            std::vector<pt::WfItem> witems;
            uint64_t slot = 0;
            for (size_t i = 0; i < wave_reqs.size(); ++i) {
                Request* r = wave_reqs[i];
                witems.push_back(pt::WfItem{(const pt::RenderParams*)r->dev, req_film(r), req_rgb(r), req_prim(r), r->npix, r->desc.spp});
                npix.push_back(r->npix);
                spp.push_back(r->desc.spp);
                depth.push_back(r->desc.max_depth);
                segs.push_back(pt::WfSegment{(uint32_t)i, 0, r->next_path, slot, wave_take[i]});
                slot += wave_take[i];
            }
            pt::wf_add_wave(plan, segs, npix, spp, depth);
            const size_t ib = up256(sizeof(pt::WfItem) * witems.size()), sb = up256(sizeof(pt::WfSegment) * plan.segments.size());
            const size_t rb = up256(sizeof(pt::WfPixels) * plan.resolve.size());
            std::memcpy(h_tables, witems.data(), sizeof(pt::WfItem) * witems.size());
            std::memcpy(h_tables + ib, plan.segments.data(), sizeof(pt::WfSegment) * plan.segments.size());
            std::memcpy(h_tables + ib + sb, plan.resolve.data(), sizeof(pt::WfPixels) * plan.resolve.size());
            std::memcpy(h_tables + ib + sb + rb, plan.finish.data(), sizeof(pt::WfPixels) * plan.finish.size());
            const size_t used = ib + sb + rb + sizeof(pt::WfPixels) * plan.finish.size();
            if (e == cudaSuccess) e = cudaMemcpyAsync(d_tables, h_tables, used, cudaMemcpyHostToDevice, stream);
            pt::WfTuning wt;
            wt.threads_per_block = cfg.tuning.threads_per_block;
            wt.queue_chunk = cfg.tuning.queue_chunk;
            wt.stack_cap = cap;
            char* dt = (char*)d_tables;
            if (e == cudaSuccess)
                e = pt::wf_launch_wave((const pt::WfItem*)dt, (const pt::WfSegment*)(dt + ib), (const pt::WfPixels*)(dt + ib + sb),
                                       (const pt::WfPixels*)(dt + ib + sb + rb), plan.waves[0], ws, wt,
                                       (unsigned long long*)d_counters + 1, stream);
        }
        unsigned long long rays = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&rays, (unsigned long long*)d_counters + 1, 8, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        const double ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
        std::vector<Request*> finished;
        {
            std::lock_guard<std::mutex> lock(mu);
            busy_ms += ms;
            ++waves;
            rays_traced += rays;
            for (size_t i = 0; i < wave_reqs.size(); ++i) {
                Request* r = wave_reqs[i];
                if (e != cudaSuccess) {
                    r->state = PT_ECUDA;
                    worker_error = std::string("serving wave: ") + cudaGetErrorString(e);
                } else if (wavefront) {
                    r->next_path += wave_take[i];
                } else {
                    r->next_px += wave_take[i];
                }
                const bool complete = wavefront ? r->next_path == r->total_paths : r->next_px == r->npix;
                if (r->state < 0 || complete) finished.push_back(r);
            }
        }
        for (Request* r : finished) {  // copy films out, release device memory
            if (r->state == 1) {
                r->rgb.resize(3 * (size_t)r->npix);
                r->prim.resize(r->npix);
                cudaError_t ce = cudaMemcpy(r->rgb.data(), req_rgb(r), 12 * (size_t)r->npix, cudaMemcpyDeviceToHost);
                if (ce == cudaSuccess) ce = cudaMemcpy(r->prim.data(), req_prim(r), 4 * (size_t)r->npix, cudaMemcpyDeviceToHost);
                r->state = ce == cudaSuccess ? 2 : PT_ECUDA;
            }
            cudaFree(r->dev);
            r->dev = nullptr;
            std::lock_guard<std::mutex> lock(mu);
            r->done = Clock::now();
            mem_in_use -= r->bytes;
            active.erase(std::remove(active.begin(), active.end(), r), active.end());
            ++completed;
        }
        if (!finished.empty()) done_cv.notify_all();
    }
}

using namespace pt;

extern "C" int pt_server_create(const pt_server_config* cfg, pt_server** out) {
    if (!cfg || !out) return fail(PT_EINVAL, "cfg or out is NULL");
    *out = nullptr;
    if (cfg->max_inflight == 0 || cfg->max_inflight > 65536) return fail(PT_EINVAL, "max_inflight must be in [1, 65536]");
    int rc = check_tuning(cfg->tuning);
    if (rc) return rc;
    std::unique_ptr<pt_server> s(new pt_server());
    s->cfg = *cfg;
    if (!s->cfg.wave_pixels) s->cfg.wave_pixels = 1u << 20;
    if (cudaGetDevice(&s->device) != cudaSuccess) return fail(PT_ECUDA, "no CUDA device available");
    s->max_items = std::min<uint32_t>(cfg->max_inflight, 4096);
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&s->d_items, sizeof(BatchItem) * s->max_items) != cudaSuccess ||
        cudaMallocHost((void**)&s->h_items, sizeof(BatchItem) * s->max_items) != cudaSuccess ||
        cudaMalloc(&s->d_counters, 16) != cudaSuccess) {
        if (s->stream) cudaStreamDestroy(s->stream);
        if (s->d_items) cudaFree(s->d_items);
        if (s->h_items) cudaFreeHost(s->h_items);
        return fail(PT_ENOMEM, "server buffers");
    }
    s->wavefront = cfg->tuning.pipeline == PT_PIPELINE_WAVEFRONT;
    if (s->wavefront) {
        const uint64_t cap_paths = std::min<uint64_t>(s->cfg.wave_pixels, 1ull << 26);
        const uint32_t n = s->max_items;
        s->table_bytes = up256(sizeof(WfItem) * n) + up256(sizeof(WfSegment) * n) + up256(sizeof(WfPixels) * 2 * n) +
                         sizeof(WfPixels) * n;
        if (cudaMalloc(&s->d_wave, wf_state_bytes((uint32_t)cap_paths)) != cudaSuccess ||
            cudaMalloc(&s->d_tables, s->table_bytes) != cudaSuccess ||
            cudaMallocHost((void**)&s->h_tables, s->table_bytes) != cudaSuccess) {
            if (s->d_wave) cudaFree(s->d_wave);
            if (s->d_tables) cudaFree(s->d_tables);
            cudaFree(s->d_items);
            cudaFree(s->d_counters);
            cudaFreeHost(s->h_items);
            cudaStreamDestroy(s->stream);
            return fail(PT_ENOMEM, "server wave buffers");
        }
        wf_state_carve(s->d_wave, (uint32_t)cap_paths, s->ws);
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
    if (desc->flags & PT_RENDER_WAVEFRONT) return fail(PT_EINVAL, "served requests run the fused pipeline");
    if (scene->device != s->device) return fail(PT_EINVAL, "scene lives on another device");
    if (!stack_cap_for(scene->max_depth, s->cfg.tuning.stack_depth)) return fail(PT_ESTACK, "tree too deep");
    std::unique_ptr<Request> r(new Request());
    r->scene = scene;
    r->desc = *desc;
    r->params = render_params(scene, desc);
    r->npix = desc->width * desc->height;
    r->total_paths = (uint64_t)r->npix * desc->spp;
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

extern "C" int pt_server_wait(pt_server* s, uint64_t ticket, uint32_t timeout_ms, int* state) {
    if (!s || !state) return fail(PT_EINVAL, "server or state is NULL");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return fail(PT_EINVAL, "unknown ticket");
    Request* r = it->second.get();
    const bool ok = s->done_cv.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] { return r->state == 2 || r->state < 0; });
    *state = r->state;
    if (!ok) return fail(PT_ETIMEOUT, "request not finished within the timeout");
    return PT_OK;
}

extern "C" int pt_server_fetch(pt_server* s, uint64_t ticket, float* rgb_out, uint32_t* primary_out) {
    if (!s) return fail(PT_EINVAL, "server is NULL");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return fail(PT_EINVAL, "unknown ticket");
    Request* r = it->second.get();
    if (r->state < 0) {
        const int st = r->state;
        s->all.erase(it);
        return fail(st, "request failed: " + s->worker_error);
    }
    if (r->state != 2) return fail(PT_EINVAL, "request not finished");
    if (rgb_out) std::memcpy(rgb_out, r->rgb.data(), r->rgb.size() * sizeof(float));
    if (primary_out) std::memcpy(primary_out, r->prim.data(), r->prim.size() * sizeof(uint32_t));
    s->all.erase(it);
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
    return PT_OK;
}

extern "C" int pt_server_destroy(pt_server* s) {
    if (!s) return PT_OK;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto& kv : s->all)
        if (kv.second->dev) cudaFree(kv.second->dev);
    cudaFree(s->d_items);
    cudaFree(s->d_counters);
    cudaFreeHost(s->h_items);
    if (s->d_wave) cudaFree(s->d_wave);
    if (s->d_tables) cudaFree(s->d_tables);
    if (s->h_tables) cudaFreeHost(s->h_tables);
    cudaStreamDestroy(s->stream);
    delete s;
    return PT_OK;
}
