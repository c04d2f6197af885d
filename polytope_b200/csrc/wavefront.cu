// wavefront.cu -- the multi-render wavefront engine (see wavefront.h).

#include <algorithm>

#include "path.cuh"
#include "wavefront.h"

namespace pt {

namespace {

__device__ __forceinline__ uint32_t find_segment(const WfSegment* segs, uint32_t n, uint64_t slot) {
    uint32_t lo = 0, hi = n - 1;  // last segment whose slot_base <= slot
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) / 2;
        if (segs[mid].slot_base <= slot) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ uint32_t find_pixels(const WfPixels* e, uint32_t n, uint64_t t) {
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) / 2;
        if (e[mid].base <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool pred) {
    const uint32_t active = __activemask();
    const uint32_t mask = __ballot_sync(active, pred);
    if (mask == 0) return 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(active, base, leader);
    return pred ? base + __popc(mask & ((1u << lane) - 1u)) : 0xFFFFFFFFu;
}

}  // namespace

__global__ void __launch_bounds__(128) wf_init_kernel(const WfItem* __restrict__ items, const WfSegment* __restrict__ segs,
                                                      uint32_t nseg, uint32_t count, WfState ws) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        ws.counters[0] = count;
        ws.counters[1] = 0;
        ws.counters[2] = 0;
    }
    if (i >= count) return;
    const WfSegment sg = segs[find_segment(segs, nseg, i)];
    const RenderParams& p = *items[sg.item].params;
    const uint64_t local = sg.local_begin + (i - sg.slot_base);
    uint32_t pixel, sample;
    F3 o, d;
    path_camera(p, local, pixel, sample, o, d);
    ws.ray_o[i] = make_float4(o.x, o.y, o.z, __uint_as_float(sg.item));
    ws.ray_d[i] = make_float4(d.x, d.y, d.z, __uint_as_float(0u));
    ws.thr[i] = make_float4(1.f, 1.f, 1.f, __uint_as_float(0u));
    ws.rad[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    ws.path[i] = local;
    ws.queue[0][i] = i;
}

// Persistent closest-hit (SHADOW = false: queue of slots) or any-hit (SHADOW = true: the shadow
// queue) traversal with per-lane refill; each lane follows its own ray's scene.
// The first kWfTraceShared stack entries of a lane live in shared memory (blocks of up to 256
// threads); kWfTraceMinBlocks is the resident-block floor given to the register allocator.
// Measured on the 256-scene batch: 4 blocks of 256 (64 registers) beat the unconstrained 72
// registers by 9 %, and 3 blocks or 5-6 blocks are slower; 16 shared entries together with the
// warp-voted walk (PT_LEAF_BATCH_WAVEFRONT) gave 2024 Mrays/s against 1806 for neither (8 or 24
// entries: 1918 / 1954 at batch 16; shared entries without the vote: no gain).
// Re-swept with the min/max box test (256-scene batch, Mrays/s): leaf batch 12 / 16 / 8: 2199 /
// 2150 / 2121; 24 shared entries: 2198; 3 / 5 blocks per SM: 1967 / 1842.
#ifndef PT_WF_TRACE_SHARED
#define PT_WF_TRACE_SHARED 16
#endif
#ifndef PT_WF_TRACE_MIN_BLOCKS
#define PT_WF_TRACE_MIN_BLOCKS 4
#endif
constexpr int kWfTraceShared = PT_WF_TRACE_SHARED;
constexpr int kWfTraceMinBlocks = PT_WF_TRACE_MIN_BLOCKS;

template <int CAP, bool SHADOW>
__global__ void __launch_bounds__(256, kWfTraceMinBlocks) wf_trace_kernel(const WfItem* __restrict__ items, WfState ws,
                                                       const uint32_t* __restrict__ queue, const uint32_t* count_ptr,
                                                       unsigned long long* fetch, uint32_t chunk,
                                                       unsigned long long* rays_traced) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t n = *count_ptr;
    uint64_t pool_next = 0, pool_end = 0;
    bool exhausted = false, active = false;
    uint32_t slot = 0, entry = 0, num_nodes = 0, rays = 0;
    const uint4* nodes = nullptr;
    const float4* tris = nullptr;
    int* err = nullptr;
    __shared__ uint32_t sstack[kWfTraceShared > 0 ? kWfTraceShared * 256 : 1];
    RayWalkT<CAP, kWfTraceShared> k;
    k.stack.base = sstack + threadIdx.x;
    k.stack.stride = blockDim.x;
    while (true) {
        const uint32_t need = __ballot_sync(0xFFFFFFFFu, !active);
        if (need && !exhausted && pool_next >= pool_end) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(fetch, (unsigned long long)chunk);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base >= n) {
                exhausted = true;
            } else {
                pool_next = base;
                pool_end = base + chunk < n ? base + chunk : n;
            }
        }
        if (need) {
            const uint64_t avail = pool_end - pool_next;
            const uint32_t rank = __popc(need & lt_mask);
            if (!active && rank < avail) {
                entry = (uint32_t)(pool_next + rank);
                float4 o4, d4;
                float tmax;
                if (SHADOW) {
                    o4 = ws.sh_o[entry];
                    d4 = ws.sh_d[entry];
                    slot = __float_as_uint(d4.w);
                    tmax = o4.w;
                } else {
                    slot = queue[entry];
                    o4 = ws.ray_o[slot];
                    d4 = ws.ray_d[slot];
                    tmax = __int_as_float(0x7F800000);
                }
                const RenderParams* p = items[__float_as_uint(SHADOW ? ws.ray_o[slot].w : o4.w)].params;
                nodes = (const uint4*)p->nodes;
                tris = (const float4*)p->tris;
                num_nodes = p->num_nodes;
                err = p->err;
                walk_begin(k, o4.x, o4.y, o4.z, d4.x, d4.y, d4.z, tmax, SHADOW, p->exact_tree != 0);
                active = true;
                ++rays;
            }
            const uint64_t took = (uint64_t)__popc(need) < avail ? (uint64_t)__popc(need) : avail;
            pool_next += took;
        }
        if (!__any_sync(0xFFFFFFFFu, active)) {
            if (exhausted) break;
            continue;
        }
        uint32_t leaf_off = 0, leaf_n = 0;
        bool ok, at_leaf;
        if constexpr (PT_LEAF_BATCH_WAVEFRONT > 0) {
            // node steps per ballot on the 256-scene batch: two 2152 vs one 2028 Mrays/s; after the
            // node-step changes three 2438 vs two 2406 (the path kernel keeps one: two measured
            // 1615 vs 1805 Msamples/s on the 6.5 M-face frame)
            walk_round<false, 3>(k, active && k.sp > 0, PT_LEAF_BATCH_WAVEFRONT, nodes, num_nodes, at_leaf, ok, leaf_off,
                                 leaf_n);
        } else {
            ok = !active || walk_to_leaf<false, CAP>(k, nodes, num_nodes, leaf_off, leaf_n);
            at_leaf = active && ok && leaf_n > 0;
        }
        if (at_leaf) walk_leaf<false, CAP>(k, tris, leaf_off, leaf_n);
        if (active) {
            if (!ok || k.done || k.sp == 0) {
                if (!ok) atomicExch(err, 1);
                if (SHADOW) {
                    if (ok && k.prim == kPrimNone) {  // one shadow ray per slot per bounce: no other writer
                        const float4 c = ws.sh_c[entry];
                        float4 l = ws.rad[slot];
                        l.x = fadd(l.x, c.x);
                        l.y = fadd(l.y, c.y);
                        l.z = fadd(l.z, c.z);
                        ws.rad[slot] = l;
                    }
                } else {
                    ws.hit[slot] = make_uint4(ok ? k.prim : kPrimNone, k.leaf, __float_as_uint(k.u), __float_as_uint(k.v));
                    ws.hit_w[slot] = k.w;
                }
                active = false;
            }
        }
    }
    if (rays_traced) {
        const uint32_t s = __reduce_add_sync(0xFFFFFFFFu, rays);
        if (lane == 0 && s) atomicAdd(rays_traced, (unsigned long long)s);
    }
}

__global__ void __launch_bounds__(128) wf_shade_kernel(const WfItem* __restrict__ items, WfState ws,
                                                       const uint32_t* __restrict__ queue, const uint32_t* count_ptr,
                                                       uint32_t* __restrict__ next_queue, uint32_t* next_count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < *count_ptr;
    bool more = false, shadow = false;
    uint32_t slot = 0;
    ShadowReq sh;
    sh.valid = false;
    if (live) {
        slot = queue[i];
        const float4 o = ws.ray_o[slot], d = ws.ray_d[slot], t = ws.thr[slot], l = ws.rad[slot];
        const uint32_t item = __float_as_uint(o.w);
        const WfItem it = items[item];
        const RenderParams& p = *it.params;
        const uint64_t local = ws.path[slot];
        const uint32_t sample = (uint32_t)(local / it.npix), pixel = (uint32_t)(local % it.npix);
        PathState s;
        s.o = f3(o.x, o.y, o.z);
        s.d = f3(d.x, d.y, d.z);
        s.src = f3(t.x, t.y, t.z);
        s.L = f3(l.x, l.y, l.z);
        s.last_lambert = __float_as_uint(t.w);
        s.bounces = __float_as_uint(d.w);
        const uint4 h = ws.hit[slot];
        if (s.bounces == 0 && sample == 0 && it.primary) it.primary[pixel] = h.x;
        more = shade_hit(p, s, h.x, h.y, __uint_as_float(h.z), __uint_as_float(h.w), ws.hit_w[slot], pixel, sample, sh);
        more = more && !throughput_is_zero(s.src);  // the loop head's is_zero test of the next bounce
        shadow = sh.valid;
        ws.rad[slot] = make_float4(s.L.x, s.L.y, s.L.z, 0.f);
        if (more) {
            ws.ray_o[slot] = make_float4(s.o.x, s.o.y, s.o.z, __uint_as_float(item));
            ws.ray_d[slot] = make_float4(s.d.x, s.d.y, s.d.z, __uint_as_float(s.bounces));
            ws.thr[slot] = make_float4(s.src.x, s.src.y, s.src.z, __uint_as_float(s.last_lambert));
        }
    }
    const uint32_t qn = warp_append(next_count, more);
    if (more) next_queue[qn] = slot;
    const uint32_t qs = warp_append(ws.counters + 2, shadow);
    if (shadow) {
        ws.sh_o[qs] = make_float4(sh.o.x, sh.o.y, sh.o.z, sh.tmax);
        ws.sh_d[qs] = make_float4(sh.wi.x, sh.wi.y, sh.wi.z, __uint_as_float(slot));
        ws.sh_c[qs] = make_float4(sh.contrib.x, sh.contrib.y, sh.contrib.z, 0.f);
    }
}

// Whole paths of several renders in one persistent launch.  Each lane runs one path at a time
// (the fused loop of path.cuh, with the same device functions in the same order, so results are
// bit-identical): its current ray, closest-hit or shadow, is walked node by node in warp rounds
// (walk_round: PT_LEAF_BATCH_PATHS lanes at a leaf, then walk_leaf), and when it ends the lane
// shades, starts the path's next ray, or
// stores the clamped radiance and takes the next slot.  Warps take slots in chunks of `chunk`
// from *fetch and refill idle lanes from the chunk, so a warp no longer waits for its longest
// path.  The first SH stack entries of a lane live in shared memory.
//
// Shading runs in batches: a lane whose ray has ended waits (idle) until at least kShadeBatch
// lanes of its warp are in the same state, or no lane is still walking, and then those lanes shade
// together, so the long shading code is not replayed by the warp for one or two lanes at a time.
// Each lane's own sequence of operations is unchanged.  16 measured best on the 6.5 M-face frame
// (with the voted walk: 1706 Msamples/s; 8: 1545, 12: 1640, 24: 1603).
constexpr int kShadeBatch = PT_SHADE_BATCH_PATHS;

// Per-lane path state that only the shading step reads or writes (the path's next ray, throughput,
// radiance, bounce count, the pending shadow contribution, the slot and its pixel, sample and
// item), parked in shared memory between shading steps: the walk loop then holds only the ray
// walk and the scene pointers in registers, so it runs at 7 or 8 blocks per SM without spilling
// that state to local memory.  Field f of lane t lives at [f * 128 + t] (consecutive lanes, consecutive
// banks).
enum ColdField : uint32_t {
    kOx, kOy, kOz, kDx, kDy, kDz, kSr, kSg, kSb, kLr, kLg, kLb, kCr, kCg, kCb,
    kBounces, kFlags, kSlot, kPixel, kSample, kItem, kColdFields,
    // kernels that walk two-level scenes also keep the world ray of the current walk (a path ray
    // or a shadow ray), which instance entries and exits carry in and out of object space
    kWox = kColdFields, kWoy, kWoz, kWdx, kWdy, kWdz,
    kFaceBase, kPrimBase, kInst,  // the instance being walked: its first face and primitive id
    kHitInst,                     // the instance of the committed hit
    kColdFieldsTwoLevel
};
constexpr uint32_t kColdShadow = 1u, kColdPending = 2u, kColdLambert = 4u, kColdExact = 8u;  // kColdExact: NaN boxes

struct ColdLane {
    uint32_t* c;  // this lane's field 0
    __device__ __forceinline__ float f(uint32_t k) const { return __uint_as_float(c[k * 128]); }
    __device__ __forceinline__ uint32_t u(uint32_t k) const { return c[k * 128]; }
    __device__ __forceinline__ void set(uint32_t k, float v) const { c[k * 128] = __float_as_uint(v); }
    __device__ __forceinline__ void set(uint32_t k, uint32_t v) const { c[k * 128] = v; }
    __device__ __forceinline__ F3 f3at(uint32_t k) const { return f3(f(k), f(k + 1), f(k + 2)); }
    __device__ __forceinline__ void set3(uint32_t k, const F3& v) const { set(k, v.x); set(k + 1, v.y); set(k + 2, v.z); }
};

// What two_level_transition needs of a lane: its walk's world ray and where to record the
// instance entered, both in the lane's shared-memory fields.
struct TwoLevelLane {
    ColdLane cold;
    __device__ __forceinline__ void world(float& ox, float& oy, float& oz, float& dx, float& dy, float& dz) const {
        ox = cold.f(kWox); oy = cold.f(kWoy); oz = cold.f(kWoz);
        dx = cold.f(kWdx); dy = cold.f(kWdy); dz = cold.f(kWdz);
    }
    __device__ __forceinline__ void set_instance(uint32_t face_base, uint32_t prim_base, uint32_t inst) const {
        cold.set(kFaceBase, face_base);
        cold.set(kPrimBase, prim_base);
        cold.set(kInst, inst);
    }
};

// PT_PATH_MIN_BLOCKS blocks of 128 per SM.  With the shading state in shared memory (see
// ColdField), at 8 blocks: on the 6.5 M-face 1920x1080x64 frame 1840-1847 Msamples/s against
// 1794-1796 with that state in registers (and spilled), and 1678 against 1584 Mrays/s on the
// 256-scene batch.  TL: the wave may hold
// two-level scenes (a lane walks its item's layout: walk_step, or two_level_node_step and
// two_level_transition).
template <int CAP, int SH, bool TL>
__global__ void __launch_bounds__(128, PT_PATH_MIN_BLOCKS) wf_path_kernel(const WfItem* __restrict__ items, const WfSegment* __restrict__ segs,
                                                      uint32_t nseg, uint32_t count, float* __restrict__ radiance,
                                                      unsigned long long* fetch, uint32_t chunk,
                                                      unsigned long long* rays_traced) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const float inf = bitsf(0x7F800000u);
    __shared__ uint32_t sstack[SH > 0 ? SH * 128 : 1];
    __shared__ uint32_t scold[(TL ? kColdFieldsTwoLevel : kColdFields) * 128];
    const ColdLane cold{scold + threadIdx.x};
    RayWalkT<CAP, SH> k;
    // two-level lanes: the instance bookkeeping lives in the lane's shared fields, so the
    // bottom-level node steps carry no extra registers
    bool two = false;
    const TwoLevelLane tl_lane{cold};
    // starts a walk of the lane's ray in its item's layout
    auto begin = [&](const F3& o, const F3& d, float tmax, bool any, bool exact) {
        if (TL && two) {
            cold.set3(kWox, o);
            cold.set3(kWdx, d);
            walk_begin_two_level(k, o.x, o.y, o.z, d.x, d.y, d.z, tmax, any, exact);
        } else {
            walk_begin(k, o.x, o.y, o.z, d.x, d.y, d.z, tmax, any, exact);
        }
    };
    k.stack.base = sstack + threadIdx.x;
    k.stack.stride = 128;
    uint32_t pool_next = 0, pool_end = 0;
    bool exhausted = false, active = false;
    uint32_t num_nodes = 0, rays = 0;
    const uint4* nodes = nullptr;
    const float4* tris = nullptr;
    bool finished = false, walk_ok = true;  // the current ray's walk has ended (and how)
    while (true) {
        const uint32_t need = __ballot_sync(0xFFFFFFFFu, !active);
        if (need && !exhausted && pool_next >= pool_end) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(fetch, (unsigned long long)chunk);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base >= count) {
                exhausted = true;
            } else {
                pool_next = (uint32_t)base;
                pool_end = base + chunk < count ? (uint32_t)base + chunk : count;
            }
        }
        if (need) {
            const uint32_t avail = pool_end - pool_next;
            const uint32_t rank = __popc(need & lt_mask);
            if (!active && rank < avail) {
                const uint32_t slot = pool_next + rank;
                const WfSegment sg = segs[find_segment(segs, nseg, slot)];
                const uint32_t item = sg.item;
                const RenderParams* p = items[item].params;
                nodes = (const uint4*)p->nodes;
                tris = (const float4*)p->tris;
                num_nodes = p->num_nodes;
                const bool exact = p->exact_tree != 0;
                uint32_t pixel, sample;
                F3 o, d;
                path_camera(*p, sg.local_begin + (slot - sg.slot_base), pixel, sample, o, d);
                cold.set3(kOx, o);
                cold.set3(kDx, d);
                cold.set3(kSr, f3(1.f, 1.f, 1.f));
                cold.set3(kLr, f3(0.f, 0.f, 0.f));
                cold.set(kBounces, 0u);
                cold.set(kFlags, exact ? kColdExact : 0u);
                cold.set(kSlot, slot);
                cold.set(kPixel, pixel);
                cold.set(kSample, sample);
                cold.set(kItem, item);
                if (TL) two = p->instances != nullptr;
                begin(o, d, inf, false, exact);
                active = true;
                finished = false;
            }
            const uint32_t took = (uint32_t)__popc(need) < avail ? (uint32_t)__popc(need) : avail;
            pool_next += took;
        }
        if (!__any_sync(0xFFFFFFFFu, active)) {
            if (exhausted) break;
            continue;
        }
        {
            uint32_t leaf_off = 0, leaf_n = 0;
            bool ok, at_leaf;
            if constexpr (TL) {
                // walk_round with each lane stepping its own layout
                at_leaf = false;
                ok = true;
                const bool walking0 = active && !finished && k.sp > 0;
                const uint32_t cand = __ballot_sync(0xFFFFFFFFu, walking0);
                const int want = __popc(cand) < PT_LEAF_BATCH_PATHS ? __popc(cand) : PT_LEAF_BATCH_PATHS;
                while (true) {
                    const bool w_now = walking0 && ok && !at_leaf && k.sp > 0;
                    const uint32_t w = __ballot_sync(0xFFFFFFFFu, w_now);
                    if (w == 0 || __popc(cand & ~w) >= want) break;
                    if (w_now) {
                        int r;
                        if (two) {
                            const uint32_t e = k.stack.get(--k.sp);
                            r = two_level_tagged(e)
                                    ? two_level_transition<false>(k, e, items[cold.u(kItem)].params, tl_lane)
                                    // the min/max box form without the per-node choice where the lane's
                                    // ray takes it: 517 against 500 Msamples/s on the two-level frame
                                    : k.box_mode == 0 ? two_level_node_step<false, true>(k, e, nodes, num_nodes, leaf_off, leaf_n)
                                                      : two_level_node_step<false>(k, e, nodes, num_nodes, leaf_off, leaf_n);
                        } else {
                            r = walk_step<false>(k, nodes, num_nodes, leaf_off, leaf_n);
                        }
                        at_leaf = r > 0;
                        ok = r >= 0;
                    }
                }
            } else if constexpr (PT_LEAF_BATCH_PATHS > 0) {
                walk_round<false, 1, true>(k, active && !finished && k.sp > 0, PT_LEAF_BATCH_PATHS, nodes, num_nodes, at_leaf,
                                     ok, leaf_off, leaf_n);
            } else {
                const bool walking = active && !finished;
                ok = !walking || walk_to_leaf<false>(k, nodes, num_nodes, leaf_off, leaf_n);
                at_leaf = walking && ok && leaf_n > 0;
            }
            if (at_leaf) {
                if (TL && two) {
                    if (walk_leaf_two_level<false>(k, tris, cold.u(kFaceBase), leaf_off, leaf_n, cold.u(kPrimBase)))
                        cold.set(kHitInst, cold.u(kInst));
                } else {
                    walk_leaf<false>(k, tris, leaf_off, leaf_n);
                }
            }
            if (active && !finished && (!ok || k.done || k.sp == 0)) {
                finished = true;
                walk_ok = ok;
            }
        }
        const uint32_t fin = __ballot_sync(0xFFFFFFFFu, active && finished);
        const uint32_t walking = __ballot_sync(0xFFFFFFFFu, active && !finished);
        if (fin && (walking == 0 || __popc(fin) >= kShadeBatch)) {
            if (active && finished) {
                finished = false;
                ++rays;
                const WfItem& it = items[cold.u(kItem)];
                const RenderParams* p = it.params;
                uint32_t flags = cold.u(kFlags);
                const bool shadow = (flags & kColdShadow) != 0;
                const bool exact = (flags & kColdExact) != 0;
                bool go = false, next_shadow = false;
                if (!walk_ok) {
                    raise_flag(p->err);
                } else if (!shadow) {
                    PathState s;
                    s.o = cold.f3at(kOx);
                    s.d = cold.f3at(kDx);
                    s.src = cold.f3at(kSr);
                    s.L = cold.f3at(kLr);
                    s.bounces = cold.u(kBounces);
                    s.last_lambert = (flags & kColdLambert) ? 1u : 0u;
                    const uint32_t pixel = cold.u(kPixel), sample = cold.u(kSample);
                    if (s.bounces == 0 && sample == 0 && it.primary) it.primary[pixel] = k.prim;
                    ShadowReq sh;
                    const bool more = (TL && two)
                                          ? shade_hit_two_level(*p, s, k.prim, k.leaf, cold.u(kHitInst), k.u, k.v, k.w, pixel,
                                                                sample, sh)
                                          : shade_hit(*p, s, k.prim, k.leaf, k.u, k.v, k.w, pixel, sample, sh);
                    cold.set3(kOx, s.o);
                    cold.set3(kDx, s.d);
                    cold.set3(kSr, s.src);
                    cold.set3(kLr, s.L);
                    cold.set(kBounces, s.bounces);
                    flags = (s.last_lambert ? kColdLambert : 0u) | (flags & kColdExact);
                    if (sh.valid) {
                        cold.set3(kCr, sh.contrib);
                        flags |= kColdShadow | (more ? kColdPending : 0u);
                        next_shadow = true;
                        begin(sh.o, sh.wi, sh.tmax, true, exact);
                    } else {
                        go = more && !throughput_is_zero(s.src);
                    }
                    cold.set(kFlags, flags);
                } else {
                    if (k.prim == kPrimNone) cold.set3(kLr, vadd(cold.f3at(kLr), cold.f3at(kCr)));
                    go = (flags & kColdPending) != 0 && !throughput_is_zero(cold.f3at(kSr));
                    cold.set(kFlags, flags & ~(kColdShadow | kColdPending));
                }
                if (!next_shadow) {
                    if (go) {
                        begin(cold.f3at(kOx), cold.f3at(kDx), inf, false, exact);
                    } else {
                        clamp_store(radiance + 3 * (size_t)cold.u(kSlot), cold.f3at(kLr));
                        active = false;
                    }
                }
            }
        }
    }
    if (rays_traced) {
        const uint32_t sum = __reduce_add_sync(0xFFFFFFFFu, rays);
        if (lane == 0 && sum) atomicAdd(rays_traced, (unsigned long long)sum);
    }
}

__global__ void wf_advance_kernel(uint32_t* counters, uint32_t consumed) {
    counters[consumed] = 0;
    counters[2] = 0;
}

__global__ void __launch_bounds__(256) wf_store_kernel(WfState ws, uint32_t count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float4 l = ws.rad[i];
    clamp_store(ws.radiance + 3 * (size_t)i, f3(l.x, l.y, l.z));
}

// film[pixel] += radiance of the pixel's samples inside the segment, in sample order.
__global__ void __launch_bounds__(256) wf_resolve_kernel(const WfItem* __restrict__ items, const WfSegment* __restrict__ segs,
                                                         const WfPixels* __restrict__ e, uint32_t ne, uint64_t total,
                                                         const float* __restrict__ radiance) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const WfPixels ent = e[find_pixels(e, ne, t)];
    const WfSegment sg = segs[ent.seg];
    const WfItem it = items[sg.item];
    const uint32_t pixel = ent.pix_begin + (uint32_t)(t - ent.base);
    const uint64_t a = sg.local_begin, b = sg.local_begin + sg.count;
    uint64_t s0 = a / it.npix;
    if (s0 * it.npix + pixel < a) ++s0;
    float* f = it.film + 3 * (size_t)pixel;
    float r = f[0], g = f[1], bl = f[2];
    for (uint64_t p = s0 * it.npix + pixel; p < b; p += it.npix) {
        const size_t k = 3 * (size_t)(sg.slot_base + (p - a));
        r = fadd(r, radiance[k]);
        g = fadd(g, radiance[k + 1]);
        bl = fadd(bl, radiance[k + 2]);
    }
    f[0] = r;
    f[1] = g;
    f[2] = bl;
}

// rgb = film * (1 / spp) for items whose last path ran in this wave (BoxFilter.cpp:65-67).
__global__ void __launch_bounds__(256) wf_finish_kernel(const WfItem* __restrict__ items, const WfPixels* __restrict__ e,
                                                        uint32_t ne, uint64_t total) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const WfPixels ent = e[find_pixels(e, ne, t)];
    const WfItem it = items[ent.item];
    const uint32_t pixel = ent.pix_begin + (uint32_t)(t - ent.base);
    const float inv = frcp((float)it.spp);
    for (int c = 0; c < 3; ++c) it.rgb[3 * (size_t)pixel + c] = fmul(it.film[3 * (size_t)pixel + c], inv);
}

// ---- host side --------------------------------------------------------------------------------

// The persistent path kernel (paths_only) needs only the radiance and the counters.
size_t wf_state_bytes(uint32_t cap, bool paths_only) {
    size_t n = 0;
    auto take = [&](size_t b) { n += (b + 255) & ~(size_t)255; };
    if (!paths_only) {
        for (int k = 0; k < 4; ++k) take(16 * (size_t)cap);  // ray_o, ray_d, thr, rad
        take(8 * (size_t)cap);                               // path
        take(16 * (size_t)cap);                              // hit
        take(4 * (size_t)cap);                               // hit_w
        take(4 * (size_t)cap);
        take(4 * (size_t)cap);                               // queues
        for (int k = 0; k < 3; ++k) take(16 * (size_t)cap);  // shadow queue
    }
    take(12 * (size_t)cap);                                  // radiance
    take(64);                                                // counters
    return n;
}

void wf_state_carve(void* base, uint32_t cap, WfState& ws, bool paths_only) {
    char* q = (char*)base;
    auto take = [&](size_t b) { char* r = q; q += (b + 255) & ~(size_t)255; return r; };
    ws = WfState{};
    if (!paths_only) {
        ws.ray_o = (float4*)take(16 * (size_t)cap);
        ws.ray_d = (float4*)take(16 * (size_t)cap);
        ws.thr = (float4*)take(16 * (size_t)cap);
        ws.rad = (float4*)take(16 * (size_t)cap);
        ws.path = (uint64_t*)take(8 * (size_t)cap);
        ws.hit = (uint4*)take(16 * (size_t)cap);
        ws.hit_w = (float*)take(4 * (size_t)cap);
        ws.queue[0] = (uint32_t*)take(4 * (size_t)cap);
        ws.queue[1] = (uint32_t*)take(4 * (size_t)cap);
        ws.sh_o = (float4*)take(16 * (size_t)cap);
        ws.sh_d = (float4*)take(16 * (size_t)cap);
        ws.sh_c = (float4*)take(16 * (size_t)cap);
    }
    ws.radiance = (float*)take(12 * (size_t)cap);
    ws.counters = (uint32_t*)take(64);
    ws.capacity = cap;
}

void wf_add_wave(WfPlan& plan, const std::vector<WfSegment>& segs, const std::vector<uint32_t>& npix,
                 const std::vector<uint32_t>& spp, const std::vector<uint32_t>& max_depth) {
    WfWave w{};
    w.seg_begin = (uint32_t)plan.segments.size();
    w.seg_count = (uint32_t)segs.size();
    w.res_begin = (uint32_t)plan.resolve.size();
    w.fin_begin = (uint32_t)plan.finish.size();
    uint64_t count = 0, res_px = 0, fin_px = 0;
    uint32_t bounces = 0;
    for (const WfSegment& sg : segs) {
        const uint32_t gseg = (uint32_t)plan.segments.size();
        plan.segments.push_back(sg);
        count += sg.count;
        bounces = std::max(bounces, max_depth[sg.item] + 1);
        const uint64_t n = npix[sg.item];
        const uint64_t a = sg.local_begin, b = sg.local_begin + sg.count;
        auto add_res = [&](uint32_t p0, uint32_t pc) {
            plan.resolve.push_back(WfPixels{gseg, p0, pc, sg.item, res_px});
            res_px += pc;
        };
        if (b - a >= n) {
            add_res(0, (uint32_t)n);
        } else {
            const uint32_t pa = (uint32_t)(a % n), pb = (uint32_t)((b - 1) % n);
            if (a / n == (b - 1) / n) {
                add_res(pa, pb - pa + 1);
            } else {
                add_res(pa, (uint32_t)n - pa);
                add_res(0, pb + 1);
            }
        }
        if (b == n * spp[sg.item]) {
            plan.finish.push_back(WfPixels{gseg, 0, (uint32_t)n, sg.item, fin_px});
            fin_px += n;
        }
    }
    w.count = (uint32_t)count;
    w.bounces = bounces;
    w.res_count = (uint32_t)plan.resolve.size() - w.res_begin;
    w.res_pixels = res_px;
    w.fin_count = (uint32_t)plan.finish.size() - w.fin_begin;
    w.fin_pixels = fin_px;
    plan.waves.push_back(w);
}

void wf_plan_all(WfPlan& plan, const std::vector<uint32_t>& npix, const std::vector<uint32_t>& spp,
                 const std::vector<uint32_t>& max_depth, uint64_t wave_paths) {
    std::vector<WfSegment> segs;
    uint64_t room = wave_paths;
    uint64_t slot = 0;
    for (uint32_t i = 0; i < npix.size(); ++i) {
        const uint64_t total = (uint64_t)npix[i] * spp[i];
        uint64_t done = 0;
        while (done < total) {
            const uint64_t take = std::min<uint64_t>(room, total - done);
            segs.push_back(WfSegment{i, 0, done, slot, take});
            done += take;
            slot += take;
            room -= take;
            if (room == 0) {
                wf_add_wave(plan, segs, npix, spp, max_depth);
                segs.clear();
                room = wave_paths;
                slot = 0;
            }
        }
    }
    if (!segs.empty()) wf_add_wave(plan, segs, npix, spp, max_depth);
}

namespace {
template <int CAP, bool SHADOW>
cudaError_t launch_trace_stage(const WfItem* items, const WfState& ws, const uint32_t* queue, const uint32_t* count_ptr,
                               unsigned long long* fetch, const WfTuning& t, unsigned long long* rays, cudaStream_t s) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wf_trace_kernel<CAP, SHADOW>, (int)t.threads_per_block, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    e = cudaMemsetAsync(fetch, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    wf_trace_kernel<CAP, SHADOW><<<(unsigned)(sms * per_sm), t.threads_per_block, 0, s>>>(items, ws, queue, count_ptr, fetch,
                                                                                         t.queue_chunk, rays);
    return cudaGetLastError();
}

template <int CAP, bool TL>
cudaError_t launch_path_stage(const WfItem* items, const WfSegment* segs, uint32_t nseg, uint32_t count, float* radiance,
                              unsigned long long* fetch, uint32_t chunk, unsigned long long* rays, cudaStream_t s) {
    constexpr int SH = 16;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wf_path_kernel<CAP, SH, TL>, 128, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    uint64_t grid = (uint64_t)sms * per_sm;
    const uint64_t grid_needed = (((uint64_t)count + chunk - 1) / chunk * 32 + 127) / 128;
    if (grid > grid_needed) grid = grid_needed ? grid_needed : 1;
    e = cudaMemsetAsync(fetch, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    wf_path_kernel<CAP, SH, TL><<<(unsigned)grid, 128, 0, s>>>(items, segs, nseg, count, radiance, fetch, chunk, rays);
    return cudaGetLastError();
}

cudaError_t path_stage(int cap, bool two_level, const WfItem* items, const WfSegment* segs, uint32_t nseg, uint32_t count,
                       float* radiance, unsigned long long* fetch, uint32_t chunk, unsigned long long* rays, cudaStream_t s) {
    if (two_level) {  // the top level, the exit marker and the bottom level share the stack: the largest capacity
        return launch_path_stage<64, true>(items, segs, nseg, count, radiance, fetch, chunk, rays, s);
    }
    switch (cap) {
        case 24: return launch_path_stage<24, false>(items, segs, nseg, count, radiance, fetch, chunk, rays, s);
        case 32: return launch_path_stage<32, false>(items, segs, nseg, count, radiance, fetch, chunk, rays, s);
        case 48: return launch_path_stage<48, false>(items, segs, nseg, count, radiance, fetch, chunk, rays, s);
        default: return launch_path_stage<64, false>(items, segs, nseg, count, radiance, fetch, chunk, rays, s);
    }
}

template <bool SHADOW>
cudaError_t trace_stage(int cap, const WfItem* items, const WfState& ws, const uint32_t* queue, const uint32_t* count_ptr,
                        unsigned long long* fetch, const WfTuning& t, unsigned long long* rays, cudaStream_t s) {
    switch (cap) {
        case 24: return launch_trace_stage<24, SHADOW>(items, ws, queue, count_ptr, fetch, t, rays, s);
        case 32: return launch_trace_stage<32, SHADOW>(items, ws, queue, count_ptr, fetch, t, rays, s);
        case 48: return launch_trace_stage<48, SHADOW>(items, ws, queue, count_ptr, fetch, t, rays, s);
        default: return launch_trace_stage<64, SHADOW>(items, ws, queue, count_ptr, fetch, t, rays, s);
    }
}
// Camera rays of the wave's slots, then per bounce: extend, shade (queue the next rays and the
// shadow rays), shadow; finally the clamped radiance of every slot.
cudaError_t bounce_stages(const WfItem* d_items, const WfSegment* d_segments, const WfWave& w, const WfState& ws,
                          const WfTuning& t, unsigned long long* rays_traced, cudaStream_t s) {
    const uint32_t blocks = (w.count + 127) / 128;
    wf_init_kernel<<<blocks, 128, 0, s>>>(d_items, d_segments + w.seg_begin, w.seg_count, w.count, ws);
    cudaError_t e = cudaGetLastError();
    unsigned long long* fetch0 = (unsigned long long*)(ws.counters + 4);
    unsigned long long* fetch1 = (unsigned long long*)(ws.counters + 6);
    uint32_t cur = 0;
    for (uint32_t b = 0; e == cudaSuccess && b < w.bounces; ++b) {
        const uint32_t nxt = cur ^ 1u;
        e = trace_stage<false>(t.stack_cap, d_items, ws, ws.queue[cur], ws.counters + cur, fetch0, t, rays_traced, s);
        if (e != cudaSuccess) break;
        wf_shade_kernel<<<blocks, 128, 0, s>>>(d_items, ws, ws.queue[cur], ws.counters + cur, ws.queue[nxt], ws.counters + nxt);
        e = cudaGetLastError();
        if (e != cudaSuccess) break;
        e = trace_stage<true>(t.stack_cap, d_items, ws, nullptr, ws.counters + 2, fetch1, t, rays_traced, s);
        if (e != cudaSuccess) break;
        wf_advance_kernel<<<1, 1, 0, s>>>(ws.counters, cur);
        e = cudaGetLastError();
        cur = nxt;
    }
    if (e != cudaSuccess) return e;
    wf_store_kernel<<<(w.count + 255) / 256, 256, 0, s>>>(ws, w.count);
    return cudaGetLastError();
}
}  // namespace

cudaError_t wf_launch_wave(const WfItem* d_items, const WfSegment* d_segments, const WfPixels* d_resolve,
                           const WfPixels* d_finish, const WfWave& w, const WfState& ws, const WfTuning& t,
                           unsigned long long* rays_traced, cudaStream_t s) {
    if (w.count == 0) return cudaSuccess;
    if (w.count > ws.capacity) return cudaErrorInvalidValue;
    if (!t.paths && !ws.ray_o) return cudaErrorInvalidValue;  // state carved for the path kernel only
    cudaError_t e = t.paths ? path_stage(t.stack_cap, t.two_level, d_items, d_segments + w.seg_begin, w.seg_count, w.count,
                                         ws.radiance, (unsigned long long*)(ws.counters + 4), t.queue_chunk, rays_traced, s)
                            : bounce_stages(d_items, d_segments, w, ws, t, rays_traced, s);
    if (e != cudaSuccess) return e;
    if (w.res_pixels)
        wf_resolve_kernel<<<(unsigned)((w.res_pixels + 255) / 256), 256, 0, s>>>(d_items, d_segments, d_resolve + w.res_begin,
                                                                                 w.res_count, w.res_pixels, ws.radiance);
    if (w.fin_pixels)
        wf_finish_kernel<<<(unsigned)((w.fin_pixels + 255) / 256), 256, 0, s>>>(d_items, d_finish + w.fin_begin, w.fin_count,
                                                                               w.fin_pixels);
    return cudaGetLastError();
}

}  // namespace pt
