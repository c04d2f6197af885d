// serve_sched.h -- the serving loop's scheduling decisions as plain host functions (no CUDA):
// which admitted requests get work in the next wave and how much, whether a request fits the
// device-memory budget, and what cancelling a request does.  server.cpp makes every one of these
// decisions through this header; tests/cpp/serve_sched_check.cpp drives them on the CPU.
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace pt {
namespace serve {

// Request states, as pt_server_poll reports them (negative values are errors).
constexpr int kQueued = 0, kAdmitted = 1, kDone = 2, kCancelled = 3;

// What the planner sees of an admitted request.
struct Work {
    int state = kQueued;
    bool cancel = false;      // being cancelled: gets no more work
    uint64_t total = 0;       // work units: pixels (fused pipeline) or paths (wave pipelines)
    uint64_t planned = 0;     // units handed to waves so far
};

struct Take {
    size_t index;             // into the active list
    uint64_t first, count;    // the request's units [first, first + count)
};

constexpr uint32_t kOldestFirst = 0, kFairShare = 1;  // PT_SERVE_OLDEST_FIRST, PT_SERVE_FAIR_SHARE

// A request that can still be given work.
inline bool open(const Work& w) { return w.state == kAdmitted && !w.cancel && w.planned < w.total; }

// The next wave's work over `active` (admission order): the oldest request first, each taking what
// it has left up to the wave's room (oldest-first), or an equal share of the room for every open
// request, at least 1024 units each (fair share); at most max_items requests.  Advances `planned`.
inline void plan_wave(std::vector<Work*>& active, uint64_t room, uint32_t policy, size_t max_items, std::vector<Take>& out) {
    out.clear();
    uint64_t share = room;
    if (policy == kFairShare) {
        size_t n = 0;
        for (const Work* w : active) n += open(*w);
        if (n) share = std::max<uint64_t>(1024, room / n);
    }
    for (size_t i = 0; i < active.size(); ++i) {
        if (out.size() >= max_items || room == 0) break;
        Work& w = *active[i];
        if (!open(w)) continue;
        const uint64_t t = std::min<uint64_t>(std::min<uint64_t>(share, w.total - w.planned), room);
        room -= t;
        out.push_back(Take{i, w.planned, t});
        w.planned += t;
    }
}

// Admission against the device-memory budget: a request fits when its bytes stay inside the budget,
// or when nothing else is admitted (a request larger than the budget then runs alone).
inline bool fits(size_t in_use, size_t need, size_t budget, bool none_admitted) {
    return none_admitted || in_use + need <= budget;
}

// pt_server_cancel: a queued request ends at once; an admitted one ends at once when no queued wave
// holds its work, else when the last such wave retires; anything else is refused.
enum class CancelAction { EndNow, EndAfterWaves, AlreadyCancelling, Refuse };
inline CancelAction on_cancel(int state, bool cancelling, uint32_t waves_queued) {
    if (state == kQueued) return CancelAction::EndNow;
    if (state != kAdmitted) return CancelAction::Refuse;
    if (cancelling) return CancelAction::AlreadyCancelling;
    return waves_queued == 0 ? CancelAction::EndNow : CancelAction::EndAfterWaves;
}

// After a wave retires (its waves_queued already decremented): a cancelled admitted request whose
// last queued wave that was ends now; an admitted request whose work is all planned and whose wave
// finished it is done.
inline bool cancel_ends_on_retire(int state, bool cancelling, uint32_t waves_queued) {
    return state == kAdmitted && cancelling && waves_queued == 0;
}

}  // namespace serve
}  // namespace pt
