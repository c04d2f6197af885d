// serve_sched_check.cpp -- the serving loop's scheduling decisions (polytope_b200/csrc/serve_sched.h)
// driven on the CPU: wave planning under both policies, admission against the memory budget, and
// cancellation of queued and admitted requests, including a simulated scheduler run in which
// requests arrive, are admitted, get waves, are cancelled at every stage and retire.
// Built and run by tests/test_serve_sched_cpu.py; prints "ok" and exits 0 when every check holds.
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <random>
#include <vector>

#include "serve_sched.h"

using namespace pt::serve;

static int failures = 0;
#define CHECK(c)                                                           \
    do {                                                                   \
        if (!(c)) {                                                        \
            std::fprintf(stderr, "%s:%d: CHECK(%s)\n", __FILE__, __LINE__, #c); \
            ++failures;                                                    \
        }                                                                  \
    } while (0)

static Work admitted(uint64_t total) {
    Work w;
    w.state = kAdmitted;
    w.total = total;
    return w;
}

static void oldest_first() {
    Work a = admitted(100), b = admitted(50), c = admitted(30);
    std::vector<Work*> act{&a, &b, &c};
    std::vector<Take> t;
    plan_wave(act, 120, kOldestFirst, 64, t);
    CHECK(t.size() == 2 && t[0].index == 0 && t[0].first == 0 && t[0].count == 100);
    CHECK(t[1].index == 1 && t[1].first == 0 && t[1].count == 20);
    plan_wave(act, 120, kOldestFirst, 64, t);
    CHECK(t.size() == 2 && t[0].index == 1 && t[0].first == 20 && t[0].count == 30);
    CHECK(t[1].index == 2 && t[1].count == 30);
    plan_wave(act, 120, kOldestFirst, 64, t);
    CHECK(t.empty());
    CHECK(a.planned == a.total && b.planned == b.total && c.planned == c.total);
}

static void fair_share() {
    Work r[4] = {admitted(10000), admitted(10000), admitted(10000), admitted(500)};
    std::vector<Work*> act{&r[0], &r[1], &r[2]};
    std::vector<Take> t;
    plan_wave(act, 4096, kFairShare, 64, t);  // 4096 / 3 = 1365 each
    CHECK(t.size() == 3);
    for (const Take& x : t) CHECK(x.count == 1365);
    std::vector<Work*> four{&r[0], &r[1], &r[2], &r[3]};
    plan_wave(four, 2048, kFairShare, 64, t);  // 512 each, raised to the 1024 floor: two requests fit
    CHECK(t.size() == 2 && t[0].count == 1024 && t[1].count == 1024);
    plan_wave(four, 1 << 20, kFairShare, 64, t);  // a small request takes only what it has left
    CHECK(t.size() == 4 && t[3].count == 500);
}

static void limits_and_skips() {
    Work r[5] = {admitted(10), admitted(10), admitted(10), admitted(10), admitted(10)};
    r[1].cancel = true;        // being cancelled: no more work
    r[2].state = kQueued;      // not admitted
    std::vector<Work*> act{&r[0], &r[1], &r[2], &r[3], &r[4]};
    std::vector<Take> t;
    plan_wave(act, 1000, kOldestFirst, 2, t);
    CHECK(t.size() == 2 && t[0].index == 0 && t[1].index == 3);
    CHECK(r[1].planned == 0 && r[2].planned == 0);
    CHECK(fits(0, 100, 50, true));       // alone, even above the budget
    CHECK(!fits(10, 100, 50, false));
    CHECK(fits(10, 40, 50, false) && !fits(11, 40, 50, false));
}

static void cancel_transitions() {
    CHECK(on_cancel(kQueued, false, 0) == CancelAction::EndNow);
    CHECK(on_cancel(kAdmitted, false, 0) == CancelAction::EndNow);
    CHECK(on_cancel(kAdmitted, false, 2) == CancelAction::EndAfterWaves);
    CHECK(on_cancel(kAdmitted, true, 1) == CancelAction::AlreadyCancelling);
    CHECK(on_cancel(kDone, false, 0) == CancelAction::Refuse);
    CHECK(on_cancel(kCancelled, false, 0) == CancelAction::Refuse);
    CHECK(on_cancel(-4, false, 0) == CancelAction::Refuse);
    CHECK(cancel_ends_on_retire(kAdmitted, true, 0));
    CHECK(!cancel_ends_on_retire(kAdmitted, true, 1));
    CHECK(!cancel_ends_on_retire(kAdmitted, false, 0));
}

// A scheduler run: requests arrive over time, are admitted under a memory budget, waves are
// planned (two kept queued, the oldest retired each step), and random requests are cancelled while
// queued, while admitted with and without queued waves, and after they finished (refused).
struct SimReq : Work {
    size_t bytes = 0;
    uint32_t waves_queued = 0;
    bool ever_planned_after_cancel = false;
};

static int total_cancelled = 0, total_refused = 0;

static void simulated_run(uint32_t policy, unsigned seed) {
    std::mt19937 rng(seed);
    std::vector<SimReq> reqs(200);
    for (auto& r : reqs) {
        r.total = 1 + rng() % 5000;
        r.bytes = 1 + rng() % 300;
    }
    std::deque<SimReq*> pending;
    std::vector<SimReq*> active;
    std::deque<std::vector<SimReq*>> queued;  // waves in flight: members
    size_t in_use = 0, budget = 1000, next_arrival = 0;
    int done = 0, cancelled = 0, refused = 0;
    for (int step = 0; step < 100000 && (done + cancelled < (int)reqs.size()); ++step) {
        if (next_arrival < reqs.size() && rng() % 2) pending.push_back(&reqs[next_arrival++]);
        // admission
        while (!pending.empty() && active.size() < 16) {
            SimReq* r = pending.front();
            if (!fits(in_use, r->bytes, budget, active.empty())) break;
            pending.pop_front();
            r->state = kAdmitted;
            in_use += r->bytes;
            active.push_back(r);
        }
        // a cancellation now and then
        if (next_arrival > 0 && rng() % 7 == 0) {
            SimReq* r = &reqs[rng() % next_arrival];
            switch (on_cancel(r->state, r->cancel, r->waves_queued)) {
                case CancelAction::EndNow:
                    if (r->state == kQueued) {
                        for (auto it = pending.begin(); it != pending.end(); ++it)
                            if (*it == r) { pending.erase(it); break; }
                    } else {
                        in_use -= r->bytes;
                        for (auto it = active.begin(); it != active.end(); ++it)
                            if (*it == r) { active.erase(it); break; }
                    }
                    r->state = kCancelled;
                    ++cancelled;
                    break;
                case CancelAction::EndAfterWaves: r->cancel = true; break;
                case CancelAction::AlreadyCancelling: break;
                case CancelAction::Refuse: ++refused; CHECK(r->state == kDone || r->state == kCancelled); break;
            }
        }
        // plan a wave
        std::vector<Work*> view(active.begin(), active.end());
        std::vector<Take> t;
        plan_wave(view, 2048, policy, 8, t);
        std::vector<SimReq*> members;
        for (const Take& x : t) {
            SimReq* r = active[x.index];
            if (r->cancel) r->ever_planned_after_cancel = true;
            CHECK(x.count > 0 && x.first + x.count <= r->total);
            ++r->waves_queued;
            members.push_back(r);
        }
        if (!members.empty()) queued.push_back(members);
        // retire the oldest wave when two are queued, or when nothing was planned
        if (!queued.empty() && (queued.size() >= 2 || members.empty())) {
            std::vector<SimReq*> w = queued.front();
            queued.pop_front();
            for (SimReq* r : w) --r->waves_queued;
            for (SimReq* r : w) {
                bool end = false;
                if (cancel_ends_on_retire(r->state, r->cancel, r->waves_queued)) {
                    r->state = kCancelled;
                    ++cancelled;
                    end = true;
                } else if (r->state == kAdmitted && !r->cancel && r->planned == r->total && r->waves_queued == 0) {
                    r->state = kDone;
                    ++done;
                    end = true;
                }
                if (end) {
                    in_use -= r->bytes;
                    for (auto it = active.begin(); it != active.end(); ++it)
                        if (*it == r) { active.erase(it); break; }
                }
            }
        }
    }
    CHECK(done + cancelled == (int)reqs.size());
    CHECK(in_use == 0 && active.empty() && pending.empty());
    for (const SimReq& r : reqs) {
        CHECK(r.state == kDone || r.state == kCancelled);
        CHECK(!r.ever_planned_after_cancel);
        CHECK(r.waves_queued == 0);
        if (r.state == kDone) CHECK(r.planned == r.total);
    }
    total_cancelled += cancelled;
    total_refused += refused;
}

int main() {
    oldest_first();
    fair_share();
    limits_and_skips();
    cancel_transitions();
    for (unsigned seed = 1; seed <= 20; ++seed) {
        simulated_run(kOldestFirst, seed);
        simulated_run(kFairShare, seed + 100);
    }
    CHECK(total_cancelled > 0 && total_refused > 0);  // the runs did cancel, and did hit finished requests
    if (failures) {
        std::fprintf(stderr, "%d checks failed\n", failures);
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
