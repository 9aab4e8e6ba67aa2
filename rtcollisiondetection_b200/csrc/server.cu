// server.cu - continuous-batching request server over resident scenes.
//
// Requests (any size, any thread) queue up.  Each of `slots` worker threads
// owns one stream and, per detector it serves, a clone of that detector (own
// workspace, shared resident robot and scene).  A worker repeatedly takes the
// oldest request it may serve plus every queued request for the same
// detector and flags that fits, merges them into one launch, runs it and
// splits the results.  Two classes of slots keep small requests fast:
//  - fast slots serve only requests of at most fast_max_units units, on the
//    highest-priority stream, with persistent kernels allowed the whole GPU;
//  - bulk slots serve anything, on normal-priority streams, with persistent
//    kernels limited to bulk_share percent of each SM, so a fast launch finds
//    room to run beside a long bulk launch instead of queueing behind it.
// A launch is admitted only while the estimated bytes of the launches in
// flight fit the memory budget.  Poses and trajectories are independent, so
// a request's result in a merged launch equals its result alone.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "../../include/rtcd.h"
#include "engine.h"

namespace rtcd {
void detector_info(rtcd_detector* d, rtcd_ctx** ctx, int* kind, rtcd_robot** robot, rtcd_scene** scene,
                   rtcd_config* cfg, uint32_t* n_links, uint32_t* n_spheres, uint32_t* dof);
}

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket = 0;
    rtcd_detector* det = nullptr;
    int kind = 0;
    uint32_t flags = 0;
    uint32_t n = 0;
    uint32_t units = 0;     // poses, or waypoints of a sweep request
    uint32_t segments = 0;  // sweep: segments of the request
    std::vector<float> q;
    std::vector<uint32_t> traj_off;
    std::vector<uint8_t> out_flags, out_seg;
    std::vector<uint32_t> out_counts;
    Clock::time_point submitted;
    double latency_ms = 0;
    bool done = false;
    int status = RTCD_OK;
    std::string error;
};

bool is_sweep(int kind) { return kind == RTCD_LINEAR_SWEEP || kind == RTCD_QUAD_SWEEP; }

uint64_t units_of(const std::vector<Request*>& batch) {
    uint64_t u = 0;
    for (const Request* r : batch) u += r->units;
    return u;
}

struct Slot {
    bool fast = false;
    uint32_t index = 0;
    std::mutex mu;                                      // held while the slot runs a launch or is prepared
    std::map<rtcd_detector*, rtcd_detector*> clones;    // user detector -> this slot's clone
};

}  // namespace

struct rtcd_server {
    rtcd_ctx* ctx = nullptr;
    rtcd_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_mem;
    std::deque<Request*> pending;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> requests;
    uint64_t next_ticket = 1;
    bool stopping = false;
    uint64_t inflight_bytes = 0;
    uint64_t submitted = 0, completed = 0, failed = 0, units_completed = 0, batches = 0, inflight_peak = 0;
    std::vector<double> latencies, queue_ms, run_ms;
    uint64_t workspace_grows = 0;
    double grow_ms = 0, run_max_ms = 0, run_max_at_s = 0;
    uint32_t run_max_kind = 0, run_max_units = 0, run_max_grows = 0, run_max_slot = 0;
    Clock::time_point stats_since = Clock::now();
    std::vector<std::unique_ptr<Slot>> slots;
    std::vector<std::thread> workers;
};

namespace {

// Bytes a launch holds on the device (inputs, per-item state, candidate buffer).
uint64_t estimate_bytes(int kind, uint64_t n, uint64_t units, uint32_t n_links, uint32_t n_spheres, uint32_t dof) {
    if (!is_sweep(kind))
        return n * (4ull * dof + 16) + n * n_links * (48ull + 1 + 4 + 1 + 4 + 8ull * 128);
    return units * (4ull * dof + 2ull * 16 * n_spheres) + n * 16 + units * 8;
}

// The slot's clone of a user detector (created on first use).
rtcd_detector* clone_for(rtcd_server* S, Slot& slot, rtcd_detector* det) {
    rtcd_detector*& c = slot.clones[det];
    if (c) return c;
    rtcd_ctx* ctx;
    int kind;
    rtcd_robot* rb;
    rtcd_scene* sc;
    rtcd_config cfg;
    uint32_t nl, ns, dof;
    rtcd::detector_info(det, &ctx, &kind, &rb, &sc, &cfg, &nl, &ns, &dof);
    if (slot.fast) {
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        cfg.stream_priority = hi;
        cfg.residency_percent = 0;
    } else {
        cfg.stream_priority = 0;
        cfg.residency_percent = S->cfg.bulk_share;
    }
    rtcd_status st = rtcd_detector_create(ctx, (rtcd_detector_kind) kind, rb, sc, &cfg, &c);
    if (st != RTCD_OK) {
        c = nullptr;
        char buf[256];
        rtcd_last_error(buf, sizeof(buf));
        rtcd::fail(st, buf);
    }
    return c;
}

// Runs one merged launch on the slot's clone; host buffers in and out.
rtcd_status run_launch(rtcd_server* S, Slot& slot, rtcd_detector* det, int kind, const std::vector<float>& q,
                       const std::vector<uint32_t>& off, uint32_t n, uint32_t flags, std::vector<uint8_t>& out_flags,
                       std::vector<uint8_t>& out_seg, std::vector<uint32_t>& out_counts, std::string& msg) {
    rtcd_detector* c = nullptr;
    try {
        c = clone_for(S, slot, det);
    } catch (const rtcd::Error& e) {
        msg = e.msg;
        return (rtcd_status) e.status;
    }
    const bool sweep = is_sweep(kind);
    const bool counts = (flags & RTCD_CHECK_COUNTS) != 0;
    rtcd_status st = rtcd_check(c, q.data(), sweep ? off.data() : nullptr, n, out_flags.data(),
                                sweep ? out_seg.data() : nullptr, counts ? out_counts.data() : nullptr,
                                (flags & (RTCD_CHECK_COUNTS | RTCD_CHECK_NO_ENDPOINTS | RTCD_CHECK_SURFACE)) |
                                    RTCD_CHECK_HOST_BUFFERS,
                                nullptr);
    if (st != RTCD_OK) {
        char buf[512];
        rtcd_last_error(buf, sizeof(buf));
        msg = buf;
    }
    return st;
}

void worker(rtcd_server* S, Slot* slot) {
    std::vector<float> q;
    std::vector<uint32_t> off, counts;
    std::vector<uint8_t> flags, seg;
    const uint32_t limit = slot->fast ? std::max(S->cfg.fast_max_units, 1u) * 2 : S->cfg.max_batch_units;
    while (true) {
        std::vector<Request*> batch;
        uint64_t bytes = 0;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            auto servable = [&](const Request* r) { return !slot->fast || r->units <= S->cfg.fast_max_units; };
            auto has_work = [&] {
                for (const Request* r : S->pending)
                    if (servable(r)) return true;
                return false;
            };
            S->cv_work.wait(lk, [&] { return S->stopping || has_work(); });
            if (!has_work()) break;  // stopping, and nothing this slot may serve is left
            auto first_it = std::find_if(S->pending.begin(), S->pending.end(), servable);
            Request* first = *first_it;
            uint64_t units = 0;
            for (auto it = first_it; it != S->pending.end();) {
                Request* r = *it;
                if (servable(r) && r->det == first->det && r->flags == first->flags &&
                    (batch.empty() || units + r->units <= limit)) {
                    batch.push_back(r);
                    units += r->units;
                    it = S->pending.erase(it);
                } else {
                    ++it;
                }
            }
            rtcd_ctx* c;
            int kind;
            rtcd_robot* rb;
            rtcd_scene* sc;
            rtcd_config dc;
            uint32_t nl, ns, dof;
            rtcd::detector_info(first->det, &c, &kind, &rb, &sc, &dc, &nl, &ns, &dof);
            uint64_t n = 0;
            for (Request* r : batch) n += r->n;
            bytes = estimate_bytes(kind, n, units, nl, ns, dof);
            S->cv_mem.wait(lk, [&] { return S->inflight_bytes == 0 || S->inflight_bytes + bytes <= S->cfg.memory_budget; });
            S->inflight_bytes += bytes;
            S->inflight_peak = std::max(S->inflight_peak, S->inflight_bytes);
            ++S->batches;
            if (!S->pending.empty()) S->cv_work.notify_all();  // others may serve what is left
        }
        // merge the inputs
        Request* r0 = batch[0];
        const bool sweep = is_sweep(r0->kind);
        size_t nq = 0, n = 0;
        uint32_t total_seg = 0;
        for (Request* r : batch) {
            nq += r->q.size();
            n += r->n;
            total_seg += r->segments;
        }
        q.resize(nq);
        size_t pos = 0;
        off.assign(1, 0);
        for (Request* r : batch) {
            std::memcpy(q.data() + pos, r->q.data(), r->q.size() * sizeof(float));
            if (sweep) {
                const uint32_t base = off.back();
                for (uint32_t i = 1; i <= r->n; ++i) off.push_back(base + r->traj_off[i]);
            }
            pos += r->q.size();
        }
        flags.assign(n, 0);
        counts.assign(n, 0);
        seg.assign(sweep ? std::max<uint32_t>(total_seg, 1) : 0, 0);
        std::string msg;
        rtcd_status st;
        const auto started = Clock::now();
        const rtcd::GrowCounter g0 = rtcd::thread_grows();
        {
            std::lock_guard<std::mutex> sl(slot->mu);
            st = run_launch(S, *slot, r0->det, r0->kind, q, off, (uint32_t) n, r0->flags, flags, seg, counts, msg);
        }
        const rtcd::GrowCounter& g1 = rtcd::thread_grows();
        const uint64_t grows = g1.grows - g0.grows;
        const double grow_ms = g1.ms - g0.ms;
        const bool want_counts = (r0->flags & RTCD_CHECK_COUNTS) != 0;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            size_t p = 0, sp = 0;
            const auto now = Clock::now();
            const double run = std::chrono::duration<double, std::milli>(now - started).count();
            S->workspace_grows += grows;
            S->grow_ms += grow_ms;
            if (run > S->run_max_ms) {
                S->run_max_ms = run;
                S->run_max_kind = (uint32_t) r0->kind;
                S->run_max_units = (uint32_t) units_of(batch);
                S->run_max_grows = (uint32_t) grows;
                S->run_max_slot = slot->index;
                S->run_max_at_s = std::chrono::duration<double>(started - S->stats_since).count();
            }
            for (Request* r : batch) {
                r->status = st;
                r->error = msg;
                if (st == RTCD_OK) {
                    r->out_flags.assign(flags.begin() + p, flags.begin() + p + r->n);
                    if (want_counts) r->out_counts.assign(counts.begin() + p, counts.begin() + p + r->n);
                    if (sweep) r->out_seg.assign(seg.begin() + sp, seg.begin() + sp + r->segments);
                    ++S->completed;
                    S->units_completed += r->n;
                } else {
                    ++S->failed;
                }
                r->latency_ms = std::chrono::duration<double, std::milli>(now - r->submitted).count();
                if (st == RTCD_OK) {
                    S->latencies.push_back(r->latency_ms);
                    S->queue_ms.push_back(std::chrono::duration<double, std::milli>(started - r->submitted).count());
                    S->run_ms.push_back(run);
                }
                r->done = true;
                p += r->n;
                sp += r->segments;
            }
            S->inflight_bytes -= bytes;
        }
        S->cv_done.notify_all();
        S->cv_mem.notify_all();
    }
}

template <class F>
rtcd_status guard(F&& f) {
    try {
        f();
        rtcd::set_last_error("");
        return RTCD_OK;
    } catch (const rtcd::Error& e) {
        rtcd::set_last_error(e.msg);
        return (rtcd_status) e.status;
    } catch (const std::exception& e) {
        rtcd::set_last_error(e.what());
        return RTCD_ERR_INTERNAL;
    }
}

}  // namespace

extern "C" {

rtcd_status rtcd_server_create(rtcd_ctx* ctx, const rtcd_server_config* config, rtcd_server** out) {
    return guard([&] {
        if (!ctx || !out) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "NULL argument");
        *out = nullptr;
        std::unique_ptr<rtcd_server> S(new rtcd_server());
        S->ctx = ctx;
        if (config) S->cfg = *config;
        rtcd_server_config& c = S->cfg;
        if (!c.slots) c.slots = 4;
        if (c.slots > 64) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "at most 64 slots");
        if (!c.max_batch_units) c.max_batch_units = 65536;
        if (!c.fast_max_units) c.fast_max_units = 4096;
        if (!c.fast_slots) c.fast_slots = c.slots > 1 ? 1 : 0;
        if (c.fast_slots >= c.slots) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "at least one slot must serve any request");
        if (!c.bulk_share) c.bulk_share = 50;
        if (c.bulk_share > 100) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "bulk_share is a percentage");
        if (!c.memory_budget) {
            size_t free_b = 0, total_b = 0;
            rtcd::cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
            c.memory_budget = free_b / 2;
        }
        for (uint32_t i = 0; i < c.slots; ++i) {
            S->slots.emplace_back(new Slot());
            S->slots.back()->fast = i < c.fast_slots;
            S->slots.back()->index = i;
        }
        for (auto& sl : S->slots) S->workers.emplace_back(worker, S.get(), sl.get());
        *out = S.release();
    });
}

rtcd_status rtcd_server_destroy(rtcd_server* S) {
    return guard([&] {
        if (!S) return;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->stopping = true;
        }
        S->cv_work.notify_all();
        for (auto& t : S->workers) t.join();
        for (auto& sl : S->slots)
            for (auto& kv : sl->clones)
                if (kv.second) rtcd_detector_destroy(kv.second);
        delete S;
    });
}

rtcd_status rtcd_server_prepare(rtcd_server* S, rtcd_detector* det, uint32_t max_units) {
    return guard([&] {
        if (!S || !det) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "NULL argument");
        rtcd_ctx* c;
        int kind;
        rtcd_robot* rb;
        rtcd_scene* sc;
        rtcd_config dc;
        uint32_t nl, ns, dof;
        rtcd::detector_info(det, &c, &kind, &rb, &sc, &dc, &nl, &ns, &dof);
        if (c != S->ctx) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "detector belongs to another context");
        // Synthetic launches (zero poses, zero trajectories) that reach every workspace a launch of up
        // to `units` units can need.  Discrete: one launch of `units` poses.  Sweeps: `units` waypoints
        // in three shapes - the shortest trajectories (the most trajectories and pieces), 16-waypoint
        // ones (many trajectories: the staged light pass), and 128-waypoint ones (the longest the weight
        // tables are prebuilt for, and few enough trajectories that the unstaged kernels and their
        // sphere-centre buffers run) - each flags-only and counting, in both sweep semantics (the
        // reference semantics also build the scene's loop-edge trees).
        const bool sweep = is_sweep(kind);
        const std::vector<uint32_t> lens =
            sweep ? std::vector<uint32_t>{kind == RTCD_QUAD_SWEEP ? 3u : 2u, 16u, 128u} : std::vector<uint32_t>{1u};
        std::vector<uint32_t> modes = {0u, (uint32_t) RTCD_CHECK_COUNTS};
        if (sweep) {
            modes.push_back(RTCD_CHECK_SURFACE);
            modes.push_back(RTCD_CHECK_SURFACE | RTCD_CHECK_COUNTS);
        }
        for (auto& sl : S->slots) {
            uint32_t units = max_units ? max_units : S->cfg.max_batch_units;
            if (sl->fast) units = std::min(units, std::max(S->cfg.fast_max_units, 1u) * 2);
            std::lock_guard<std::mutex> lk(sl->mu);
            for (uint32_t len : lens) {
                const uint32_t n = std::max(1u, units / len);
                const uint32_t u = sweep ? len * n : n;
                std::vector<uint32_t> off;
                if (sweep) {
                    off.resize(n + 1);
                    for (uint32_t i = 0; i <= n; ++i) off[i] = len * i;
                }
                std::vector<float> q((size_t) u * dof, 0.0f);
                std::vector<uint8_t> fl(n), seg(sweep ? (size_t) u + 2 * n : 0);
                std::vector<uint32_t> cnt(n);
                std::string msg;
                for (uint32_t mode : modes) {
                    rtcd_status st = run_launch(S, *sl, det, kind, q, off, n, mode, fl, seg, cnt, msg);
                    if (st != RTCD_OK) rtcd::fail(st, msg);
                }
            }
        }
    });
}

rtcd_status rtcd_server_submit(rtcd_server* S, rtcd_detector* det, const float* q, const uint32_t* traj_offsets,
                               uint32_t n, uint32_t flags, uint64_t* ticket) {
    return guard([&] {
        if (!S || !det || !ticket || (n && !q)) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "NULL argument");
        if (flags & ~(uint32_t) (RTCD_CHECK_COUNTS | RTCD_CHECK_NO_ENDPOINTS | RTCD_CHECK_SURFACE))
            rtcd::fail(RTCD_ERR_INVALID_ARGUMENT,
                       "server requests accept RTCD_CHECK_COUNTS, RTCD_CHECK_NO_ENDPOINTS and RTCD_CHECK_SURFACE");
        rtcd_ctx* c;
        int kind;
        rtcd_robot* rb;
        rtcd_scene* sc;
        rtcd_config dc;
        uint32_t nl, ns, dof;
        rtcd::detector_info(det, &c, &kind, &rb, &sc, &dc, &nl, &ns, &dof);
        if (c != S->ctx) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "detector belongs to another context");
        std::unique_ptr<Request> r(new Request());
        r->det = det;
        r->kind = kind;
        r->flags = flags;
        r->n = n;
        if (is_sweep(kind)) {
            if (!traj_offsets) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "traj_offsets required for sweep detectors");
            if (traj_offsets[0] != 0) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "traj_offsets must start at 0");
            std::vector<uint32_t> seg(n + 1);
            rtcd_status st = rtcd_segment_offsets((rtcd_detector_kind) kind, traj_offsets, n, flags, seg.data());
            if (st != RTCD_OK) rtcd::fail(st, "bad traj_offsets");
            r->traj_off.assign(traj_offsets, traj_offsets + n + 1);
            r->units = traj_offsets[n];
            r->segments = seg[n];
        } else {
            r->units = n;
        }
        r->q.assign(q, q + (size_t) r->units * dof);
        r->submitted = Clock::now();
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stopping) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "server is stopping");
        r->ticket = S->next_ticket++;
        *ticket = r->ticket;
        ++S->submitted;
        S->pending.push_back(r.get());
        S->requests[r->ticket] = std::move(r);
        S->cv_work.notify_all();
    });
}

rtcd_status rtcd_server_wait(rtcd_server* S, uint64_t ticket, int32_t timeout_ms, uint8_t* flags_out,
                             uint8_t* seg_flags_out, uint32_t* counts_out, double* latency_ms) {
    return guard([&] {
        if (!S) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "NULL server");
        std::unique_lock<std::mutex> lk(S->mu);
        if (S->requests.find(ticket) == S->requests.end()) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "unknown ticket");
        // the ticket is looked up afresh after every wake-up: another thread
        // waiting on the same ticket may have collected and released it
        auto ready = [&] {
            auto j = S->requests.find(ticket);
            return j == S->requests.end() || j->second->done;
        };
        if (timeout_ms < 0)
            S->cv_done.wait(lk, ready);
        else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
            rtcd::fail(RTCD_ERR_DEVICE_TIMEOUT, "request not finished yet");
        auto it = S->requests.find(ticket);
        if (it == S->requests.end())
            rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "unknown ticket (collected by another waiter)");
        Request* r = it->second.get();
        if (r->status != RTCD_OK) {
            std::string m = r->error;
            int st = r->status;
            S->requests.erase(it);
            S->cv_done.notify_all();  // other waiters on this ticket learn it is gone
            rtcd::fail(st, m);
        }
        if (flags_out) std::memcpy(flags_out, r->out_flags.data(), r->out_flags.size());
        if (seg_flags_out && !r->out_seg.empty()) std::memcpy(seg_flags_out, r->out_seg.data(), r->out_seg.size());
        if (counts_out && !r->out_counts.empty())
            std::memcpy(counts_out, r->out_counts.data(), 4 * r->out_counts.size());
        if (latency_ms) *latency_ms = r->latency_ms;
        S->requests.erase(it);
        S->cv_done.notify_all();
    });
}

rtcd_status rtcd_server_get_stats(rtcd_server* S, rtcd_server_stats* out) {
    return guard([&] {
        if (!S || !out) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "NULL argument");
        std::memset(out, 0, sizeof(*out));
        std::vector<double> lat, qms, rms;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            out->submitted = S->submitted;
            out->completed = S->completed;
            out->failed = S->failed;
            out->units_completed = S->units_completed;
            out->batches = S->batches;
            out->inflight_bytes_peak = S->inflight_peak;
            out->queue_depth = (uint32_t) S->pending.size();
            lat = S->latencies;
            qms = S->queue_ms;
            rms = S->run_ms;
        }
        auto pct = [](std::vector<double>& v, double p) {
            if (v.empty()) return 0.0;
            size_t k = std::min(v.size() - 1, (size_t) (p * (double) (v.size() - 1) + 0.5));
            std::nth_element(v.begin(), v.begin() + (long) k, v.end());
            return v[k];
        };
        if (!lat.empty()) {
            out->p50_ms = pct(lat, 0.50);
            out->p99_ms = pct(lat, 0.99);
            double s = 0, mx = 0;
            for (double v : lat) {
                s += v;
                mx = std::max(mx, v);
            }
            out->mean_ms = s / (double) lat.size();
            out->max_ms = mx;
        }
        out->queue_p50_ms = pct(qms, 0.50);
        out->queue_p99_ms = pct(qms, 0.99);
        out->run_p99_ms = pct(rms, 0.99);
        std::lock_guard<std::mutex> lk(S->mu);
        out->workspace_grows = S->workspace_grows;
        out->grow_ms = S->grow_ms;
        out->run_max_ms = S->run_max_ms;
        out->run_max_kind = S->run_max_kind;
        out->run_max_units = S->run_max_units;
        out->run_max_grows = S->run_max_grows;
        out->run_max_slot = S->run_max_slot;
        out->run_max_at_s = S->run_max_at_s;
    });
}

rtcd_status rtcd_server_reset_stats(rtcd_server* S) {
    return guard([&] {
        if (!S) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "NULL server");
        std::lock_guard<std::mutex> lk(S->mu);
        S->submitted = S->completed = S->failed = S->units_completed = S->batches = 0;
        S->inflight_peak = S->inflight_bytes;
        S->latencies.clear();
        S->queue_ms.clear();
        S->run_ms.clear();
        S->workspace_grows = 0;
        S->grow_ms = S->run_max_ms = S->run_max_at_s = 0;
        S->run_max_kind = S->run_max_units = S->run_max_grows = S->run_max_slot = 0;
        S->stats_since = Clock::now();
    });
}

}  // extern "C"
