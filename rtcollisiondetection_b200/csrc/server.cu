// server.cu - continuous-batching request server over resident scenes.
//
// Requests (any size, any thread) queue up; each of `slots` worker threads
// owns one stream and its own workspace (a clone of every detector it serves,
// sharing the resident robot and scene) and repeatedly takes the oldest
// request plus every queued request for the same detector and flags, up to
// max_batch_units, merges them into one launch, runs it, and splits the
// flags back.  A launch is admitted only while the estimated bytes of the
// launches in flight fit the memory budget.  Poses and trajectories are
// independent, so a request's result in a merged launch equals its result
// alone.
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
    uint32_t units = 0;            // poses, or waypoints of a sweep request
    uint32_t segments = 0;         // sweep: segments of the request
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
    // statistics
    uint64_t submitted = 0, completed = 0, failed = 0, units_completed = 0, batches = 0, inflight_peak = 0;
    std::vector<double> latencies;
    std::vector<std::thread> workers;
};

namespace {

// Bytes a launch holds on the device (inputs, per-item state, candidate buffer).
uint64_t estimate_bytes(int kind, uint64_t n, uint64_t units, uint32_t n_links, uint32_t n_spheres, uint32_t dof) {
    if (!is_sweep(kind))
        return n * (4ull * dof + 16) + n * n_links * (48ull + 1 + 4 + 1 + 4 + 8ull * 128);
    return units * (4ull * dof + 2ull * 16 * n_spheres) + n * 16 + units * 8;
}

void worker(rtcd_server* S) {
    std::map<std::pair<rtcd_detector*, uint32_t>, rtcd_detector*> clones;
    std::vector<float> q;
    std::vector<uint32_t> off, counts, seg_off;
    std::vector<uint8_t> flags, seg;
    while (true) {
        std::vector<Request*> batch;
        uint64_t bytes = 0;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] { return S->stopping || !S->pending.empty(); });
            if (S->pending.empty()) break;  // stopping and drained
            Request* first = S->pending.front();
            uint64_t units = 0;
            for (auto it = S->pending.begin(); it != S->pending.end();) {
                Request* r = *it;
                if (r->det == first->det && r->flags == first->flags &&
                    (batch.empty() || units + r->units <= S->cfg.max_batch_units)) {
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
            // admission: wait while other launches hold the budget
            S->cv_mem.wait(lk, [&] { return S->inflight_bytes == 0 || S->inflight_bytes + bytes <= S->cfg.memory_budget; });
            S->inflight_bytes += bytes;
            S->inflight_peak = std::max(S->inflight_peak, S->inflight_bytes);
            ++S->batches;
        }
        // merge the inputs
        Request* r0 = batch[0];
        const bool sweep = is_sweep(r0->kind);
        size_t nq = 0, n = 0;
        for (Request* r : batch) {
            nq += r->q.size();
            n += r->n;
        }
        q.resize(nq);
        size_t pos = 0;
        off.assign(1, 0);
        for (Request* r : batch) {
            std::memcpy(q.data() + pos, r->q.data(), r->q.size() * sizeof(float));
            if (sweep) {
                uint32_t base = off.back();
                for (uint32_t i = 1; i <= r->n; ++i) off.push_back(base + r->traj_off[i]);
            }
            pos += r->q.size();
        }
        flags.assign(n, 0);
        counts.assign(n, 0);
        const bool want_counts = (r0->flags & RTCD_CHECK_COUNTS) != 0;
        uint32_t total_seg = 0;
        for (Request* r : batch) total_seg += r->segments;
        seg.assign(sweep ? std::max<uint32_t>(total_seg, 1) : 0, 0);
        rtcd_detector*& clone = clones[{r0->det, r0->flags}];
        rtcd_status st = RTCD_OK;
        std::string msg;
        if (!clone) {
            rtcd_ctx* c;
            int kind;
            rtcd_robot* rb;
            rtcd_scene* sc;
            rtcd_config dc;
            uint32_t nl, ns, dof;
            rtcd::detector_info(r0->det, &c, &kind, &rb, &sc, &dc, &nl, &ns, &dof);
            st = rtcd_detector_create(c, (rtcd_detector_kind) kind, rb, sc, &dc, &clone);
        }
        if (st == RTCD_OK)
            st = rtcd_check(clone, q.data(), sweep ? off.data() : nullptr, (uint32_t) n, flags.data(),
                            sweep ? seg.data() : nullptr, want_counts ? counts.data() : nullptr,
                            (r0->flags & (RTCD_CHECK_COUNTS | RTCD_CHECK_NO_ENDPOINTS)) | RTCD_CHECK_HOST_BUFFERS,
                            nullptr);
        if (st != RTCD_OK) {
            char buf[512];
            rtcd_last_error(buf, sizeof(buf));
            msg = buf;
        }
        // split the results
        {
            std::lock_guard<std::mutex> lk(S->mu);
            size_t p = 0, sp = 0;
            auto now = Clock::now();
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
                if (st == RTCD_OK) S->latencies.push_back(r->latency_ms);
                r->done = true;
                p += r->n;
                sp += r->segments;
            }
            S->inflight_bytes -= bytes;
        }
        S->cv_done.notify_all();
        S->cv_mem.notify_all();
    }
    for (auto& kv : clones)
        if (kv.second) rtcd_detector_destroy(kv.second);
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
        if (!S->cfg.slots) S->cfg.slots = 4;
        if (S->cfg.slots > 64) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "at most 64 slots");
        if (!S->cfg.max_batch_units) S->cfg.max_batch_units = 65536;
        if (!S->cfg.memory_budget) {
            size_t free_b = 0, total_b = 0;
            rtcd::cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
            S->cfg.memory_budget = free_b / 2;
        }
        for (uint32_t i = 0; i < S->cfg.slots; ++i) S->workers.emplace_back(worker, S.get());
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
        delete S;
    });
}

rtcd_status rtcd_server_submit(rtcd_server* S, rtcd_detector* det, const float* q, const uint32_t* traj_offsets,
                               uint32_t n, uint32_t flags, uint64_t* ticket) {
    return guard([&] {
        if (!S || !det || !ticket || (n && !q)) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "NULL argument");
        if (flags & ~(uint32_t) (RTCD_CHECK_COUNTS | RTCD_CHECK_NO_ENDPOINTS))
            rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "server requests accept RTCD_CHECK_COUNTS and RTCD_CHECK_NO_ENDPOINTS");
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
            std::vector<uint32_t> seg(n + 1);
            rtcd_status st = rtcd_segment_offsets((rtcd_detector_kind) kind, traj_offsets, n, flags, seg.data());
            if (st != RTCD_OK) rtcd::fail(st, "bad traj_offsets");
            if (traj_offsets[0] != 0) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "traj_offsets must start at 0");
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
        S->cv_work.notify_one();
    });
}

rtcd_status rtcd_server_wait(rtcd_server* S, uint64_t ticket, int32_t timeout_ms, uint8_t* flags_out,
                             uint8_t* seg_flags_out, uint32_t* counts_out, double* latency_ms) {
    return guard([&] {
        if (!S) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "NULL server");
        std::unique_lock<std::mutex> lk(S->mu);
        auto it = S->requests.find(ticket);
        if (it == S->requests.end()) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "unknown ticket");
        Request* r = it->second.get();
        auto ready = [&] { return r->done; };
        if (timeout_ms < 0)
            S->cv_done.wait(lk, ready);
        else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
            rtcd::fail(RTCD_ERR_DEVICE_TIMEOUT, "request not finished yet");
        if (r->status != RTCD_OK) {
            std::string m = r->error;
            int st = r->status;
            S->requests.erase(it);
            rtcd::fail(st, m);
        }
        if (flags_out) std::memcpy(flags_out, r->out_flags.data(), r->out_flags.size());
        if (seg_flags_out && !r->out_seg.empty()) std::memcpy(seg_flags_out, r->out_seg.data(), r->out_seg.size());
        if (counts_out && !r->out_counts.empty())
            std::memcpy(counts_out, r->out_counts.data(), 4 * r->out_counts.size());
        if (latency_ms) *latency_ms = r->latency_ms;
        S->requests.erase(it);
    });
}

rtcd_status rtcd_server_get_stats(rtcd_server* S, rtcd_server_stats* out) {
    return guard([&] {
        if (!S || !out) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "NULL argument");
        std::memset(out, 0, sizeof(*out));
        std::vector<double> lat;
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
        }
        if (!lat.empty()) {
            auto pct = [&](double p) {
                size_t k = std::min(lat.size() - 1, (size_t) (p * (double) (lat.size() - 1) + 0.5));
                std::nth_element(lat.begin(), lat.begin() + (long) k, lat.end());
                return lat[k];
            };
            out->p50_ms = pct(0.50);
            out->p99_ms = pct(0.99);
            double s = 0, mx = 0;
            for (double v : lat) {
                s += v;
                mx = std::max(mx, v);
            }
            out->mean_ms = s / (double) lat.size();
            out->max_ms = mx;
        }
    });
}

rtcd_status rtcd_server_reset_stats(rtcd_server* S) {
    return guard([&] {
        if (!S) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "NULL server");
        std::lock_guard<std::mutex> lk(S->mu);
        S->submitted = S->completed = S->failed = S->units_completed = S->batches = 0;
        S->inflight_peak = S->inflight_bytes;
        S->latencies.clear();
    });
}

}  // extern "C"
