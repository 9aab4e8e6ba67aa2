// api.cu - the C ABI (include/rtcd.h) over the device engine.
//
// Host-side responsibilities: validate inputs, extract unique edges and fit
// PCA OBBs (RTCD/Meshes/mesh.h:200-216, RTCD/Meshes/Obb.h:29-114), build and
// keep the robot and scene LBVHs resident, size the per-detector workspaces,
// stage host buffers through pinned memory, and launch the query pipeline on a
// stream without any host round trip (the plain path adds one per frame, the
// shape of the upstream check(), RTCD/CollisionDetector/CollisionDetector.h:
// 354-471).
#include <algorithm>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_set>

#include "../../include/rtcd.h"
#include "kernels.h"

namespace rtcd {

static thread_local std::string g_last_error;

void fail(int status, const std::string& msg) { throw Error{status, msg}; }

void set_last_error(const std::string& msg) { g_last_error = msg; }

void cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    cudaGetLastError();
    int st = (e == cudaErrorMemoryAllocation) ? RTCD_ERR_OUT_OF_MEMORY : RTCD_ERR_CUDA;
    fail(st, std::string(what) + ": " + cudaGetErrorString(e));
}

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

// Growth is geometric (at least 1.5x): cudaFree synchronises the device, so a
// workspace that follows slowly rising batch sizes must not re-allocate often.
GrowCounter& thread_grows() {
    static thread_local GrowCounter c;
    return c;
}

namespace {
// Counts one re-allocation on this thread and the time from construction to destruction.
struct GrowTimer {
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    ~GrowTimer() {
        GrowCounter& c = thread_grows();
        ++c.grows;
        c.ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};
}  // namespace

void DevBuf::ensure(size_t n) {
    if (n <= bytes && p) return;
    GrowTimer timer;
    size_t want = std::max<size_t>(std::max<size_t>(n, 256), bytes + bytes / 2);
    release();
    cuda_check(cudaMalloc(&p, want), "cudaMalloc");
    bytes = want;
}

void HostBuf::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
}

void HostBuf::ensure(size_t n) {
    if (n <= bytes && p) return;
    GrowTimer timer;
    size_t want = std::max<size_t>(std::max<size_t>(n, 256), bytes + bytes / 2);
    release();
    cuda_check(cudaMallocHost(&p, want), "cudaMallocHost");
    bytes = want;
}

int device_sm_count() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 1;
}

// ---------------------------------------------------------------- host geometry
// Unique undirected edges in first-seen orientation (RTCD/Meshes/mesh.h:200-216).
static std::vector<uint32_t> unique_edges(const uint32_t* tris, size_t n_tris) {
    std::vector<uint32_t> out;
    out.reserve(n_tris * 3);
    std::unordered_set<uint64_t> seen;
    seen.reserve(n_tris * 3);
    for (size_t t = 0; t < n_tris; ++t)
        for (int k = 0; k < 3; ++k) {
            uint32_t a = tris[3 * t + k], b = tris[3 * t + (k + 1) % 3];
            uint64_t key = ((uint64_t) std::min(a, b) << 32) | std::max(a, b);
            if (seen.insert(key).second) {
                out.push_back(a);
                out.push_back(b);
            }
        }
    return out;
}

// Symmetric 3x3 eigen-decomposition by cyclic Jacobi rotations.
static void jacobi3(double A[3][3], double V[3][3], double w[3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) V[i][j] = (i == j);
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = std::fabs(A[0][1]) + std::fabs(A[0][2]) + std::fabs(A[1][2]);
        if (off < 1e-300) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (std::fabs(A[p][q]) < 1e-300) continue;
                double theta = (A[q][q] - A[p][p]) / (2 * A[p][q]);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                double c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    double akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - s * akq;
                    A[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - s * aqk;
                    A[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < 3; ++i) w[i] = A[i][i];
}

// PCA-fitted OBB of a point set (RTCD/Meshes/Obb.h:29-114): principal axes
// by decreasing variance, right-handed, extents from the projections.  The
// float result is then grown until it contains every input point and padded
// by `pad`.  out: centre(3), half(3), axes x/y/z (9), bounding radius.
static void fit_obb(const float* pts, const std::vector<uint32_t>& idx, float pad, float* out) {
    std::memset(out, 0, 16 * sizeof(float));
    out[6] = 1; out[10] = 1; out[14] = 1;
    if (idx.empty()) return;
    double mean[3] = {0, 0, 0};
    for (uint32_t i : idx)
        for (int k = 0; k < 3; ++k) mean[k] += pts[3 * i + k];
    for (int k = 0; k < 3; ++k) mean[k] /= (double) idx.size();
    double C[3][3] = {{0}};
    for (uint32_t i : idx) {
        double d[3] = {pts[3 * i] - mean[0], pts[3 * i + 1] - mean[1], pts[3 * i + 2] - mean[2]};
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) C[a][b] += d[a] * d[b];
    }
    double V[3][3], w[3];
    jacobi3(C, V, w);
    int order[3] = {0, 1, 2};
    std::sort(order, order + 3, [&](int a, int b) { return w[a] > w[b]; });
    double ax[3][3];
    for (int a = 0; a < 3; ++a)
        for (int k = 0; k < 3; ++k) ax[a][k] = V[k][order[a]];
    double det = ax[0][0] * (ax[1][1] * ax[2][2] - ax[1][2] * ax[2][1]) -
                 ax[0][1] * (ax[1][0] * ax[2][2] - ax[1][2] * ax[2][0]) +
                 ax[0][2] * (ax[1][0] * ax[2][1] - ax[1][1] * ax[2][0]);
    if (det < 0)
        for (int k = 0; k < 3; ++k) ax[2][k] = -ax[2][k];
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (uint32_t i : idx)
        for (int a = 0; a < 3; ++a) {
            double v = ax[a][0] * pts[3 * i] + ax[a][1] * pts[3 * i + 1] + ax[a][2] * pts[3 * i + 2];
            lo[a] = std::min(lo[a], v);
            hi[a] = std::max(hi[a], v);
        }
    double c[3] = {0, 0, 0};
    for (int a = 0; a < 3; ++a)
        for (int k = 0; k < 3; ++k) c[k] += ax[a][k] * 0.5 * (lo[a] + hi[a]);
    float fc[3], fh[3], fa[9];
    for (int k = 0; k < 3; ++k) fc[k] = (float) c[k];
    for (int a = 0; a < 3; ++a) {
        fh[a] = (float) (0.5 * (hi[a] - lo[a]));
        for (int k = 0; k < 3; ++k) fa[3 * a + k] = (float) ax[a][k];
    }
    // grow the float box until it holds every point (checked in double on the float box)
    for (uint32_t i : idx)
        for (int a = 0; a < 3; ++a) {
            double v = 0;
            for (int k = 0; k < 3; ++k) v += (double) fa[3 * a + k] * ((double) pts[3 * i + k] - fc[k]);
            double need = std::fabs(v) * (1 + 1e-6) + 1e-7;
            if (need > fh[a]) fh[a] = (float) need;
        }
    for (int a = 0; a < 3; ++a) fh[a] += pad;
    for (int k = 0; k < 3; ++k) out[k] = fc[k];
    for (int a = 0; a < 3; ++a) out[3 + a] = fh[a];
    for (int k = 0; k < 9; ++k) out[6 + k] = fa[k];
    out[15] = std::sqrt(fh[0] * fh[0] + fh[1] * fh[1] + fh[2] * fh[2]);
}

// Directed loop edges (RTCD/Meshes/mesh.h:378-620): every triangle's three
// edges, in the directions kept, run around it as a loop; an edge two
// neighbours need in opposite directions is kept in both.  The sweep
// detectors cast these under the entering-ray semantics (a closed triangle
// boundary that crosses the swept surface crosses it inwards somewhere along
// its loop).  The directions follow the upstream breadth-first walk: from the
// first unprocessed triangle, pop a triangle, complete its loop from the
// directions already chosen (see complete_loop), queue its unprocessed
// neighbours (per edge in increasing triangle index).  Output: triangles in
// index order, each triangle's edges in order, forward before reverse, each
// directed edge once.  Fails when a triangle does not end up a loop (the
// upstream throws: the mesh is not watertight).
namespace {
enum class Dir : uint8_t { none, fwd, bwd, both };

struct LoopBuilder {
    std::unordered_set<uint64_t> chosen;  // directed edges a -> b
    static uint64_t key(uint32_t a, uint32_t b) { return ((uint64_t) a << 32) | b; }
    bool has(uint32_t a, uint32_t b) const { return chosen.count(key(a, b)) != 0; }
    void add(uint32_t a, uint32_t b) { chosen.insert(key(a, b)); }
    Dir dir(uint32_t a, uint32_t b) const {
        const bool f = has(a, b), r = has(b, a);
        return f && r ? Dir::both : f ? Dir::fwd : r ? Dir::bwd : Dir::none;
    }
    // Adds directions so the triangle (v[0] v[1] v[2]) becomes a loop, by the
    // upstream rules for 3, 2, 1 and 0 edges already directed.
    void complete_loop(const uint32_t v[4]) {
        Dir d[3];
        int fwd = 0, bwd = 0, set = 0;
        for (int i = 0; i < 3; ++i) {
            d[i] = dir(v[i], v[i + 1]);
            fwd += d[i] == Dir::fwd || d[i] == Dir::both;
            bwd += d[i] == Dir::bwd || d[i] == Dir::both;
            set += d[i] != Dir::none;
        }
        auto orient = [&](int i, Dir w) {  // edge i in direction w
            if (w == Dir::fwd) add(v[i], v[i + 1]); else add(v[i + 1], v[i]);
        };
        auto first = [&](auto pred) {
            for (int i = 0; i < 3; ++i)
                if (pred(d[i])) return i;
            return -1;
        };
        const auto one_way = [](Dir x) { return x == Dir::fwd || x == Dir::bwd; };
        if (set == 3) {
            if (fwd == 3 || bwd == 3) return;
            // the rule breaker gets its other direction too
            const int i = fwd == bwd ? first([](Dir x) { return x != Dir::both; })
                          : fwd < bwd ? first([](Dir x) { return x == Dir::fwd; })
                                      : first([](Dir x) { return x == Dir::bwd; });
            if (i >= 0) orient(i, d[i] == Dir::fwd ? Dir::bwd : Dir::fwd);
        } else if (set == 2) {
            const int open = first([](Dir x) { return x == Dir::none; });
            Dir w = Dir::fwd;  // both decided edges two-way: forward (the upstream leaves this unset)
            const int i = first(one_way);
            if (fwd != 2 && bwd != 2) {  // one forward, one backward: double the first, follow the other
                orient(i, d[i] == Dir::fwd ? Dir::bwd : Dir::fwd);
                w = d[i] == Dir::fwd ? Dir::bwd : Dir::fwd;
            } else if (i >= 0) {
                w = d[i];
            }
            orient(open, w);
        } else if (set == 1) {
            const int i = first([](Dir x) { return x != Dir::none; });
            const Dir w = d[i] == Dir::fwd ? Dir::fwd : Dir::bwd;  // two-way counts as backward, as upstream
            for (int k = 0; k < 3; ++k)
                if (d[k] == Dir::none) orient(k, w);
        } else {
            for (int k = 0; k < 3; ++k) orient(k, Dir::fwd);
        }
    }
};
}  // namespace

std::vector<uint32_t> loop_edges(const uint32_t* tris, size_t n_tris) {
    std::vector<uint32_t> out;
    if (!n_tris) return out;
    // triangles around each undirected edge, ascending
    std::vector<std::pair<uint64_t, uint32_t>> adj;
    adj.reserve(3 * n_tris);
    for (size_t t = 0; t < n_tris; ++t)
        for (int k = 0; k < 3; ++k) {
            const uint32_t a = tris[3 * t + k], b = tris[3 * t + (k + 1) % 3];
            adj.emplace_back(LoopBuilder::key(std::min(a, b), std::max(a, b)), (uint32_t) t);
        }
    std::sort(adj.begin(), adj.end());
    adj.erase(std::unique(adj.begin(), adj.end()), adj.end());
    LoopBuilder L;
    L.chosen.reserve(4 * n_tris);
    std::vector<uint8_t> done(n_tris, 0);
    std::deque<uint32_t> open;
    size_t start = 0;
    while (true) {
        while (start < n_tris && done[start]) ++start;
        if (start == n_tris) break;
        open.push_back((uint32_t) start);
        while (!open.empty()) {
            const uint32_t cur = open.front();
            open.pop_front();
            if (done[cur]) continue;
            const uint32_t v[4] = {tris[3ull * cur], tris[3ull * cur + 1], tris[3ull * cur + 2], tris[3ull * cur]};
            L.complete_loop(v);
            done[cur] = 1;
            for (int i = 0; i < 3; ++i) {
                const uint64_t k = LoopBuilder::key(std::min(v[i], v[i + 1]), std::max(v[i], v[i + 1]));
                auto it = std::lower_bound(adj.begin(), adj.end(), std::make_pair(k, 0u));
                for (; it != adj.end() && it->first == k; ++it)
                    if (it->second != cur && !done[it->second]) open.push_back(it->second);
            }
        }
    }
    out.reserve(2 * L.chosen.size());
    for (size_t t = 0; t < n_tris; ++t) {
        const uint32_t v[4] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2], tris[3 * t]};
        int fwd = 0, bwd = 0;
        for (int i = 0; i < 3; ++i) {
            fwd += L.has(v[i], v[i + 1]);
            bwd += L.has(v[i + 1], v[i]);
        }
        if (fwd != 3 && bwd != 3) fail(RTCD_ERR_INVALID_ARGUMENT, "loop edges: a triangle does not close a loop");
    }
    for (size_t t = 0; t < n_tris; ++t) {
        const uint32_t v[4] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2], tris[3 * t]};
        for (int i = 0; i < 3; ++i)
            for (int rev = 0; rev < 2; ++rev) {
                const uint32_t a = rev ? v[i + 1] : v[i], b = rev ? v[i] : v[i + 1];
                if (L.chosen.erase(LoopBuilder::key(a, b))) {
                    out.push_back(a);
                    out.push_back(b);
                }
            }
    }
    return out;
}

// Device LBVH over triangles or edges, concatenated over several groups
// (links); returns per-group roots.
struct GroupedBvh {
    DevBuf nodes, prims;
    std::vector<uint32_t> roots;
    uint32_t max_depth = 0;
};

static void build_grouped(bool tris, const float* d_verts, const std::vector<uint32_t>& vert_off, const uint32_t* d_idx,
                          const std::vector<uint32_t>& prim_off, uint32_t* d_err, cudaStream_t s, GroupedBvh& out,
                          const uint32_t* d_tag = nullptr) {
    size_t groups = prim_off.size() - 1;
    uint32_t total = prim_off.back();
    size_t total_nodes = 0;
    for (size_t g = 0; g < groups; ++g) {
        uint32_t n = prim_off[g + 1] - prim_off[g];
        total_nodes += n > 1 ? n - 1 : 0;
    }
    out.nodes.ensure(64 * std::max<size_t>(total_nodes, 1));
    out.prims.ensure((tris ? 48 : 32) * (size_t) std::max<uint32_t>(total, 1));
    out.roots.assign(groups, kNone);
    DevBuf lo, hi, perm;
    lo.ensure(16ull * std::max<uint32_t>(total, 1));
    hi.ensure(16ull * std::max<uint32_t>(total, 1));
    perm.ensure(4ull * std::max<uint32_t>(total, 1));
    uint32_t node_off = 0;
    const int per = tris ? 3 : 2;
    for (size_t g = 0; g < groups; ++g) {
        uint32_t p0 = prim_off[g], n = prim_off[g + 1] - p0;
        if (!n) continue;
        const float* v = d_verts + 3ull * vert_off[g];
        const uint32_t* ix = d_idx + (size_t) per * p0;
        float4* l = lo.as<float4>() + p0;
        float4* h = hi.as<float4>() + p0;
        if (tris) tri_boxes(v, ix, n, l, h, s); else edge_boxes(v, ix, n, l, h, s);
        LbvhResult r = build_lbvh(l, h, n, out.nodes.as<float4>() + 4ull * node_off, perm.as<uint32_t>() + p0, node_off,
                                  p0, d_err, s);
        out.roots[g] = r.root;
        out.max_depth = std::max(out.max_depth, r.depth);
        if (tris)
            gather_tris(v, ix, perm.as<uint32_t>() + p0, n, p0, (uint32_t) g, d_tag ? d_tag + p0 : nullptr,
                        out.prims.as<float4>() + 3ull * p0, s);
        else
            gather_edges(v, ix, perm.as<uint32_t>() + p0, n, p0, (uint32_t) g, out.prims.as<float4>() + 2ull * p0, s);
        node_off += n > 1 ? n - 1 : 0;
    }
    cuda_check(cudaStreamSynchronize(s), "grouped bvh");
}

}  // namespace rtcd

using namespace rtcd;

struct rtcd_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    DevBuf err;
    DevBuf knn_w2;  // squared neighbour-search weights
    std::mutex mu;  // guards knn_w2
};

struct rtcd_robot {
    rtcd_ctx* ctx = nullptr;
    RobotDev dev{};
    GroupedBvh tri, edge;
    DevBuf verts, tris, edges, spheres, sphere_link;
    std::vector<uint32_t> edge_off;
    uint32_t dof = 0;
};

struct rtcd_scene {
    rtcd_ctx* ctx = nullptr;
    SceneDev dev{};
    GroupedBvh tri, edge;
    DevBuf verts, tris, edges, obbs, tri_obs, obs_box, obs_point;
    DevBuf tri_wide, edge_wide, tri_cut, edge_cut;  // 4-wide copies of the two scene trees and their top cuts
    uint32_t n_tris = 0, n_edges = 0, n_obs = 0;
    // the directed loop edges and their trees, built on the first surface-semantics sweep
    std::mutex loop_mu;
    bool loop_built = false;
    SceneDev dev_loop{};  // dev with the edge fields pointing at the loop-edge trees
    GroupedBvh loop;
    DevBuf loop_edges, loop_wide, loop_cut;
    uint32_t n_loop = 0;
};

// Host threads of the plain path: worker i runs the frames handed to it on
// stream i (the upstream ThreadPool, RTCD/CollisionDetector/threadPool.h:
// 10-92, one task per frame).  run() hands each worker its job for one
// group and returns when all have finished.
struct PlainPool {
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv, cv_done;
    std::vector<std::function<void()>> jobs;
    uint64_t generation = 0;
    size_t pending = 0;
    bool stop = false;
    std::exception_ptr error;

    explicit PlainPool(size_t n) : jobs(n) {
        for (size_t i = 0; i < n; ++i) threads.emplace_back([this, i] { work(i); });
    }
    ~PlainPool() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
        for (auto& t : threads) t.join();
    }
    void work(size_t i) {
        uint64_t seen = 0;
        while (true) {
            std::function<void()> job;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || (generation != seen && jobs[i]); });
                if (stop) return;
                seen = generation;
                job.swap(jobs[i]);
            }
            std::exception_ptr ep;
            try {
                job();
            } catch (...) {
                ep = std::current_exception();
            }
            std::lock_guard<std::mutex> lk(mu);
            if (ep && !error) error = ep;
            if (--pending == 0) cv_done.notify_all();
        }
    }
    // jobs_in[i] (empty: worker i idles this group)
    void run(std::vector<std::function<void()>>& jobs_in) {
        {
            std::lock_guard<std::mutex> lk(mu);
            pending = 0;
            for (size_t i = 0; i < jobs.size(); ++i)
                if (jobs_in[i]) {
                    jobs[i] = std::move(jobs_in[i]);
                    ++pending;
                }
            ++generation;
            error = nullptr;
        }
        cv.notify_all();
        std::unique_lock<std::mutex> lk(mu);
        cv_done.wait(lk, [&] { return pending == 0; });
        if (error) std::rethrow_exception(error);
    }
};

struct rtcd_detector {
    rtcd_ctx* ctx = nullptr;
    rtcd_detector_kind kind = RTCD_OBS_TO_ROBOT;
    rtcd_robot* robot = nullptr;
    rtcd_scene* scene = nullptr;
    rtcd_config cfg{};
    std::mutex mu;
    cudaStream_t stream = nullptr;
    cudaEvent_t staged = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // stage timing: start, prepared, culled, traversed
    cudaEvent_t ev_end = nullptr;
    cudaEvent_t ev_first = nullptr;      // after the first traversal kernel (RTCD_CHECK_TIMING)
    bool timed = false;
    cudaStream_t last_stream = nullptr;  // stream of the last check (stats read on it)
    cudaGraph_t graph = nullptr;         // captured launch sequence (RTCD_CHECK_GRAPH)
    cudaGraphExec_t graph_exec = nullptr;
    uint64_t graph_key[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool timed_total_only = false;       // the last check timed only ev[0] -> ev_end (graph path)
    uint32_t blocks = 0;
    // discrete workspace
    DevBuf q, T, mask, items, count, pose_hit, counts, edge_bits, flags, seg_flags, work, err, stats, contain;
    DevBuf cand, item_overflow, overflow_items, wave_counts, sub;  // wavefront traversal
    uint32_t blocks_a = 0, blocks_b = 0, blocks_a_full = 0;
    uint32_t threads = 128;  // traversal launch shape (stage B / sweep kernel)
    ScanScratch scan;
    // sweep workspace
    DevBuf centers, ctrl, aux, piece_hit, W, W_off, heavy, split;
    DevBuf edge_q, edge_pose_flags;  // edge checks: interpolated configurations, per-configuration flags
    std::vector<uint32_t> edge_off;
    std::vector<float> W_host;
    std::vector<uint32_t> W_off_host;
    uint32_t W_max = 0;
    HostBuf pin_in, pin_out, pin_aux;
    DevBuf hq, hflags, hseg, hcounts;  // device sides of a graph replay with host buffers
    uint64_t last_items = 0, last_culled = 0;
    uint32_t last_path_flags = 0;  // rtcd_stats.path_flags of the last check
    // plain path: one clone of this detector per stream (own stream and workspace) and their threads
    std::vector<rtcd_detector*> plain_clones;
    std::unique_ptr<PlainPool> plain_pool;
};

namespace {
void ensure_weights(rtcd_detector* d, uint32_t max_wp);
extern const uint32_t kWeightsPrebuilt;
}  // namespace

static rtcd_status finish(const std::exception_ptr& ep) {
    try {
        std::rethrow_exception(ep);
    } catch (const Error& e) {
        g_last_error = e.msg;
        return (rtcd_status) e.status;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return RTCD_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return RTCD_ERR_INTERNAL;
    } catch (...) {
        g_last_error = "unknown error";
        return RTCD_ERR_INTERNAL;
    }
}

template <class F>
static rtcd_status guarded(F&& f) {
    try {
        g_last_error.clear();
        f();
        return RTCD_OK;
    } catch (...) {
        return finish(std::current_exception());
    }
}

#define RTCD_REQUIRE(cond, msg) \
    do {                        \
        if (!(cond)) fail(RTCD_ERR_INVALID_ARGUMENT, msg); \
    } while (0)

// Traversal launch shape from the detector config: threads per block (64, 128
// or 256) and resident blocks per SM (0 or more than fit: as many as fit).
static void apply_launch_shape(rtcd_detector* d) {
    uint32_t t = d->cfg.traverse_threads ? d->cfg.traverse_threads : 128;
    if (t != 64 && t != 128 && t != 256) fail(RTCD_ERR_INVALID_ARGUMENT, "traverse_threads must be 64, 128 or 256");
    const bool discrete = d->kind == RTCD_OBS_TO_ROBOT || d->kind == RTCD_ROBOT_TO_OBS;
    uint32_t fit = discrete ? stage_b_max_blocks_per_sm(d->kind == RTCD_ROBOT_TO_OBS, t)
                            : sweep_max_blocks_per_sm(d->kind == RTCD_QUAD_SWEEP, t);
    uint32_t per_sm = d->cfg.traverse_blocks_per_sm ? std::min(d->cfg.traverse_blocks_per_sm, fit) : fit;
    const uint32_t pct = d->cfg.residency_percent;
    if (pct > 100) fail(RTCD_ERR_INVALID_ARGUMENT, "residency_percent must be at most 100");
    if (d->cfg.stage_b_form > 4) fail(RTCD_ERR_INVALID_ARGUMENT, "stage_b_form must be 0 to 4");
    if (d->cfg.stage_b_chunk > 4096) fail(RTCD_ERR_INVALID_ARGUMENT, "stage_b_chunk must be at most 4096");
    const uint32_t sms = (uint32_t) device_sm_count();
    if (pct) per_sm = std::max(1u, per_sm * pct / 100);
    d->threads = t;
    if (discrete) {
        d->blocks_b = per_sm * sms;
        if (pct) d->blocks_a = std::max(sms, d->blocks_a_full * pct / 100);
    } else {
        d->blocks = per_sm * sms;
    }
}

struct DeviceScope {
    int prev = 0;
    explicit DeviceScope(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cuda_check(cudaSetDevice(dev), "cudaSetDevice");
    }
    ~DeviceScope() {
        int cur = 0;
        cudaGetDevice(&cur);
        if (cur != prev) cudaSetDevice(prev);
    }
};

extern "C" {

int rtcd_abi_version(void) { return RTCD_ABI_VERSION; }

rtcd_status rtcd_last_error(char* buf, size_t n) {
    if (buf && n) {
        size_t k = std::min(n - 1, g_last_error.size());
        std::memcpy(buf, g_last_error.data(), k);
        buf[k] = 0;
    }
    return RTCD_OK;
}

rtcd_status rtcd_context_create(int device, rtcd_ctx** out) {
    return guarded([&] {
        RTCD_REQUIRE(out, "out is NULL");
        *out = nullptr;
        int n = 0;
        cuda_check(cudaGetDeviceCount(&n), "cudaGetDeviceCount");
        RTCD_REQUIRE(device >= 0 && device < n, "no such CUDA device");
        DeviceScope ds(device);
        auto* c = new rtcd_ctx();
        c->device = device;
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete c;
            cuda_check(e, "cudaStreamCreate");
        }
        c->err.ensure(4);
        cuda_check(cudaMemset(c->err.p, 0, 4), "memset");
        *out = c;
    });
}

rtcd_status rtcd_context_destroy(rtcd_ctx* ctx) {
    return guarded([&] {
        if (!ctx) return;
        DeviceScope ds(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
        ctx->err.release();
        delete ctx;
    });
}

rtcd_status rtcd_robot_create(rtcd_ctx* ctx, const rtcd_robot_desc* d, rtcd_robot** out) {
    return guarded([&] {
        RTCD_REQUIRE(ctx && d && out, "NULL argument");
        *out = nullptr;
        RTCD_REQUIRE(d->dof >= 1 && d->dof <= (uint32_t) kMaxDof, "dof must be in [1, 15]");
        RTCD_REQUIRE(d->base_tf && d->cos_mask && d->sin_mask && d->one_mask, "chain masks are required");
        RTCD_REQUIRE(d->link_verts && d->link_vert_offsets && d->link_tris && d->link_tri_offsets,
                     "link meshes are required");
        DeviceScope ds(ctx->device);
        const uint32_t L = d->dof + 1;
        std::vector<uint32_t> voff(d->link_vert_offsets, d->link_vert_offsets + L + 1);
        std::vector<uint32_t> toff(d->link_tri_offsets, d->link_tri_offsets + L + 1);
        RTCD_REQUIRE(voff[0] == 0 && toff[0] == 0, "offsets must start at 0");
        for (uint32_t l = 0; l < L; ++l)
            RTCD_REQUIRE(voff[l + 1] >= voff[l] && toff[l + 1] >= toff[l], "offsets must be non-decreasing");
        for (uint32_t l = 0; l < L; ++l)
            for (uint32_t t = toff[l]; t < toff[l + 1]; ++t)
                for (int k = 0; k < 3; ++k)
                    RTCD_REQUIRE(d->link_tris[3ull * t + k] < voff[l + 1] - voff[l],
                                 "link triangle index out of range");
        std::unique_ptr<rtcd_robot> r(new rtcd_robot());
        r->ctx = ctx;
        r->dof = d->dof;
        // edges
        std::vector<uint32_t> edges, eoff(L + 1, 0);
        if (d->link_edges) {
            RTCD_REQUIRE(d->link_edge_offsets, "link_edge_offsets required with link_edges");
            eoff.assign(d->link_edge_offsets, d->link_edge_offsets + L + 1);
            RTCD_REQUIRE(eoff[0] == 0, "edge offsets must start at 0");
            for (uint32_t l = 0; l < L; ++l) RTCD_REQUIRE(eoff[l + 1] >= eoff[l], "edge offsets must be non-decreasing");
            edges.assign(d->link_edges, d->link_edges + 2ull * eoff[L]);
            for (uint32_t l = 0; l < L; ++l)
                for (uint32_t e = eoff[l]; e < eoff[l + 1]; ++e)
                    RTCD_REQUIRE(edges[2 * e] < voff[l + 1] - voff[l] && edges[2 * e + 1] < voff[l + 1] - voff[l],
                                 "link edge index out of range");
        } else {
            for (uint32_t l = 0; l < L; ++l) {
                auto e = unique_edges(d->link_tris + 3ull * toff[l], toff[l + 1] - toff[l]);
                edges.insert(edges.end(), e.begin(), e.end());
                eoff[l + 1] = (uint32_t) (edges.size() / 2);
            }
        }
        r->edge_off = eoff;
        // chain
        Chain& ch = r->dev.chain;
        std::memset(&ch, 0, sizeof(ch));
        ch.dof = (int) d->dof;
        std::memcpy(ch.base, d->base_tf, 12 * sizeof(float));
        std::memcpy(ch.cm, d->cos_mask, 12ull * d->dof * sizeof(float));
        std::memcpy(ch.sm, d->sin_mask, 12ull * d->dof * sizeof(float));
        std::memcpy(ch.om, d->one_mask, 12ull * d->dof * sizeof(float));
        r->dev.n_links = L;
        r->dev.first_link = d->skip_base ? 1 : 0;
        for (uint32_t l = 0; l < L; ++l) {  // the containment test's ray start: the link's first vertex
            const float* v = d->link_verts + 3ull * voff[l];
            r->dev.link_point[l] = voff[l + 1] > voff[l] ? make_float4(v[0], v[1], v[2], 0.f) : make_float4(0, 0, 0, 0);
        }
        // OBBs (link frames)
        for (uint32_t l = 0; l < L; ++l) {
            float* o = r->dev.obb[l];
            if (d->link_obbs) {
                std::memcpy(o, d->link_obbs + 15ull * l, 15 * sizeof(float));
                o[3] += 1e-5f; o[4] += 1e-5f; o[5] += 1e-5f;
                o[15] = std::sqrt(o[3] * o[3] + o[4] * o[4] + o[5] * o[5]);
            } else {
                std::vector<uint32_t> idx(voff[l + 1] - voff[l]);
                for (size_t k = 0; k < idx.size(); ++k) idx[k] = voff[l] + (uint32_t) k;
                fit_obb(d->link_verts, idx, 1e-5f, o);
            }
        }
        cudaStream_t s = ctx->stream;
        upload(r->verts, d->link_verts, 3ull * voff[L], s);
        upload(r->tris, d->link_tris, 3ull * toff[L], s);
        upload(r->edges, edges.data(), edges.size(), s);
        build_grouped(true, r->verts.as<float>(), voff, r->tris.as<uint32_t>(), toff, ctx->err.as<uint32_t>(), s, r->tri);
        build_grouped(false, r->verts.as<float>(), voff, r->edges.as<uint32_t>(), eoff, ctx->err.as<uint32_t>(), s,
                      r->edge);
        r->dev.tri_nodes = r->tri.nodes.as<float4>();
        r->dev.tri_prims = r->tri.prims.as<float4>();
        r->dev.edge_nodes = r->edge.nodes.as<float4>();
        r->dev.edge_prims = r->edge.prims.as<float4>();
        for (uint32_t l = 0; l < (uint32_t) kMaxLinks; ++l) {
            r->dev.tri_root[l] = l < L ? r->tri.roots[l] : kNone;
            r->dev.edge_root[l] = l < L ? r->edge.roots[l] : kNone;
        }
        r->dev.n_edges_total = eoff[L];
        // spheres
        r->dev.n_spheres = d->n_spheres;
        if (d->n_spheres) {
            RTCD_REQUIRE(d->sphere_centers && d->sphere_radii && d->sphere_links, "sphere arrays required");
            std::vector<float4> sp(d->n_spheres);
            for (uint32_t i = 0; i < d->n_spheres; ++i) {
                RTCD_REQUIRE(d->sphere_links[i] < L, "sphere link out of range");
                RTCD_REQUIRE(d->sphere_radii[i] >= 0, "negative sphere radius");
                sp[i] = make_float4(d->sphere_centers[3 * i], d->sphere_centers[3 * i + 1], d->sphere_centers[3 * i + 2],
                                    d->sphere_radii[i]);
            }
            upload(r->spheres, sp.data(), sp.size(), s);
            upload(r->sphere_link, d->sphere_links, d->n_spheres, s);
        } else {
            r->spheres.ensure(16);
            r->sphere_link.ensure(4);
        }
        r->dev.spheres = r->spheres.as<float4>();
        r->dev.sphere_link = r->sphere_link.as<uint32_t>();
        cuda_check(cudaStreamSynchronize(s), "robot upload");
        *out = r.release();
    });
}

rtcd_status rtcd_robot_destroy(rtcd_robot* r) {
    return guarded([&] {
        if (!r) return;
        DeviceScope ds(r->ctx->device);
        cudaStreamSynchronize(r->ctx->stream);
        delete r;
    });
}

rtcd_status rtcd_scene_create(rtcd_ctx* ctx, const float* verts, uint32_t n_verts, const uint32_t* tris, uint32_t n_tris,
                              const uint32_t* obstacle_tri_offsets, uint32_t n_obstacles, rtcd_scene** out) {
    return guarded([&] {
        RTCD_REQUIRE(ctx && out, "NULL argument");
        *out = nullptr;
        RTCD_REQUIRE(n_tris == 0 || (verts && tris), "vertex and triangle arrays required");
        for (size_t i = 0; i < 3ull * n_tris; ++i) RTCD_REQUIRE(tris[i] < n_verts, "triangle index out of range");
        std::vector<uint32_t> off;
        if (obstacle_tri_offsets && n_obstacles) {
            off.assign(obstacle_tri_offsets, obstacle_tri_offsets + n_obstacles + 1);
            RTCD_REQUIRE(off[0] == 0 && off.back() == n_tris, "obstacle offsets must span [0, n_tris]");
            for (uint32_t i = 0; i < n_obstacles; ++i) RTCD_REQUIRE(off[i + 1] >= off[i], "obstacle offsets decrease");
        } else {
            off = {0, n_tris};
        }
        DeviceScope ds(ctx->device);
        std::unique_ptr<rtcd_scene> sc(new rtcd_scene());
        sc->ctx = ctx;
        auto edges = unique_edges(tris, n_tris);
        sc->n_tris = n_tris;
        sc->n_edges = (uint32_t) (edges.size() / 2);
        // obstacle OBBs
        uint32_t nob = (uint32_t) off.size() - 1;
        std::vector<float> obbs(16ull * nob);
        for (uint32_t o = 0; o < nob; ++o) {
            std::vector<uint32_t> idx;
            idx.reserve(3ull * (off[o + 1] - off[o]));
            for (uint32_t t = off[o]; t < off[o + 1]; ++t)
                for (int k = 0; k < 3; ++k) idx.push_back(tris[3ull * t + k]);
            std::sort(idx.begin(), idx.end());
            idx.erase(std::unique(idx.begin(), idx.end()), idx.end());
            fit_obb(verts, idx, 1e-5f, obbs.data() + 16ull * o);
        }
        sc->n_obs = nob;
        // per obstacle: the exact box of its vertices and one of its vertices (the
        // containment test's ray start); per triangle: its obstacle
        std::vector<uint32_t> tri_obs(std::max<uint32_t>(n_tris, 1), 0);
        std::vector<float> obs_box(8ull * std::max<uint32_t>(nob, 1), 0.f), obs_point(4ull * std::max<uint32_t>(nob, 1), 0.f);
        for (uint32_t o = 0; o < nob; ++o) {
            float lo[3] = {3e38f, 3e38f, 3e38f}, hi[3] = {-3e38f, -3e38f, -3e38f};
            for (uint32_t t = off[o]; t < off[o + 1]; ++t) {
                tri_obs[t] = o;
                for (int k = 0; k < 3; ++k)
                    for (int a = 0; a < 3; ++a) {
                        const float v = verts[3ull * tris[3ull * t + k] + a];
                        lo[a] = std::min(lo[a], v);
                        hi[a] = std::max(hi[a], v);
                    }
            }
            for (int a = 0; a < 3; ++a) {
                obs_box[8ull * o + a] = lo[a];
                obs_box[8ull * o + 4 + a] = hi[a];
            }
            if (off[o + 1] > off[o])
                for (int a = 0; a < 3; ++a) obs_point[4ull * o + a] = verts[3ull * tris[3ull * off[o]] + a];
        }
        cudaStream_t s = ctx->stream;
        upload(sc->verts, verts, 3ull * n_verts, s);
        upload(sc->tris, tris, 3ull * n_tris, s);
        upload(sc->edges, edges.data(), edges.size(), s);
        upload(sc->obbs, obbs.data(), obbs.size(), s);
        upload(sc->tri_obs, tri_obs.data(), tri_obs.size(), s);
        upload(sc->obs_box, obs_box.data(), obs_box.size(), s);
        upload(sc->obs_point, obs_point.data(), obs_point.size(), s);
        std::vector<uint32_t> v0 = {0, 0};
        std::vector<uint32_t> toff = {0, n_tris}, eoff = {0, sc->n_edges};
        build_grouped(true, sc->verts.as<float>(), v0, sc->tris.as<uint32_t>(), toff, ctx->err.as<uint32_t>(), s, sc->tri,
                      sc->tri_obs.as<uint32_t>());
        build_grouped(false, sc->verts.as<float>(), v0, sc->edges.as<uint32_t>(), eoff, ctx->err.as<uint32_t>(), s,
                      sc->edge);
        const auto node_count = [](uint32_t n) { return n > 1 ? n - 1 : 0u; };
        const WideResult wt = build_wide(sc->tri.nodes.as<float4>(), node_count(n_tris), sc->tri.roots[0], sc->tri_wide, s);
        const WideResult we =
            build_wide(sc->edge.nodes.as<float4>(), node_count(sc->n_edges), sc->edge.roots[0], sc->edge_wide, s);
        SceneDev& dv = sc->dev;
        dv.tri_wide = sc->tri_wide.as<float4>();
        dv.tri_wide_root = wt.root;
        dv.edge_wide = sc->edge_wide.as<float4>();
        dv.edge_wide_root = we.root;
        dv.wide_front = wide_frontier(std::max(wt.depth, we.depth));
        upload(sc->tri_cut, wt.cut.data(), wt.cut.size(), s);
        upload(sc->edge_cut, we.cut.data(), we.cut.size(), s);
        dv.tri_cut = sc->tri_cut.as<float4>();
        dv.edge_cut = sc->edge_cut.as<float4>();
        dv.n_tri_cut = (uint32_t) wt.cut.size() / 2;
        dv.n_tri_wide = wt.nodes;
        dv.n_edge_wide = we.nodes;
        dv.n_edge_cut = (uint32_t) we.cut.size() / 2;
        // a depth-first lane descent keeps at most 3 siblings per level plus the last node's 4 children
        dv.edge_wide_lane = (kWide - 1) * we.depth + kWide <= (uint32_t) kStack ? 1u : 0u;
        dv.tri_nodes = sc->tri.nodes.as<float4>();
        dv.tri_prims = sc->tri.prims.as<float4>();
        dv.tri_root = sc->tri.roots[0];
        dv.n_tris = n_tris;
        dv.edge_nodes = sc->edge.nodes.as<float4>();
        dv.edge_prims = sc->edge.prims.as<float4>();
        dv.edge_root = sc->edge.roots[0];
        dv.n_edges = sc->n_edges;
        dv.obbs = sc->obbs.as<float>();
        dv.obs_box = sc->obs_box.as<float4>();
        dv.obs_point = sc->obs_point.as<float4>();
        dv.n_obs = nob;
        cuda_check(cudaStreamSynchronize(s), "scene upload");
        *out = sc.release();
    });
}

rtcd_status rtcd_scene_destroy(rtcd_scene* sc) {
    return guarded([&] {
        if (!sc) return;
        DeviceScope ds(sc->ctx->device);
        cudaStreamSynchronize(sc->ctx->stream);
        delete sc;
    });
}

rtcd_status rtcd_scene_info(const rtcd_scene* sc, uint32_t* n_tris, uint32_t* n_edges, uint32_t* n_obstacles) {
    return guarded([&] {
        RTCD_REQUIRE(sc, "NULL scene");
        if (n_tris) *n_tris = sc->n_tris;
        if (n_edges) *n_edges = sc->n_edges;
        if (n_obstacles) *n_obstacles = sc->n_obs;
    });
}

rtcd_status rtcd_loop_edges(const uint32_t* tris, uint32_t n_tris, uint32_t* edges_out, uint32_t max_edges,
                            uint32_t* n_edges) {
    return guarded([&] {
        RTCD_REQUIRE(n_edges && (n_tris == 0 || tris), "NULL argument");
        const std::vector<uint32_t> e = loop_edges(tris, n_tris);
        *n_edges = (uint32_t) (e.size() / 2);
        if (!edges_out) return;
        RTCD_REQUIRE(e.size() / 2 <= max_edges, "edges_out too small");
        std::copy(e.begin(), e.end(), edges_out);
    });
}

rtcd_status rtcd_detector_create(rtcd_ctx* ctx, rtcd_detector_kind kind, rtcd_robot* robot, rtcd_scene* scene,
                                 const rtcd_config* config, rtcd_detector** out) {
    return guarded([&] {
        RTCD_REQUIRE(ctx && robot && scene && out, "NULL argument");
        *out = nullptr;
        RTCD_REQUIRE(kind >= RTCD_OBS_TO_ROBOT && kind <= RTCD_QUAD_SWEEP, "unknown detector kind");
        RTCD_REQUIRE(robot->ctx == ctx && scene->ctx == ctx, "robot and scene must belong to the context");
        if (kind == RTCD_LINEAR_SWEEP || kind == RTCD_QUAD_SWEEP)
            RTCD_REQUIRE(robot->dev.n_spheres > 0, "sweep detectors need a sphere model");
        DeviceScope ds(ctx->device);
        std::unique_ptr<rtcd_detector> d(new rtcd_detector());
        d->ctx = ctx;
        d->kind = kind;
        d->robot = robot;
        d->scene = scene;
        if (config) d->cfg = *config;
        if (!d->cfg.frame_size) d->cfg.frame_size = 1024;
        if (!d->cfg.plain_streams) d->cfg.plain_streams = 4;
        RTCD_REQUIRE(d->cfg.plain_streams <= 16, "plain_streams must be at most 16");
        RTCD_REQUIRE(d->cfg.top_nodes_shared <= 256, "top_nodes_shared must be at most 256");
        int lo_prio = 0, hi_prio = 0;
        cuda_check(cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio), "cudaDeviceGetStreamPriorityRange");
        const int prio = std::min(lo_prio, std::max(hi_prio, (int) d->cfg.stream_priority));
        cuda_check(cudaStreamCreateWithPriority(&d->stream, cudaStreamNonBlocking, prio), "cudaStreamCreate");
        cuda_check(cudaEventCreateWithFlags(&d->staged, cudaEventDisableTiming), "cudaEventCreate");
        for (auto& e : d->ev) cuda_check(cudaEventCreate(&e), "cudaEventCreate");
        cuda_check(cudaEventCreate(&d->ev_end), "cudaEventCreate");
        cuda_check(cudaEventCreate(&d->ev_first), "cudaEventCreate");
        if (kind == RTCD_OBS_TO_ROBOT || kind == RTCD_ROBOT_TO_OBS) {
            d->blocks = discrete_persistent_blocks(kind == RTCD_ROBOT_TO_OBS);
            d->blocks_a = d->blocks_a_full = stage_a_blocks(kind == RTCD_ROBOT_TO_OBS);
        }
        apply_launch_shape(d.get());
        d->err.ensure(4);
        d->stats.ensure(8 * kStatWords);
        d->work.ensure(32);  // [0] work counter, [1] heavy units appended, [2] heavy-pass counter, [3..4] split pass
        d->count.ensure(4);
        cuda_check(cudaMemset(d->err.p, 0, 4), "memset");
        cuda_check(cudaMemset(d->stats.p, 0, 8 * kStatWords), "memset");
        if (kind == RTCD_QUAD_SWEEP) ensure_weights(d.get(), kWeightsPrebuilt);
        *out = d.release();
    });
}

}  // extern "C"

namespace rtcd {
void detector_info(rtcd_detector* d, rtcd_ctx** ctx, int* kind, rtcd_robot** robot, rtcd_scene** scene,
                   rtcd_config* cfg, uint32_t* n_links, uint32_t* n_spheres, uint32_t* dof) {
    *ctx = d->ctx;
    *kind = (int) d->kind;
    *robot = d->robot;
    *scene = d->scene;
    *cfg = d->cfg;
    *n_links = d->robot->dev.n_links;
    *n_spheres = d->robot->dev.n_spheres;
    *dof = d->robot->dof;
}
}  // namespace rtcd

extern "C" {

rtcd_status rtcd_detector_destroy(rtcd_detector* d) {
    return guarded([&] {
        if (!d) return;
        DeviceScope ds(d->ctx->device);
        cudaStreamSynchronize(d->stream);
        d->plain_pool.reset();
        for (rtcd_detector* c : d->plain_clones) rtcd_detector_destroy(c);
        if (d->graph_exec) cudaGraphExecDestroy(d->graph_exec);
        if (d->graph) cudaGraphDestroy(d->graph);
        cudaEventDestroy(d->staged);
        for (auto& e : d->ev) cudaEventDestroy(e);
        cudaEventDestroy(d->ev_end);
        cudaEventDestroy(d->ev_first);
        cudaStreamDestroy(d->stream);
        delete d;
    });
}

}  // extern "C"

// ---------------------------------------------------------------- query paths
namespace {

uint32_t quad_ctrl_count(uint32_t n_wp) { return std::max<uint32_t>(3, (n_wp + 1) / 2); }

// The scene as the surface-semantics sweeps see it: the edge trees replaced
// by trees over the directed loop edges, built on first use (the triangles
// are read back from the device, the loop edges computed on the host, both
// trees built on the scene's context stream; synchronous, once per scene).
const SceneDev& scene_loop(rtcd_scene* sc) {
    std::lock_guard<std::mutex> lk(sc->loop_mu);
    if (sc->loop_built) return sc->dev_loop;
    cudaStream_t s = sc->ctx->stream;
    std::vector<uint32_t> tris(3ull * sc->n_tris);
    if (sc->n_tris)
        cuda_check(cudaMemcpyAsync(tris.data(), sc->tris.p, 4ull * tris.size(), cudaMemcpyDeviceToHost, s), "tris");
    cuda_check(cudaStreamSynchronize(s), "tris");
    const std::vector<uint32_t> e = loop_edges(tris.data(), sc->n_tris);
    sc->n_loop = (uint32_t) (e.size() / 2);
    upload(sc->loop_edges, e.data(), e.size(), s);
    const std::vector<uint32_t> v0 = {0, 0}, off = {0, sc->n_loop};
    build_grouped(false, sc->verts.as<float>(), v0, sc->loop_edges.as<uint32_t>(), off, sc->ctx->err.as<uint32_t>(), s,
                  sc->loop);
    const WideResult w =
        build_wide(sc->loop.nodes.as<float4>(), sc->n_loop > 1 ? sc->n_loop - 1 : 0, sc->loop.roots[0], sc->loop_wide, s);
    upload(sc->loop_cut, w.cut.data(), w.cut.size(), s);
    SceneDev dv = sc->dev;
    dv.edge_nodes = sc->loop.nodes.as<float4>();
    dv.edge_prims = sc->loop.prims.as<float4>();
    dv.edge_root = sc->loop.roots[0];
    dv.n_edges = sc->n_loop;
    dv.edge_wide = sc->loop_wide.as<float4>();
    dv.edge_wide_root = w.root;
    dv.edge_cut = sc->loop_cut.as<float4>();
    dv.n_edge_cut = (uint32_t) w.cut.size() / 2;
    dv.n_edge_wide = w.nodes;
    dv.edge_wide_lane = (kWide - 1) * w.depth + kWide <= (uint32_t) kStack ? 1u : 0u;
    dv.wide_front = std::max(dv.wide_front, wide_frontier(w.depth));
    cuda_check(cudaStreamSynchronize(s), "loop-edge trees");
    sc->dev_loop = dv;
    sc->loop_built = true;
    return sc->dev_loop;
}

uint32_t pieces_of(rtcd_detector_kind kind, uint32_t n_wp, uint32_t flags) {
    if (kind == RTCD_LINEAR_SWEEP) return n_wp > 0 ? n_wp - 1 : 0;
    return quad_ctrl_count(n_wp) - 2 + ((flags & (RTCD_CHECK_NO_ENDPOINTS | RTCD_CHECK_SURFACE)) ? 0 : 2);
}

// Least-squares quadratic B-spline fit W = (B^T B)^{-1} B^T (nc x nt), with B
// the uniform unclamped quadratic basis sampled at u = linspace(2, nc, nt);
// the shipped weight tables (RTCD/data/weights/quad/normal/) are this matrix.
// Each row of B has three consecutive nonzeros, so G = B^T B is pentadiagonal
// and its Cholesky factor has two subdiagonals: the factor and the nt solves
// touch only the band (the entries a dense factorisation would compute outside
// it are exact zeros, so the result is the same).
std::vector<double> fit_weights(uint32_t nc, uint32_t nt) {
    constexpr uint32_t kBand = 2;
    std::vector<double> B((size_t) nt * nc, 0.0), W((size_t) nc * nt, 0.0);
    for (uint32_t t = 0; t < nt; ++t) {
        double x = nt > 1 ? 2.0 + (double) (nc - 2) * t / (nt - 1) : 2.0;
        int seg = std::min<int>((int) std::floor(x) - 2, (int) nc - 3);
        seg = std::max(seg, 0);
        double s = x - (seg + 2);
        B[(size_t) t * nc + seg] += 0.5 * (1 - s) * (1 - s);
        B[(size_t) t * nc + seg + 1] += 0.5 + s - s * s;
        B[(size_t) t * nc + seg + 2] += 0.5 * s * s;
    }
    // L[i][i - k], k = 0..2, in G's band
    std::vector<double> L((size_t) nc * (kBand + 1), 0.0);
    auto Lr = [&](uint32_t i, uint32_t j) -> double& { return L[(size_t) i * (kBand + 1) + (i - j)]; };
    for (uint32_t i = 0; i < nc; ++i)
        for (uint32_t j = (i >= kBand ? i - kBand : 0); j <= i; ++j) {
            double acc = 0;
            for (uint32_t t = 0; t < nt; ++t) acc += B[(size_t) t * nc + i] * B[(size_t) t * nc + j];
            Lr(i, j) = acc;
        }
    for (uint32_t j = 0; j < nc; ++j) {
        double dg = Lr(j, j);
        for (uint32_t k = (j >= kBand ? j - kBand : 0); k < j; ++k) dg -= Lr(j, k) * Lr(j, k);
        if (dg <= 0) fail(RTCD_ERR_INVALID_ARGUMENT, "spline fit is singular");
        dg = std::sqrt(dg);
        Lr(j, j) = dg;
        for (uint32_t i = j + 1; i < nc && i <= j + kBand; ++i) {
            double v = Lr(i, j);
            for (uint32_t k = (i >= kBand ? i - kBand : 0); k < j; ++k) v -= Lr(i, k) * Lr(j, k);
            Lr(i, j) = v / dg;
        }
    }
    std::vector<double> y(nc);
    for (uint32_t t = 0; t < nt; ++t) {
        for (uint32_t i = 0; i < nc; ++i) {
            double v = B[(size_t) t * nc + i];
            for (uint32_t k = (i >= kBand ? i - kBand : 0); k < i; ++k) v -= Lr(i, k) * y[k];
            y[i] = v / Lr(i, i);
        }
        for (int i = (int) nc - 1; i >= 0; --i) {
            double v = y[i];
            for (uint32_t k = i + 1; k < nc && k <= (uint32_t) i + kBand; ++k) v -= Lr(k, i) * y[k];
            y[i] = v / Lr(i, i);
        }
        for (uint32_t i = 0; i < nc; ++i) W[(size_t) i * nt + t] = y[i];
    }
    return W;
}

// Process-wide cache of the FP32 tables by waypoint count (they depend on n only).
const std::vector<float>& weight_table(uint32_t n) {
    static std::mutex mu;
    static std::map<uint32_t, std::vector<float>> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(n);
    if (it != cache.end()) return it->second;
    std::vector<float> f;
    if (n >= 3) {
        auto W = fit_weights(quad_ctrl_count(n), n);
        f.assign(W.begin(), W.end());
    }
    return cache.emplace(n, std::move(f)).first->second;
}

// Tables for every waypoint count up to max_wp on the device.  Growth is
// geometric (the stream is synchronised before the buffer is replaced), and
// detectors start with tables up to kWeightsPrebuilt waypoints.
extern const uint32_t kWeightsPrebuilt = 128;

void ensure_weights(rtcd_detector* d, uint32_t max_wp) {
    if (max_wp <= d->W_max) return;
    max_wp = std::max(max_wp, d->W_max + d->W_max / 2);
    if (d->W_off_host.empty()) d->W_off_host.assign(1, 0);
    d->W_off_host.resize(max_wp + 2, 0);
    for (uint32_t n = d->W_max + 1; n <= max_wp; ++n) {
        d->W_off_host[n] = (uint32_t) d->W_host.size();
        const std::vector<float>& w = weight_table(n);
        d->W_host.insert(d->W_host.end(), w.begin(), w.end());
    }
    d->W_max = max_wp;
    cuda_check(cudaStreamSynchronize(d->stream), "weights sync");
    upload(d->W, d->W_host.data(), std::max<size_t>(d->W_host.size(), 1), d->stream);
    upload(d->W_off, d->W_off_host.data(), d->W_off_host.size(), d->stream);
    cuda_check(cudaStreamSynchronize(d->stream), "weights upload");
}

// True when p is page-locked host memory (cudaHostAlloc, cudaMallocHost,
// cudaHostRegister): the upload then reads it by DMA directly instead of
// copying it into the detector's pinned staging first.
static bool host_pinned(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

void check_device_errors(rtcd_detector* d, cudaStream_t s) {
    uint32_t e = 0;
    cuda_check(cudaMemcpyAsync(&e, d->err.p, 4, cudaMemcpyDeviceToHost, s), "error readback");
    cuda_check(cudaStreamSynchronize(s), "sync");
    if (e) {
        cudaMemsetAsync(d->err.p, 0, 4, s);
        cudaStreamSynchronize(s);
        if (e & kErrLookback) fail(RTCD_ERR_DEVICE_TIMEOUT, "device look-back wait ran out");
        if (e & kErrStack) fail(RTCD_ERR_CAPACITY, "traversal stack overflow");
        fail(RTCD_ERR_INTERNAL, "device range check failed");
    }
}

// One discrete pass over poses [0, n) of d_q.  When `plain`, the item count
// is read back and the traversal grid sized to it (the upstream shape).
// The traversal of one direction over the items of the current pass.
// The first kernel counts into stats bank 0 (and is followed by ev_first,
// when given), the later passes into bank 1.
static void traverse(rtcd_detector* d, bool r2o, const DiscreteArgs& A, uint32_t n, bool plain, uint32_t blocks,
                     uint32_t flags, cudaStream_t s, cudaEvent_t ev_first) {
    RobotDev& R = d->robot->dev;
    const uint32_t L = R.n_links;
    cuda_check(cudaMemsetAsync(d->work.p, 0, 8, s), "memset");
    if (flags & RTCD_CHECK_FUSED) {
        launch_discrete(r2o, R, d->scene->dev, A, blocks, s);
        if (ev_first) cuda_check(cudaEventRecord(ev_first, s), "event");
        return;
    }
    // stage A (+ B) -> heavy pass -> the thread-per-item kernel over items whose candidates overflowed
    const size_t items_max = (size_t) n * L;
    const uint32_t cap = (uint32_t) std::min<size_t>(std::max<size_t>(items_max * 128, 1u << 16), 1u << 26);
    d->cand.ensure(8ull * cap);
    d->item_overflow.ensure(items_max + 4);  // marked a word at a time
    d->overflow_items.ensure(4ull * items_max);
    d->wave_counts.ensure(8 * 4);
    cuda_check(cudaMemsetAsync(d->item_overflow.p, 0, items_max + 4, s), "memset");
    cuda_check(cudaMemsetAsync(d->wave_counts.p, 0, 32, s), "memset");
    // [0] candidates, [1] overflowed items, [2] fallback work, [3] heavy, [4..7] subtree pass
    uint32_t* wc = d->wave_counts.as<uint32_t>();
    WaveArgs W{};
    W.d = A;
    W.top_nodes = d->cfg.top_nodes_shared;
    W.cand = d->cand.as<uint2>();
    W.cand_count = wc;
    W.cand_cap = cap;
    W.item_overflow = d->item_overflow.as<uint8_t>();
    W.overflow_items = d->overflow_items.as<uint32_t>();
    W.overflow_count = wc + 1;
    const bool fused_form = d->cfg.stage_b_form == 0 || d->cfg.stage_b_form >= 3;
    // lanes / packets: the chunk; fused forms: stage_b_chunk is the item's stage-B step budget
    W.chunk = (!fused_form && d->cfg.stage_b_chunk) ? d->cfg.stage_b_chunk : (d->cfg.stage_b_form == 2 ? 4u : 64u);
    W.item_steps = fused_form ? (d->cfg.stage_b_chunk ? d->cfg.stage_b_chunk : 8u) : 0xFFFFFFFFu;
    W.light_steps = d->cfg.light_steps == 0xFFFFFFFFu ? 0u
                    : d->cfg.light_steps                ? d->cfg.light_steps
                                                              : 32u;
    if (W.light_steps) {
        const uint32_t hcap = std::min<uint32_t>(cap, 1u << 24);
        d->heavy.ensure(8ull * hcap);
        W.heavy = d->heavy.as<uint2>();
        W.heavy_cap = hcap;
        W.heavy_count = wc + 3;
        W.heavy_work = d->work.as<uint32_t>() + 1;
    }
    if (fused_form) {
        const uint32_t scap = (uint32_t) std::min<size_t>(std::max<size_t>(items_max * 8, 1u << 16), 1u << 24);
        d->sub.ensure(2 * 8ull * scap);
        W.sub = d->sub.as<uint2>();
        W.sub_cap = scap;
        W.sub_count = wc + 4;
    }
    uint32_t ba = plain ? std::max<uint32_t>(1, blocks * kTravThreads / (kStageAWarps * 32)) : d->blocks_a;
    const uint32_t share = d->cfg.residency_percent ? d->cfg.residency_percent : 100;
    WaveArgs W1 = W;  // the later passes count into bank 1
    W1.d.stats = A.stats + kStatBank;
    if (fused_form) {
        const bool packets = d->cfg.stage_b_form == 4;
        const uint32_t full = stage_ab_blocks(r2o, packets, d->scene->dev);
        launch_stage_ab(r2o, packets, R, d->scene->dev, W, plain ? std::min(ba, full) : std::max(1u, full * share / 100),
                        s);
        if (ev_first) cuda_check(cudaEventRecord(ev_first, s), "event");
        // the rest of the crowded items' descents, the one-lane pass over the candidates they
        // deferred, then the heavy pass
        launch_subtree(r2o, R, d->scene->dev, W1, share, s);
        launch_stage_b(r2o, R, d->scene->dev, W1, d->blocks_b, d->threads, share, false, s);
    } else {
        launch_stage_a(r2o, R, d->scene->dev, W, std::min(ba, d->blocks_a), s);
        if (ev_first) cuda_check(cudaEventRecord(ev_first, s), "event");
        launch_stage_b(r2o, R, d->scene->dev, W1, d->blocks_b, d->threads, share, d->cfg.stage_b_form == 2, s);
    }
    DiscreteArgs F = A;
    F.stats = A.stats + kStatBank;
    F.items = d->overflow_items.as<uint32_t>();  // item words
    F.link_major = 0;
    F.n_items = wc + 1;
    F.work_counter = wc + 2;
    launch_discrete(r2o, R, d->scene->dev, F, d->blocks, s);
}

// One discrete pass over poses [0, n) of d_q.  When `plain`, the item count
// is read back and the traversal grid sized to it (the upstream shape).  With
// RTCD_CHECK_TWO_WAY both directions run over the same items (ObsToRobot
// first, so RobotToObs skips the poses it decided; with counts RobotToObs
// first, its edge counts then ObsToRobot's hits added); with
// RTCD_CHECK_CONTAINMENT the containment test runs over the poses left.
void discrete_pass(rtcd_detector* d, const float* d_q, uint32_t n, uint32_t* d_hit, uint32_t* d_counts,
                   uint32_t* d_bits, uint32_t* d_contain, uint32_t flags, bool plain, cudaStream_t s) {
    RobotDev& R = d->robot->dev;
    const uint32_t L = R.n_links;
    const bool counts = (flags & RTCD_CHECK_COUNTS) != 0;
    const bool two_way = (flags & RTCD_CHECK_TWO_WAY) != 0;
    d->T.ensure(48ull * n * L);
    d->mask.ensure((size_t) n * L);
    d->items.ensure(4ull * n * L);
    const bool timed = (flags & RTCD_CHECK_TIMING) && !plain;
    if (timed) cuda_check(cudaEventRecord(d->ev[0], s), "event");
    launch_fk_poses(R.chain, d_q, n, d->T.as<float4>(), s);
    if (timed) cuda_check(cudaEventRecord(d->ev[1], s), "event");
    if (flags & RTCD_CHECK_NO_CULL) {
        launch_all_items(R, n, d->items.as<uint32_t>(), d->count.as<uint32_t>(), s);
    } else {
        launch_cull(R, d->scene->dev, d->T.as<float4>(), n, d->mask.as<uint8_t>(), true, d->stats.as<unsigned long long>(),
                    s);
        select_u8(d->mask.as<uint8_t>(), n * L, d->items.as<uint32_t>(), d->count.as<uint32_t>(), d->scan,
                  d->err.as<uint32_t>(), s);
    }
    uint32_t blocks = d->blocks;
    if (plain) {
        uint32_t cnt = 0;
        cuda_check(cudaMemcpyAsync(&cnt, d->count.p, 4, cudaMemcpyDeviceToHost, s), "count readback");
        cuda_check(cudaStreamSynchronize(s), "frame sync");
        d->last_items += cnt;
        if (!cnt) return;
        blocks = (cnt + kTravThreads - 1) / kTravThreads;
    }
    DiscreteArgs A{};
    A.T = d->T.as<float4>();
    A.items = d->items.as<uint32_t>();
    A.link_major = 1u;
    A.n_items = d->count.as<uint32_t>();
    A.n_poses = n;
    A.pose_hit = d_hit;
    A.edge_words = (R.n_edges_total + 31) / 32;
    A.work_counter = d->work.as<uint32_t>();
    A.err = d->err.as<uint32_t>();
    A.stats = d->stats.as<unsigned long long>();
    A.want_counts = counts ? 1 : 0;
    if (timed) cuda_check(cudaEventRecord(d->ev[2], s), "event");
    const bool own_r2o = d->kind == RTCD_ROBOT_TO_OBS;
    // the directions to run, in order
    bool dirs[2] = {own_r2o, !own_r2o};
    int n_dirs = 1;
    if (two_way) {
        n_dirs = 2;
        dirs[0] = counts;  // counts: RobotToObs first (its popcount writes the counts), else ObsToRobot first
        dirs[1] = !counts;
    }
    for (int k = 0; k < n_dirs; ++k) {
        const bool r2o = dirs[k];
        DiscreteArgs Ad = A;
        Ad.counts = (counts && !r2o) ? d_counts : nullptr;
        Ad.edge_bits = (counts && r2o) ? d_bits : nullptr;
        traverse(d, r2o, Ad, n, plain, blocks, flags, s, timed && k == 0 ? d->ev_first : nullptr);
        if (counts && r2o) launch_popcount_rows(d_bits, A.edge_words, n, d_counts, s);
    }
    if (d_contain) launch_contain(R, d->scene->dev, A, d_contain, s);
    if (timed) cuda_check(cudaEventRecord(d->ev[3], s), "event");
    d->timed = timed;
}

void check_discrete(rtcd_detector* d, const float* q, uint32_t n, uint8_t* flags_out, uint32_t* counts_out,
                    uint32_t flags, cudaStream_t s) {
    const bool host = (flags & RTCD_CHECK_HOST_BUFFERS) != 0;
    const bool counts = (flags & RTCD_CHECK_COUNTS) != 0;
    const uint32_t dof = d->robot->dof;
    RobotDev& R = d->robot->dev;
    const float* d_q = q;
    if (host) {
        d->q.ensure(4ull * n * dof);
        const void* src = q;
        if (!host_pinned(q)) {
            d->pin_in.ensure(4ull * n * dof);
            std::memcpy(d->pin_in.p, q, 4ull * n * dof);
            src = d->pin_in.p;
        }
        cuda_check(cudaMemcpyAsync(d->q.p, src, 4ull * n * dof, cudaMemcpyHostToDevice, s), "q upload");
        d_q = d->q.as<float>();
    }
    d->pose_hit.ensure(4ull * n);
    cuda_check(cudaMemsetAsync(d->pose_hit.p, 0, 4ull * n, s), "memset");
    uint32_t* d_counts = nullptr;
    uint32_t* d_bits = nullptr;
    uint32_t words = (R.n_edges_total + 31) / 32;
    if (counts) {
        if (host || !counts_out) {
            d->counts.ensure(4ull * n);
            d_counts = d->counts.as<uint32_t>();
        } else {
            d_counts = counts_out;
        }
        cuda_check(cudaMemsetAsync(d_counts, 0, 4ull * n, s), "memset");
        if (d->kind == RTCD_ROBOT_TO_OBS || (flags & RTCD_CHECK_TWO_WAY)) {
            d->edge_bits.ensure(4ull * n * words);
            d_bits = d->edge_bits.as<uint32_t>();
            cuda_check(cudaMemsetAsync(d_bits, 0, 4ull * n * words, s), "memset");
        }
    }
    uint32_t* d_contain = nullptr;
    if (flags & RTCD_CHECK_CONTAINMENT) {
        d->contain.ensure(4ull * n);
        d_contain = d->contain.as<uint32_t>();
        cuda_check(cudaMemsetAsync(d_contain, 0, 4ull * n, s), "memset");
    }
    d->last_items = 0;
    if (flags & RTCD_CHECK_PLAIN) {
        // The upstream check() shape (RTCD/CollisionDetector/CollisionDetector.h:354-433): frames of
        // frame_size poses, frame f on stream f % plain_streams, each stream driven by its own host
        // thread; a frame reads its culled item count back to the host before its traversal (the
        // upstream compaction round trip, RTCD/Robot/batchRayRobot.h:467); after every group of
        // plain_streams frames the call waits for the group's streams.
        const uint32_t fs = d->cfg.frame_size, ns = d->cfg.plain_streams;
        if (d->plain_clones.size() != ns) {
            d->plain_pool.reset();
            for (rtcd_detector* c : d->plain_clones) rtcd_detector_destroy(c);
            d->plain_clones.clear();
            rtcd_config cc = d->cfg;
            cc.plain_streams = 1;
            for (uint32_t i = 0; i < ns; ++i) {
                rtcd_detector* c = nullptr;
                if (rtcd_detector_create(d->ctx, d->kind, d->robot, d->scene, &cc, &c) != RTCD_OK)
                    fail(RTCD_ERR_INTERNAL, "plain path: " + g_last_error);
                d->plain_clones.push_back(c);
            }
            d->plain_pool.reset(new PlainPool(ns));
        }
        cuda_check(cudaStreamSynchronize(s), "plain staging");  // inputs and cleared outputs ready
        const int dev = d->ctx->device;
        for (uint32_t start = 0; start < n; start += fs * ns) {
            std::vector<std::function<void()>> jobs(ns);
            for (uint32_t i = 0; i < ns && start + i * fs < n; ++i) {
                const uint32_t a = start + i * fs, m = std::min(fs, n - a);
                rtcd_detector* c = d->plain_clones[i];
                jobs[i] = [=] {
                    cuda_check(cudaSetDevice(dev), "cudaSetDevice");
                    c->last_items = 0;
                    discrete_pass(c, d_q + (size_t) a * dof, m, d->pose_hit.as<uint32_t>() + a,
                                  d_counts ? d_counts + a : nullptr, d_bits ? d_bits + (size_t) a * words : nullptr,
                                  d_contain ? d_contain + a : nullptr, flags, true, c->stream);
                };
            }
            d->plain_pool->run(jobs);
            for (uint32_t i = 0; i < ns && start + i * fs < n; ++i) {
                rtcd_detector* c = d->plain_clones[i];
                check_device_errors(c, c->stream);  // waits for the frame's stream
                d->last_items += c->last_items;
            }
        }
    } else {
        discrete_pass(d, d_q, n, d->pose_hit.as<uint32_t>(), d_counts, d_bits, d_contain, flags, false, s);
    }
    uint8_t* d_flags = flags_out;
    if (host || !flags_out) {
        d->flags.ensure(n);
        d_flags = d->flags.as<uint8_t>();
    }
    launch_flags(d->pose_hit.as<uint32_t>(), n, d_flags, s, d_contain);
    if (host) {
        d->pin_out.ensure(5ull * n + 16);
        uint8_t* pf = d->pin_out.as<uint8_t>();
        uint32_t* pc = reinterpret_cast<uint32_t*>(pf + ((n + 15) & ~15u));
        cuda_check(cudaMemcpyAsync(pf, d_flags, n, cudaMemcpyDeviceToHost, s), "flags download");
        if (counts && counts_out)
            cuda_check(cudaMemcpyAsync(pc, d_counts, 4ull * n, cudaMemcpyDeviceToHost, s), "counts download");
        cuda_check(cudaStreamSynchronize(s), "check sync");
        if (flags_out) std::memcpy(flags_out, pf, n);
        if (counts && counts_out) std::memcpy(counts_out, pc, 4ull * n);
    } else if (counts && counts_out && d_counts != counts_out) {
        cuda_check(cudaMemcpyAsync(counts_out, d_counts, 4ull * n, cudaMemcpyDeviceToDevice, s), "counts copy");
    }
}

void check_sweep(rtcd_detector* d, const float* q, const uint32_t* traj_off, uint32_t n, uint8_t* flags_out,
                 uint8_t* seg_out, uint32_t* counts_out, uint32_t flags, cudaStream_t s) {
    RTCD_REQUIRE(traj_off, "traj_offsets required for sweep detectors");
    RTCD_REQUIRE(!(flags & (RTCD_CHECK_CONTAINMENT | RTCD_CHECK_TWO_WAY)),
                 "containment and two-way checks are for the discrete detectors");
    const bool host = (flags & RTCD_CHECK_HOST_BUFFERS) != 0;
    const bool counts = (flags & RTCD_CHECK_COUNTS) != 0;
    const bool quad = d->kind == RTCD_QUAD_SWEEP;
    const bool want_pieces = seg_out != nullptr;
    RobotDev& R = d->robot->dev;
    const uint32_t dof = d->robot->dof, ns = R.n_spheres;
    RTCD_REQUIRE(traj_off[0] == 0, "traj_offsets must start at 0");
    uint32_t max_wp = 0;
    uint64_t pieces = 0, ctrl_total = 0;
    for (uint32_t i = 0; i < n; ++i) {
        RTCD_REQUIRE(traj_off[i + 1] >= traj_off[i], "traj_offsets must be non-decreasing");
        uint32_t w = traj_off[i + 1] - traj_off[i];
        RTCD_REQUIRE(w >= (quad ? 3u : 2u), quad ? "quadratic trajectories need >= 3 waypoints"
                                                : "linear trajectories need >= 2 waypoints");
        max_wp = std::max(max_wp, w);
        pieces += pieces_of(d->kind, w, flags);
        if (quad) ctrl_total += quad_ctrl_count(w);
    }
    RTCD_REQUIRE(pieces * ns < (1ull << 32), "too many sweep units in one call");
    const uint32_t total_wp = traj_off[n];
    if (quad) ensure_weights(d, max_wp);
    // auxiliary tables: wp_off | piece_off | ctrl_off | piece_traj
    const size_t aux_words = 3ull * (n + 1) + pieces;
    // under graph capture the staging buffer is idle (synchronised before the
    // capture) and replays never rewrite it, so no staging event is recorded
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cuda_check(cudaStreamIsCapturing(s, &cap), "cudaStreamIsCapturing");
    const bool capturing = cap != cudaStreamCaptureStatusNone;
    if (!capturing) cuda_check(cudaEventSynchronize(d->staged), "staging reuse");
    d->pin_aux.ensure(4 * aux_words);
    uint32_t* a = d->pin_aux.as<uint32_t>();
    uint32_t* wp_off = a;
    uint32_t* piece_off = a + (n + 1);
    uint32_t* ctrl_off = a + 2 * (n + 1);
    uint32_t* piece_traj = a + 3 * (n + 1);
    wp_off[0] = piece_off[0] = ctrl_off[0] = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t w = traj_off[i + 1] - traj_off[i];
        uint32_t p = pieces_of(d->kind, w, flags);
        wp_off[i + 1] = traj_off[i + 1];
        piece_off[i + 1] = piece_off[i] + p;
        ctrl_off[i + 1] = ctrl_off[i] + (quad ? quad_ctrl_count(w) : 0);
        for (uint32_t k = 0; k < p; ++k) piece_traj[piece_off[i] + k] = i;
    }
    d->aux.ensure(4 * aux_words);
    cuda_check(cudaMemcpyAsync(d->aux.p, a, 4 * aux_words, cudaMemcpyHostToDevice, s), "aux upload");
    const float* d_q = q;
    if (host) {
        d->q.ensure(4ull * total_wp * dof);
        const void* src = q;
        if (!host_pinned(q)) {
            d->pin_in.ensure(4ull * total_wp * dof);
            std::memcpy(d->pin_in.p, q, 4ull * total_wp * dof);
            src = d->pin_in.p;
        }
        cuda_check(cudaMemcpyAsync(d->q.p, src, 4ull * total_wp * dof, cudaMemcpyHostToDevice, s), "q upload");
        d_q = d->q.as<float>();
    }
    if (!capturing) cuda_check(cudaEventRecord(d->staged, s), "event");
    const uint32_t* dwp = d->aux.as<uint32_t>();
    const uint32_t* dpo = dwp + (n + 1);
    const uint32_t* dco = dwp + 2 * (n + 1);
    const uint32_t* dpt = dwp + 3 * (n + 1);
    // the staged light pass runs each trajectory's FK (and fit) in shared memory; when the longest
    // trajectory does not fit there, centres and control points go through global memory
    uint32_t max_pieces = 0;
    for (uint32_t i = 0; i < n; ++i) max_pieces = std::max(max_pieces, piece_off[i + 1] - piece_off[i]);
    const uint32_t max_nc = quad ? quad_ctrl_count(max_wp) : 0;
    // A staged block works on one trajectory at a time, so the staged pass needs several trajectories
    // per resident block to keep the GPU busy: a batch of a few trajectories would run on a few
    // blocks (one trajectory of 128 waypoints is 8,128 units for one block) where the unstaged pass
    // spreads its units over the whole grid.
    const bool staged = !d->cfg.sweep_unstaged && n >= 4 * d->blocks &&
                        sweep_staged_smem(quad, R.n_links, max_wp, max_nc, max_pieces) != 0;
    d->last_path_flags = staged ? 1u : 0u;
    const bool timed = (flags & RTCD_CHECK_TIMING) != 0;
    d->timed = timed;
    if (timed) cuda_check(cudaEventRecord(d->ev[0], s), "event");
    if (!staged) {
        d->centers.ensure(16ull * total_wp * ns);
        launch_fk_spheres(R, d_q, total_wp, d->centers.as<float4>(), s);
        if (quad) {
            d->ctrl.ensure(16ull * ctrl_total * ns);
            launch_fit(d->centers.as<float4>(), dwp, dco, d->W.as<float>(), d->W_off.as<uint32_t>(), n, ns,
                       d->ctrl.as<float4>(), s);
        }
    }
    d->pose_hit.ensure(4ull * n);
    cuda_check(cudaMemsetAsync(d->pose_hit.p, 0, 4ull * n, s), "memset");
    if (want_pieces) {
        d->piece_hit.ensure(4ull * pieces);
        cuda_check(cudaMemsetAsync(d->piece_hit.p, 0, 4ull * pieces, s), "memset");
    }
    uint32_t* d_counts = nullptr;
    if (counts) {
        d->counts.ensure(4ull * n);
        d_counts = d->counts.as<uint32_t>();
        cuda_check(cudaMemsetAsync(d_counts, 0, 4ull * n, s), "memset");
    }
    cuda_check(cudaMemsetAsync(d->work.p, 0, 20, s), "memset");  // [0..4]: the sweep passes' counters
    SweepArgs A{};
    A.centers = staged ? nullptr : d->centers.as<float4>();
    A.ctrl = quad && !staged ? d->ctrl.as<float4>() : nullptr;
    A.q = d_q;
    A.W = d->W.as<float>();
    A.W_off = d->W_off.as<uint32_t>();
    A.max_wp = max_wp;
    A.max_nc = max_nc;
    A.max_pieces = max_pieces;
    A.group = d->cfg.sweep_group;
    A.traj_piece_off = dpo;
    A.traj_wp_off = dwp;
    A.traj_ctrl_off = dco;
    A.piece_traj = dpt;
    A.n_traj = n;
    A.n_spheres = ns;
    A.total_units = (uint32_t) (pieces * ns);
    A.quad = quad;
    A.endpoints = !(flags & (RTCD_CHECK_NO_ENDPOINTS | RTCD_CHECK_SURFACE));
    A.surface = (flags & RTCD_CHECK_SURFACE) != 0;
    A.traj_hit = d->pose_hit.as<uint32_t>();
    A.piece_hit = want_pieces ? d->piece_hit.as<uint32_t>() : nullptr;
    A.counts = d_counts;
    A.work_counter = d->work.as<uint32_t>();
    A.err = d->err.as<uint32_t>();
    A.stats = d->stats.as<unsigned long long>();
    A.want_counts = counts;
    A.want_pieces = want_pieces;
    A.light_steps = d->cfg.light_steps == 0xFFFFFFFFu ? 0u
                    : d->cfg.light_steps                ? d->cfg.light_steps
                                                              : 16u;
    A.heavy_wide = d->cfg.sweep_heavy_wide ? 1 : 0;
    A.descend_cap = d->cfg.sweep_descend_cap == 0xFFFFFFFFu ? 0u
                    : d->cfg.sweep_descend_cap                ? d->cfg.sweep_descend_cap
                                                                  : 3u;
    if (A.light_steps) {
        // room for every unit (near dense geometry most units of a piece can spill)
        const uint32_t cap = (uint32_t) std::min<uint64_t>(std::max<uint64_t>(pieces * ns, 1024), 1u << 20);
        d->heavy.ensure(sizeof(SweepRec) * cap);
        A.heavy = d->heavy.as<SweepRec>();
        A.heavy_cap = cap;
        A.heavy_count = d->work.as<uint32_t>() + 1;
        A.heavy_work = d->work.as<uint32_t>() + 2;
        // the split pass: room for one frontier entry per unit the light pass could defer
        A.heavy_steps = d->cfg.sweep_heavy_steps == 0xFFFFFFFFu ? 0u
                        : d->cfg.sweep_heavy_steps                ? d->cfg.sweep_heavy_steps
                                                                      : 32u;
        d->split.ensure(sizeof(uint2) * cap);
        A.split = d->split.as<uint2>();
        A.split_cap = cap;
        A.split_count = d->work.as<uint32_t>() + 3;
        A.split_work = d->work.as<uint32_t>() + 4;
    }
    d->last_items = A.total_units;
    if (timed) {
        cuda_check(cudaEventRecord(d->ev[1], s), "event");
        cuda_check(cudaEventRecord(d->ev[2], s), "event");
    }
    A.binary_tree = d->cfg.stage_b_form == 1 ? 1 : 0;
    if (A.total_units)
        launch_sweep(A.surface ? scene_loop(d->scene) : d->scene->dev, R, A, d->blocks, d->threads,
                     d->cfg.residency_percent ? d->cfg.residency_percent : 100, staged, s,
                     timed ? d->ev_first : nullptr);
    else if (timed)
        cuda_check(cudaEventRecord(d->ev_first, s), "event");
    if (timed) cuda_check(cudaEventRecord(d->ev[3], s), "event");
    // outputs
    uint8_t* d_flags = (host || !flags_out) ? (d->flags.ensure(n), d->flags.as<uint8_t>()) : flags_out;
    launch_flags(d->pose_hit.as<uint32_t>(), n, d_flags, s);
    uint8_t* d_seg = nullptr;
    if (want_pieces) {
        d_seg = host ? (d->seg_flags.ensure(pieces), d->seg_flags.as<uint8_t>()) : seg_out;
        launch_flags(d->piece_hit.as<uint32_t>(), (uint32_t) pieces, d_seg, s);
    }
    if (host) {
        size_t fpad = (n + 15) & ~15ull, ppad = (pieces + 15) & ~15ull;
        d->pin_out.ensure(fpad + ppad + 4ull * n + 16);
        uint8_t* pf = d->pin_out.as<uint8_t>();
        uint8_t* pp = pf + fpad;
        uint32_t* pc = reinterpret_cast<uint32_t*>(pp + ppad);
        cuda_check(cudaMemcpyAsync(pf, d_flags, n, cudaMemcpyDeviceToHost, s), "flags download");
        if (want_pieces) cuda_check(cudaMemcpyAsync(pp, d_seg, pieces, cudaMemcpyDeviceToHost, s), "seg download");
        if (counts && counts_out)
            cuda_check(cudaMemcpyAsync(pc, d_counts, 4ull * n, cudaMemcpyDeviceToHost, s), "counts download");
        cuda_check(cudaStreamSynchronize(s), "check sync");
        if (flags_out) std::memcpy(flags_out, pf, n);
        if (want_pieces) std::memcpy(seg_out, pp, pieces);
        if (counts && counts_out) std::memcpy(counts_out, pc, 4ull * n);
    } else if (counts && counts_out) {
        cuda_check(cudaMemcpyAsync(counts_out, d_counts, 4ull * n, cudaMemcpyDeviceToDevice, s), "counts copy");
    }
}

}  // namespace

extern "C" {

rtcd_status rtcd_check(rtcd_detector* d, const float* q, const uint32_t* traj_offsets, uint32_t n, uint8_t* flags_out,
                       uint8_t* seg_flags_out, uint32_t* counts_out, uint32_t flags, void* stream) {
    return guarded([&] {
        RTCD_REQUIRE(d, "NULL detector");
        RTCD_REQUIRE(n == 0 || q, "q is NULL");
        std::lock_guard<std::mutex> lock(d->mu);
        DeviceScope ds(d->ctx->device);
        cudaStream_t s = stream ? (cudaStream_t) stream : d->stream;
        d->timed = false;
        d->timed_total_only = false;
        d->last_stream = s;
        if (n) cuda_check(cudaMemsetAsync(d->stats.p, 0, 8 * kStatWords, s), "stats reset");
        if (n == 0) return;
        if (flags & RTCD_CHECK_GRAPH) {
            const bool discrete = d->kind == RTCD_OBS_TO_ROBOT || d->kind == RTCD_ROBOT_TO_OBS;
            const bool host = (flags & RTCD_CHECK_HOST_BUFFERS) != 0;
            RTCD_REQUIRE(!(flags & RTCD_CHECK_PLAIN), "graph replay needs the batched path");
            RTCD_REQUIRE(!discrete || !seg_flags_out, "segment flags exist only for sweep detectors");
            RTCD_REQUIRE(discrete || traj_offsets, "traj_offsets required for sweep detectors");
            RTCD_REQUIRE(flags_out, "graph replay needs a flags buffer");
            // events recorded inside a graph cannot be timed: a replay is timed as a whole
            const bool want_time = (flags & RTCD_CHECK_TIMING) != 0;
            const uint32_t f = flags & ~(RTCD_CHECK_GRAPH | RTCD_CHECK_TIMING);
            // sweeps: the graph holds the trajectory tables built from traj_offsets, so
            // their contents are part of the key (FNV-1a over the n + 1 offsets)
            uint64_t h = 1469598103934665603ull;
            if (!discrete)
                for (uint32_t i = 0; i <= n; ++i) h = (h ^ traj_offsets[i]) * 1099511628211ull;
            // host buffers: the graph runs between the pinned staging and device mirrors; the
            // copies from and to the caller's arrays stay outside it
            const float* gq = q;
            uint8_t* gflags = flags_out;
            uint8_t* gseg = seg_flags_out;
            uint32_t* gcounts = counts_out;
            size_t in_bytes = 0, n_seg = 0, seg_at = 0, counts_at = 0, err_at = 0;
            const void* up_src = nullptr;  // host: the caller's page-locked array or the pinned staging
            if (host) {
                in_bytes = 4ull * (discrete ? n : traj_offsets[n]) * d->robot->dof;
                if (seg_flags_out)
                    for (uint32_t i = 0; i < n; ++i) n_seg += pieces_of(d->kind, traj_offsets[i + 1] - traj_offsets[i], f);
                d->hq.ensure(std::max<size_t>(in_bytes, 16));
                if (host_pinned(q)) {  // the graph's upload reads the caller's page-locked array itself
                    up_src = q;
                } else {
                    d->pin_in.ensure(std::max<size_t>(in_bytes, 16));
                    std::memcpy(d->pin_in.p, q, in_bytes);
                    up_src = d->pin_in.p;
                }
                gq = d->hq.as<float>();
                d->hflags.ensure(n);
                gflags = d->hflags.as<uint8_t>();
                if (seg_flags_out) {
                    d->hseg.ensure(std::max<size_t>(n_seg, 1));
                    gseg = d->hseg.as<uint8_t>();
                }
                if (counts_out) {
                    d->hcounts.ensure(4ull * n);
                    gcounts = d->hcounts.as<uint32_t>();
                }
                // pinned results: flags | segment flags | counts | the device error word
                seg_at = (n + 15) & ~size_t(15);
                counts_at = seg_at + ((n_seg + 15) & ~size_t(15));
                err_at = counts_at + (counts_out ? 4ull * n : 0);
                d->pin_out.ensure(err_at + 16);
                for (uint64_t v : {(uint64_t) up_src, (uint64_t) d->pin_out.p}) h = (h ^ v) * 1099511628211ull;
            }
            const uint64_t key[8] = {(uint64_t) gq, n, (uint64_t) gflags, (uint64_t) gcounts, f, (uint64_t) s,
                                     (uint64_t) gseg, h};
            uint8_t* po = d->pin_out.as<uint8_t>();
            auto run = [&] {
                const uint32_t fd = f & ~RTCD_CHECK_HOST_BUFFERS;
                if (host) cuda_check(cudaMemcpyAsync(d->hq.p, up_src, in_bytes, cudaMemcpyHostToDevice, s), "q upload");
                if (discrete)
                    check_discrete(d, gq, n, gflags, gcounts, fd, s);
                else
                    check_sweep(d, gq, traj_offsets, n, gflags, gseg, gcounts, fd, s);
                if (host) {
                    cuda_check(cudaMemcpyAsync(po, gflags, n, cudaMemcpyDeviceToHost, s), "flags download");
                    if (gseg) cuda_check(cudaMemcpyAsync(po + seg_at, gseg, n_seg, cudaMemcpyDeviceToHost, s), "download");
                    if (counts_out)
                        cuda_check(cudaMemcpyAsync(po + counts_at, gcounts, 4ull * n, cudaMemcpyDeviceToHost, s), "download");
                    cuda_check(cudaMemcpyAsync(po + err_at, d->err.p, 4, cudaMemcpyDeviceToHost, s), "error readback");
                }
            };
            // host buffers: wait for the download, report a device error, hand the results over
            auto finish = [&] {
                if (!host) return;
                cuda_check(cudaStreamSynchronize(s), "check sync");
                uint32_t e = 0;
                std::memcpy(&e, po + err_at, 4);
                if (e) check_device_errors(d, s);  // resets the word and reports it
                std::memcpy(flags_out, po, n);
                if (seg_flags_out) std::memcpy(seg_flags_out, po + seg_at, n_seg);
                if (counts_out) std::memcpy(counts_out, po + counts_at, 4ull * n);
            };
            if (d->graph_exec && std::equal(key, key + 8, d->graph_key)) {
                if (want_time) cuda_check(cudaEventRecord(d->ev[0], s), "event");
                cuda_check(cudaGraphLaunch(d->graph_exec, s), "cudaGraphLaunch");
                if (want_time) cuda_check(cudaEventRecord(d->ev_end, s), "event");
                d->timed_total_only = want_time;
                finish();
                return;
            }
            // run once normally (this also sizes every workspace), then capture the
            // same sequence - which now allocates nothing - for the next calls
            if (want_time) cuda_check(cudaEventRecord(d->ev[0], s), "event");
            run();
            if (want_time) cuda_check(cudaEventRecord(d->ev_end, s), "event");
            d->timed_total_only = want_time;
            cuda_check(cudaStreamSynchronize(s), "pre-capture sync");  // staging buffers idle before capture
            if (d->graph_exec) cudaGraphExecDestroy(d->graph_exec);
            if (d->graph) cudaGraphDestroy(d->graph);
            d->graph_exec = nullptr;
            d->graph = nullptr;
            cuda_check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
            try {
                run();
            } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(s, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            cuda_check(cudaStreamEndCapture(s, &d->graph), "cudaStreamEndCapture");
            cuda_check(cudaGraphInstantiate(&d->graph_exec, d->graph, 0), "cudaGraphInstantiate");
            std::copy(key, key + 8, d->graph_key);
            finish();  // the results of the run before the capture
            return;
        }
        if (d->graph_exec) {  // this call may grow (move) workspaces the graph points into
            cuda_check(cudaStreamSynchronize(s), "graph retire");
            cudaGraphExecDestroy(d->graph_exec);
            cudaGraphDestroy(d->graph);
            d->graph_exec = nullptr;
            d->graph = nullptr;
        }
        if (d->kind == RTCD_OBS_TO_ROBOT || d->kind == RTCD_ROBOT_TO_OBS) {
            RTCD_REQUIRE(!seg_flags_out, "segment flags exist only for sweep detectors");
            check_discrete(d, q, n, flags_out, counts_out, flags, s);
        } else {
            RTCD_REQUIRE(!(flags & RTCD_CHECK_PLAIN), "the plain frame path is for the discrete detectors");
            check_sweep(d, q, traj_offsets, n, flags_out, seg_flags_out, counts_out, flags, s);
        }
        if (d->timed) cuda_check(cudaEventRecord(d->ev_end, s), "event");
        if (flags & RTCD_CHECK_HOST_BUFFERS) check_device_errors(d, s);
    });
}

rtcd_status rtcd_sync(rtcd_detector* d, void* stream) {
    return guarded([&] {
        RTCD_REQUIRE(d, "NULL detector");
        std::lock_guard<std::mutex> lock(d->mu);
        DeviceScope ds(d->ctx->device);
        cudaStream_t s = stream ? (cudaStream_t) stream : d->stream;
        check_device_errors(d, s);
    });
}

rtcd_status rtcd_segment_offsets(rtcd_detector_kind kind, const uint32_t* traj_offsets, uint32_t n, uint32_t flags,
                                 uint32_t* offsets_out) {
    return guarded([&] {
        RTCD_REQUIRE(kind == RTCD_LINEAR_SWEEP || kind == RTCD_QUAD_SWEEP, "segments exist only for sweep kinds");
        RTCD_REQUIRE(traj_offsets && offsets_out, "NULL argument");
        offsets_out[0] = 0;
        for (uint32_t i = 0; i < n; ++i) {
            RTCD_REQUIRE(traj_offsets[i + 1] >= traj_offsets[i], "traj_offsets must be non-decreasing");
            offsets_out[i + 1] = offsets_out[i] + pieces_of(kind, traj_offsets[i + 1] - traj_offsets[i], flags);
        }
    });
}

rtcd_status rtcd_last_stats(rtcd_detector* d, rtcd_stats* out) {
    return guarded([&] {
        RTCD_REQUIRE(d && out, "NULL argument");
        std::lock_guard<std::mutex> lock(d->mu);
        DeviceScope ds(d->ctx->device);
        std::memset(out, 0, sizeof(*out));
        unsigned long long sb[kStatWords] = {0}, st[kStatBank] = {0};
        uint32_t cnt = 0;
        cudaStream_t s = d->last_stream ? d->last_stream : d->stream;
        cuda_check(cudaMemcpyAsync(sb, d->stats.p, sizeof(sb), cudaMemcpyDeviceToHost, s), "stats");
        cuda_check(cudaMemcpyAsync(&cnt, d->count.p, 4, cudaMemcpyDeviceToHost, s), "stats");
        const bool discrete = d->kind == RTCD_OBS_TO_ROBOT || d->kind == RTCD_ROBOT_TO_OBS;
        uint32_t cand = 0, wave[4] = {0, 0, 0, 0}, work[2] = {0, 0};
        if (d->wave_counts.p)
            cuda_check(cudaMemcpyAsync(wave, d->wave_counts.p, sizeof(wave), cudaMemcpyDeviceToHost, s), "stats");
        if (!discrete && d->work.p)
            cuda_check(cudaMemcpyAsync(work, d->work.p, sizeof(work), cudaMemcpyDeviceToHost, s), "stats");
        cuda_check(cudaStreamSynchronize(s), "stats sync");
        cand = wave[0];
        // the heavy list's append counter: [3] of the discrete wave counters, [1] of the sweep work words
        out->deferred = discrete ? wave[3] : work[1];
        for (int k = 0; k < kStatBank; ++k) st[k] = sb[k] + sb[kStatBank + k];
        out->path_flags = d->last_path_flags;
        out->first_node_tests = sb[7];
        out->first_exact_tests = sb[4];
        out->cull_sphere_tests = sb[kStatCullSpheres];
        out->cull_sat_tests = sb[kStatCullSats];
        out->fp64_retests = st[0];
        // discrete: the candidate buffer's count, or the fused form's in-warp count
        out->candidates = discrete ? (st[6] ? st[6] : cand) : st[5];
        out->exact_tests = st[4];
        out->skipped = st[2];
        out->node_tests = st[7];
        if (d->timed) {
            cuda_check(cudaEventElapsedTime(&out->ms_prepare, d->ev[0], d->ev[1]), "elapsed");
            cuda_check(cudaEventElapsedTime(&out->ms_cull, d->ev[1], d->ev[2]), "elapsed");
            cuda_check(cudaEventElapsedTime(&out->ms_traverse, d->ev[2], d->ev[3]), "elapsed");
            cuda_check(cudaEventElapsedTime(&out->ms_first_pass, d->ev[2], d->ev_first), "elapsed");
            cuda_check(cudaEventElapsedTime(&out->ms_total, d->ev[0], d->ev_end), "elapsed");
        } else if (d->timed_total_only) {
            cuda_check(cudaEventElapsedTime(&out->ms_total, d->ev[0], d->ev_end), "elapsed");
        }
        out->work_items = (d->kind == RTCD_OBS_TO_ROBOT || d->kind == RTCD_ROBOT_TO_OBS) && !d->last_items ? cnt
                                                                                                          : d->last_items;
    });
}

rtcd_status rtcd_detector_autotune(rtcd_detector* d, const float* q_dev, const uint32_t* traj_offsets, uint32_t n,
                                   void* stream, rtcd_config* best_out, float* best_ms) {
    return guarded([&] {
        RTCD_REQUIRE(d && q_dev && n, "NULL argument");
        DeviceScope ds(d->ctx->device);
        cudaStream_t s = stream ? (cudaStream_t) stream : d->stream;
        const bool discrete = d->kind == RTCD_OBS_TO_ROBOT || d->kind == RTCD_ROBOT_TO_OBS;
        DevBuf flags, seg;
        flags.ensure(n);
        uint32_t n_seg = 0;
        if (!discrete) {  // sweeps are tuned with segment flags on (no trajectory-level early exit)
            std::vector<uint32_t> so(n + 1);
            rtcd_status st = rtcd_segment_offsets(d->kind, traj_offsets, n, 0, so.data());
            if (st != RTCD_OK) fail(st, g_last_error);
            n_seg = so[n];
            seg.ensure(std::max(n_seg, 1u));
        }
        const rtcd_config saved = d->cfg;
        rtcd_config best = saved;
        float best_t = 3.0e38f;
        std::vector<std::pair<float, rtcd_config>> tried;
        // Each candidate is timed as a caller running a stream of checks sees it: the whole check
        // replayed as a CUDA graph (no host launch gaps, which dominate small batches when kernels
        // are launched one by one), after a write larger than the L2 (the previous check's tree
        // nodes are not left cached) when the device has the memory to spare for it.
        DevBuf flush;
        size_t flush_bytes = 0;
        {
            int l2 = 0;
            cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, d->ctx->device);
            size_t free_b = 0, total_b = 0;
            cudaMemGetInfo(&free_b, &total_b);
            const size_t want = 2ull * (size_t) std::max(l2, 0);
            if (want && free_b > 8 * want) {
                flush.ensure(want);
                flush_bytes = want;
            }
        }
        // a graph captured under another configuration must not be replayed for this one
        auto retire_graph = [&] {
            std::lock_guard<std::mutex> lock(d->mu);
            if (!d->graph_exec) return;
            cuda_check(cudaStreamSynchronize(s), "graph retire");
            cudaGraphExecDestroy(d->graph_exec);
            cudaGraphDestroy(d->graph);
            d->graph_exec = nullptr;
            d->graph = nullptr;
        };
        // median of `reps` timed replays after a warm-up run (which captures the graph)
        auto measure = [&](const rtcd_config& c, int reps) {
            retire_graph();
            d->cfg = c;
            apply_launch_shape(d);
            float ms[16];
            for (int rep = 0; rep <= reps; ++rep) {
                if (flush_bytes) cuda_check(cudaMemsetAsync(flush.p, rep & 255, flush_bytes, s), "L2 flush");
                rtcd_status st = rtcd_check(d, q_dev, traj_offsets, n, flags.as<uint8_t>(),
                                            discrete ? nullptr : seg.as<uint8_t>(), nullptr,
                                            RTCD_CHECK_TIMING | RTCD_CHECK_GRAPH, s);
                rtcd_stats stt;
                if (st == RTCD_OK) st = rtcd_last_stats(d, &stt);
                if (st != RTCD_OK) {
                    retire_graph();
                    d->cfg = saved;
                    apply_launch_shape(d);
                    fail(st, g_last_error);
                }
                ms[rep] = stt.ms_total;
            }
            std::sort(ms + 1, ms + reps + 1);
            return ms[1 + reps / 2];
        };
        auto time_cfg = [&](const rtcd_config& c) {
            const float t = measure(c, 3);
            tried.emplace_back(t, c);
            if (t < best_t) {
                best_t = t;
                best = c;
            }
        };
        // coordinate descent: the launch shape, then the light-pass budget, then the stage B
        // form and its chunk length (discrete) or the tree and staging (sweeps), then the launch
        // shape again under the settings found (the best shape depends on them)
        auto shape_pass = [&](const rtcd_config& base) {
            for (uint32_t t : {64u, 128u, 256u}) {
                uint32_t fit = discrete ? stage_b_max_blocks_per_sm(d->kind == RTCD_ROBOT_TO_OBS, t)
                                        : sweep_max_blocks_per_sm(d->kind == RTCD_QUAD_SWEEP, t);
                std::vector<uint32_t> shapes = {std::max(1u, fit / 4), std::max(1u, fit / 2), fit};
                shapes.erase(std::unique(shapes.begin(), shapes.end()), shapes.end());
                for (uint32_t per_sm : shapes) {
                    rtcd_config c = base;
                    c.traverse_threads = t;
                    c.traverse_blocks_per_sm = per_sm;
                    time_cfg(c);
                }
            }
        };
        auto light_pass = [&](const rtcd_config& base) {
            for (uint32_t light : {0u, 16u, 32u, 64u}) {  // 0: the kind's default budget
                rtcd_config c = base;
                c.light_steps = light;
                time_cfg(c);
            }
        };
        auto form_pass = [&](const rtcd_config& base) {
            if (!discrete) {  // the binary or the wide edge tree, staged or unstaged centres, grouping
                rtcd_config c = base;
                c.stage_b_form = base.stage_b_form == 1 ? 0u : 1u;
                time_cfg(c);
                c = base;
                c.sweep_unstaged = base.sweep_unstaged ? 0u : 1u;
                time_cfg(c);
                c = base;
                c.sweep_group = base.sweep_group == 1 ? 0u : 1u;
                time_cfg(c);
                c = base;
                c.sweep_heavy_wide = base.sweep_heavy_wide ? 0u : 1u;
                time_cfg(c);
                for (uint32_t cap : {2u, 4u, 6u}) {  // visits per descent (0: the default, 3)
                    c = base;
                    c.sweep_descend_cap = base.sweep_descend_cap == cap ? 0u : cap;
                    time_cfg(c);
                }
                return;
            }
            for (uint32_t form : {1u, 2u, 3u, 4u})
                for (uint32_t chunk : {1u, 16u, 64u, 256u}) {
                    rtcd_config c = base;
                    c.stage_b_form = form;
                    // lanes: candidates per lane; packets: groups per warp; fused: the item's
                    // stage-B step budget (1, 4, 16, 64)
                    c.stage_b_chunk = form == 2 ? std::max(1u, chunk / 16) : (form >= 3 ? std::max(1u, chunk / 4) : chunk);
                    time_cfg(c);
                }
            if (best.stage_b_form == 0 || best.stage_b_form >= 3) {  // the fused form: top levels in shared memory
                rtcd_config c = best;
                c.top_nodes_shared = best.top_nodes_shared ? 0u : 85u;  // 1 + 4 + 16 + 64: the first four levels
                time_cfg(c);
            }
        };
        // rounds of descent over the three groups of settings until a round changes nothing (the
        // best light budget and stage-B form depend on the launch shape and back)
        shape_pass(saved);
        for (int round = 0; round < 3; ++round) {
            const rtcd_config start = best;
            light_pass(best);
            form_pass(best);
            shape_pass(best);
            if (std::memcmp(&start, &best, sizeof(rtcd_config)) == 0) break;
        }
        // run-to-run noise is of the order of the differences between the leading shapes: the
        // three fastest are timed again, longer, and the fastest of that round is kept
        std::stable_sort(tried.begin(), tried.end(),
                         [](const std::pair<float, rtcd_config>& x, const std::pair<float, rtcd_config>& y) {
                             return x.first < y.first;
                         });
        best_t = 3.0e38f;
        for (size_t k = 0; k < std::min<size_t>(3, tried.size()); ++k) {
            const float t = measure(tried[k].second, 9);
            if (t < best_t) {
                best_t = t;
                best = tried[k].second;
            }
        }
        retire_graph();
        d->cfg = best;
        apply_launch_shape(d);
        if (best_out) *best_out = best;
        if (best_ms) *best_ms = best_t;
    });
}

rtcd_status rtcd_quad_fit_weights(uint32_t n_ctrl, uint32_t n_wp, float* W_out) {
    return guarded([&] {
        RTCD_REQUIRE(W_out, "NULL argument");
        RTCD_REQUIRE(n_ctrl >= 3 && n_wp >= n_ctrl, "need 3 <= n_ctrl <= n_wp");
        const std::vector<double> W = fit_weights(n_ctrl, n_wp);
        for (size_t i = 0; i < W.size(); ++i) W_out[i] = (float) W[i];
    });
}

rtcd_status rtcd_knn(rtcd_ctx* ctx, const float* points_dev, uint32_t n, uint32_t dim, const float* weights,
                     uint32_t k, const uint8_t* mask_dev, uint32_t* idx_dev, float* dist_dev, void* stream) {
    return guarded([&] {
        RTCD_REQUIRE(ctx && (n == 0 || (points_dev && idx_dev && dist_dev)), "NULL argument");
        RTCD_REQUIRE(dim >= 1 && dim <= kKnnMaxDim, "dim must be 1..16");
        RTCD_REQUIRE(k >= 1 && k <= kKnnMaxK, "k must be 1..32");
        DeviceScope ds(ctx->device);
        cudaStream_t s = stream ? (cudaStream_t) stream : ctx->stream;
        std::lock_guard<std::mutex> lk(ctx->mu);
        float w2[kKnnMaxDim];
        for (uint32_t d = 0; d < dim; ++d) w2[d] = weights ? weights[d] * weights[d] : 1.0f;
        ctx->knn_w2.ensure(sizeof(w2));
        cuda_check(cudaStreamSynchronize(s), "knn weights");  // the previous call's kernel may still read them
        cuda_check(cudaMemcpy(ctx->knn_w2.p, w2, dim * sizeof(float), cudaMemcpyHostToDevice), "knn weights");
        launch_knn(points_dev, n, dim, ctx->knn_w2.as<float>(), k, mask_dev, idx_dev, dist_dev, s);
    });
}

rtcd_status rtcd_check_edges(rtcd_detector* d, const float* nodes_dev, uint32_t n_nodes, const uint32_t* edges_dev,
                             uint32_t n_edges, uint32_t n_wp, uint8_t* flags_dev, uint32_t flags, void* stream) {
    return guarded([&] {
        RTCD_REQUIRE(d && (n_edges == 0 || (nodes_dev && edges_dev && flags_dev)), "NULL argument");
        RTCD_REQUIRE(n_wp >= 2, "an edge needs at least 2 configurations");
        RTCD_REQUIRE(!(flags & ~(uint32_t) (RTCD_CHECK_NO_ENDPOINTS | RTCD_CHECK_TWO_WAY | RTCD_CHECK_CONTAINMENT)),
                     "edge checks accept RTCD_CHECK_NO_ENDPOINTS, RTCD_CHECK_TWO_WAY and RTCD_CHECK_CONTAINMENT");
        const bool discrete = d->kind == RTCD_OBS_TO_ROBOT || d->kind == RTCD_ROBOT_TO_OBS;
        RTCD_REQUIRE(discrete || !(flags & (RTCD_CHECK_TWO_WAY | RTCD_CHECK_CONTAINMENT)),
                     "two-way and containment are for the discrete detectors");
        RTCD_REQUIRE(d->kind != RTCD_QUAD_SWEEP || n_wp >= 3, "quadratic edges need at least 3 configurations");
        RTCD_REQUIRE((uint64_t) n_edges * n_wp < (1ull << 32), "too many configurations in one call");
        if (!n_edges) return;
        // one critical section: the interpolated configurations live in the detector's workspace
        std::lock_guard<std::mutex> lock(d->mu);
        DeviceScope ds(d->ctx->device);
        cudaStream_t s = stream ? (cudaStream_t) stream : d->stream;
        d->timed = false;
        d->timed_total_only = false;
        d->last_stream = s;
        if (d->graph_exec) {  // this call may grow (move) workspaces the graph points into
            cuda_check(cudaStreamSynchronize(s), "graph retire");
            cudaGraphExecDestroy(d->graph_exec);
            cudaGraphDestroy(d->graph);
            d->graph_exec = nullptr;
            d->graph = nullptr;
        }
        cuda_check(cudaMemsetAsync(d->stats.p, 0, 8 * kStatWords, s), "stats reset");
        const uint32_t dof = d->robot->dof;
        const uint32_t total = n_edges * n_wp;
        d->edge_q.ensure(4ull * total * dof);
        launch_interp_edges(nodes_dev, n_nodes, dof, edges_dev, n_edges, n_wp, d->edge_q.as<float>(),
                            d->err.as<uint32_t>(), s);
        if (discrete) {
            d->edge_pose_flags.ensure(total);
            check_discrete(d, d->edge_q.as<float>(), total, d->edge_pose_flags.as<uint8_t>(), nullptr, flags, s);
            launch_or_rows(d->edge_pose_flags.as<uint8_t>(), n_edges, n_wp, flags_dev, s);
        } else {
            d->edge_off.resize(n_edges + 1);
            for (uint32_t e = 0; e <= n_edges; ++e) d->edge_off[e] = e * n_wp;
            check_sweep(d, d->edge_q.as<float>(), d->edge_off.data(), n_edges, flags_dev, nullptr, nullptr, flags, s);
        }
    });
}

rtcd_status rtcd_robot_fk(rtcd_robot* r, const float* q_dev, uint32_t n, float* T_dev, void* stream) {
    return guarded([&] {
        RTCD_REQUIRE(r && (n == 0 || (q_dev && T_dev)), "NULL argument");
        DeviceScope ds(r->ctx->device);
        cudaStream_t s = stream ? (cudaStream_t) stream : r->ctx->stream;
        launch_fk_poses(r->dev.chain, q_dev, n, reinterpret_cast<float4*>(T_dev), s);
    });
}

rtcd_status rtcd_exclusive_scan_u32(rtcd_ctx* ctx, const uint32_t* in_dev, uint32_t* out_dev, uint32_t n,
                                    uint32_t* total_dev, void* stream) {
    return guarded([&] {
        RTCD_REQUIRE(ctx && (n == 0 || (in_dev && out_dev)), "NULL argument");
        RTCD_REQUIRE(in_dev != out_dev, "in and out must differ");
        DeviceScope ds(ctx->device);
        cudaStream_t s = stream ? (cudaStream_t) stream : ctx->stream;
        ScanScratch sc;
        scan_u32(in_dev, out_dev, n, total_dev, sc, ctx->err.as<uint32_t>(), s);
        cuda_check(cudaStreamSynchronize(s), "scan");  // the scratch is released on return
    });
}

rtcd_status rtcd_select_flags_u8(rtcd_ctx* ctx, const uint8_t* mask_dev, uint32_t n, uint32_t* idx_dev,
                                 uint32_t* count_dev, void* stream) {
    return guarded([&] {
        RTCD_REQUIRE(ctx && count_dev && (n == 0 || (mask_dev && idx_dev)), "NULL argument");
        DeviceScope ds(ctx->device);
        cudaStream_t s = stream ? (cudaStream_t) stream : ctx->stream;
        ScanScratch sc;
        select_u8(mask_dev, n, idx_dev, count_dev, sc, ctx->err.as<uint32_t>(), s);
        cuda_check(cudaStreamSynchronize(s), "select");
    });
}

rtcd_status rtcd_exact_test_probe(rtcd_ctx* ctx, int test, const float* a_dev, const float* b_dev, uint32_t n,
                                  float* f32_dev, double* f64_dev, void* stream) {
    return guarded([&] {
        RTCD_REQUIRE(ctx && (n == 0 || (a_dev && b_dev && f32_dev && f64_dev)), "NULL argument");
        RTCD_REQUIRE(test >= 0 && test <= 2, "test must be 0 (segment-triangle), 1 (capsule) or 2 (quadratic)");
        DeviceScope ds(ctx->device);
        cudaStream_t s = stream ? (cudaStream_t) stream : ctx->stream;
        if (test == 0) launch_probe_segtri(a_dev, b_dev, n, f32_dev, f64_dev, s);
        else launch_probe_sweep(test == 2, a_dev, b_dev, n, f32_dev, f64_dev, s);
    });
}

rtcd_status rtcd_selftest_lookback_timeout(rtcd_ctx* ctx, uint32_t n, uint32_t spin_limit) {
    return guarded([&] {
        RTCD_REQUIRE(ctx, "NULL context");
        RTCD_REQUIRE(n >= 1 && n <= (1u << 20), "n must be 1 to 1048576");
        RTCD_REQUIRE(spin_limit >= 1 && spin_limit <= (1u << 16), "spin_limit must be 1 to 65536");
        DeviceScope ds(ctx->device);
        cudaStream_t s = ctx->stream;
        DevBuf mask, words;
        mask.ensure(n);
        words.ensure(16);  // [0] output index, [1] count, [2] error word
        cuda_check(cudaMemsetAsync(mask.p, 0, n, s), "memset");
        cuda_check(cudaMemsetAsync(words.p, 0, 16, s), "memset");
        ScanScratch sc;
        uint32_t* w = words.as<uint32_t>();
        lookback_timeout_probe(mask.as<uint8_t>(), n, spin_limit, w, w + 1, sc, w + 2, s);
        uint32_t e = 0;
        cuda_check(cudaMemcpyAsync(&e, w + 2, 4, cudaMemcpyDeviceToHost, s), "error word read");
        cuda_check(cudaStreamSynchronize(s), "selftest");
        if (e & kErrLookback) fail(RTCD_ERR_DEVICE_TIMEOUT, "look-back wait ran out (expected by this self-test)");
        fail(RTCD_ERR_INTERNAL, "the look-back waits did not run out");
    });
}

rtcd_status rtcd_lbvh_build(rtcd_ctx* ctx, const float* lo, const float* hi, uint32_t n, uint32_t* codes_out,
                            uint32_t* perm_out, uint32_t* child_out, float* node_lo, float* node_hi,
                            uint32_t* depth_out) {
    return guarded([&] {
        RTCD_REQUIRE(ctx && (n == 0 || (lo && hi)), "NULL argument");
        DeviceScope ds(ctx->device);
        cudaStream_t s = ctx->stream;
        std::vector<float4> hl(n), hh(n);
        for (uint32_t i = 0; i < n; ++i) {
            hl[i] = make_float4(lo[3 * i], lo[3 * i + 1], lo[3 * i + 2], 0.f);
            hh[i] = make_float4(hi[3 * i], hi[3 * i + 1], hi[3 * i + 2], 0.f);
        }
        DevBuf dl, dh, nodes, perm;
        upload(dl, hl.data(), n, s);
        upload(dh, hh.data(), n, s);
        nodes.ensure(64ull * std::max<uint32_t>(n, 2));
        perm.ensure(4ull * std::max<uint32_t>(n, 1));
        std::vector<uint32_t> codes, child;
        LbvhResult res = build_lbvh(dl.as<float4>(), dh.as<float4>(), n, nodes.as<float4>(), perm.as<uint32_t>(), 0, 0,
                                    ctx->err.as<uint32_t>(), s, &codes, &child);
        if (depth_out) *depth_out = res.depth;
        if (codes_out && n) std::memcpy(codes_out, codes.data(), 4ull * n);
        if (perm_out && n) cuda_check(cudaMemcpy(perm_out, perm.p, 4ull * n, cudaMemcpyDeviceToHost), "perm");
        if (child_out && n > 1) std::memcpy(child_out, child.data(), 8ull * (n - 1));
        if ((node_lo || node_hi) && n > 1) {
            std::vector<float4> pk(4ull * (n - 1));
            cuda_check(cudaMemcpy(pk.data(), nodes.p, 64ull * (n - 1), cudaMemcpyDeviceToHost), "nodes");
            // a node's own box is the union of the two child boxes packed in it
            for (uint32_t i = 0; i < n - 1; ++i) {
                const float4* p = &pk[4ull * i];
                float l[3] = {std::min(p[0].x, p[1].z), std::min(p[0].y, p[1].w), std::min(p[0].z, p[2].x)};
                float h[3] = {std::max(p[0].w, p[2].y), std::max(p[1].x, p[2].z), std::max(p[1].y, p[2].w)};
                for (int k = 0; k < 3; ++k) {
                    if (node_lo) node_lo[3ull * i + k] = l[k];
                    if (node_hi) node_hi[3ull * i + k] = h[k];
                }
            }
        }
    });
}

}  // extern "C"
