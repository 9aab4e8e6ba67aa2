// planner.cu - the planner-side caller of the detectors: roadmap samples,
// nearest-neighbour edges and batched straight-line edge checks.
//
// The reference's planner tooling samples the configuration space with a
// Halton sequence (RTCD/Planner/sampler/sampler.h:11-82), links every sample
// to its K weighted nearest neighbours on the GPU (RTCD/Planner/KNN/
// knnCUDA.cu: all-pairs weighted squared distances, self and masked points
// excluded, a partial insertion sort, square roots), and turns each edge
// into a straight line of evenly spaced configurations that it checks as a
// trajectory (RTCD/Utils/Test/poseUtils.h:115-141).  Here the neighbour search
// is one warp per query (each lane keeps its own K best, the warp merges
// them), and an edge check interpolates the edges on the device and runs the
// detector over them in one call.
#include <algorithm>
#include <cfloat>
#include <vector>

#include "../../include/rtcd.h"
#include "kernels.h"

namespace rtcd {

constexpr int kKnnWarps = 4;

// One warp per query point.  Each lane scans every 32nd reference point and
// keeps its own K smallest (distance, index) pairs, ordered; the warp then
// pops the smallest head K times.  Pairs compare by distance, then by index,
// which is the order the reference's insertion sort settles ties in.
__global__ void __launch_bounds__(kKnnWarps * 32) k_knn(const float* __restrict__ pts, uint32_t n, uint32_t dim,
                                                         const float* __restrict__ w2, uint32_t k,
                                                         const uint8_t* __restrict__ mask, uint32_t* __restrict__ idx,
                                                         float* __restrict__ dist) {
    const int lane = threadIdx.x & 31;
    const uint32_t q = blockIdx.x * kKnnWarps + (threadIdx.x >> 5);
    if (q >= n) return;  // warp-uniform
    float qp[kKnnMaxDim], ww[kKnnMaxDim];
    for (uint32_t d = 0; d < dim; ++d) {
        qp[d] = pts[(size_t) q * dim + d];
        ww[d] = w2[d];
    }
    float bd[kKnnMaxK];
    uint32_t bi[kKnnMaxK];
    for (uint32_t j = 0; j < k; ++j) {
        bd[j] = FLT_MAX;
        bi[j] = 0xFFFFFFFFu;
    }
    const bool qmasked = mask && mask[q];
    for (uint32_t r = lane; r < n; r += 32) {
        if (r == q || qmasked || (mask && mask[r])) continue;  // not a candidate
        float s = 0.f;
        for (uint32_t d = 0; d < dim; ++d) {
            const float t = pts[(size_t) r * dim + d] - qp[d];
            s += t * t * ww[d];
        }
        // insert into this lane's ordered list when better than its last entry
        if (s < bd[k - 1] || (s == bd[k - 1] && r < bi[k - 1])) {
            int j = (int) k - 1;
            while (j > 0 && (s < bd[j - 1] || (s == bd[j - 1] && r < bi[j - 1]))) {
                bd[j] = bd[j - 1];
                bi[j] = bi[j - 1];
                --j;
            }
            bd[j] = s;
            bi[j] = r;
        }
    }
    // merge: k rounds of a warp arg-min over the lanes' heads
    uint32_t head = 0;
    for (uint32_t out = 0; out < k; ++out) {
        float v = head < k ? bd[head] : FLT_MAX;
        uint32_t i = head < k ? bi[head] : 0xFFFFFFFFu;
        float bv = v;
        uint32_t bidx = i;
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const uint32_t oi = __shfl_xor_sync(0xffffffffu, bidx, o);
            if (ov < bv || (ov == bv && oi < bidx)) {
                bv = ov;
                bidx = oi;
            }
        }
        if (v == bv && i == bidx && head < k) ++head;  // the winning lane advances (indices are unique)
        if (lane == 0) {
            idx[(size_t) q * k + out] = bidx;
            dist[(size_t) q * k + out] = bv < FLT_MAX ? sqrtf(bv) : FLT_MAX;
        }
    }
}

// Edge e = (a, b) as n_wp evenly spaced configurations a + (b - a) / (n_wp - 1) * i.
__global__ void k_interp_edges(const float* __restrict__ nodes, uint32_t n_nodes, uint32_t dof,
                               const uint32_t* __restrict__ edges, uint32_t n_edges, uint32_t n_wp,
                               float* __restrict__ q, uint32_t* __restrict__ err) {
    const size_t total = (size_t) n_edges * n_wp;
    for (size_t t = blockIdx.x * (size_t) blockDim.x + threadIdx.x; t < total; t += (size_t) gridDim.x * blockDim.x) {
        const uint32_t e = (uint32_t) (t / n_wp), i = (uint32_t) (t - (size_t) e * n_wp);
        const uint32_t a = edges[2ull * e], b = edges[2ull * e + 1];
        if (a >= n_nodes || b >= n_nodes) {
            atomicOr(err, kErrRange);
            for (uint32_t d = 0; d < dof; ++d) q[t * dof + d] = 0.f;
            continue;
        }
        for (uint32_t d = 0; d < dof; ++d) {
            const float s = nodes[(size_t) a * dof + d];
            const float span = (nodes[(size_t) b * dof + d] - s) / (float) (n_wp - 1);
            q[t * dof + d] = s + span * (float) i;
        }
    }
}

// flags[e] = OR of the pose flags of edge e's n_wp configurations
__global__ void k_or_rows(const uint8_t* __restrict__ pose_flags, uint32_t n_edges, uint32_t n_wp,
                          uint8_t* __restrict__ flags) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_edges) return;
    uint8_t f = 0;
    for (uint32_t i = 0; i < n_wp; ++i) f |= pose_flags[(size_t) e * n_wp + i];
    flags[e] = f;
}

void launch_knn(const float* pts, uint32_t n, uint32_t dim, const float* w2_dev, uint32_t k, const uint8_t* mask,
                uint32_t* idx, float* dist, cudaStream_t s) {
    if (!n) return;
    k_knn<<<(n + kKnnWarps - 1) / kKnnWarps, kKnnWarps * 32, 0, s>>>(pts, n, dim, w2_dev, k, mask, idx, dist);
    cuda_check(cudaGetLastError(), "k_knn");
}

void launch_interp_edges(const float* nodes, uint32_t n_nodes, uint32_t dof, const uint32_t* edges, uint32_t n_edges,
                         uint32_t n_wp, float* q, uint32_t* err, cudaStream_t s) {
    const size_t total = (size_t) n_edges * n_wp;
    if (!total) return;
    const uint32_t blocks = (uint32_t) std::min<size_t>((total + 255) / 256, 148u * 16u);
    k_interp_edges<<<blocks, 256, 0, s>>>(nodes, n_nodes, dof, edges, n_edges, n_wp, q, err);
    cuda_check(cudaGetLastError(), "k_interp_edges");
}

void launch_or_rows(const uint8_t* pose_flags, uint32_t n_edges, uint32_t n_wp, uint8_t* flags, cudaStream_t s) {
    if (!n_edges) return;
    k_or_rows<<<(n_edges + 255) / 256, 256, 0, s>>>(pose_flags, n_edges, n_wp, flags);
    cuda_check(cudaGetLastError(), "k_or_rows");
}

}  // namespace rtcd

namespace {

// The reference's Halton radical inverse, with its float arithmetic
// (RTCD/Planner/sampler/sampler.h:11-25).
float halton(int n, int b) {
    float hn = 0;
    int n0 = n;
    float f = 1 / ((float) b);
    while (n0 > 0) {
        float n1 = (float) (n0 / b);
        int r = n0 - (int) (n1 * (float) b);
        hn += f * (float) r;
        f = f / (float) b;
        n0 = (int) n1;
    }
    return hn;
}

}  // namespace

extern "C" {

rtcd_status rtcd_halton_samples(uint32_t n, uint32_t dim, uint32_t skip, const float* lower, const float* upper,
                                float* out) {
    static const int kPrimes[25] = {2,  3,  5,  7,  11, 13, 17, 19, 23, 29, 31, 37, 41,
                                    43, 47, 53, 59, 61, 67, 71, 73, 79, 83, 89, 97};
    try {
        if (!lower || !upper || (n && !out)) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "NULL argument");
        if (skip + dim > 25) rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "skip + dim must be at most 25 (prime bases)");
        for (uint32_t d = 0; d < dim; ++d)
            for (uint32_t i = 0; i < n; ++i)
                out[(size_t) i * dim + d] = halton((int) i, kPrimes[d + skip]) * (upper[d] - lower[d]) + lower[d];
        rtcd::set_last_error("");
        return RTCD_OK;
    } catch (const rtcd::Error& e) {
        rtcd::set_last_error(e.msg);
        return (rtcd_status) e.status;
    }
}

}  // extern "C"
