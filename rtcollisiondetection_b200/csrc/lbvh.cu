// lbvh.cu - device LBVH builder and the shared scan/select launchers.
//
// Replaces the OptiX GAS/IAS builds of the upstream path (optixAccelBuild in
// RTCD/Meshes/mesh.h:725-740, :798-815, RTCD/CollisionScenes/scene.h:138-145).
// The tree is the canonical one: 30-bit Morton codes of the float centroids
// normalised by the centroid bounds, a stable sort by (code, index), the
// Karras 2012 hierarchy ("Maximizing Parallelism in the Construction of BVHs,
// Octrees, and k-d Trees") with index tie-breaks for equal codes, one
// primitive per leaf and an atomic bottom-up box fit.  Every float step uses
// explicitly rounded intrinsics so the tree is bit-identical to the CPU
// restatement in the oracle.
#include <algorithm>
#include <cstring>

#include "engine.h"
#include "scan.cuh"

namespace rtcd {

// ---------------------------------------------------------------- scan glue
void ScanScratch::prepare(uint32_t n_items, cudaStream_t s) {
    uint32_t tiles = std::max<uint32_t>(1, scan_tiles(n_items));
    status.ensure(sizeof(unsigned long long) * tiles);
    counter.ensure(sizeof(uint32_t));
    cuda_check(cudaMemsetAsync(status.p, 0, sizeof(unsigned long long) * tiles, s), "scan status memset");
    cuda_check(cudaMemsetAsync(counter.p, 0, sizeof(uint32_t), s), "scan counter memset");
}

void scan_u32(const uint32_t* d_in, uint32_t* d_out, uint32_t n, uint32_t* d_total, ScanScratch& sc, uint32_t* d_err,
              cudaStream_t s) {
    sc.prepare(n, s);
    uint32_t tiles = std::max<uint32_t>(1, scan_tiles(n));
    ScanState st{sc.status.as<unsigned long long>(), sc.counter.as<uint32_t>(), d_err, kLookbackSpinLimit};
    k_scan_u32<<<tiles, kScanThreads, 0, s>>>(d_in, d_out, n, st, d_total);
    cuda_check(cudaGetLastError(), "k_scan_u32");
}

void select_u8(const uint8_t* d_mask, uint32_t n, uint32_t* d_out, uint32_t* d_count, ScanScratch& sc, uint32_t* d_err,
               cudaStream_t s) {
    sc.prepare(n, s);
    uint32_t tiles = std::max<uint32_t>(1, scan_tiles(n));
    ScanState st{sc.status.as<unsigned long long>(), sc.counter.as<uint32_t>(), d_err, kLookbackSpinLimit};
    k_select_u8<<<tiles, kScanThreads, 0, s>>>(d_mask, n, d_out, d_count, st);
    cuda_check(cudaGetLastError(), "k_select_u8");
}

void select_u8_raw(const uint8_t* d_mask, uint32_t n, uint32_t* d_out, uint32_t* d_count,
                   unsigned long long* d_status, uint32_t* d_counter, uint32_t* d_err, cudaStream_t s) {
    uint32_t tiles = std::max<uint32_t>(1, scan_tiles(n));
    ScanState st{d_status, d_counter, d_err, kLookbackSpinLimit};
    k_select_u8<<<tiles, kScanThreads, 0, s>>>(d_mask, n, d_out, d_count, st);
    cuda_check(cudaGetLastError(), "k_select_u8");
}

// The compaction of n zero flags with tile 0's look-back word never
// published: the tile counter starts at 1, so no block takes tile 0 and every
// tile's look-back waits on a word nothing writes.  Each wait gives up after
// spin_limit polls and sets kErrLookback in *d_err; the tiles then publish
// and return.  Every access stays in bounds: tiles 1..T (T = tiles of n) use
// status words 1..T of the T + 1 zeroed here, read no flags past n and write
// no indices (no flag is set).  d_mask: n zero bytes; d_out, d_count: one
// word each; *d_err zeroed by the caller.
void lookback_timeout_probe(const uint8_t* d_mask, uint32_t n, uint32_t spin_limit, uint32_t* d_out,
                            uint32_t* d_count, ScanScratch& sc, uint32_t* d_err, cudaStream_t s) {
    const uint32_t tiles = std::max<uint32_t>(1, scan_tiles(n));
    sc.prepare((tiles + 1) * (uint32_t) kScanTile, s);  // tiles + 1 zeroed words, counter 0
    static const uint32_t one = 1;
    cuda_check(cudaMemcpyAsync(sc.counter.p, &one, sizeof(one), cudaMemcpyHostToDevice, s), "counter seed");
    ScanState st{sc.status.as<unsigned long long>(), sc.counter.as<uint32_t>(), d_err, spin_limit};
    k_select_u8<<<tiles, kScanThreads, 0, s>>>(d_mask, n, d_out, d_count, st);
    cuda_check(cudaGetLastError(), "k_select_u8 (timeout probe)");
}

// ---------------------------------------------------------------- prim boxes
__global__ void k_tri_boxes(const float* __restrict__ v, const uint32_t* __restrict__ t, uint32_t n, float4* lo,
                            float4* hi) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = v + 3ull * t[3ull * i];
    const float* b = v + 3ull * t[3ull * i + 1];
    const float* c = v + 3ull * t[3ull * i + 2];
    lo[i] = make_float4(fminf(a[0], fminf(b[0], c[0])), fminf(a[1], fminf(b[1], c[1])), fminf(a[2], fminf(b[2], c[2])), 0.f);
    hi[i] = make_float4(fmaxf(a[0], fmaxf(b[0], c[0])), fmaxf(a[1], fmaxf(b[1], c[1])), fmaxf(a[2], fmaxf(b[2], c[2])), 0.f);
}

__global__ void k_edge_boxes(const float* __restrict__ v, const uint32_t* __restrict__ e, uint32_t n, float4* lo,
                             float4* hi) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = v + 3ull * e[2ull * i];
    const float* b = v + 3ull * e[2ull * i + 1];
    lo[i] = make_float4(fminf(a[0], b[0]), fminf(a[1], b[1]), fminf(a[2], b[2]), 0.f);
    hi[i] = make_float4(fmaxf(a[0], b[0]), fmaxf(a[1], b[1]), fmaxf(a[2], b[2]), 0.f);
}

void tri_boxes(const float* d_verts, const uint32_t* d_tris, uint32_t n, float4* d_lo, float4* d_hi, cudaStream_t s) {
    if (!n) return;
    k_tri_boxes<<<(n + 255) / 256, 256, 0, s>>>(d_verts, d_tris, n, d_lo, d_hi);
    cuda_check(cudaGetLastError(), "k_tri_boxes");
}

void edge_boxes(const float* d_verts, const uint32_t* d_edges, uint32_t n, float4* d_lo, float4* d_hi, cudaStream_t s) {
    if (!n) return;
    k_edge_boxes<<<(n + 255) / 256, 256, 0, s>>>(d_verts, d_edges, n, d_lo, d_hi);
    cuda_check(cudaGetLastError(), "k_edge_boxes");
}

__global__ void k_gather_tris(const float* __restrict__ v, const uint32_t* __restrict__ t,
                              const uint32_t* __restrict__ perm, uint32_t n, uint32_t id_base, uint32_t group,
                              const uint32_t* __restrict__ tag, float4* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t p = perm[i];
    const float* a = v + 3ull * t[3ull * p];
    const float* b = v + 3ull * t[3ull * p + 1];
    const float* c = v + 3ull * t[3ull * p + 2];
    out[3ull * i] = make_float4(a[0], a[1], a[2], __uint_as_float(id_base + p));
    out[3ull * i + 1] = make_float4(b[0], b[1], b[2], __uint_as_float(group));
    out[3ull * i + 2] = make_float4(c[0], c[1], c[2], __uint_as_float(tag ? tag[p] : 0u));
}

__global__ void k_gather_edges(const float* __restrict__ v, const uint32_t* __restrict__ e,
                               const uint32_t* __restrict__ perm, uint32_t n, uint32_t id_base, uint32_t group,
                               float4* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t p = perm[i];
    const float* a = v + 3ull * e[2ull * p];
    const float* b = v + 3ull * e[2ull * p + 1];
    out[2ull * i] = make_float4(a[0], a[1], a[2], __uint_as_float(id_base + p));
    out[2ull * i + 1] = make_float4(b[0], b[1], b[2], __uint_as_float(group));
}

void gather_tris(const float* d_verts, const uint32_t* d_tris, const uint32_t* d_perm, uint32_t n, uint32_t id_base,
                 uint32_t group, const uint32_t* d_tag, float4* d_out, cudaStream_t s) {
    if (!n) return;
    k_gather_tris<<<(n + 255) / 256, 256, 0, s>>>(d_verts, d_tris, d_perm, n, id_base, group, d_tag, d_out);
    cuda_check(cudaGetLastError(), "k_gather_tris");
}

void gather_edges(const float* d_verts, const uint32_t* d_edges, const uint32_t* d_perm, uint32_t n, uint32_t id_base,
                  uint32_t group, float4* d_out, cudaStream_t s) {
    if (!n) return;
    k_gather_edges<<<(n + 255) / 256, 256, 0, s>>>(d_verts, d_edges, d_perm, n, id_base, group, d_out);
    cuda_check(cudaGetLastError(), "k_gather_edges");
}

// ---------------------------------------------------------------- Morton codes
__device__ __forceinline__ uint32_t fenc(float f) {
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float fdec(uint32_t e) {
    uint32_t b = (e & 0x80000000u) ? (e & 0x7fffffffu) : ~e;
    return __uint_as_float(b);
}

__device__ __forceinline__ float centroid(float lo, float hi) { return __fmul_rn(0.5f, __fadd_rn(lo, hi)); }

// bounds[0..2] = encoded min, bounds[3..5] = encoded max of the centroids
__global__ void k_centroid_bounds(const float4* __restrict__ lo, const float4* __restrict__ hi, uint32_t n,
                                  uint32_t* bounds) {
    uint32_t mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 a = lo[i], b = hi[i];
        uint32_t c[3] = {fenc(centroid(a.x, b.x)), fenc(centroid(a.y, b.y)), fenc(centroid(a.z, b.z))};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            mn[k] = min(mn[k], c[k]);
            mx[k] = max(mx[k], c[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
            mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            atomicMin(bounds + k, mn[k]);
            atomicMax(bounds + 3 + k, mx[k]);
        }
    }
}

__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__device__ __forceinline__ uint32_t quantize(float c, float lo, float ext) {
    float t = ext > 0.0f ? __fdiv_rn(__fsub_rn(c, lo), ext) : 0.0f;
    float v = __fmul_rn(t, 1024.0f);
    if (!(v >= 0.0f)) v = 0.0f;
    uint32_t q = (uint32_t) floorf(v);
    return q > 1023u ? 1023u : q;
}

__global__ void k_morton(const float4* __restrict__ lo, const float4* __restrict__ hi, uint32_t n,
                         const uint32_t* __restrict__ bounds, uint32_t* codes, uint32_t* idx) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float clo[3], ext[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        clo[k] = fdec(bounds[k]);
        ext[k] = __fsub_rn(fdec(bounds[3 + k]), clo[k]);
    }
    float4 a = lo[i], b = hi[i];
    uint32_t qx = quantize(centroid(a.x, b.x), clo[0], ext[0]);
    uint32_t qy = quantize(centroid(a.y, b.y), clo[1], ext[1]);
    uint32_t qz = quantize(centroid(a.z, b.z), clo[2], ext[2]);
    codes[i] = (expand_bits(qx) << 2) | (expand_bits(qy) << 1) | expand_bits(qz);
    idx[i] = i;
}

// ---------------------------------------------------------------- radix sort
// Stable LSD radix sort of (code, index) pairs in the Onesweep form (Adinets
// and Merrill, "Onesweep: A Faster Least Significant Digit Radix Sort for
// GPUs", 2022): one kernel counts the digits of every pass at once, then each
// 8-bit pass is a single kernel - a tile (2048 keys, its index taken from an
// atomic counter) ranks its keys stably, publishes its per-digit counts,
// looks back over the tiles before it for each digit's running prefix
// (decoupled look-back, one thread per digit) and scatters.  No per-pass
// histogram or scan kernel, no host round trip.
constexpr int kRsThreads = 256;
constexpr int kRsRounds = 8;
constexpr int kRsTile = kRsThreads * kRsRounds;
constexpr int kRsPasses = 4;  // 30-bit codes: digits at bits 0, 8, 16, 24
constexpr uint32_t kRsAgg = 1u << 30, kRsInc = 2u << 30, kRsCount = (1u << 30) - 1u;

// Digit counts of every pass: ghist[pass][digit].
__global__ void __launch_bounds__(kRsThreads) k_rs_hist_all(const uint32_t* __restrict__ keys, uint32_t n,
                                                           uint32_t* __restrict__ ghist) {
    __shared__ uint32_t h[kRsPasses][256];
    for (int p = 0; p < kRsPasses; ++p) h[p][threadIdx.x] = 0;
    __syncthreads();
    for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x) {
        const uint32_t k = keys[i];
#pragma unroll
        for (int p = 0; p < kRsPasses; ++p) atomicAdd(&h[p][(k >> (8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int p = 0; p < kRsPasses; ++p)
        if (h[p][threadIdx.x]) atomicAdd(ghist + p * 256 + threadIdx.x, h[p][threadIdx.x]);
}

// One pass.  status: [tile][256] words (flag << 30 | count), zeroed before
// the pass; counter: the pass's tile counter, zeroed.
__global__ void __launch_bounds__(kRsThreads) k_rs_onesweep(const uint32_t* __restrict__ kin,
                                                           const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
                                                           uint32_t* __restrict__ vout, uint32_t n, int pass,
                                                           const uint32_t* __restrict__ ghist, uint32_t* status,
                                                           uint32_t* counter, uint32_t* err) {
    constexpr int W = kRsThreads / 32;
    __shared__ uint32_t s_tile;
    __shared__ uint32_t run[256];
    __shared__ uint32_t wcnt[W][256];
    __shared__ uint32_t s_start[256];  // first position of each digit in this pass's output
    __shared__ uint32_t s_warp[W];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, shift = 8 * pass;
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1u);
    // exclusive scan of the pass's digit counts (256 digits, one per thread)
    {
        const uint32_t c = ghist[pass * 256 + threadIdx.x];
        uint32_t inc = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        if (lane == 31) s_warp[warp] = inc;
        run[threadIdx.x] = 0;
        __syncthreads();
        uint32_t before = 0;
        for (int w = 0; w < warp; ++w) before += s_warp[w];
        s_start[threadIdx.x] = before + inc - c;
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    const size_t base = (size_t) tile * kRsTile;
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t key[kRsRounds], val[kRsRounds], rank[kRsRounds];
    // stable ranks inside the tile: round by round, warp by warp, lane by lane
#pragma unroll
    for (int r = 0; r < kRsRounds; ++r) {
#pragma unroll
        for (int w = 0; w < W; ++w) wcnt[w][threadIdx.x] = 0;
        __syncthreads();
        const size_t i = base + (size_t) r * kRsThreads + threadIdx.x;
        const bool valid = i < n;
        key[r] = valid ? kin[i] : 0u;
        val[r] = valid ? vin[i] : 0u;
        const uint32_t d = valid ? ((key[r] >> shift) & 255u) : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        rank[r] = __popc(peers & lt);
        if (valid && rank[r] == 0) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        {
            const uint32_t dd = threadIdx.x;
            uint32_t acc = run[dd];
#pragma unroll
            for (int w = 0; w < W; ++w) {
                const uint32_t t = wcnt[w][dd];
                wcnt[w][dd] = acc;
                acc += t;
            }
            run[dd] = acc;
        }
        __syncthreads();
        if (valid) rank[r] += wcnt[warp][d];
        __syncthreads();  // wcnt is cleared by the next round
    }
    // publish this tile's count of digit d, look back for the count of d in the tiles before it
    {
        const uint32_t d = threadIdx.x, cnt = run[d];
        volatile uint32_t* st = status;
        uint32_t excl = 0;
        if (tile == 0) {
            atomicExch(status + d, kRsInc | cnt);
        } else {
            atomicExch(status + (size_t) tile * 256 + d, kRsAgg | cnt);
            long long p = (long long) tile - 1;
            uint32_t spins = 0;
            while (p >= 0) {
                const uint32_t w = st[(size_t) p * 256 + d];
                if ((w & ~kRsCount) == 0) {
                    if (++spins > kLookbackSpinLimit) {
                        atomicOr(err, kErrLookback);
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                excl += w & kRsCount;
                if (w & kRsInc) break;
                --p;
            }
            atomicExch(status + (size_t) tile * 256 + d, kRsInc | (excl + cnt));
        }
        run[d] = s_start[d] + excl;  // the tile's first position for digit d
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRsRounds; ++r) {
        const size_t i = base + (size_t) r * kRsThreads + threadIdx.x;
        if (i < n) {
            const uint32_t pos = run[(key[r] >> shift) & 255u] + rank[r];
            kout[pos] = key[r];
            vout[pos] = val[r];
        }
    }
}

// ---------------------------------------------------------------- hierarchy
__device__ __forceinline__ int kdelta(const uint32_t* codes, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint32_t x = codes[i] ^ codes[j];
    if (x) return __clz(x);
    return 32 + __clz((uint32_t) i ^ (uint32_t) j);
}

// child refs: internal node index, or kLeaf | sorted position; parent[n-1+s] for leaves.
__global__ void k_karras(const uint32_t* __restrict__ codes, int n, uint32_t* child, uint32_t* parent) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (kdelta(codes, n, i, i + 1) - kdelta(codes, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = kdelta(codes, n, i, i - d);
    int lmax = 2;
    while (kdelta(codes, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (kdelta(codes, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = kdelta(codes, n, i, j);
    int s = 0;
    for (int div = 2;; div *= 2) {
        int t = (l + div - 1) / div;
        if (kdelta(codes, n, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    int g = i + s * d + (d < 0 ? -1 : 0);
    int lo = min(i, j), hi = max(i, j);
    uint32_t left = (lo == g) ? (kLeaf | (uint32_t) g) : (uint32_t) g;
    uint32_t right = (hi == g + 1) ? (kLeaf | (uint32_t) (g + 1)) : (uint32_t) (g + 1);
    child[2 * i] = left;
    child[2 * i + 1] = right;
    parent[(left & kLeaf) ? (n - 1 + (left & ~kLeaf)) : left] = (uint32_t) i;
    parent[(right & kLeaf) ? (n - 1 + (right & ~kLeaf)) : right] = (uint32_t) i;
}

__device__ __forceinline__ void child_box(uint32_t ref, const uint32_t* perm, const float4* plo, const float4* phi,
                                          const float4* nlo, const float4* nhi, float4& lo, float4& hi) {
    if (ref & kLeaf) {
        uint32_t p = perm[ref & ~kLeaf];
        lo = plo[p];
        hi = phi[p];
    } else {
        lo = __ldcg(nlo + ref);
        hi = __ldcg(nhi + ref);
    }
}

// Bottom-up fit: the second thread to reach a node computes its box.
__global__ void k_fit(const uint32_t* __restrict__ child, const uint32_t* __restrict__ parent,
                      const uint32_t* __restrict__ perm, const float4* __restrict__ plo, const float4* __restrict__ phi,
                      int n, float4* nlo, float4* nhi, uint32_t* visits) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    uint32_t node = parent[n - 1 + s];
    for (int guard = 0; guard < 2 * n + 2; ++guard) {
        __threadfence();
        if (atomicAdd(visits + node, 1u) == 0) return;
        float4 al, ah, bl, bh;
        child_box(child[2 * node], perm, plo, phi, nlo, nhi, al, ah);
        child_box(child[2 * node + 1], perm, plo, phi, nlo, nhi, bl, bh);
        float4 lo = make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), 0.f);
        float4 hi = make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.f);
        __stcg(nlo + node, lo);
        __stcg(nhi + node, hi);
        if (node == 0) return;
        node = parent[node];
    }
}

__global__ void k_leaf_depth(const uint32_t* __restrict__ parent, int n, uint32_t* max_depth) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    uint32_t node = parent[n - 1 + s], d = 1;
    while (node != 0 && d < 4096u) {
        node = parent[node];
        ++d;
    }
    atomicMax(max_depth, d);
}

__global__ void k_pack(const uint32_t* __restrict__ child, const uint32_t* __restrict__ perm,
                       const float4* __restrict__ plo, const float4* __restrict__ phi, const float4* __restrict__ nlo,
                       const float4* __restrict__ nhi, int n, uint32_t node_offset, uint32_t prim_offset,
                       float4* nodes) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    uint32_t cl = child[2 * i], cr = child[2 * i + 1];
    float4 al, ah, bl, bh;
    child_box(cl, perm, plo, phi, nlo, nhi, al, ah);
    child_box(cr, perm, plo, phi, nlo, nhi, bl, bh);
    uint32_t rl = (cl & kLeaf) ? (kLeaf | (prim_offset + (cl & ~kLeaf))) : (node_offset + cl);
    uint32_t rr = (cr & kLeaf) ? (kLeaf | (prim_offset + (cr & ~kLeaf))) : (node_offset + cr);
    float4* o = nodes + 4ull * i;
    o[0] = make_float4(al.x, al.y, al.z, ah.x);
    o[1] = make_float4(ah.y, ah.z, bl.x, bl.y);
    o[2] = make_float4(bl.z, bh.x, bh.y, bh.z);
    o[3] = make_float4(__uint_as_float(rl), __uint_as_float(rr), 0.f, 0.f);
}

LbvhResult build_lbvh(const float4* d_lo, const float4* d_hi, uint32_t n, float4* d_nodes, uint32_t* d_perm,
                      uint32_t node_offset, uint32_t prim_offset, uint32_t* d_err, cudaStream_t s,
                      std::vector<uint32_t>* codes_out, std::vector<uint32_t>* child_out) {
    LbvhResult r;
    if (n == 0) return r;
    if (n >= (1u << 30)) fail(5, "LBVH: too many primitives");
    DevBuf bounds, codes_a, codes_b, idx_a, idx_b, hist, child, parent, nlo, nhi, visits, depth;
    bounds.ensure(6 * sizeof(uint32_t));
    uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    cuda_check(cudaMemcpyAsync(bounds.p, init, sizeof(init), cudaMemcpyHostToDevice, s), "bounds init");
    int sms = device_sm_count();
    k_centroid_bounds<<<std::max(1, std::min<int>((n + 255) / 256, sms * 4)), 256, 0, s>>>(d_lo, d_hi, n,
                                                                                           bounds.as<uint32_t>());
    codes_a.ensure(4ull * n); codes_b.ensure(4ull * n); idx_a.ensure(4ull * n); idx_b.ensure(4ull * n);
    k_morton<<<(n + 255) / 256, 256, 0, s>>>(d_lo, d_hi, n, bounds.as<uint32_t>(), codes_a.as<uint32_t>(),
                                             idx_a.as<uint32_t>());
    cuda_check(cudaGetLastError(), "k_morton");
    const uint32_t tiles = (n + kRsTile - 1) / kRsTile;
    // one zeroed block: the digit counts of every pass [4][256], the tile counters [4] and the
    // look-back words of every pass [4][tiles][256]
    const size_t words = (size_t) kRsPasses * 256 + kRsPasses + (size_t) kRsPasses * tiles * 256;
    hist.ensure(4 * words);
    cuda_check(cudaMemsetAsync(hist.p, 0, 4 * words, s), "radix memset");
    uint32_t* ghist = hist.as<uint32_t>();
    uint32_t* counters = ghist + kRsPasses * 256;
    uint32_t* status = counters + kRsPasses;
    uint32_t *ka = codes_a.as<uint32_t>(), *kb = codes_b.as<uint32_t>(), *va = idx_a.as<uint32_t>(),
             *vb = idx_b.as<uint32_t>();
    k_rs_hist_all<<<std::max(1, std::min<int>((int) tiles, sms * 4)), kRsThreads, 0, s>>>(ka, n, ghist);
    for (int pass = 0; pass < kRsPasses; ++pass) {
        k_rs_onesweep<<<tiles, kRsThreads, 0, s>>>(ka, va, kb, vb, n, pass, ghist, status + (size_t) pass * tiles * 256,
                                                  counters + pass, d_err);
        cuda_check(cudaGetLastError(), "radix pass");
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    cuda_check(cudaMemcpyAsync(d_perm, va, 4ull * n, cudaMemcpyDeviceToDevice, s), "perm copy");
    if (codes_out) {
        codes_out->resize(n);
        cuda_check(cudaMemcpyAsync(codes_out->data(), ka, 4ull * n, cudaMemcpyDeviceToHost, s), "codes download");
    }
    if (n == 1) {
        cuda_check(cudaStreamSynchronize(s), "lbvh sync");
        r.root = kLeaf | prim_offset;
        r.depth = 0;
        return r;
    }
    child.ensure(8ull * (n - 1));
    parent.ensure(4ull * (2 * n - 1));
    nlo.ensure(16ull * (n - 1));
    nhi.ensure(16ull * (n - 1));
    visits.ensure(4ull * (n - 1));
    depth.ensure(4);
    cuda_check(cudaMemsetAsync(visits.p, 0, 4ull * (n - 1), s), "visits memset");
    cuda_check(cudaMemsetAsync(depth.p, 0, 4, s), "depth memset");
    k_karras<<<(n - 1 + 255) / 256, 256, 0, s>>>(ka, (int) n, child.as<uint32_t>(), parent.as<uint32_t>());
    k_fit<<<(n + 255) / 256, 256, 0, s>>>(child.as<uint32_t>(), parent.as<uint32_t>(), d_perm, d_lo, d_hi, (int) n,
                                          nlo.as<float4>(), nhi.as<float4>(), visits.as<uint32_t>());
    k_leaf_depth<<<(n + 255) / 256, 256, 0, s>>>(parent.as<uint32_t>(), (int) n, depth.as<uint32_t>());
    k_pack<<<(n - 1 + 255) / 256, 256, 0, s>>>(child.as<uint32_t>(), d_perm, d_lo, d_hi, nlo.as<float4>(),
                                               nhi.as<float4>(), (int) n, node_offset, prim_offset, d_nodes);
    cuda_check(cudaGetLastError(), "lbvh hierarchy");
    if (child_out) {
        child_out->resize(2ull * (n - 1));
        cuda_check(cudaMemcpyAsync(child_out->data(), child.p, 8ull * (n - 1), cudaMemcpyDeviceToHost, s),
                   "child download");
    }
    uint32_t dep = 0;
    cuda_check(cudaMemcpyAsync(&dep, depth.p, 4, cudaMemcpyDeviceToHost, s), "depth download");
    cuda_check(cudaStreamSynchronize(s), "lbvh sync");
    r.root = node_offset;
    r.depth = dep;
    if (dep > (uint32_t) kMaxTreeDepth) fail(5, "LBVH deeper than the traversal stack (" + std::to_string(dep) + ")");
    return r;
}

// ------------------------------------------------------------ 4-wide tree
// Greedy surface-area collapse of a binary tree into a 4-wide one: a wide
// node starts from a binary node's two children and repeatedly opens its
// largest internal child (by box surface area) until it holds four children
// or only leaves.  Wide nodes are numbered breadth-first, so the top levels
// share cache lines.  The tree is built once per scene on the host from the
// downloaded binary nodes (about a million node visits for a 430k-triangle
// scene).
static inline uint32_t host_f2u(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
static inline float host_u2f(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

WideResult build_wide(const float4* d_nodes, uint32_t n_nodes, uint32_t root, DevBuf& out, cudaStream_t s) {
    WideResult r;
    r.root = root;
    if (root == kNone || (root & kLeaf)) return r;  // empty, or one primitive: no wide nodes
    std::vector<float4> h(4ull * n_nodes);
    cuda_check(cudaMemcpyAsync(h.data(), d_nodes, 64ull * n_nodes, cudaMemcpyDeviceToHost, s), "binary nodes download");
    cuda_check(cudaStreamSynchronize(s), "binary nodes download");
    struct Kid {
        uint32_t ref;
        float lo[3], hi[3];
    };
    auto kids_of = [&](uint32_t i, Kid* k) {
        if (i >= n_nodes) fail(5, "4-wide build: binary child reference out of range");
        const float4 a = h[4ull * i], b = h[4ull * i + 1], c = h[4ull * i + 2], d = h[4ull * i + 3];
        k[0] = {host_f2u(d.x), {a.x, a.y, a.z}, {a.w, b.x, b.y}};
        k[1] = {host_f2u(d.y), {b.z, b.w, c.x}, {c.y, c.z, c.w}};
    };
    auto area = [](const Kid& k) {
        const float dx = std::max(0.f, k.hi[0] - k.lo[0]), dy = std::max(0.f, k.hi[1] - k.lo[1]),
                    dz = std::max(0.f, k.hi[2] - k.lo[2]);
        return dx * dy + dy * dz + dz * dx;
    };
    std::vector<std::pair<uint32_t, uint32_t>> queue;  // (binary node, wide depth)
    queue.reserve(n_nodes / 2 + 1);
    queue.emplace_back(root, 0u);
    std::vector<float4> wide;
    wide.reserve(4ull * n_nodes);
    for (size_t qi = 0; qi < queue.size(); ++qi) {
        const uint32_t depth = queue[qi].second;
        r.depth = std::max(r.depth, depth);
        Kid k[kWide];
        int nk = 2;
        kids_of(queue[qi].first, k);
        while (nk < kWide) {
            int best = -1;
            float best_area = -1.f;
            for (int j = 0; j < nk; ++j)
                if (!(k[j].ref & kLeaf) && area(k[j]) > best_area) {
                    best = j;
                    best_area = area(k[j]);
                }
            if (best < 0) break;
            Kid two[2];
            kids_of(k[best].ref, two);
            k[best] = two[0];
            k[nk++] = two[1];
        }
        for (int j = 0; j < kWide; ++j) {
            if (j >= nk) {  // empty slot: an inverted box and no reference
                wide.push_back(make_float4(3e38f, 3e38f, 3e38f, -3e38f));
                wide.push_back(make_float4(-3e38f, -3e38f, host_u2f(kNone), 0.f));
                continue;
            }
            uint32_t ref = k[j].ref;
            if (!(ref & kLeaf)) {
                if (queue.size() >= (size_t) kLeaf) fail(5, "4-wide build: too many nodes");
                queue.emplace_back(ref, depth + 1);
                ref = (uint32_t) (queue.size() - 1);
            }
            wide.push_back(make_float4(k[j].lo[0], k[j].lo[1], k[j].lo[2], k[j].hi[0]));
            wide.push_back(make_float4(k[j].hi[1], k[j].hi[2], host_u2f(ref), 0.f));
        }
    }
    r.nodes = (uint32_t) queue.size();
    r.root = 0;
    // the top cut: the root's records, each internal one replaced by its node's records, level
    // by level while the list stays within kWideCut records
    std::vector<uint32_t> cut;  // record indices (node * kWide + slot)
    for (int j = 0; j < kWide; ++j)
        if (host_f2u(wide[2 * j + 1].z) != kNone) cut.push_back((uint32_t) j);
    while (true) {
        std::vector<uint32_t> next;
        bool opened = false;
        for (uint32_t rec : cut) {
            const uint32_t ref = host_f2u(wide[2ull * rec + 1].z);
            if (ref & kLeaf) {
                next.push_back(rec);
                continue;
            }
            opened = true;
            for (int j = 0; j < kWide; ++j)
                if (host_f2u(wide[2ull * (kWide * ref + j) + 1].z) != kNone) next.push_back(kWide * ref + j);
        }
        if (!opened || next.size() > (size_t) kWideCut) break;
        cut.swap(next);
    }
    for (uint32_t rec : cut) {
        r.cut.push_back(wide[2ull * rec]);
        r.cut.push_back(wide[2ull * rec + 1]);
    }
    out.ensure(wide.size() * sizeof(float4));
    cuda_check(cudaMemcpyAsync(out.p, wide.data(), wide.size() * sizeof(float4), cudaMemcpyHostToDevice, s),
               "wide nodes upload");
    cuda_check(cudaStreamSynchronize(s), "wide nodes upload");
    return r;
}

}  // namespace rtcd
