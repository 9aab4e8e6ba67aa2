// scan.cuh - single-pass exclusive scan and stream compaction with decoupled
// look-back (Merrill & Garland, "Single-pass Parallel Prefix Scan with
// Decoupled Look-back", 2016).
//
// Replaces the upstream scan/compaction steps: the three-pass uint4 scan and
// the CUB ExclusiveSum wrapper (RTCD/Utils/cuda/cudaAlgorithms.cu:18-220), the
// flag compaction copies (RTCD/Utils/cuda/streamCompact.inl:12-89) and the
// CUB DeviceSelect::FlaggedIf calls (RTCD/Robot/robot.cu:502-529).  Unlike the
// upstream path, the compacted count stays on the device: no host round trip.
//
// Tiles take their index from an atomic counter so a tile only ever waits on
// tiles that started before it; every wait is bounded and reports kErrLookback.
#pragma once
#include "rtcd_internal.cuh"

namespace rtcd {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr uint32_t kLookbackSpinLimit = 1u << 24;

struct ScanState {
    unsigned long long* status;  // one word per tile: flag << 32 | value; zeroed before launch
    uint32_t* tile_counter;      // zeroed before launch
    uint32_t* error;             // device error word
    uint32_t spin_limit;         // polls of a predecessor's word before the wait gives up (kLookbackSpinLimit)
};

__device__ __forceinline__ unsigned long long scan_pack(uint32_t flag, uint32_t v) {
    return ((unsigned long long) flag << 32) | v;
}

__device__ __forceinline__ uint32_t warp_inclusive(uint32_t v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__device__ __forceinline__ uint32_t warp_sum(uint32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Exclusive prefix of `thread_sum` across the block; returns it, writes the block total.
__device__ __forceinline__ uint32_t block_exclusive(uint32_t thread_sum, uint32_t& block_total, uint32_t* smem32) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = warp_inclusive(thread_sum, lane);
    if (lane == 31) smem32[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (kScanThreads / 32) ? smem32[lane] : 0;
        uint32_t wi = warp_inclusive(w, lane);
        if (lane < (kScanThreads / 32)) smem32[lane] = wi - w;
        if (lane == (kScanThreads / 32) - 1) smem32[kScanThreads / 32] = wi;
    }
    __syncthreads();
    block_total = smem32[kScanThreads / 32];
    return smem32[warp] + inc - thread_sum;
}

// Warp 0 of the block: publish the tile aggregate, look back for the exclusive
// prefix, publish the inclusive prefix.  Returns the exclusive prefix (lane 0..31).
__device__ __forceinline__ uint32_t tile_lookback(const ScanState& st, uint32_t tile, uint32_t aggregate) {
    const int lane = threadIdx.x & 31;
    volatile unsigned long long* status = st.status;
    if (tile == 0) {
        if (lane == 0) atomicExch(st.status, scan_pack(2, aggregate));
        return 0;
    }
    if (lane == 0) atomicExch(st.status + tile, scan_pack(1, aggregate));
    uint32_t excl = 0;
    long long pred = (long long) tile - 1;
    uint32_t spins = 0;
    while (true) {
        long long idx = pred - lane;
        unsigned long long s = idx >= 0 ? status[idx] : scan_pack(2, 0);
        uint32_t flag = (uint32_t) (s >> 32);
        if (__any_sync(0xffffffffu, flag == 0)) {
            if (++spins > st.spin_limit) {
                if (lane == 0) atomicOr(st.error, kErrLookback);
                break;
            }
            __nanosleep(32);
            continue;
        }
        uint32_t inc_mask = __ballot_sync(0xffffffffu, flag == 2);
        uint32_t v = (uint32_t) s;
        if (inc_mask) {
            int first = __ffs(inc_mask) - 1;
            excl += warp_sum(lane <= first ? v : 0u);
            break;
        }
        excl += warp_sum(v);
        pred -= 32;
    }
    if (lane == 0) atomicExch(st.status + tile, scan_pack(2, excl + aggregate));
    return excl;
}

// Exclusive scan of n uint32 values; *total (optional) receives the sum.
__global__ void __launch_bounds__(kScanThreads) k_scan_u32(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                          uint32_t n, ScanState st, uint32_t* total) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[kScanThreads / 32 + 1];
    __shared__ uint32_t s_prefix;
    if (threadIdx.x == 0) s_tile = atomicAdd(st.tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const size_t base = (size_t) tile * kScanTile + (size_t) threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0u;
        sum += v[k];
    }
    uint32_t agg;
    uint32_t texcl = block_exclusive(sum, agg, s_warp);
    if (threadIdx.x < 32) {
        uint32_t e = tile_lookback(st, tile, agg);
        if (threadIdx.x == 0) s_prefix = e;
    }
    __syncthreads();
    uint32_t run = s_prefix + texcl;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (total && (size_t) (tile + 1) * kScanTile >= n && threadIdx.x == kScanThreads - 1) *total = s_prefix + agg;
}

// Stable compaction: out_idx receives every i with mask[i] != 0, in order;
// *count receives how many.
__global__ void __launch_bounds__(kScanThreads) k_select_u8(const uint8_t* __restrict__ mask, uint32_t n,
                                                           uint32_t* __restrict__ out_idx, uint32_t* count,
                                                           ScanState st) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[kScanThreads / 32 + 1];
    __shared__ uint32_t s_prefix;
    if (threadIdx.x == 0) s_tile = atomicAdd(st.tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const size_t base = (size_t) tile * kScanTile + (size_t) threadIdx.x * kScanItems;
    uint32_t bits = 0, sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        uint32_t f = (base + k < n) ? (mask[base + k] != 0) : 0u;
        bits |= f << k;
        sum += f;
    }
    uint32_t agg;
    uint32_t texcl = block_exclusive(sum, agg, s_warp);
    if (threadIdx.x < 32) {
        uint32_t e = tile_lookback(st, tile, agg);
        if (threadIdx.x == 0) s_prefix = e;
    }
    __syncthreads();
    uint32_t pos = s_prefix + texcl;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (bits & (1u << k)) out_idx[pos++] = (uint32_t) (base + k);
    if ((size_t) (tile + 1) * kScanTile >= n && threadIdx.x == kScanThreads - 1) *count = s_prefix + agg;
}

inline uint32_t scan_tiles(uint32_t n) { return (n + kScanTile - 1) / kScanTile; }

}  // namespace rtcd
