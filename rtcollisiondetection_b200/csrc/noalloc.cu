// noalloc.cu - stream compaction that allocates nothing.
//
// Some callers cannot allocate device memory at the moment they need a
// query: a robot control loop with a hard deadline cannot afford cudaMalloc
// or cudaFree (both may synchronise the whole device and take unbounded
// time), and a host process whose device memory is handed out by another
// owner (a fixed pool partitioned at start-up) has no allocation rights at
// all.  rtcd_select_flags_u8_noalloc gives them the look-back compaction of
// rtcd_select_flags_u8 with its scratch (one look-back word per 2048 flags, a
// tile counter and an error word) in a fixed file-scope device array instead
// of a cudaMalloc'd buffer.  The array is part of the library's device image:
// every GPU that loads the library holds it (131 KB) until the process exits.
#include <mutex>

#include "../../include/rtcd.h"
#include "engine.h"

namespace {

constexpr uint32_t kMaxTiles = 16384;                               // look-back words
constexpr uint64_t kMaxFlags = (uint64_t) kMaxTiles * rtcd::kSelectTileFlags;  // 33,554,432

// [0, kMaxTiles): look-back status words; [kMaxTiles]: tile counter (low
// half); [kMaxTiles + 1]: device error word (low half).
static __device__ __align__(256) unsigned long long g_select_scratch[kMaxTiles + 2];

std::mutex g_mu;  // serialises calls of this process

}  // namespace

extern "C" RTCD_API rtcd_status rtcd_select_flags_u8_noalloc(const uint8_t* mask_dev, uint32_t n, uint32_t* idx_dev,
                                                             uint32_t* count_dev, void* stream) {
    try {
        if (!count_dev || (n && (!mask_dev || !idx_dev)))
            rtcd::fail(RTCD_ERR_INVALID_ARGUMENT, "rtcd_select_flags_u8_noalloc: NULL argument");
        if ((uint64_t) n > kMaxFlags)
            rtcd::fail(RTCD_ERR_CAPACITY, "rtcd_select_flags_u8_noalloc: n = " + std::to_string(n) +
                                              " exceeds the static scratch limit of 33554432 flags");
        cudaStream_t s = (cudaStream_t) stream;
        std::lock_guard<std::mutex> lock(g_mu);
        // The host-side name of the array is not a device address: ask the
        // runtime for the address on the calling (current) device.  The lookup
        // is repeated on every call rather than cached, so a context that was
        // torn down and re-created (cudaDeviceReset) never leaves a stale
        // address behind; on a device's first call it may also load this
        // library's device code there.
        void* p = nullptr;
        rtcd::cuda_check(cudaGetSymbolAddress(&p, g_select_scratch), "cudaGetSymbolAddress");
        unsigned long long* base = static_cast<unsigned long long*>(p);
        uint32_t tiles = n ? (uint32_t) ((n + rtcd::kSelectTileFlags - 1) / rtcd::kSelectTileFlags) : 1u;
        // the previous call left its words behind: clear the ones this call uses
        rtcd::cuda_check(cudaMemsetAsync(base, 0, sizeof(unsigned long long) * tiles, s), "scratch clear");
        rtcd::cuda_check(cudaMemsetAsync(base + kMaxTiles, 0, 2 * sizeof(unsigned long long), s), "scratch clear");
        uint32_t* counter = reinterpret_cast<uint32_t*>(base + kMaxTiles);
        uint32_t* err = reinterpret_cast<uint32_t*>(base + kMaxTiles + 1);
        rtcd::select_u8_raw(mask_dev, n, idx_dev, count_dev, base, counter, err, s);
        uint32_t e = 0;
        rtcd::cuda_check(cudaMemcpyAsync(&e, err, sizeof(e), cudaMemcpyDeviceToHost, s), "error word read");
        rtcd::cuda_check(cudaStreamSynchronize(s), "stream sync");
        if (e) rtcd::fail(RTCD_ERR_DEVICE_TIMEOUT, "rtcd_select_flags_u8_noalloc: look-back wait ran out");
        rtcd::set_last_error("");
        return RTCD_OK;
    } catch (const rtcd::Error& e) {
        rtcd::set_last_error(e.msg);
        return (rtcd_status) e.status;
    } catch (...) {
        rtcd::set_last_error("rtcd_select_flags_u8_noalloc: unexpected error");
        return RTCD_ERR_INTERNAL;
    }
}
