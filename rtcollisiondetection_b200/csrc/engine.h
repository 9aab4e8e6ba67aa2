// engine.h - host-side internals shared by the translation units of the engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "rtcd_internal.cuh"

namespace rtcd {

// Raised inside the engine; converted to an rtcd_status at the ABI boundary.
struct Error {
    int status;
    std::string msg;
};

[[noreturn]] void fail(int status, const std::string& msg);
void set_last_error(const std::string& msg);  // the message rtcd_last_error returns on this thread
void cuda_check(cudaError_t e, const char* what);

// Re-allocations made by DevBuf::ensure / HostBuf::ensure on the calling
// thread, and the host milliseconds they took (release + allocation).
struct GrowCounter {
    uint64_t grows = 0;
    double ms = 0;
};
GrowCounter& thread_grows();

// Grow-only device allocation.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release();
    void ensure(size_t n);  // at least n bytes; contents are lost when it grows
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// Grow-only pinned host allocation.
struct HostBuf {
    void* p = nullptr;
    size_t bytes = 0;
    HostBuf() = default;
    HostBuf(const HostBuf&) = delete;
    HostBuf& operator=(const HostBuf&) = delete;
    ~HostBuf() { release(); }
    void release();
    void ensure(size_t n);
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

template <class T>
void upload(DevBuf& b, const T* src, size_t count, cudaStream_t s) {
    b.ensure(sizeof(T) * (count ? count : 1));
    if (count) cuda_check(cudaMemcpyAsync(b.p, src, sizeof(T) * count, cudaMemcpyHostToDevice, s), "upload");
}

// Scratch for the decoupled look-back scan / select kernels.
struct ScanScratch {
    DevBuf status, counter;
    void prepare(uint32_t n_items, cudaStream_t s);  // zeroes status + counter for one launch
};

// Exclusive scan (in != out); *d_total optional.
void scan_u32(const uint32_t* d_in, uint32_t* d_out, uint32_t n, uint32_t* d_total, ScanScratch& sc, uint32_t* d_err,
              cudaStream_t s);
// Stable compaction of the indices of nonzero mask bytes.
void select_u8(const uint8_t* d_mask, uint32_t n, uint32_t* d_out, uint32_t* d_count, ScanScratch& sc, uint32_t* d_err,
               cudaStream_t s);

// The same compaction with caller-provided look-back scratch: d_status needs
// one zeroed word per 2048 flags (at least one), d_counter and d_err zeroed.
void select_u8_raw(const uint8_t* d_mask, uint32_t n, uint32_t* d_out, uint32_t* d_count,
                   unsigned long long* d_status, uint32_t* d_counter, uint32_t* d_err, cudaStream_t s);
constexpr uint32_t kSelectTileFlags = 2048;  // flags per look-back tile of the compaction kernel

// Self-test of the bounded look-back wait: a compaction whose tile 0 never
// publishes, so every wait runs out after spin_limit polls (lbvh.cu).
void lookback_timeout_probe(const uint8_t* d_mask, uint32_t n, uint32_t spin_limit, uint32_t* d_out,
                            uint32_t* d_count, ScanScratch& sc, uint32_t* d_err, cudaStream_t s);

// A packed LBVH over one primitive set.
struct LbvhResult {
    uint32_t root = kNone;  // child reference of the root
    uint32_t depth = 0;     // edges on the longest root-leaf path
};

// Builds the canonical LBVH (30-bit Morton codes of float centroids, stable
// LSD radix sort by (code, index), Karras 2012 hierarchy, bottom-up box fit)
// over n boxes.  Writes (n - 1) packed nodes at d_nodes (4 float4 each) and
// the sorted-position -> primitive permutation to d_perm.  Child references
// are offset by node_offset (internal) and prim_offset (leaves) so several
// trees can share one node/primitive array.  Synchronises `s`.
LbvhResult build_lbvh(const float4* d_lo, const float4* d_hi, uint32_t n, float4* d_nodes, uint32_t* d_perm,
                      uint32_t node_offset, uint32_t prim_offset, uint32_t* d_err, cudaStream_t s,
                      std::vector<uint32_t>* codes_out = nullptr, std::vector<uint32_t>* child_out = nullptr);

// A 4-wide tree collapsed from a binary one (lbvh.cu).  Node i is 8 float4 =
// 4 child records of 32 bytes: (lo.x, lo.y, lo.z, hi.x), (hi.y, hi.z,
// bits(ref), 0); ref = wide node index, kLeaf | sorted primitive (the binary
// tree's leaf reference), or kNone in an empty slot (whose box is inverted).
struct WideResult {
    uint32_t root = kNone;  // 0, or the binary root when it is empty or a single leaf
    uint32_t depth = 0;     // depth of the deepest wide node (root = 0)
    uint32_t nodes = 0;
    // The top cut: at most kWideCut child records (2 float4 each) that cover
    // every root-leaf path - the root's records, opened level by level while
    // they fit; a descent starts by testing these instead of the root.
    std::vector<float4> cut;
};
WideResult build_wide(const float4* d_nodes, uint32_t n_nodes, uint32_t root, DevBuf& out, cudaStream_t s);

// Primitive boxes and gathers (lbvh.cu).
void tri_boxes(const float* d_verts, const uint32_t* d_tris, uint32_t n, float4* d_lo, float4* d_hi, cudaStream_t s);
void edge_boxes(const float* d_verts, const uint32_t* d_edges, uint32_t n, float4* d_lo, float4* d_hi, cudaStream_t s);
// Sorted triangles: 3 float4 per triangle (v0 | id, v1 | group, v2 | 0).
// Triangles in tree order: 3 float4, w = original index, group, tag[index] (0 without tags).
void gather_tris(const float* d_verts, const uint32_t* d_tris, const uint32_t* d_perm, uint32_t n, uint32_t id_base,
                 uint32_t group, const uint32_t* d_tag, float4* d_out, cudaStream_t s);
// Sorted edges: 2 float4 per edge (a | id, b | group).
void gather_edges(const float* d_verts, const uint32_t* d_edges, const uint32_t* d_perm, uint32_t n, uint32_t id_base,
                  uint32_t group, float4* d_out, cudaStream_t s);

int device_sm_count();

}  // namespace rtcd
