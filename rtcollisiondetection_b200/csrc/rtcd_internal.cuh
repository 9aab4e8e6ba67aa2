// rtcd_internal.cuh - shared device structures and helpers of the B200 engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace rtcd {

constexpr int kMaxDof = 15;
constexpr int kMaxLinks = kMaxDof + 1;
constexpr int kStack = 64;                 // per-lane traversal stack entries
constexpr uint32_t kLeaf = 0x80000000u;    // child reference: leaf flag | sorted primitive index
constexpr uint32_t kNone = 0xFFFFFFFFu;    // empty tree
constexpr int kMaxTreeDepth = kStack - 2;  // builders reject deeper trees
constexpr int kWide = 4;                    // children per node of the scene's wide trees
constexpr int kWideCut = 64;                // child records in a wide tree's top cut

// Entries a 32-wide LIFO frontier over a kWide-ary tree can hold when every
// step pops min(size, 32) entries and pushes their internal children, for a
// tree whose deepest internal node is at depth `depth`: each step's pushes
// are one segment of at most 32 * kWide entries; the step after it pops 32 of
// them (or all), so every segment below the top keeps at most
// 32 * (kWide - 1); and the smallest depth in each live segment exceeds the
// one below it, so at most depth + 1 segments are live.  A descent that
// starts from a top cut of at most kWideCut <= 32 * kWide records obeys the
// same bound.
__host__ __device__ constexpr uint32_t wide_frontier(uint32_t depth) {
    return 32u * (kWide - 1) * depth + 32u * kWide;
}

// device error word bits
constexpr uint32_t kErrStack = 1u << 0;
constexpr uint32_t kErrLookback = 1u << 1;
constexpr uint32_t kErrRange = 1u << 2;

// Packed LBVH node (64 B): the boxes of both children live in the parent so
// one 64-byte load decides both descents.
//   n[0] = (L.lo.x, L.lo.y, L.lo.z, L.hi.x)
//   n[1] = (L.hi.y, L.hi.z, R.lo.x, R.lo.y)
//   n[2] = (R.lo.z, R.hi.x, R.hi.y, R.hi.z)
//   n[3] = (bits(left ref), bits(right ref), 0, 0)
struct Box {
    float lo[3], hi[3];
};

__device__ __forceinline__ void load_node(const float4* __restrict__ nodes, uint32_t i, Box& l, Box& r, uint32_t& cl,
                                          uint32_t& cr) {
    const float4* p = nodes + 4ull * i;
    float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
    l.lo[0] = a.x; l.lo[1] = a.y; l.lo[2] = a.z; l.hi[0] = a.w;
    l.hi[1] = b.x; l.hi[2] = b.y; r.lo[0] = b.z; r.lo[1] = b.w;
    r.lo[2] = c.x; r.hi[0] = c.y; r.hi[1] = c.z; r.hi[2] = c.w;
    cl = __float_as_uint(d.x);
    cr = __float_as_uint(d.y);
}

// Adds a per-lane count to a device counter with one atomic per warp, none
// when the warp's total is zero (per-thread atomics on one address at the
// end of a large grid serialise in L2 for a noticeable time).  Every lane of
// the warp must call it; per-lane counts fit 32 bits.
// Work counters of a check (64-bit words on the device).  Two banks of
// kStatBank words with the same layout: bank 0 for the first traversal kernel
// of a check (the fused or stage-A discrete kernel, the light sweep pass) and
// the cull, bank 1 for the passes that follow (subtree, deferred and heavy
// candidates, the overflow fallback, the heavy sweep pass).
constexpr int kStatBank = 16;
constexpr int kStatWords = 2 * kStatBank;
constexpr int kStatCullSpheres = 8;   // bank 0: bounding-sphere tests of the OBB cull
constexpr int kStatCullSats = 9;      // bank 0: 15-axis SATs the cull evaluated

__device__ __forceinline__ void warp_count(unsigned long long* p, unsigned long long v) {
    const unsigned total = __reduce_add_sync(0xffffffffu, (unsigned) v);
    if ((threadIdx.x & 31) == 0 && total) atomicAdd(p, (unsigned long long) total);
}

__device__ __forceinline__ bool box_overlap(const Box& b, const float* lo, const float* hi) {
    return !(lo[0] > b.hi[0] || hi[0] < b.lo[0] || lo[1] > b.hi[1] || hi[1] < b.lo[1] || lo[2] > b.hi[2] ||
             hi[2] < b.lo[2]);
}

// Robot chain, passed by value as a kernel parameter (lives in the constant bank).
struct Chain {
    int dof;
    float base[12];
    float cm[kMaxDof * 12], sm[kMaxDof * 12], om[kMaxDof * 12];
};

// 3x4 affine product R = A * L (L's translation added after rotation).
__device__ __forceinline__ void affine_mul(const float* A, const float* L, float* R) {
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float v = A[r * 4 + 0] * L[c] + A[r * 4 + 1] * L[4 + c] + A[r * 4 + 2] * L[8 + c];
            if (c == 3) v += A[r * 4 + 3];
            R[r * 4 + c] = v;
        }
    }
}

// Forward kinematics of one configuration; T receives (dof + 1) transforms.
__device__ __forceinline__ void fk_chain(const Chain& ch, const float* q, float (*T)[12]) {
#pragma unroll
    for (int k = 0; k < 12; ++k) T[0][k] = ch.base[k];
    for (int i = 0; i < ch.dof; ++i) {
        float s, c;
        sincosf(q[i], &s, &c);
        float L[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) L[k] = c * ch.cm[i * 12 + k] + s * ch.sm[i * 12 + k] + ch.om[i * 12 + k];
        affine_mul(T[i], L, T[i + 1]);
    }
}

struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ f3 f3of(float4 v) { return mk(v.x, v.y, v.z); }

struct d3 {
    double x, y, z;
};
__device__ __forceinline__ d3 dk(double x, double y, double z) { return d3{x, y, z}; }
__device__ __forceinline__ d3 operator-(d3 a, d3 b) { return dk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ d3 operator+(d3 a, d3 b) { return dk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ d3 operator*(d3 a, double s) { return dk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 cross(d3 a, d3 b) {
    return dk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ d3 d3of(f3 a) { return dk(a.x, a.y, a.z); }

// x_world = T x (T: 3 rows of float4 [R | t])
__device__ __forceinline__ f3 xf(const float4* T, f3 p) {
    return mk(T[0].x * p.x + T[0].y * p.y + T[0].z * p.z + T[0].w, T[1].x * p.x + T[1].y * p.y + T[1].z * p.z + T[1].w,
              T[2].x * p.x + T[2].y * p.y + T[2].z * p.z + T[2].w);
}
// x_local = R^T (x - t)
__device__ __forceinline__ f3 xf_inv(const float4* T, f3 p) {
    f3 q = mk(p.x - T[0].w, p.y - T[1].w, p.z - T[2].w);
    return mk(T[0].x * q.x + T[1].x * q.y + T[2].x * q.z, T[0].y * q.x + T[1].y * q.y + T[2].y * q.z,
              T[0].z * q.x + T[1].z * q.y + T[2].z * q.z);
}
__device__ __forceinline__ d3 xf_d(const float4* T, f3 p) {
    d3 q = d3of(p);
    return dk((double) T[0].x * q.x + (double) T[0].y * q.y + (double) T[0].z * q.z + (double) T[0].w,
              (double) T[1].x * q.x + (double) T[1].y * q.y + (double) T[1].z * q.z + (double) T[1].w,
              (double) T[2].x * q.x + (double) T[2].y * q.y + (double) T[2].z * q.z + (double) T[2].w);
}

}  // namespace rtcd
