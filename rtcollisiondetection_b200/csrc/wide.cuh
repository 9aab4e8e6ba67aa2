// wide.cuh - a warp's descent of a 4-wide tree through a shared LIFO
// frontier (the scene trees' wide copies), generic in the node-box test.
#pragma once
#include "rtcd_internal.cuh"

namespace rtcd {

constexpr int kWideBatch = 2;  // child records a lane loads before testing them (2 beat 4: fewer spills)

// One round of a wide descent: every lane tests one child record (a, b) -
// (lo.x, lo.y, lo.z, hi.x), (hi.y, hi.z, bits(ref), 0); ref kNone in an empty
// slot or a lane without a record - with test(box); overlapping internal
// children are pushed on the frontier fr[0, sp), leaves appended to cb[nc,
// ...).  Returns false, with the error flag set, if the frontier would
// overflow (which its size, derived from the tree depth, rules out).
template <class Test>
__device__ __forceinline__ bool wide_round(const float4& a, const float4& b, uint32_t* fr, int& sp, uint32_t* cb,
                                           int& nc, const Test& test, uint32_t front_cap, uint32_t* err,
                                           unsigned long long& n_node, unsigned long long& n_cand) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t ref = __float_as_uint(b.z);
    bool h = false;
    if (ref != kNone) {
        ++n_node;
        Box bx;
        bx.lo[0] = a.x; bx.lo[1] = a.y; bx.lo[2] = a.z;
        bx.hi[0] = a.w; bx.hi[1] = b.x; bx.hi[2] = b.y;
        h = test(bx);
    }
    const bool push = h && !(ref & kLeaf), emit = h && (ref & kLeaf);
    const uint32_t mp = __ballot_sync(0xffffffffu, push), me = __ballot_sync(0xffffffffu, emit);
    const int npush = __popc(mp);
    if (sp + npush > (int) front_cap) {
        if (lane == 0) atomicOr(err, kErrStack);
        return false;
    }
    if (push) fr[sp + __popc(mp & lt)] = ref;
    if (emit) cb[nc + __popc(me & lt)] = ref & ~kLeaf;
    sp += npush;
    const int nemit = __popc(me);
    nc += nemit;
    n_cand += lane == 0 ? (unsigned long long) nemit : 0ull;
    return true;
}

// One step of a warp's descent of a scene wide tree through its shared LIFO
// frontier fr[0, sp): pops up to 32 nodes and spreads their children over
// the lanes (4 lanes per node when at most 8 are waiting, 2 when at most 16,
// else one lane tests all four children of its node, so a step costs about
// one box test per lane); at most 32 * kWide leaves are appended per step.
// TOP: top / n_top are a shared-memory copy of the tree's first n_top nodes
// (they are numbered breadth-first, so these are its top levels), and records
// of those nodes are read from it instead of global memory; without TOP the
// loads are plain global loads with no branch between them.
template <bool TOP = false, class Test>
__device__ __forceinline__ bool wide_step(const float4* __restrict__ wn, uint32_t* fr, int& sp, uint32_t* cb, int& nc,
                                          const Test& test, uint32_t front_cap, uint32_t* err,
                                          unsigned long long& n_node, unsigned long long& n_cand,
                                          const float4* top = nullptr, uint32_t n_top = 0) {
    const int lane = threadIdx.x & 31;
    const int lg = sp <= 8 ? 2 : (sp <= 16 ? 1 : 0), g = 1 << lg;
    const int take = min(sp, 32 >> lg);
    sp -= take;
    const int j = lane >> lg;
    const uint32_t node = j < take ? fr[sp + j] : kNone;
    __syncwarp();
    // this lane's kWide / g child records, kWideBatch loads issued before the first test of
    // each batch (the records of one node share a 128-byte line, but each is its own sector)
    const int c0 = lane & (g - 1), rounds = kWide >> lg;
    bool ok = true;
#pragma unroll
    for (int r0 = 0; r0 < kWide; r0 += kWideBatch) {
        if (r0 >= rounds) break;  // warp-uniform
        float4 ra[kWideBatch], rb[kWideBatch];
#pragma unroll
        for (int r = 0; r < kWideBatch; ++r) {
            ra[r] = make_float4(0.f, 0.f, 0.f, 0.f);
            rb[r] = make_float4(0.f, 0.f, __uint_as_float(kNone), 0.f);
            if (r0 + r < rounds && node != kNone) {
                const size_t at = 2ull * (kWide * (size_t) node + c0 + (r0 + r) * g);
                if (TOP && node < n_top) {
                    ra[r] = top[at];
                    rb[r] = top[at + 1];
                } else {
                    ra[r] = __ldg(wn + at);
                    rb[r] = __ldg(wn + at + 1);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < kWideBatch; ++r) {
            if (r0 + r >= rounds) break;  // warp-uniform
            if (!wide_round(ra[r], rb[r], fr, sp, cb, nc, test, front_cap, err, n_node, n_cand)) {
                ok = false;
                break;
            }
        }
        if (!ok) break;
    }
    __syncwarp();
    return ok;
}

// The first step of a descent: the tree's top cut (at most kWideCut child
// records that cover every root-leaf path), one record per lane.
template <class Test>
__device__ __forceinline__ bool cut_step(const float4* __restrict__ cut, uint32_t n_cut, uint32_t* fr, int& sp,
                                         uint32_t* cb, int& nc, const Test& test, uint32_t front_cap, uint32_t* err,
                                         unsigned long long& n_node, unsigned long long& n_cand) {
    const int lane = threadIdx.x & 31;
    float4 ra[kWideCut / 32], rb[kWideCut / 32];
#pragma unroll
    for (int r = 0; r < kWideCut / 32; ++r) {
        const uint32_t i = 32u * r + lane;
        ra[r] = make_float4(0.f, 0.f, 0.f, 0.f);
        rb[r] = make_float4(0.f, 0.f, __uint_as_float(kNone), 0.f);
        if (i < n_cut) {
            ra[r] = __ldg(cut + 2ull * i);
            rb[r] = __ldg(cut + 2ull * i + 1);
        }
    }
    bool ok = true;
#pragma unroll
    for (int r = 0; r < kWideCut / 32; ++r) {
        if (32u * r >= n_cut) break;  // warp-uniform
        if (!wide_round(ra[r], rb[r], fr, sp, cb, nc, test, front_cap, err, n_node, n_cand)) {
            ok = false;
            break;
        }
    }
    __syncwarp();
    return ok;
}

}  // namespace rtcd
