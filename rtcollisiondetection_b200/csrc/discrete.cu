// discrete.cu - forward kinematics, OBB prefilter and the mesh-to-mesh
// traversal of the two discrete detectors.
//
// Upstream path (RTCD/CollisionDetector/CollisionDetector.h:919-983): FK
// (RTCD/Robot/robot.cu:202-241), OBB transform (robot.cu:407-464), all-pairs
// OBB SAT (RTCD/CollisionDetector/BBCollisionDetection.cu:4-37, :70-98), a host
// round trip to compact the surviving links, a per-batch IAS rebuild, then one
// RT-core ray per edge (CCCuda.cu:56-77 ObsToRobot, CCRay.cu:74-116
// RobotToObs).
//
// Here a work item is one (pose, link) pair that survived the cull.  One lane
// owns one item and runs a two-stage query in a persistent loop:
//   A. the link's world OBB descends the scene LBVH (triangles for
//      RobotToObs, obstacle edges for ObsToRobot); each overlapping scene
//      primitive becomes a candidate;
//   B. the candidate is moved into the link frame (x_l = R^T (x - t)) and
//      descends the static link LBVH (link edges for RobotToObs, link
//      triangles for ObsToRobot); each overlapping pair gets the exact
//      segment-triangle test.
// Both sides are instanced - no per-batch acceleration structure is built -
// and the result is the same predicate the upstream rays evaluate: some edge
// of the source mesh crosses some triangle of the target mesh.  Lanes fetch new
// items from a device counter as they finish (persistent threads), so uneven
// items do not idle a warp.  Without counts, a pose stops as soon as one
// of its items hits.
#include <cooperative_groups.h>

#include <algorithm>

#include "kernels.h"

namespace cg = cooperative_groups;

namespace rtcd {

// ---------------------------------------------------------------- kinematics
// Upstream: 12 threads per pose with 7 shared-memory barriers
// (fkineKernelAdj, robot.cu:202-231).  Here one thread keeps the whole chain in
// registers; accurate sincosf replaces the __sincosf intrinsic.
__global__ void __launch_bounds__(kFkThreads) k_fk_poses(const Chain ch, const float* __restrict__ q, uint32_t n,
                                                        float4* __restrict__ T) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float qq[kMaxDof];
    for (int k = 0; k < ch.dof; ++k) qq[k] = q[(size_t) i * ch.dof + k];
    float Tl[kMaxLinks][12];
    fk_chain(ch, qq, Tl);
    float4* out = T + (size_t) i * (ch.dof + 1) * 3;
    for (int l = 0; l <= ch.dof; ++l) {
        out[l * 3 + 0] = make_float4(Tl[l][0], Tl[l][1], Tl[l][2], Tl[l][3]);
        out[l * 3 + 1] = make_float4(Tl[l][4], Tl[l][5], Tl[l][6], Tl[l][7]);
        out[l * 3 + 2] = make_float4(Tl[l][8], Tl[l][9], Tl[l][10], Tl[l][11]);
    }
}

void launch_fk_poses(const Chain& ch, const float* d_q, uint32_t n, float4* d_T, cudaStream_t s) {
    if (!n) return;
    k_fk_poses<<<(n + kFkThreads - 1) / kFkThreads, kFkThreads, 0, s>>>(ch, d_q, n, d_T);
    cuda_check(cudaGetLastError(), "k_fk_poses");
}

// ---------------------------------------------------------------- OBB cull
struct ObbW {
    f3 c, h, ax[3];
};

__device__ __forceinline__ ObbW world_obb(const float* lo, const float4* T) {
    ObbW o;
    o.c = xf(T, mk(lo[0], lo[1], lo[2]));
    o.h = mk(lo[3], lo[4], lo[5]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        f3 v = mk(lo[6 + 3 * a], lo[7 + 3 * a], lo[8 + 3 * a]);
        o.ax[a] = mk(T[0].x * v.x + T[0].y * v.y + T[0].z * v.z, T[1].x * v.x + T[1].y * v.y + T[1].z * v.z,
                     T[2].x * v.x + T[2].y * v.y + T[2].z * v.z);
    }
    return o;
}

// 15-axis separating-axis test (Gottschalk et al. 1996), the test of the
// upstream checkOBBCollision (BBCollisionDetection.cu:4-37).  kPar guards the
// cross-product axes of near-parallel edges; kTol keeps the test conservative
// against rounding.  Returns true when the boxes may overlap.
__device__ __forceinline__ bool obb_overlap(const ObbW& A, const float* B) {
    constexpr float kPar = 1e-6f, kTol = 2e-5f;
    f3 bc = mk(B[0], B[1], B[2]);
    float bh[3] = {B[3], B[4], B[5]};
    f3 bax[3] = {mk(B[6], B[7], B[8]), mk(B[9], B[10], B[11]), mk(B[12], B[13], B[14])};
    float ah[3] = {A.h.x + kTol, A.h.y + kTol, A.h.z + kTol};
    float Rm[3][3], AR[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Rm[i][j] = dot(A.ax[i], bax[j]);
            AR[i][j] = fabsf(Rm[i][j]) + kPar;
        }
    f3 d = bc - A.c;
    float t[3] = {dot(d, A.ax[0]), dot(d, A.ax[1]), dot(d, A.ax[2])};
#pragma unroll
    for (int i = 0; i < 3; ++i)
        if (fabsf(t[i]) > ah[i] + bh[0] * AR[i][0] + bh[1] * AR[i][1] + bh[2] * AR[i][2]) return false;
#pragma unroll
    for (int j = 0; j < 3; ++j)
        if (fabsf(t[0] * Rm[0][j] + t[1] * Rm[1][j] + t[2] * Rm[2][j]) >
            ah[0] * AR[0][j] + ah[1] * AR[1][j] + ah[2] * AR[2][j] + bh[j])
            return false;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            float ra = ah[i1] * AR[i2][j] + ah[i2] * AR[i1][j];
            float rb = bh[j1] * AR[i][j2] + bh[j2] * AR[i][j1];
            if (fabsf(t[i2] * Rm[i1][j] - t[i1] * Rm[i2][j]) > ra + rb) return false;
        }
    }
    return true;
}

constexpr int kCullChunk = 256;  // obstacle OBBs staged in shared memory per pass

// One thread per (pose, link): the link OBB against every obstacle OBB, with a
// bounding-sphere reject before the full test.
__global__ void __launch_bounds__(256) k_cull(const RobotDev R, const float* __restrict__ sobb, uint32_t n_obs,
                                             const float4* __restrict__ T, uint32_t n, uint8_t* __restrict__ mask) {
    __shared__ float s_obb[kCullChunk * 16];
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t pose = i / R.n_links, link = i % R.n_links;
    bool active = pose < n && link >= R.first_link;
    ObbW A;
    float arad = 0.f;
    if (active) {
        A = world_obb(R.obb[link], T + ((size_t) pose * R.n_links + link) * 3);
        arad = sqrtf(dot(A.h, A.h)) + 2e-5f;
    }
    bool hit = false;
    for (uint32_t base = 0; base < n_obs; base += kCullChunk) {
        uint32_t m = min((uint32_t) kCullChunk, n_obs - base);
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < m * 16; k += blockDim.x) s_obb[k] = sobb[(size_t) base * 16 + k];
        __syncthreads();
        if (active && !hit) {
            for (uint32_t o = 0; o < m; ++o) {
                const float* B = s_obb + o * 16;
                f3 d = mk(B[0], B[1], B[2]) - A.c;
                float rr = arad + B[15];
                if (dot(d, d) > rr * rr) continue;
                if (obb_overlap(A, B)) {
                    hit = true;
                    break;
                }
            }
        }
    }
    if (pose < n) mask[i] = hit ? 1 : 0;
}

void launch_cull(const RobotDev& R, const SceneDev& S, const float4* d_T, uint32_t n, uint8_t* d_mask, cudaStream_t s) {
    uint32_t total = n * R.n_links;
    if (!total) return;
    k_cull<<<(total + 255) / 256, 256, 0, s>>>(R, S.obbs, S.n_obs, d_T, n, d_mask);
    cuda_check(cudaGetLastError(), "k_cull");
}

__global__ void k_all_items(uint32_t n_links, uint32_t first, uint32_t n, uint32_t* items, uint32_t* count) {
    uint32_t per = n_links - first;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *count = n * per;
    if (i >= n * per) return;
    items[i] = (i / per) * n_links + first + (i % per);
}

void launch_all_items(const RobotDev& R, uint32_t n, uint32_t* d_items, uint32_t* d_count, cudaStream_t s) {
    uint32_t total = std::max<uint32_t>(1, n * (R.n_links - R.first_link));
    k_all_items<<<(total + 255) / 256, 256, 0, s>>>(R.n_links, R.first_link, n, d_items, d_count);
    cuda_check(cudaGetLastError(), "k_all_items");
}

// ---------------------------------------------------------------- exact tests
// Segment pq against triangle abc, FP32 with an error filter.
// 0 = certain miss, 1 = certain hit, 2 = too close to call in FP32.
// Five signed volumes decide the crossing: the endpoint sides of the plane
// and the three edge volumes of the segment's line (Plucker sides).  A value
// within kRel of its magnitude bound is uncertain; the bound covers both the
// FP32 rounding here and the rounding of the frame change before it.
__device__ __forceinline__ float l1(f3 v) { return fabsf(v.x) + fabsf(v.y) + fabsf(v.z); }

__device__ __forceinline__ int sgn_tol(float v, float tol) { return v > tol ? 1 : (v < -tol ? -1 : 0); }

__device__ __forceinline__ int seg_tri_f32(f3 p, f3 q, f3 a, f3 b, f3 c) {
    constexpr float kRel = 1e-4f;
    f3 e1 = b - a, e2 = c - a, n = cross(e1, e2);
    f3 pa = p - a, qa = q - a;
    float nl = l1(n);
    int sp = sgn_tol(dot(n, pa), kRel * nl * l1(pa));
    int sq = sgn_tol(dot(n, qa), kRel * nl * l1(qa));
    if (sp == sq && sp != 0) return 0;
    f3 d = q - p, ap = a - p, bp = b - p, cp = c - p;
    float dl = l1(d), al = l1(ap), bl = l1(bp), cl = l1(cp);
    int s1 = sgn_tol(dot(d, cross(ap, bp)), kRel * dl * al * bl);
    int s2 = sgn_tol(dot(d, cross(bp, cp)), kRel * dl * bl * cl);
    int s3 = sgn_tol(dot(d, cross(cp, ap)), kRel * dl * cl * al);
    bool pos = s1 > 0 || s2 > 0 || s3 > 0, neg = s1 < 0 || s2 < 0 || s3 < 0;
    if (pos && neg) return 0;
    if (sp != 0 && sq != 0 && s1 != 0 && s2 != 0 && s3 != 0) return 1;
    return 2;
}

__device__ __forceinline__ double orient2(double ax, double ay, double bx, double by, double cx, double cy) {
    return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}

__device__ __forceinline__ bool seg_seg_2d(double px, double py, double qx, double qy, double ax, double ay, double bx,
                                           double by) {
    double o1 = orient2(px, py, qx, qy, ax, ay), o2 = orient2(px, py, qx, qy, bx, by);
    double o3 = orient2(ax, ay, bx, by, px, py), o4 = orient2(ax, ay, bx, by, qx, qy);
    if (((o1 > 0 && o2 < 0) || (o1 < 0 && o2 > 0)) && ((o3 > 0 && o4 < 0) || (o3 < 0 && o4 > 0))) return true;
    auto on = [](double ax_, double ay_, double bx_, double by_, double x, double y) {
        return x >= fmin(ax_, bx_) && x <= fmax(ax_, bx_) && y >= fmin(ay_, by_) && y <= fmax(ay_, by_);
    };
    if (o1 == 0 && on(px, py, qx, qy, ax, ay)) return true;
    if (o2 == 0 && on(px, py, qx, qy, bx, by)) return true;
    if (o3 == 0 && on(ax, ay, bx, by, px, py)) return true;
    if (o4 == 0 && on(ax, ay, bx, by, qx, qy)) return true;
    return false;
}

// FP64 re-test of a candidate in the FP32 inflation band: the same five
// volumes in double precision, on coordinates rebuilt from the stored floats.
__device__ __noinline__ bool seg_tri_f64(d3 p, d3 q, d3 a, d3 b, d3 c) {
    d3 n = cross(b - a, c - a);
    double dp = dot(n, p - a), dq = dot(n, q - a);
    if ((dp > 0 && dq > 0) || (dp < 0 && dq < 0)) return false;
    d3 d = q - p, ap = a - p, bp = b - p, cp = c - p;
    double v1 = dot(d, cross(ap, bp)), v2 = dot(d, cross(bp, cp)), v3 = dot(d, cross(cp, ap));
    if ((v1 > 0 || v2 > 0 || v3 > 0) && (v1 < 0 || v2 < 0 || v3 < 0)) return false;
    if (!(dp == 0 && dq == 0) && !(v1 == 0 && v2 == 0 && v3 == 0)) return true;
    // coplanar: 2D test on the plane, dropping the dominant normal axis
    double ax_ = fabs(n.x), ay_ = fabs(n.y), az_ = fabs(n.z);
    if (ax_ + ay_ + az_ == 0) return false;
    int drop = (ax_ >= ay_ && ax_ >= az_) ? 0 : (ay_ >= az_ ? 1 : 2);
    auto U = [&](d3 v) { return drop == 0 ? v.y : v.x; };
    auto V = [&](d3 v) { return drop == 2 ? v.y : v.z; };
    double o1 = orient2(U(a), V(a), U(b), V(b), U(p), V(p));
    double o2 = orient2(U(b), V(b), U(c), V(c), U(p), V(p));
    double o3 = orient2(U(c), V(c), U(a), V(a), U(p), V(p));
    if ((o1 >= 0 && o2 >= 0 && o3 >= 0) || (o1 <= 0 && o2 <= 0 && o3 <= 0)) return true;
    return seg_seg_2d(U(p), V(p), U(q), V(q), U(a), V(a), U(b), V(b)) ||
           seg_seg_2d(U(p), V(p), U(q), V(q), U(b), V(b), U(c), V(c)) ||
           seg_seg_2d(U(p), V(p), U(q), V(q), U(c), V(c), U(a), V(a));
}

// Conservative OBB-vs-AABB test: the box's projection on the three world axes
// and on the three OBB axes (6 of the 15 SAT axes).
__device__ __forceinline__ bool obb_aabb(const Box& b, const ObbW& o, const f3& ext) {
    float cx = 0.5f * (b.lo[0] + b.hi[0]), cy = 0.5f * (b.lo[1] + b.hi[1]), cz = 0.5f * (b.lo[2] + b.hi[2]);
    float hx = 0.5f * (b.hi[0] - b.lo[0]), hy = 0.5f * (b.hi[1] - b.lo[1]), hz = 0.5f * (b.hi[2] - b.lo[2]);
    f3 d = mk(o.c.x - cx, o.c.y - cy, o.c.z - cz);
    if (fabsf(d.x) > hx + ext.x || fabsf(d.y) > hy + ext.y || fabsf(d.z) > hz + ext.z) return false;
    float h[3] = {o.h.x, o.h.y, o.h.z};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float r = hx * fabsf(o.ax[i].x) + hy * fabsf(o.ax[i].y) + hz * fabsf(o.ax[i].z);
        if (fabsf(dot(d, o.ax[i])) > h[i] + r) return false;
    }
    return true;
}

__device__ __forceinline__ uint32_t ld_flag(const uint32_t* p) { return __ldcg(p); }

// ---------------------------------------------------------------- traversal
template <bool R2O>
__global__ void __launch_bounds__(kTravThreads) k_discrete(const RobotDev R, const SceneDev S, const DiscreteArgs A) {
    constexpr float kBoxTol = 2e-5f;
    const float4* __restrict__ wn = R2O ? S.tri_nodes : S.edge_nodes;
    const float4* __restrict__ wp = R2O ? S.tri_prims : S.edge_prims;
    const uint32_t wroot = R2O ? S.tri_root : S.edge_root;
    const float4* __restrict__ ln = R2O ? R.edge_nodes : R.tri_nodes;
    const float4* __restrict__ lp = R2O ? R.edge_prims : R.tri_prims;
    const uint32_t n_items = *A.n_items;

    uint32_t stA[kStack], stB[kStack];
    int spA = 0, spB = 0;
    int state = 0;  // 0: fetch an item, 1: scene descent, 2: link descent
    uint32_t pose = 0, link = 0, cand = 0;
    float4 T[3];
    ObbW ob;
    f3 ext;
    f3 c0, c1, c2;  // candidate in the link frame (c2 unused for edges)
    float blo[3], bhi[3];

    while (true) {
        if (state == 0) {
            cg::coalesced_group g = cg::coalesced_threads();
            uint32_t base = 0;
            if (g.thread_rank() == 0) base = atomicAdd(A.work_counter, g.size());
            base = g.shfl(base, 0);
            uint32_t it = base + g.thread_rank();
            if (it >= n_items) break;
            uint32_t item = A.items[it];
            pose = item / R.n_links;
            link = item - pose * R.n_links;
            if (pose >= A.n_poses || wroot == kNone) {
                if (pose >= A.n_poses) atomicOr(A.err, kErrRange);
                continue;
            }
            if (!A.want_counts && ld_flag(A.pose_hit + pose)) continue;
            const float4* tp = A.T + ((size_t) pose * R.n_links + link) * 3;
            T[0] = tp[0]; T[1] = tp[1]; T[2] = tp[2];
            ob = world_obb(R.obb[link], T);
            ob.h = mk(ob.h.x + kBoxTol, ob.h.y + kBoxTol, ob.h.z + kBoxTol);
            ext = mk(fabsf(ob.ax[0].x) * ob.h.x + fabsf(ob.ax[1].x) * ob.h.y + fabsf(ob.ax[2].x) * ob.h.z,
                     fabsf(ob.ax[0].y) * ob.h.x + fabsf(ob.ax[1].y) * ob.h.y + fabsf(ob.ax[2].y) * ob.h.z,
                     fabsf(ob.ax[0].z) * ob.h.x + fabsf(ob.ax[1].z) * ob.h.y + fabsf(ob.ax[2].z) * ob.h.z);
            stA[0] = wroot;
            spA = 1;
            state = 1;
            continue;
        }
        if (state == 1) {
            if (spA == 0) {
                state = 0;
                continue;
            }
            uint32_t ref = stA[--spA];
            if (ref & kLeaf) {
                if (!A.want_counts && ld_flag(A.pose_hit + pose)) {
                    state = 0;
                    continue;
                }
                cand = ref & ~kLeaf;
                uint32_t lroot = R2O ? R.edge_root[link] : R.tri_root[link];
                if (lroot == kNone) continue;
                if (R2O) {
                    const float4* t = wp + 3ull * cand;
                    c0 = xf_inv(T, f3of(__ldg(t)));
                    c1 = xf_inv(T, f3of(__ldg(t + 1)));
                    c2 = xf_inv(T, f3of(__ldg(t + 2)));
                    blo[0] = fminf(c0.x, fminf(c1.x, c2.x)); bhi[0] = fmaxf(c0.x, fmaxf(c1.x, c2.x));
                    blo[1] = fminf(c0.y, fminf(c1.y, c2.y)); bhi[1] = fmaxf(c0.y, fmaxf(c1.y, c2.y));
                    blo[2] = fminf(c0.z, fminf(c1.z, c2.z)); bhi[2] = fmaxf(c0.z, fmaxf(c1.z, c2.z));
                } else {
                    const float4* e = wp + 2ull * cand;
                    c0 = xf_inv(T, f3of(__ldg(e)));
                    c1 = xf_inv(T, f3of(__ldg(e + 1)));
                    blo[0] = fminf(c0.x, c1.x); bhi[0] = fmaxf(c0.x, c1.x);
                    blo[1] = fminf(c0.y, c1.y); bhi[1] = fmaxf(c0.y, c1.y);
                    blo[2] = fminf(c0.z, c1.z); bhi[2] = fmaxf(c0.z, c1.z);
                }
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    blo[k] -= kBoxTol;
                    bhi[k] += kBoxTol;
                }
                stB[0] = lroot;
                spB = 1;
                state = 2;
                continue;
            }
            Box bl, br;
            uint32_t rl, rr;
            load_node(wn, ref, bl, br, rl, rr);
            bool hr = obb_aabb(br, ob, ext), hl = obb_aabb(bl, ob, ext);
            if (spA + 2 > kStack) {
                atomicOr(A.err, kErrStack);
                hr = hl = false;
            }
            if (hr) stA[spA++] = rr;
            if (hl) stA[spA++] = rl;
            continue;
        }
        // state 2: link-side descent for the current candidate
        if (spB == 0) {
            state = 1;
            continue;
        }
        uint32_t ref = stB[--spB];
        if (ref & kLeaf) {
            uint32_t li = ref & ~kLeaf;
            int r;
            f3 p, q, a, b, c;
            if (R2O) {
                const float4* e = lp + 2ull * li;
                p = f3of(__ldg(e)); q = f3of(__ldg(e + 1));
                a = c0; b = c1; c = c2;
            } else {
                const float4* t = lp + 3ull * li;
                p = c0; q = c1;
                a = f3of(__ldg(t)); b = f3of(__ldg(t + 1)); c = f3of(__ldg(t + 2));
            }
            r = seg_tri_f32(p, q, a, b, c);
            if (r == 2) {
                atomicAdd(A.stats, 1ull);
                bool h;
                if (R2O) {
                    const float4* e = lp + 2ull * li;
                    const float4* t = wp + 3ull * cand;
                    h = seg_tri_f64(xf_d(T, f3of(__ldg(e))), xf_d(T, f3of(__ldg(e + 1))), d3of(f3of(__ldg(t))),
                                    d3of(f3of(__ldg(t + 1))), d3of(f3of(__ldg(t + 2))));
                } else {
                    const float4* e = wp + 2ull * cand;
                    const float4* t = lp + 3ull * li;
                    h = seg_tri_f64(d3of(f3of(__ldg(e))), d3of(f3of(__ldg(e + 1))), xf_d(T, f3of(__ldg(t))),
                                    xf_d(T, f3of(__ldg(t + 1))), xf_d(T, f3of(__ldg(t + 2))));
                }
                r = h ? 1 : 0;
            }
            if (r == 1) {
                if (!A.want_counts) {
                    atomicExch(A.pose_hit + pose, 1u);
                    state = 0;
                    continue;
                }
                A.pose_hit[pose] = 1u;
                if (R2O) {
                    uint32_t eid = __float_as_uint(__ldg(lp + 2ull * li).w);
                    atomicOr(A.edge_bits + (size_t) pose * A.edge_words + (eid >> 5), 1u << (eid & 31));
                } else {
                    atomicAdd(A.counts + pose, 1u);
                }
            }
            continue;
        }
        Box bl, br;
        uint32_t rl, rr;
        load_node(ln, ref, bl, br, rl, rr);
        bool hr = box_overlap(br, blo, bhi), hl = box_overlap(bl, blo, bhi);
        if (spB + 2 > kStack) {
            atomicOr(A.err, kErrStack);
            hr = hl = false;
        }
        if (hr) stB[spB++] = rr;
        if (hl) stB[spB++] = rl;
    }
}

uint32_t discrete_persistent_blocks(bool robot_to_obs) {
    int per_sm = 0;
    if (robot_to_obs)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_discrete<true>, kTravThreads, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_discrete<false>, kTravThreads, 0);
    return (uint32_t) std::max(1, per_sm) * (uint32_t) device_sm_count();
}

void launch_discrete(bool robot_to_obs, const RobotDev& R, const SceneDev& S, const DiscreteArgs& A, uint32_t blocks,
                     cudaStream_t s) {
    if (robot_to_obs)
        k_discrete<true><<<blocks, kTravThreads, 0, s>>>(R, S, A);
    else
        k_discrete<false><<<blocks, kTravThreads, 0, s>>>(R, S, A);
    cuda_check(cudaGetLastError(), "k_discrete");
}

__global__ void k_popcount_rows(const uint32_t* __restrict__ bits, uint32_t words, uint32_t rows, uint32_t* out) {
    uint32_t row = blockIdx.x;
    if (row >= rows) return;
    uint32_t acc = 0;
    for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) acc += __popc(bits[(size_t) row * words + w]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ uint32_t s[32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int k = 0; k < (int) (blockDim.x / 32); ++k) t += s[k];
        out[row] = t;
    }
}

void launch_popcount_rows(const uint32_t* d_bits, uint32_t words, uint32_t rows, uint32_t* d_out, cudaStream_t s) {
    if (!rows) return;
    k_popcount_rows<<<rows, 128, 0, s>>>(d_bits, words, rows, d_out);
    cuda_check(cudaGetLastError(), "k_popcount_rows");
}

__global__ void k_flags(const uint32_t* __restrict__ hit, uint32_t n, uint8_t* __restrict__ flags) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[i] = hit[i] ? 1 : 0;
}

void launch_flags(const uint32_t* d_hit, uint32_t n, uint8_t* d_flags, cudaStream_t s) {
    if (!n) return;
    k_flags<<<(n + 255) / 256, 256, 0, s>>>(d_hit, n, d_flags);
    cuda_check(cudaGetLastError(), "k_flags");
}

}  // namespace rtcd
