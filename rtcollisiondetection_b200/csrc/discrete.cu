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
#include "wide.cuh"

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
// The culled items are compacted link by link, the last (most distal) link
// of every pose first, then every pose's next-to-last, ...: in flags mode a
// pose hit through one link is decided before most of its other links' items
// start, and those stop at their first check instead of running beside it.
// The distal links sweep most of the workspace and decide most colliding
// poses, so they go first (the 65,536-pose dense scene: 2.07 ms pose-major,
// 1.51 ms base link first, 1.20 ms last link first).  item_word turns a
// compacted index back into pose * n_links + link.
__device__ __forceinline__ uint32_t link_slot(uint32_t link, uint32_t n_links) { return n_links - 1 - link; }
__device__ __forceinline__ uint32_t item_word(const DiscreteArgs& A, uint32_t n_links, uint32_t j) {
    if (!A.link_major) return j;
    const uint32_t slot = j / A.n_poses, pose = j - slot * A.n_poses;
    return pose * n_links + link_slot(slot, n_links);
}

// One thread per (pose, link): the link OBB against every obstacle OBB, with a
// bounding-sphere reject before the full test.
__global__ void __launch_bounds__(256) k_cull(const RobotDev R, const float* __restrict__ sobb, uint32_t n_obs,
                                             const float4* __restrict__ T, uint32_t n, uint8_t* __restrict__ mask,
                                             bool link_major, unsigned long long* stats) {
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
    unsigned long long n_sphere = 0, n_sat = 0;  // bounding-sphere tests, then the SATs they let through
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
                ++n_sphere;
                if (dot(d, d) > rr * rr) continue;
                ++n_sat;
                if (obb_overlap(A, B)) {
                    hit = true;
                    break;
                }
            }
        }
    }
    if (pose < n) mask[link_major ? (size_t) link_slot(link, R.n_links) * n + pose : i] = hit ? 1 : 0;
    warp_count(stats + kStatCullSpheres, n_sphere);
    warp_count(stats + kStatCullSats, n_sat);
}

void launch_cull(const RobotDev& R, const SceneDev& S, const float4* d_T, uint32_t n, uint8_t* d_mask, bool link_major,
                 unsigned long long* d_stats, cudaStream_t s) {
    uint32_t total = n * R.n_links;
    if (!total) return;
    k_cull<<<(total + 255) / 256, 256, 0, s>>>(R, S.obbs, S.n_obs, d_T, n, d_mask, link_major, d_stats);
    cuda_check(cudaGetLastError(), "k_cull");
}

// Every item, in the link-major order of the culled list (item_word): the
// slots of links n_links - 1 down to first_link, each over all poses.
__global__ void k_all_items(uint32_t n_links, uint32_t first, uint32_t n, uint32_t* items, uint32_t* count) {
    uint32_t per = n_links - first;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *count = n * per;
    if (i >= n * per) return;
    items[i] = i;
}

void launch_all_items(const RobotDev& R, uint32_t n, uint32_t* d_items, uint32_t* d_count, cudaStream_t s) {
    uint32_t total = std::max<uint32_t>(1, n * (R.n_links - R.first_link));
    k_all_items<<<(total + 255) / 256, 256, 0, s>>>(R.n_links, R.first_link, n, d_items, d_count);
    cuda_check(cudaGetLastError(), "k_all_items");
}

// ---------------------------------------------------------------- exact tests
// Segment pq against triangle abc, FP32 with an error filter.
// 0 = certain miss, 1 = certain hit, 2 = too close to call in FP32.
// Five signed volumes decide the crossing: the endpoint sides of the plane,
// n.(p - a) and n.(q - a), and the three edge volumes of the segment's line,
// d.((a - p) x (b - a)) and its two rotations (Plucker sides, written with the
// short triangle edges so no large cross product cancels).  Each volume is a
// distance times known lengths; it is uncertain when that distance is below
// kDist plus a relative rounding term.  kDist (1 um) is twenty times the
// coordinate error of the frame change before the test and far below the
// 1e-5 m parity band, so FP32 decides everything outside the band and the
// FP64 re-test only sees true near-degeneracies.
__device__ __forceinline__ float l1(f3 v) { return fabsf(v.x) + fabsf(v.y) + fabsf(v.z); }

__device__ __forceinline__ int sgn_tol(float v, float tol) { return v > tol ? 1 : (v < -tol ? -1 : 0); }

__device__ __forceinline__ int seg_tri_f32(f3 p, f3 q, f3 a, f3 b, f3 c) {
    constexpr float kDist = 1e-6f, kRel = 4e-6f;
    f3 ab = b - a, bc = c - b, ca = a - c;
    f3 n = cross(ab, c - a);
    f3 pa = p - a, qa = q - a;
    float nl = l1(n);
    int sp = sgn_tol(dot(n, pa), nl * (kDist + kRel * l1(pa)));
    int sq = sgn_tol(dot(n, qa), nl * (kDist + kRel * l1(qa)));
    if (sp == sq && sp != 0) return 0;
    f3 d = q - p, ap = a - p, bp = b - p, cp = c - p;
    float dl = l1(d);
    int s1 = sgn_tol(dot(d, cross(ap, ab)), dl * l1(ab) * (kDist + kRel * l1(ap)));
    int s2 = sgn_tol(dot(d, cross(bp, bc)), dl * l1(bc) * (kDist + kRel * l1(bp)));
    int s3 = sgn_tol(dot(d, cross(cp, ca)), dl * l1(ca) * (kDist + kRel * l1(cp)));
    bool pos = s1 > 0 || s2 > 0 || s3 > 0, neg = s1 < 0 || s2 < 0 || s3 < 0;
    if (pos && neg) return 0;
    if (sp != 0 && sq != 0 && s1 != 0 && s2 != 0 && s3 != 0) return 1;
    return 2;
}

// Segment p + t d, t in [0, 1], against a box (slab test); inv = 1 / d per axis
// (infinite for a zero component), boxes padded by `pad`.
__device__ __forceinline__ bool seg_box(const f3& p, const f3& inv, const Box& b, float pad) {
    float t0x = (b.lo[0] - pad - p.x) * inv.x, t1x = (b.hi[0] + pad - p.x) * inv.x;
    float t0y = (b.lo[1] - pad - p.y) * inv.y, t1y = (b.hi[1] + pad - p.y) * inv.y;
    float t0z = (b.lo[2] - pad - p.z) * inv.z, t1z = (b.hi[2] + pad - p.z) * inv.z;
    float tmin = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), 0.0f));
    float tmax = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fminf(fmaxf(t0z, t1z), 1.0f));
    return tmin <= tmax;
}

// A box that straddles (or touches, within pad) the plane n.x = w.
__device__ __forceinline__ bool plane_box(const f3& n, float w, const Box& b, float pad) {
    float cx = 0.5f * (b.lo[0] + b.hi[0]), cy = 0.5f * (b.lo[1] + b.hi[1]), cz = 0.5f * (b.lo[2] + b.hi[2]);
    float r = fabsf(n.x) * (0.5f * (b.hi[0] - b.lo[0]) + pad) + fabsf(n.y) * (0.5f * (b.hi[1] - b.lo[1]) + pad) +
              fabsf(n.z) * (0.5f * (b.hi[2] - b.lo[2]) + pad);
    return fabsf(n.x * cx + n.y * cy + n.z * cz - w) <= r;
}

__device__ __forceinline__ float safe_inv(float v) { return v != 0.0f ? 1.0f / v : copysignf(3.0e38f, v); }

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

// The FP64 re-test of one (scene primitive, link primitive) pair, rebuilt in
// the world frame from the stored floats and the link transform (out of line
// so its double registers do not weigh on the traversal loop).
// R2O: link edge li against scene triangle wi; else scene edge wi against link triangle li.
template <bool R2O>
__device__ __noinline__ bool retest_f64(const float4* T, const float4* __restrict__ lp, uint32_t li,
                                        const float4* __restrict__ wp, uint32_t wi) {
    if (R2O) {
        const float4* e = lp + 2ull * li;
        const float4* t = wp + 3ull * wi;
        return seg_tri_f64(xf_d(T, f3of(__ldg(e))), xf_d(T, f3of(__ldg(e + 1))), d3of(f3of(__ldg(t))),
                           d3of(f3of(__ldg(t + 1))), d3of(f3of(__ldg(t + 2))));
    }
    const float4* e = wp + 2ull * wi;
    const float4* t = lp + 3ull * li;
    return seg_tri_f64(d3of(f3of(__ldg(e))), d3of(f3of(__ldg(e + 1))), xf_d(T, f3of(__ldg(t))),
                       xf_d(T, f3of(__ldg(t + 1))), xf_d(T, f3of(__ldg(t + 2))));
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
    f3 cn, cinv;    // candidate triangle normal (RobotToObs) / inverse segment direction (ObsToRobot)
    float cw = 0.f; // plane offset n.c0 of the candidate triangle
    float blo[3], bhi[3];

    while (true) {
        if (state == 0) {
            cg::coalesced_group g = cg::coalesced_threads();
            uint32_t base = 0;
            if (g.thread_rank() == 0) base = atomicAdd(A.work_counter, g.size());
            base = g.shfl(base, 0);
            uint32_t it = base + g.thread_rank();
            if (it >= n_items) break;
            uint32_t item = item_word(A, R.n_links, A.items[it]);
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
                // link OBB in its own frame: the candidate must reach it
                const float* lo = R.obb[link];
                const f3 oc = mk(lo[0], lo[1], lo[2]);
                const f3 u0 = mk(lo[6], lo[7], lo[8]), u1 = mk(lo[9], lo[10], lo[11]), u2 = mk(lo[12], lo[13], lo[14]);
                if (R2O) {
                    const float4* t = wp + 3ull * cand;
                    c0 = xf_inv(T, f3of(__ldg(t)));
                    c1 = xf_inv(T, f3of(__ldg(t + 1)));
                    c2 = xf_inv(T, f3of(__ldg(t + 2)));
                    cn = cross(c1 - c0, c2 - c0);
                    cw = dot(cn, c0);
                    // the triangle's plane must cut the link OBB
                    float rr = (lo[3] + kBoxTol) * fabsf(dot(cn, u0)) + (lo[4] + kBoxTol) * fabsf(dot(cn, u1)) +
                               (lo[5] + kBoxTol) * fabsf(dot(cn, u2));
                    if (fabsf(dot(cn, oc) - cw) > rr) continue;
                    blo[0] = fminf(c0.x, fminf(c1.x, c2.x)); bhi[0] = fmaxf(c0.x, fmaxf(c1.x, c2.x));
                    blo[1] = fminf(c0.y, fminf(c1.y, c2.y)); bhi[1] = fmaxf(c0.y, fmaxf(c1.y, c2.y));
                    blo[2] = fminf(c0.z, fminf(c1.z, c2.z)); bhi[2] = fmaxf(c0.z, fmaxf(c1.z, c2.z));
                } else {
                    const float4* e = wp + 2ull * cand;
                    c0 = xf_inv(T, f3of(__ldg(e)));
                    c1 = xf_inv(T, f3of(__ldg(e + 1)));
                    f3 d = c1 - c0;
                    cinv = mk(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
                    // the segment must pass through the link OBB (slab test in the OBB frame)
                    f3 pr = c0 - oc;
                    f3 po = mk(dot(pr, u0), dot(pr, u1), dot(pr, u2));
                    f3 dd = mk(dot(d, u0), dot(d, u1), dot(d, u2));
                    Box ob_local;
                    ob_local.lo[0] = -lo[3]; ob_local.lo[1] = -lo[4]; ob_local.lo[2] = -lo[5];
                    ob_local.hi[0] = lo[3]; ob_local.hi[1] = lo[4]; ob_local.hi[2] = lo[5];
                    if (!seg_box(po, mk(safe_inv(dd.x), safe_inv(dd.y), safe_inv(dd.z)), ob_local, kBoxTol)) continue;
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
                r = retest_f64<R2O>(T, lp, li, wp, cand) ? 1 : 0;
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
        bool hr, hl;
        if (R2O) {  // node box overlaps the triangle's box and straddles its plane
            hr = box_overlap(br, blo, bhi) && plane_box(cn, cw, br, kBoxTol);
            hl = box_overlap(bl, blo, bhi) && plane_box(cn, cw, bl, kBoxTol);
        } else {    // the segment passes through the node box
            hr = seg_box(c0, cinv, br, kBoxTol);
            hl = seg_box(c0, cinv, bl, kBoxTol);
        }
        if (spB + 2 > kStack) {
            atomicOr(A.err, kErrStack);
            hr = hl = false;
        }
        if (hr) stB[spB++] = rr;
        if (hl) stB[spB++] = rl;
    }
}

// ---------------------------------------------------------------- wavefront form
// Stage A: one warp per (pose, link) item.  The warp descends the scene LBVH
// with the link's world OBB through a shared LIFO frontier: each step the
// lanes take up to 32 nodes off the top, test both children, push the
// internal survivors and emit the leaf survivors as candidates - contiguously
// per item, so stage B's neighbouring lanes share a link and a transform.
template <bool R2O>
__global__ void __launch_bounds__(kStageAWarps * 32) k_stage_a(const RobotDev R, const SceneDev S, const WaveArgs W) {
    constexpr float kBoxTol = 2e-5f;
    __shared__ uint32_t s_front[kStageAWarps][kFrontier];
    const DiscreteArgs& A = W.d;
    const int lane = threadIdx.x & 31;
    uint32_t* fr = s_front[threadIdx.x >> 5];
    const uint32_t lt = (1u << lane) - 1u;
    const float4* __restrict__ wn = R2O ? S.tri_nodes : S.edge_nodes;
    const uint32_t wroot = R2O ? S.tri_root : S.edge_root;
    const uint32_t n_items = *A.n_items;
    unsigned long long n_node = 0;
    while (true) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(A.work_counter, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= n_items) break;
        const uint32_t item = item_word(A, R.n_links, A.items[it]);
        const uint32_t pose = item / R.n_links, link = item - pose * R.n_links;
        if (pose >= A.n_poses) {
            if (lane == 0) atomicOr(A.err, kErrRange);
            continue;
        }
        if (wroot == kNone || (!A.want_counts && ld_flag(A.pose_hit + pose))) continue;
        float4 T[3];
        const float4* tp = A.T + ((size_t) pose * R.n_links + link) * 3;
        T[0] = tp[0]; T[1] = tp[1]; T[2] = tp[2];
        ObbW ob = world_obb(R.obb[link], T);
        ob.h = mk(ob.h.x + kBoxTol, ob.h.y + kBoxTol, ob.h.z + kBoxTol);
        const f3 ext = mk(fabsf(ob.ax[0].x) * ob.h.x + fabsf(ob.ax[1].x) * ob.h.y + fabsf(ob.ax[2].x) * ob.h.z,
                          fabsf(ob.ax[0].y) * ob.h.x + fabsf(ob.ax[1].y) * ob.h.y + fabsf(ob.ax[2].y) * ob.h.z,
                          fabsf(ob.ax[0].z) * ob.h.x + fabsf(ob.ax[1].z) * ob.h.y + fabsf(ob.ax[2].z) * ob.h.z);
        int sp = 1;
        if (lane == 0) fr[0] = wroot;
        __syncwarp();
        bool overflow = false;
        while (sp > 0 && !overflow) {
            const int take = min(sp, 32);
            sp -= take;
            uint32_t ref = lane < take ? fr[sp + lane] : kNone;
            __syncwarp();
            bool hl = false, hr = false;
            uint32_t rl = kNone, rr = kNone;
            if (ref != kNone) {
                if (ref & kLeaf) {  // a one-primitive scene: the root itself is a leaf
                    hl = true;
                    rl = ref;
                } else {
                    Box bl, br;
                    load_node(wn, ref, bl, br, rl, rr);
                    n_node += 2;
                    hl = obb_aabb(bl, ob, ext);
                    hr = obb_aabb(br, ob, ext);
                }
            }
            const bool pl = hl && !(rl & kLeaf), pr = hr && !(rr & kLeaf);
            const bool el = hl && (rl & kLeaf), er = hr && (rr & kLeaf);
            const uint32_t mpl = __ballot_sync(0xffffffffu, pl), mpr = __ballot_sync(0xffffffffu, pr);
            const int npush = __popc(mpl) + __popc(mpr);
            if (sp + npush > kFrontier) {  // cannot happen for trees within the depth limit
                if (lane == 0) atomicOr(A.err, kErrStack);
                break;
            }
            if (pl) fr[sp + __popc(mpl & lt)] = rl;
            if (pr) fr[sp + __popc(mpl) + __popc(mpr & lt)] = rr;
            sp += npush;
            const uint32_t mel = __ballot_sync(0xffffffffu, el), mer = __ballot_sync(0xffffffffu, er);
            const int nemit = __popc(mel) + __popc(mer);
            if (nemit) {
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(W.cand_count, (uint32_t) nemit);
                base = __shfl_sync(0xffffffffu, base, 0);
                if (base + (uint32_t) nemit > W.cand_cap) {
                    // slots below the capacity still get written (as blanks) so stage B
                    // never reads an unwritten candidate
                    overflow = true;
                    const uint32_t pl_ = base + __popc(mel & lt), pr_ = base + __popc(mel) + __popc(mer & lt);
                    if (el && pl_ < W.cand_cap) W.cand[pl_] = make_uint2(kNone, kNone);
                    if (er && pr_ < W.cand_cap) W.cand[pr_] = make_uint2(kNone, kNone);
                } else {
                    if (el) W.cand[base + __popc(mel & lt)] = make_uint2(item, rl & ~kLeaf);
                    if (er) W.cand[base + __popc(mel) + __popc(mer & lt)] = make_uint2(item, rr & ~kLeaf);
                }
            }
            __syncwarp();
        }
        if (overflow && lane == 0) {
            W.item_overflow[item] = 1;
            W.overflow_items[atomicAdd(W.overflow_count, 1u)] = item;
        }
    }
    warp_count(A.stats + 7, n_node);
}

// Stage B works on one candidate (item, scene primitive) at a time: move the
// scene primitive into the link frame, reject it against the link OBB,
// descend the link LBVH and run the exact segment-triangle test at the leaves.
constexpr float kBigTri = 0.03f;  // m: triangles whose box is longer get the edge-axis node test

struct StageBCand {
    float4 T[3];
    f3 c0, c1, c2, cn, cinv;  // primitive in the link frame; triangle normal (R2O) / 1 / segment (O2R)
    float cw;                 // plane offset n.c0 (R2O)
    float blo[3], bhi[3];     // triangle box (R2O)
    uint32_t pose, lroot, prim;
    bool big;                 // R2O: a triangle large enough for the edge-axis node test
};

// 0: nothing to do (blank, decided, overflowed item, empty link, OBB reject); 1: descend.
// Every outcome but "decided" is a function of the inputs alone, so a warp
// that sets up one candidate on all lanes (check_decided false) agrees.
template <bool R2O>
__device__ __forceinline__ int stage_b_setup(const RobotDev& R, const SceneDev& S, const WaveArgs& W, uint2 cd,
                                             StageBCand& C, unsigned long long& n_skip, unsigned long long& n_rej,
                                             bool check_decided = true) {
    constexpr float kBoxTol = 2e-5f;
    const DiscreteArgs& A = W.d;
    if (cd.x == kNone) return 0;  // blank slot of an overflowed emission
    const uint32_t item = cd.x;
    const uint32_t pose = item / R.n_links, link = item - pose * R.n_links;
    if (check_decided && !A.want_counts && ld_flag(A.pose_hit + pose)) {
        ++n_skip;
        return 0;
    }
    if (W.item_overflow[item]) return 0;  // the fused kernel re-runs this item
    C.lroot = R2O ? R.edge_root[link] : R.tri_root[link];
    if (C.lroot == kNone) return 0;
    C.pose = pose;
    C.prim = cd.y;
    const float4* tp = A.T + ((size_t) pose * R.n_links + link) * 3;
    C.T[0] = tp[0]; C.T[1] = tp[1]; C.T[2] = tp[2];
    const float* lo = R.obb[link];
    const f3 oc = mk(lo[0], lo[1], lo[2]);
    const f3 u0 = mk(lo[6], lo[7], lo[8]), u1 = mk(lo[9], lo[10], lo[11]), u2 = mk(lo[12], lo[13], lo[14]);
    const float4* __restrict__ wp = R2O ? S.tri_prims : S.edge_prims;
    C.c2 = C.cn = C.cinv = mk(0.f, 0.f, 0.f);
    C.cw = 0.f;
    C.big = false;
    if (R2O) {
        const float4* t = wp + 3ull * cd.y;
        C.c0 = xf_inv(C.T, f3of(__ldg(t)));
        C.c1 = xf_inv(C.T, f3of(__ldg(t + 1)));
        C.c2 = xf_inv(C.T, f3of(__ldg(t + 2)));
        C.cn = cross(C.c1 - C.c0, C.c2 - C.c0);
        C.cw = dot(C.cn, C.c0);
        const float rr = (lo[3] + kBoxTol) * fabsf(dot(C.cn, u0)) + (lo[4] + kBoxTol) * fabsf(dot(C.cn, u1)) +
                         (lo[5] + kBoxTol) * fabsf(dot(C.cn, u2));
        if (fabsf(dot(C.cn, oc) - C.cw) > rr) {
            ++n_rej;
            return 0;
        }
        C.blo[0] = fminf(C.c0.x, fminf(C.c1.x, C.c2.x)) - kBoxTol; C.bhi[0] = fmaxf(C.c0.x, fmaxf(C.c1.x, C.c2.x)) + kBoxTol;
        C.blo[1] = fminf(C.c0.y, fminf(C.c1.y, C.c2.y)) - kBoxTol; C.bhi[1] = fmaxf(C.c0.y, fmaxf(C.c1.y, C.c2.y)) + kBoxTol;
        C.blo[2] = fminf(C.c0.z, fminf(C.c1.z, C.c2.z)) - kBoxTol; C.bhi[2] = fmaxf(C.c0.z, fmaxf(C.c1.z, C.c2.z)) + kBoxTol;
        C.big = fmaxf(fmaxf(C.bhi[0] - C.blo[0], C.bhi[1] - C.blo[1]), C.bhi[2] - C.blo[2]) > kBigTri;
    } else {
        const float4* e = wp + 2ull * cd.y;
        C.c0 = xf_inv(C.T, f3of(__ldg(e)));
        C.c1 = xf_inv(C.T, f3of(__ldg(e + 1)));
        const f3 d = C.c1 - C.c0;
        C.cinv = mk(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
        const f3 pr = C.c0 - oc;
        const f3 po = mk(dot(pr, u0), dot(pr, u1), dot(pr, u2));
        const f3 dd = mk(dot(d, u0), dot(d, u1), dot(d, u2));
        Box obl;
        obl.lo[0] = -lo[3]; obl.lo[1] = -lo[4]; obl.lo[2] = -lo[5];
        obl.hi[0] = lo[3]; obl.hi[1] = lo[4]; obl.hi[2] = lo[5];
        if (!seg_box(po, mk(safe_inv(dd.x), safe_inv(dd.y), safe_inv(dd.z)), obl, kBoxTol)) {
            ++n_rej;
            return 0;
        }
    }
    return 1;
}

// Node test: the box overlaps the triangle's box and straddles its plane
// (R2O), or the segment passes through the box (O2R).
// The nine edge-cross separating axes of a triangle and a box (edge i x world
// axis k), the box grown by pad: false when one separates them.  Together
// with the box overlap and the plane straddle this is the full 13-axis
// triangle-box test; it prunes the link-tree nodes near a large triangle's
// plane but beyond its edges.
__device__ __forceinline__ bool tri_box_edges(const f3& c0, const f3& c1, const f3& c2, const Box& b, float pad) {
    const f3 m = mk(0.5f * (b.lo[0] + b.hi[0]), 0.5f * (b.lo[1] + b.hi[1]), 0.5f * (b.lo[2] + b.hi[2]));
    const float hx = 0.5f * (b.hi[0] - b.lo[0]) + pad, hy = 0.5f * (b.hi[1] - b.lo[1]) + pad,
                hz = 0.5f * (b.hi[2] - b.lo[2]) + pad;
    const f3 v0 = c0 - m, v1 = c1 - m, v2 = c2 - m;
    const f3 f[3] = {v1 - v0, v2 - v1, v0 - v2};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const f3 e = f[i];
        // x cross e = (0, -e.z, e.y)
        float p0 = -e.z * v0.y + e.y * v0.z, p1 = -e.z * v1.y + e.y * v1.z, p2 = -e.z * v2.y + e.y * v2.z;
        float r = hy * fabsf(e.z) + hz * fabsf(e.y);
        if (fminf(p0, fminf(p1, p2)) > r || fmaxf(p0, fmaxf(p1, p2)) < -r) return false;
        // y cross e = (e.z, 0, -e.x)
        p0 = e.z * v0.x - e.x * v0.z; p1 = e.z * v1.x - e.x * v1.z; p2 = e.z * v2.x - e.x * v2.z;
        r = hx * fabsf(e.z) + hz * fabsf(e.x);
        if (fminf(p0, fminf(p1, p2)) > r || fmaxf(p0, fmaxf(p1, p2)) < -r) return false;
        // z cross e = (-e.y, e.x, 0)
        p0 = -e.y * v0.x + e.x * v0.y; p1 = -e.y * v1.x + e.x * v1.y; p2 = -e.y * v2.x + e.x * v2.y;
        r = hx * fabsf(e.y) + hy * fabsf(e.x);
        if (fminf(p0, fminf(p1, p2)) > r || fmaxf(p0, fmaxf(p1, p2)) < -r) return false;
    }
    return true;
}

// EDGES: large triangles also get the edge axes (the fused and heavy passes;
// the one-lane pass over deferred candidates is faster without them).
template <bool R2O, bool EDGES = true>
__device__ __forceinline__ bool stage_b_node(const StageBCand& C, const Box& b) {
    constexpr float kBoxTol = 2e-5f;
    if (R2O)
        return box_overlap(b, C.blo, C.bhi) && plane_box(C.cn, C.cw, b, kBoxTol) &&
               (!EDGES || !C.big || tri_box_edges(C.c0, C.c1, C.c2, b, kBoxTol));
    return seg_box(C.c0, C.cinv, b, kBoxTol);
}

// Exact test of link primitive li against the candidate: FP32 with the FP64
// re-test of the undecided band.
template <bool R2O>
__device__ __forceinline__ bool stage_b_leaf(const float4* __restrict__ lp, const float4* __restrict__ wp,
                                             uint32_t li, const StageBCand& C, unsigned long long* stats) {
    f3 p, q, a, b, c;
    if (R2O) {
        const float4* e = lp + 2ull * li;
        p = f3of(__ldg(e)); q = f3of(__ldg(e + 1));
        a = C.c0; b = C.c1; c = C.c2;
    } else {
        const float4* t = lp + 3ull * li;
        p = C.c0; q = C.c1;
        a = f3of(__ldg(t)); b = f3of(__ldg(t + 1)); c = f3of(__ldg(t + 2));
    }
    int r = seg_tri_f32(p, q, a, b, c);
    if (r == 2) {
        atomicAdd(stats, 1ull);
        r = retest_f64<R2O>(C.T, lp, li, wp, C.prim) ? 1 : 0;
    }
    return r == 1;
}

// Stage B, light pass: one lane per candidate (grid-stride, so neighbouring
// lanes take neighbouring candidates of the same item).  A candidate still
// open after W.light_steps node and leaf visits goes to the heavy pass (hits
// already found stay: pose flags and edge bits are idempotent; ObsToRobot
// hit counts are added only when the candidate finishes here).  A candidate
// carries its (pose, link) item word, so one whose pose is already decided
// costs two loads.
template <bool R2O, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_stage_b(const RobotDev R, const SceneDev S, const WaveArgs W) {
    const DiscreteArgs& A = W.d;
    const float4* __restrict__ wp = R2O ? S.tri_prims : S.edge_prims;
    const float4* __restrict__ ln = R2O ? R.edge_nodes : R.tri_nodes;
    const float4* __restrict__ lp = R2O ? R.edge_prims : R.tri_prims;
    const uint32_t total = min(*W.cand_count, W.cand_cap);
    const uint32_t budget = W.light_steps ? W.light_steps : 0xFFFFFFFFu;
    uint32_t st[kStack];
    unsigned long long n_acc = 0, n_skip = 0, n_rej = 0, n_leaf = 0, n_node = 0;
    // each lane takes up to W.chunk consecutive candidates in order: a pose's
    // candidates spread over a few lanes that each stop at its first hit,
    // instead of over many lanes that all start before any hit is known.
    // A batch smaller than the grid keeps one candidate per lane (latency).
    const uint32_t K = max(1u, min(W.chunk, total / (gridDim.x * blockDim.x)));
    for (uint32_t cc = (blockIdx.x * blockDim.x + threadIdx.x) * K; cc < total; cc += gridDim.x * blockDim.x * K)
    for (uint32_t c = cc; c < min(cc + K, total); ++c) {
        StageBCand C;
        const uint2 cd = W.cand[c];
        if (!stage_b_setup<R2O>(R, S, W, cd, C, n_skip, n_rej)) continue;
        ++n_acc;
        int sp = 0;
        st[sp++] = C.lroot;
        uint32_t steps = 0, hits = 0;
        while (sp > 0) {
            if (++steps > budget) {
                const uint32_t slot = atomicAdd(W.heavy_count, 1u);
                if (slot < W.heavy_cap) {
                    W.heavy[slot] = cd;
                    hits = 0;
                    break;
                }
                steps = 0;  // the heavy list is full: finish the candidate here
            }
            const uint32_t ref = st[--sp];
            if (ref & kLeaf) {
                ++n_leaf;
                const uint32_t li = ref & ~kLeaf;
                if (stage_b_leaf<R2O>(lp, wp, li, C, A.stats)) {
                    if (!A.want_counts) {
                        atomicExch(A.pose_hit + C.pose, 1u);
                        break;
                    }
                    A.pose_hit[C.pose] = 1u;
                    if (R2O) {
                        const uint32_t eid = __float_as_uint(__ldg(lp + 2ull * li).w);
                        atomicOr(A.edge_bits + (size_t) C.pose * A.edge_words + (eid >> 5), 1u << (eid & 31));
                    } else {
                        ++hits;
                    }
                }
                continue;
            }
            Box bl, br;
            uint32_t rl, rr;
            load_node(ln, ref, bl, br, rl, rr);
            n_node += 2;
            const bool hr = stage_b_node<R2O, false>(C, br), hl = stage_b_node<R2O, false>(C, bl);
            if (sp + 2 > kStack) {
                atomicOr(A.err, kErrStack);
                break;
            }
            if (hr) st[sp++] = rr;
            if (hl) st[sp++] = rl;
        }
        if (hits) atomicAdd(A.counts + C.pose, hits);
    }
    warp_count(A.stats + 1, n_acc);
    warp_count(A.stats + 2, n_skip);
    warp_count(A.stats + 3, n_rej);
    warp_count(A.stats + 4, n_leaf);
    warp_count(A.stats + 7, n_node);
}

// Stage B, light pass in packets: a warp takes 32 consecutive candidates and
// splits them by item (stage A emits each item's candidates in contiguous
// runs, so a group is one item or a few).  The lanes of one item share the
// link LBVH and the pose: they descend it together as a packet - one node
// load per step for the whole warp, each lane testing the node against its
// own scene primitive, the node visited when any lane needs it - and test
// each reached leaf against their own primitives in one converged step.
// A packet still open after 4 * W.light_steps steps hands its candidates to
// the heavy pass.
template <bool R2O, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_stage_b_packet(const RobotDev R, const SceneDev S, const WaveArgs W) {
    const DiscreteArgs& A = W.d;
    const float4* __restrict__ wp = R2O ? S.tri_prims : S.edge_prims;
    const float4* __restrict__ ln = R2O ? R.edge_nodes : R.tri_nodes;
    const float4* __restrict__ lp = R2O ? R.edge_prims : R.tri_prims;
    const uint32_t total = min(*W.cand_count, W.cand_cap);
    const uint32_t budget = W.light_steps ? 4u * W.light_steps : 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t n_groups = (total + 31) / 32;
    const uint32_t warps = gridDim.x * (BLOCK / 32);
    uint32_t st[kStack];
    unsigned long long n_acc = 0, n_skip = 0, n_rej = 0, n_leaf = 0, n_node = 0;
    const uint32_t K = max(1u, min(W.chunk, n_groups / warps));  // consecutive groups per warp, in order
    for (uint32_t gg = (blockIdx.x * (BLOCK / 32) + (threadIdx.x >> 5)) * K; gg < n_groups; gg += warps * K)
    for (uint32_t g = gg; g < min(gg + K, n_groups); ++g) {
        const uint32_t c = g * 32 + lane;
        StageBCand C;
        uint2 cd = make_uint2(kNone, kNone);
        bool live = false;
        if (c < total) {
            cd = W.cand[c];
            live = stage_b_setup<R2O>(R, S, W, cd, C, n_skip, n_rej) != 0;
        }
        if (live) ++n_acc;
        const uint32_t same = __match_any_sync(0xffffffffu, live ? cd.x : kNone);
        uint32_t pending = __ballot_sync(0xffffffffu, live);
        while (pending) {
            const int leader = __ffs(pending) - 1;
            const uint32_t grp = __shfl_sync(0xffffffffu, same, leader) & pending;
            pending &= ~grp;
            const bool in = (grp >> lane) & 1u;
            const uint32_t pose = __shfl_sync(0xffffffffu, C.pose, leader);
            int sp = 0;
            st[sp++] = __shfl_sync(0xffffffffu, C.lroot, leader);
            uint32_t steps = 0, hits = 0;
            bool spilled = false;
            while (sp > 0) {
                if (++steps > budget) {
                    const uint32_t n = __popc(grp);
                    uint32_t base = 0;
                    if (lane == leader) base = atomicAdd(W.heavy_count, n);
                    base = __shfl_sync(0xffffffffu, base, leader);
                    if (base + n <= W.heavy_cap) {
                        if (in) W.heavy[base + __popc(grp & lt)] = cd;
                        spilled = true;
                        break;
                    }
                    // the heavy list is full: blank the reserved slots below the
                    // capacity (the heavy pass reads up to it) and finish here
                    if (in && base + __popc(grp & lt) < W.heavy_cap)
                        W.heavy[base + __popc(grp & lt)] = make_uint2(kNone, kNone);
                    steps = 0;
                }
                if (!A.want_counts && (steps & 15) == 0) {  // decided meanwhile by another candidate?
                    uint32_t dec = 0;
                    if (lane == leader) dec = ld_flag(A.pose_hit + pose);
                    if (__shfl_sync(0xffffffffu, dec, leader)) break;
                }
                const uint32_t ref = st[--sp];
                if (ref & kLeaf) {
                    const uint32_t li = ref & ~kLeaf;
                    bool hit = false;
                    if (in) {
                        ++n_leaf;
                        hit = stage_b_leaf<R2O>(lp, wp, li, C, A.stats);
                    }
                    const uint32_t hm = __ballot_sync(0xffffffffu, hit);
                    if (hm) {
                        if (!A.want_counts) {
                            if (lane == leader) atomicExch(A.pose_hit + pose, 1u);
                            break;
                        }
                        if (lane == leader) A.pose_hit[pose] = 1u;
                        if (hit) {
                            if (R2O) {
                                const uint32_t eid = __float_as_uint(__ldg(lp + 2ull * li).w);
                                atomicOr(A.edge_bits + (size_t) pose * A.edge_words + (eid >> 5), 1u << (eid & 31));
                            } else {
                                ++hits;
                            }
                        }
                    }
                    continue;
                }
                Box bl, br;
                uint32_t rl, rr;
                load_node(ln, ref, bl, br, rl, rr);
                if (in) n_node += 2;
                const bool hr = in && stage_b_node<R2O>(C, br), hl = in && stage_b_node<R2O>(C, bl);
                const bool any_r = __any_sync(0xffffffffu, hr), any_l = __any_sync(0xffffffffu, hl);
                if (sp + 2 > kStack) {
                    if (lane == leader) atomicOr(A.err, kErrStack);
                    break;
                }
                if (any_r) st[sp++] = rr;
                if (any_l) st[sp++] = rl;
            }
            if (hits && !spilled) atomicAdd(A.counts + pose, hits);
        }
    }
    warp_count(A.stats + 1, n_acc);
    warp_count(A.stats + 2, n_skip);
    warp_count(A.stats + 3, n_rej);
    warp_count(A.stats + 4, n_leaf);
    warp_count(A.stats + 7, n_node);
}

// Stages A and B in one warp per (pose, link) item.  The warp descends the
// scene's 4-wide tree with the link's OBB through a shared LIFO frontier
// (each step pops up to 32 nodes and spreads their children over the lanes:
// 4 lanes per node when at most 8 are waiting, 2 when at most 16, else one
// lane tests all four children of its node, so a step costs about one box
// test per lane and the descent half the dependent node loads of a binary
// tree), keeps the leaf survivors in a shared buffer and, 32 at a time, runs
// them through stage B at once (one lane per candidate, bounded by the light
// budget; longer candidates are written to the candidate buffer and handed
// to the heavy pass).  An item whose pose is found in collision stops
// generating candidates: most colliding items are decided after their first
// few candidates, so most of stage A's traversal and candidate traffic is
// never spent on them.  PACKET: the 32 buffered candidates (one item, so one
// link tree) descend the link LBVH together - one node load per step for the
// warp, each lane testing its own primitive - which shares the top levels of
// the link tree when many small scene primitives crowd one link.
constexpr int kAbWarps = 4;
constexpr int kCandBuf = 32 + 32 * kWide;  // < 32 waiting + up to 32 * kWide added by one frontier step

// The link OBB of an item in the world frame, padded by the box tolerance,
// and its world-axis half extents.
__device__ __forceinline__ void item_box(const RobotDev& R, const DiscreteArgs& A, uint32_t pose, uint32_t link,
                                         ObbW& ob, f3& ext) {
    constexpr float kBoxTol = 2e-5f;
    float4 T[3];
    const float4* tp = A.T + ((size_t) pose * R.n_links + link) * 3;
    T[0] = tp[0]; T[1] = tp[1]; T[2] = tp[2];
    ob = world_obb(R.obb[link], T);
    ob.h = mk(ob.h.x + kBoxTol, ob.h.y + kBoxTol, ob.h.z + kBoxTol);
    ext = mk(fabsf(ob.ax[0].x) * ob.h.x + fabsf(ob.ax[1].x) * ob.h.y + fabsf(ob.ax[2].x) * ob.h.z,
             fabsf(ob.ax[0].y) * ob.h.x + fabsf(ob.ax[1].y) * ob.h.y + fabsf(ob.ax[2].y) * ob.h.z,
             fabsf(ob.ax[0].z) * ob.h.x + fabsf(ob.ax[1].z) * ob.h.y + fabsf(ob.ax[2].z) * ob.h.z);
}

// Marks an item for the thread-per-item fallback once, however many warps
// give up on it (one byte per item in a word-aligned buffer with 3 spare bytes).
__device__ __forceinline__ void mark_overflow(const WaveArgs& W, uint32_t item) {
    unsigned* word = reinterpret_cast<unsigned*>(W.item_overflow + (item & ~3u));
    const unsigned bit = 1u << (8 * (item & 3u));
    if (!(atomicOr(word, bit) & bit)) W.overflow_items[atomicAdd(W.overflow_count, 1u)] = item;
}

// The OBB test of the wide descents (wide.cuh) of the fused and subtree kernels.
struct ObbTest {
    const ObbW& ob;
    const f3& ext;
    __device__ __forceinline__ bool operator()(const Box& b) const { return obb_aabb(b, ob, ext); }
};

// Register caps (measured on the 65,536-pose dense workload and the dense
// shelf): RobotToObs at 5 resident blocks per SM (96 registers, a few spills;
// more warps to hide the node-load latency: 4 blocks at 128 registers was 7 %
// slower), ObsToRobot at 4 (128 registers, no spills: 2-4 % faster than 5).
// TOP: the first W.top_nodes wide nodes are staged in shared memory after the
// frontiers and read from there (a separate instantiation, so the default
// kernel's node loads carry no branch).
template <bool R2O, bool PACKET, bool TOP>
__global__ void __launch_bounds__(kAbWarps * 32, R2O ? 5 : 4) k_stage_ab(const RobotDev R, const SceneDev S, const WaveArgs W) {
    extern __shared__ uint32_t s_front[];  // [kAbWarps][S.wide_front], then (TOP) the staged wide nodes
    __shared__ uint32_t s_cand[kAbWarps][kCandBuf];
    __shared__ uint32_t s_hits[kAbWarps];  // a lane of the warp's current stage-B step hit its pose
    const DiscreteArgs& A = W.d;
    const int lane = threadIdx.x & 31;
    uint32_t* fr = s_front + (threadIdx.x >> 5) * S.wide_front;
    uint32_t* cb = s_cand[threadIdx.x >> 5];
    volatile uint32_t* s_hit = s_hits + (threadIdx.x >> 5);
    const uint32_t lt = (1u << lane) - 1u;
    const float4* __restrict__ wn = R2O ? S.tri_wide : S.edge_wide;
    const float4* __restrict__ wp = R2O ? S.tri_prims : S.edge_prims;
    const uint32_t wroot = R2O ? S.tri_wide_root : S.edge_wide_root;
    const float4* __restrict__ ln = R2O ? R.edge_nodes : R.tri_nodes;
    const float4* __restrict__ lp = R2O ? R.edge_prims : R.tri_prims;
    const uint32_t n_items = *A.n_items;
    const uint32_t budget = W.light_steps ? W.light_steps : 0xFFFFFFFFu;
    // the tree's top levels in shared memory (its first nodes, breadth-first), read by every descent
    const uint32_t n_top = TOP ? min(W.top_nodes, R2O ? S.n_tri_wide : S.n_edge_wide) : 0u;
    float4* s_top = reinterpret_cast<float4*>(s_front + ((kAbWarps * S.wide_front + 3u) & ~3u));
    if constexpr (TOP) {
        for (uint32_t k = threadIdx.x; k < n_top * 2 * kWide; k += blockDim.x) s_top[k] = __ldg(wn + k);
        __syncthreads();
    }
    uint32_t st[kStack];
    unsigned long long n_acc = 0, n_skip = 0, n_rej = 0, n_leaf = 0, n_cand = 0, n_node = 0;
    while (true) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(A.work_counter, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= n_items) break;
        const uint32_t item = item_word(A, R.n_links, A.items[it]);
        const uint32_t pose = item / R.n_links, link = item - pose * R.n_links;
        if (pose >= A.n_poses) {
            if (lane == 0) atomicOr(A.err, kErrRange);
            continue;
        }
        uint32_t dec = 0;
        if (lane == 0 && !A.want_counts) dec = ld_flag(A.pose_hit + pose);
        if (wroot == kNone || __shfl_sync(0xffffffffu, dec, 0)) continue;
        ObbW ob;
        f3 ext;
        item_box(R, A, pose, link, ob, ext);
        // the descent starts with the tree's top cut; a one-primitive scene's root is its only candidate
        int sp = 0, nc = 0;
        uint32_t nbs = 0;  // stage-B steps this item ran in its warp
        bool overflow = false;
        if (wroot & kLeaf) {
            if (lane == 0) cb[0] = wroot & ~kLeaf;
            nc = 1;
            __syncwarp();
        } else if (!cut_step(R2O ? S.tri_cut : S.edge_cut, R2O ? S.n_tri_cut : S.n_edge_cut, fr, sp, cb, nc,
                             ObbTest{ob, ext}, S.wide_front, A.err, n_node, n_cand)) {
            continue;
        }
        while (true) {
            if (nc >= 32 || (sp == 0 && nc > 0)) {  // stage B on up to 32 buffered candidates
                const int take = min(nc, 32);
                nc -= take;
                const uint32_t prim = lane < take ? cb[nc + lane] : kNone;
                __syncwarp();
                if (!A.want_counts && nbs >= W.item_steps) {
                    // a crowded item: its further candidates go to the one-lane pass, which
                    // spreads them over the whole GPU instead of this warp's serial steps
                    uint32_t base = 0, d2 = 0;
                    if (lane == 0) {
                        d2 = ld_flag(A.pose_hit + pose);  // decided by another item: stop enumerating
                        if (!d2) base = atomicAdd(W.cand_count, (uint32_t) take);
                    }
                    if (__shfl_sync(0xffffffffu, d2, 0)) break;
                    base = __shfl_sync(0xffffffffu, base, 0);
                    if (base + (uint32_t) take <= W.cand_cap) {
                        if (prim != kNone) W.cand[base + lane] = make_uint2(item, prim);
                        if (sp > 0) {
                            // and the rest of its descent to the subtree pass, one warp per frontier
                            // node, so no single warp walks a crowded item's whole overlap
                            uint32_t sb = 0;
                            if (lane == 0) sb = atomicAdd(W.sub_count, (uint32_t) sp);
                            sb = __shfl_sync(0xffffffffu, sb, 0);
                            const bool fits = sb + (uint32_t) sp <= W.sub_cap;
                            for (int i = lane; i < sp; i += 32)  // slots below the capacity are always written
                                if (sb + i < W.sub_cap) W.sub[sb + i] = fits ? make_uint2(item, fr[i]) : make_uint2(kNone, kNone);
                            __syncwarp();
                            if (!fits) {
                                overflow = true;
                                break;
                            }
                            sp = 0;
                        }
                        continue;
                    }
                    // no room: blank the reserved slots below the capacity and hand the whole
                    // item to the thread-per-item kernel (flags only, so re-running is safe)
                    if (prim != kNone && base + lane < W.cand_cap) W.cand[base + lane] = make_uint2(kNone, kNone);
                    overflow = true;
                    break;
                }
                ++nbs;
                bool hit = false;
                StageBCand C;
                if (lane == 0) *s_hit = 0u;
                __syncwarp();
                if (PACKET) {
                    const bool live =
                        prim != kNone && stage_b_setup<R2O>(R, S, W, make_uint2(item, prim), C, n_skip, n_rej, false);
                    const uint32_t grp = __ballot_sync(0xffffffffu, live);
                    if (live) ++n_acc;
                    if (grp) {
                        int bsp = 0;
                        st[bsp++] = R2O ? R.edge_root[link] : R.tri_root[link];
                        uint32_t steps = 0, hits = 0;
                        bool spilled = false;
                        const uint32_t rank = __popc(grp & lt), np = __popc(grp);
                        while (bsp > 0) {
                            if (++steps > 4u * budget) {  // hand the packet's candidates to the heavy pass
                                uint32_t hbase = 0;
                                if (lane == 0) hbase = atomicAdd(W.heavy_count, np);
                                hbase = __shfl_sync(0xffffffffu, hbase, 0);
                                const bool fits = hbase + np <= W.heavy_cap;
                                // heavy slots below the capacity are always written (blank when the
                                // packet stays here), since the heavy pass reads up to it
                                if (live && hbase + rank < W.heavy_cap)
                                    W.heavy[hbase + rank] = fits ? make_uint2(item, prim) : make_uint2(kNone, kNone);
                                if (fits) {
                                    spilled = true;
                                    break;
                                }
                                steps = 0;  // no room: finish the packet here
                            }
                            const uint32_t ref = st[--bsp];
                            if (ref & kLeaf) {
                                const uint32_t li = ref & ~kLeaf;
                                bool h = false;
                                if (live) {
                                    ++n_leaf;
                                    h = stage_b_leaf<R2O>(lp, wp, li, C, A.stats);
                                }
                                if (__any_sync(0xffffffffu, h)) {
                                    hit = true;
                                    if (!A.want_counts) break;
                                    if (h) {
                                        if (R2O) {
                                            const uint32_t eid = __float_as_uint(__ldg(lp + 2ull * li).w);
                                            atomicOr(A.edge_bits + (size_t) pose * A.edge_words + (eid >> 5),
                                                     1u << (eid & 31));
                                        } else {
                                            ++hits;
                                        }
                                    }
                                }
                                continue;
                            }
                            Box bl, br;
                            uint32_t rl, rr;
                            load_node(ln, ref, bl, br, rl, rr);
                            if (live) n_node += 2;
                            const bool hr = live && stage_b_node<R2O>(C, br), hl = live && stage_b_node<R2O>(C, bl);
                            const bool any_r = __any_sync(0xffffffffu, hr), any_l = __any_sync(0xffffffffu, hl);
                            if (bsp + 2 > kStack) {
                                if (lane == 0) atomicOr(A.err, kErrStack);
                                break;
                            }
                            if (any_r) st[bsp++] = rr;
                            if (any_l) st[bsp++] = rl;
                        }
                        if (hits && !spilled) atomicAdd(A.counts + pose, hits);
                    }
                } else if (prim != kNone && stage_b_setup<R2O>(R, S, W, make_uint2(item, prim), C, n_skip, n_rej, false)) {
                    ++n_acc;
                    int bsp = 0;
                    st[bsp++] = C.lroot;
                    uint32_t steps = 0, hits = 0;
                    bool spilled = false;
                    while (bsp > 0) {
                        // flags only: another lane of this step has hit the pose, so the rest is moot
                        if (!A.want_counts && *s_hit) break;
                        if (++steps > budget) {
                            const uint32_t h = atomicAdd(W.heavy_count, 1u);
                            if (h < W.heavy_cap) {
                                W.heavy[h] = make_uint2(item, prim);
                                spilled = true;
                                break;
                            }
                            steps = 0;  // no room: finish the candidate here
                        }
                        const uint32_t ref = st[--bsp];
                        if (ref & kLeaf) {
                            ++n_leaf;
                            const uint32_t li = ref & ~kLeaf;
                            if (stage_b_leaf<R2O>(lp, wp, li, C, A.stats)) {
                                hit = true;
                                if (!A.want_counts) {
                                    *s_hit = 1u;
                                    break;
                                }
                                if (R2O) {
                                    const uint32_t eid = __float_as_uint(__ldg(lp + 2ull * li).w);
                                    atomicOr(A.edge_bits + (size_t) pose * A.edge_words + (eid >> 5), 1u << (eid & 31));
                                } else {
                                    ++hits;
                                }
                            }
                            continue;
                        }
                        Box bl, br;
                        uint32_t rl, rr;
                        load_node(ln, ref, bl, br, rl, rr);
                        n_node += 2;
                        const bool hr = stage_b_node<R2O>(C, br), hl = stage_b_node<R2O>(C, bl);
                        if (bsp + 2 > kStack) {
                            atomicOr(A.err, kErrStack);
                            break;
                        }
                        if (hr) st[bsp++] = rr;
                        if (hl) st[bsp++] = rl;
                    }
                    if (hits && !spilled) atomicAdd(A.counts + pose, hits);
                }
                const bool any = __any_sync(0xffffffffu, hit);
                if (any) {
                    if (lane == 0) {
                        if (A.want_counts) A.pose_hit[pose] = 1u;
                        else atomicExch(A.pose_hit + pose, 1u);
                    }
                    if (!A.want_counts) break;
                }
                if (!A.want_counts) {  // decided meanwhile by another item?
                    uint32_t d2 = 0;
                    if (lane == 0) d2 = ld_flag(A.pose_hit + pose);
                    if (__shfl_sync(0xffffffffu, d2, 0)) break;
                }
                continue;
            }
            if (sp == 0) break;
            if (!wide_step<TOP>(wn, fr, sp, cb, nc, ObbTest{ob, ext}, S.wide_front, A.err, n_node, n_cand, s_top, n_top))
                break;
        }
        if (overflow && lane == 0) mark_overflow(W, item);
        __syncwarp();
    }
    warp_count(A.stats + 1, n_acc);
    warp_count(A.stats + 2, n_skip);
    warp_count(A.stats + 3, n_rej);
    warp_count(A.stats + 4, n_leaf);
    warp_count(A.stats + 7, n_node);
    warp_count(A.stats + 6, n_cand);
}

// The subtree pass: the rest of a crowded item's scene descent, one warp
// per frontier node the fused kernel handed over.  Every leaf that overlaps
// the item's OBB is appended to the candidate buffer for the one-lane pass
// (32 or more at a time); a subtree stops when its pose is decided.  When the
// buffer is full the item goes to the thread-per-item fallback (flags only,
// like every deferral).  It runs twice.  The first launch (SPLIT) takes the
// fused kernel's nodes and descends breadth-first - while at most 32 nodes
// wait, every step pops them all, so the frontier holds one level - and as
// soon as a level is wider than 32 nodes hands those nodes to the second
// launch, which descends each to the end: a large subtree becomes many
// pieces of equal depth on as many warps instead of one warp's serial walk.
template <bool R2O, bool SPLIT>
__global__ void __launch_bounds__(kAbWarps * 32) k_subtree(const RobotDev R, const SceneDev S, const WaveArgs W) {
    extern __shared__ uint32_t s_front[];  // [kAbWarps][S.wide_front]
    __shared__ uint32_t s_cand[kAbWarps][kCandBuf];
    const DiscreteArgs& A = W.d;
    const int lane = threadIdx.x & 31;
    uint32_t* fr = s_front + (threadIdx.x >> 5) * S.wide_front;
    uint32_t* cb = s_cand[threadIdx.x >> 5];
    const float4* __restrict__ wn = R2O ? S.tri_wide : S.edge_wide;
    const uint2* src = SPLIT ? W.sub : W.sub + W.sub_cap;  // the second half holds the split pieces
    const uint32_t n_sub = min(SPLIT ? W.sub_count[0] : W.sub_count[2], W.sub_cap);
    uint32_t* work = SPLIT ? W.sub_count + 1 : W.sub_count + 3;
    unsigned long long n_node = 0, n_cand = 0;
    while (true) {
        uint32_t h = 0;
        if (lane == 0) h = atomicAdd(work, 1u);
        h = __shfl_sync(0xffffffffu, h, 0);
        if (h >= n_sub) break;
        const uint2 pr = src[h];
        if (pr.x == kNone) continue;  // a blanked slot of a reservation that did not fit
        const uint32_t item = pr.x, pose = item / R.n_links, link = item - pose * R.n_links;
        if (pose >= A.n_poses) {
            if (lane == 0) atomicOr(A.err, kErrRange);
            continue;
        }
        uint32_t skip = 0;
        if (lane == 0) skip = W.item_overflow[item] | ld_flag(A.pose_hit + pose);
        if (__shfl_sync(0xffffffffu, skip, 0)) continue;  // re-run whole by the fallback, or decided
        ObbW ob;
        f3 ext;
        item_box(R, A, pose, link, ob, ext);
        int sp = 1, nc = 0;
        if (lane == 0) fr[0] = pr.y;
        __syncwarp();
        while (true) {
            if (nc >= 32 || (sp == 0 && nc > 0)) {  // flush every buffered candidate
                uint32_t base = 0, dec = 0;
                if (lane == 0) {
                    dec = ld_flag(A.pose_hit + pose);
                    if (!dec) base = atomicAdd(W.cand_count, (uint32_t) nc);
                }
                if (__shfl_sync(0xffffffffu, dec, 0)) break;
                base = __shfl_sync(0xffffffffu, base, 0);
                const bool fits = base + (uint32_t) nc <= W.cand_cap;
                for (int i = lane; i < nc; i += 32)  // slots below the capacity are always written
                    if (base + i < W.cand_cap) W.cand[base + i] = fits ? make_uint2(item, cb[i]) : make_uint2(kNone, kNone);
                __syncwarp();
                nc = 0;
                if (!fits) {
                    if (lane == 0) mark_overflow(W, item);
                    break;
                }
                continue;
            }
            if (sp == 0) break;
            if (SPLIT && sp > 32) {  // one level wider than a step: hand its nodes to the second launch
                uint32_t sb = 0;
                if (lane == 0) sb = atomicAdd(W.sub_count + 2, (uint32_t) sp);
                sb = __shfl_sync(0xffffffffu, sb, 0);
                const bool fits = sb + (uint32_t) sp <= W.sub_cap;
                uint2* dst = W.sub + W.sub_cap;
                for (int i = lane; i < sp; i += 32)  // slots below the capacity are always written
                    if (sb + i < W.sub_cap) dst[sb + i] = fits ? make_uint2(item, fr[i]) : make_uint2(kNone, kNone);
                __syncwarp();
                if (!fits && lane == 0) mark_overflow(W, item);
                sp = 0;
                if (!fits) break;
                continue;  // flush what is buffered, then the item is done here
            }
            if (!wide_step(wn, fr, sp, cb, nc, ObbTest{ob, ext}, S.wide_front, A.err, n_node, n_cand)) break;
        }
        __syncwarp();
    }
    warp_count(A.stats + 7, n_node);
    warp_count(A.stats + 6, n_cand);
}

// Stage B, heavy pass: one warp per spilled candidate.  The warp descends the
// link LBVH through a shared LIFO frontier (up to 32 nodes a step) and tests
// the surviving leaves 32 at a time, one per lane.
constexpr int kHeavyWarps = 4;
constexpr int kLeafBuf = 96;  // < 32 waiting + up to 64 added by one node step

template <bool R2O>
__global__ void __launch_bounds__(kHeavyWarps * 32) k_stage_b_heavy(const RobotDev R, const SceneDev S,
                                                                   const WaveArgs W) {
    __shared__ uint32_t s_front[kHeavyWarps][kFrontier];
    __shared__ uint32_t s_leaf[kHeavyWarps][kLeafBuf];
    const DiscreteArgs& A = W.d;
    const float4* __restrict__ wp = R2O ? S.tri_prims : S.edge_prims;
    const float4* __restrict__ ln = R2O ? R.edge_nodes : R.tri_nodes;
    const float4* __restrict__ lp = R2O ? R.edge_prims : R.tri_prims;
    const int lane = threadIdx.x & 31;
    uint32_t* fr = s_front[threadIdx.x >> 5];
    uint32_t* lf = s_leaf[threadIdx.x >> 5];
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t n_heavy = min(*W.heavy_count, W.heavy_cap);
    unsigned long long n_skip = 0, n_rej = 0, n_leaf = 0, n_node = 0;
    while (true) {
        uint32_t h = 0;
        if (lane == 0) h = atomicAdd(W.heavy_work, 1u);
        h = __shfl_sync(0xffffffffu, h, 0);
        if (h >= n_heavy) break;
        const uint2 cd = W.heavy[h];
        if (cd.x == kNone) continue;  // a blanked slot of a reservation that did not fit
        StageBCand C;
        if (!stage_b_setup<R2O>(R, S, W, cd, C, n_skip, n_rej, false)) continue;  // warp-uniform
        if (!A.want_counts) {  // decided meanwhile? (one lane reads, all follow)
            uint32_t dec = 0;
            if (lane == 0) dec = ld_flag(A.pose_hit + C.pose);
            if (__shfl_sync(0xffffffffu, dec, 0)) continue;
        }
        if (lane == 0) fr[0] = C.lroot;
        __syncwarp();
        int sp = 1, nl = 0, step = 0;
        uint32_t hits = 0;
        while (true) {
            if (nl >= 32 || (sp == 0 && nl > 0)) {  // leaf step
                const int take = min(nl, 32);
                nl -= take;
                const uint32_t li = lane < take ? lf[nl + lane] : kNone;
                __syncwarp();
                bool hit = false;
                if (li != kNone) {
                    ++n_leaf;
                    hit = stage_b_leaf<R2O>(lp, wp, li, C, A.stats);
                }
                const uint32_t mh = __ballot_sync(0xffffffffu, hit);
                if (mh) {
                    if (!A.want_counts) {
                        if (lane == 0) atomicExch(A.pose_hit + C.pose, 1u);
                        break;
                    }
                    if (lane == 0) A.pose_hit[C.pose] = 1u;
                    if (R2O) {
                        if (hit) {
                            const uint32_t eid = __float_as_uint(__ldg(lp + 2ull * li).w);
                            atomicOr(A.edge_bits + (size_t) C.pose * A.edge_words + (eid >> 5), 1u << (eid & 31));
                        }
                    } else {
                        hits += __popc(mh);
                    }
                }
                continue;
            }
            if (sp == 0) break;
            if (!A.want_counts && (++step & 7) == 0) {  // decided meanwhile by another candidate?
                uint32_t dec = 0;
                if (lane == 0) dec = ld_flag(A.pose_hit + C.pose);
                if (__shfl_sync(0xffffffffu, dec, 0)) break;
            }
            const int take = min(sp, 32);
            sp -= take;
            const uint32_t ref = lane < take ? fr[sp + lane] : kNone;
            __syncwarp();
            bool hl = false, hr = false;
            uint32_t rl = kNone, rr = kNone;
            if (ref != kNone) {
                if (ref & kLeaf) {  // a one-primitive link: the root itself is a leaf
                    hl = true;
                    rl = ref;
                } else {
                    Box bl, br;
                    load_node(ln, ref, bl, br, rl, rr);
                    n_node += 2;
                    hl = stage_b_node<R2O>(C, bl);
                    hr = stage_b_node<R2O>(C, br);
                }
            }
            const bool pl = hl && !(rl & kLeaf), pr = hr && !(rr & kLeaf);
            const bool el = hl && (rl & kLeaf), er = hr && (rr & kLeaf);
            const uint32_t mpl = __ballot_sync(0xffffffffu, pl), mpr = __ballot_sync(0xffffffffu, pr);
            const uint32_t mel = __ballot_sync(0xffffffffu, el), mer = __ballot_sync(0xffffffffu, er);
            const int npush = __popc(mpl) + __popc(mpr);
            if (sp + npush > kFrontier) {  // cannot happen for trees within the depth limit
                if (lane == 0) atomicOr(A.err, kErrStack);
                break;
            }
            if (pl) fr[sp + __popc(mpl & lt)] = rl;
            if (pr) fr[sp + __popc(mpl) + __popc(mpr & lt)] = rr;
            sp += npush;
            if (el) lf[nl + __popc(mel & lt)] = rl & ~kLeaf;
            if (er) lf[nl + __popc(mel) + __popc(mer & lt)] = rr & ~kLeaf;
            nl += __popc(mel) + __popc(mer);
            __syncwarp();
        }
        if (lane == 0 && hits) atomicAdd(A.counts + C.pose, hits);
        __syncwarp();
    }
    warp_count(A.stats + 4, n_leaf);
    warp_count(A.stats + 7, n_node);
}

template <class K>
static uint32_t grid_for(K kernel, int threads) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
    return (uint32_t) std::max(1, per_sm) * (uint32_t) device_sm_count();
}

uint32_t stage_a_blocks(bool r2o) {
    return r2o ? grid_for(k_stage_a<true>, kStageAWarps * 32) : grid_for(k_stage_a<false>, kStageAWarps * 32);
}
template <bool R2O>
static int stage_b_per_sm(int threads) {
    int per_sm = 0;
    if (threads == 64)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stage_b<R2O, 64>, 64, 0);
    else if (threads == 256)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stage_b<R2O, 256>, 256, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stage_b<R2O, 128>, 128, 0);
    return std::max(1, per_sm);
}

uint32_t stage_b_max_blocks_per_sm(bool r2o, uint32_t threads) {
    return (uint32_t) (r2o ? stage_b_per_sm<true>((int) threads) : stage_b_per_sm<false>((int) threads));
}

uint32_t stage_b_blocks(bool r2o) { return stage_b_max_blocks_per_sm(r2o, kTravThreads) * device_sm_count(); }

void launch_stage_a(bool r2o, const RobotDev& R, const SceneDev& S, const WaveArgs& W, uint32_t blocks,
                    cudaStream_t s) {
    if (r2o)
        k_stage_a<true><<<blocks, kStageAWarps * 32, 0, s>>>(R, S, W);
    else
        k_stage_a<false><<<blocks, kStageAWarps * 32, 0, s>>>(R, S, W);
    cuda_check(cudaGetLastError(), "k_stage_a");
}

template <bool R2O>
static void stage_b_dispatch(const RobotDev& R, const SceneDev& S, const WaveArgs& W, uint32_t blocks,
                             uint32_t threads, bool packets, cudaStream_t s) {
    if (packets) {
        if (threads == 64)
            k_stage_b_packet<R2O, 64><<<blocks, 64, 0, s>>>(R, S, W);
        else if (threads == 256)
            k_stage_b_packet<R2O, 256><<<blocks, 256, 0, s>>>(R, S, W);
        else
            k_stage_b_packet<R2O, 128><<<blocks, 128, 0, s>>>(R, S, W);
        return;
    }
    if (threads == 64)
        k_stage_b<R2O, 64><<<blocks, 64, 0, s>>>(R, S, W);
    else if (threads == 256)
        k_stage_b<R2O, 256><<<blocks, 256, 0, s>>>(R, S, W);
    else
        k_stage_b<R2O, 128><<<blocks, 128, 0, s>>>(R, S, W);
}

void launch_stage_b(bool r2o, const RobotDev& R, const SceneDev& S, const WaveArgs& W, uint32_t blocks,
                    uint32_t threads, uint32_t heavy_share, bool packets, cudaStream_t s) {
    if (r2o)
        stage_b_dispatch<true>(R, S, W, blocks, threads, packets, s);
    else
        stage_b_dispatch<false>(R, S, W, blocks, threads, packets, s);
    cuda_check(cudaGetLastError(), "k_stage_b");
    launch_stage_b_heavy(r2o, R, S, W, heavy_share, s);
}

void launch_stage_b_heavy(bool r2o, const RobotDev& R, const SceneDev& S, const WaveArgs& W, uint32_t heavy_share,
                          cudaStream_t s) {
    if (!W.light_steps) return;
    static const uint32_t full_r2o = grid_for(k_stage_b_heavy<true>, kHeavyWarps * 32);
    static const uint32_t full_o2r = grid_for(k_stage_b_heavy<false>, kHeavyWarps * 32);
    const uint32_t hb = std::max(1u, (r2o ? full_r2o : full_o2r) * heavy_share / 100);
    if (r2o)
        k_stage_b_heavy<true><<<hb, kHeavyWarps * 32, 0, s>>>(R, S, W);
    else
        k_stage_b_heavy<false><<<hb, kHeavyWarps * 32, 0, s>>>(R, S, W);
    cuda_check(cudaGetLastError(), "k_stage_b_heavy");
}

// The fused kernel's frontier lives in dynamic shared memory, sized from the
// scene's wide-tree depth.
static size_t stage_ab_smem(const SceneDev& S) { return sizeof(uint32_t) * kAbWarps * (size_t) S.wide_front; }
// with top_nodes wide nodes staged after the frontiers (16-byte aligned)
static size_t stage_ab_smem(const SceneDev& S, uint32_t top_nodes) {
    return ((stage_ab_smem(S) + 15) & ~size_t(15)) + (size_t) top_nodes * 2 * kWide * sizeof(float4);
}

template <class K>
static uint32_t stage_ab_grid(K kernel, size_t smem) {
    // beyond the default 48 KB a block needs the opt-in (trees deeper than ~44 wide levels;
    // the deepest accepted tree needs about 96 KB)
    if (smem + sizeof(uint32_t) * kAbWarps * kCandBuf > 48 * 1024)
        cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem),
                   "k_stage_ab shared memory");
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kAbWarps * 32, smem);
    return (uint32_t) std::max(1, per_sm) * (uint32_t) device_sm_count();
}

// Runs f with the k_stage_ab instantiation for (r2o, packets, top).
template <class F>
static auto with_stage_ab(bool r2o, bool packets, bool top, F&& f) {
    if (top) {
        if (packets) return r2o ? f(k_stage_ab<true, true, true>) : f(k_stage_ab<false, true, true>);
        return r2o ? f(k_stage_ab<true, false, true>) : f(k_stage_ab<false, false, true>);
    }
    if (packets) return r2o ? f(k_stage_ab<true, true, false>) : f(k_stage_ab<false, true, false>);
    return r2o ? f(k_stage_ab<true, false, false>) : f(k_stage_ab<false, false, false>);
}

uint32_t stage_ab_blocks(bool r2o, bool packets, const SceneDev& S) {
    const size_t smem = stage_ab_smem(S);
    return with_stage_ab(r2o, packets, false, [&](auto kernel) { return stage_ab_grid(kernel, smem); });
}

void launch_subtree(bool r2o, const RobotDev& R, const SceneDev& S, const WaveArgs& W, uint32_t share, cudaStream_t s) {
    const size_t smem = stage_ab_smem(S);
    const uint32_t full = r2o ? stage_ab_grid(k_subtree<true, true>, smem) : stage_ab_grid(k_subtree<false, true>, smem);
    const uint32_t blocks = std::max(1u, full * share / 100);
    if (r2o) {
        stage_ab_grid(k_subtree<true, false>, smem);
        k_subtree<true, true><<<blocks, kAbWarps * 32, smem, s>>>(R, S, W);
        k_subtree<true, false><<<blocks, kAbWarps * 32, smem, s>>>(R, S, W);
    } else {
        stage_ab_grid(k_subtree<false, false>, smem);
        k_subtree<false, true><<<blocks, kAbWarps * 32, smem, s>>>(R, S, W);
        k_subtree<false, false><<<blocks, kAbWarps * 32, smem, s>>>(R, S, W);
    }
    cuda_check(cudaGetLastError(), "k_subtree");
}

void launch_stage_ab(bool r2o, bool packets, const RobotDev& R, const SceneDev& S, const WaveArgs& W, uint32_t blocks,
                     cudaStream_t s) {
    const uint32_t top = std::min(W.top_nodes, r2o ? S.n_tri_wide : S.n_edge_wide);
    const size_t smem = stage_ab_smem(S, top);
    with_stage_ab(r2o, packets, top != 0, [&](auto kernel) {
        // sets the shared-memory limit before the first launch, and caps the grid at what fits
        const uint32_t b = std::min(blocks, stage_ab_grid(kernel, smem));
        kernel<<<b, kAbWarps * 32, smem, s>>>(R, S, W);
        return 0;
    });
    cuda_check(cudaGetLastError(), "k_stage_ab");
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

// Diagnostics of the segment-triangle arithmetic: per pair the FP32 filter's
// class (0 certain miss, 1 certain hit, 2 handed to FP64) and the FP64
// re-test's decision, on pairs given in world coordinates.
__global__ void k_probe_segtri(const float* __restrict__ seg, const float* __restrict__ tri, uint32_t n,
                               float* __restrict__ cls, double* __restrict__ dec) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* e = seg + 6ull * i;
    const float* t = tri + 9ull * i;
    const f3 p = mk(e[0], e[1], e[2]), q = mk(e[3], e[4], e[5]);
    const f3 a = mk(t[0], t[1], t[2]), b = mk(t[3], t[4], t[5]), c = mk(t[6], t[7], t[8]);
    cls[i] = (float) seg_tri_f32(p, q, a, b, c);
    dec[i] = seg_tri_f64(d3of(p), d3of(q), d3of(a), d3of(b), d3of(c)) ? 1.0 : 0.0;
}

void launch_probe_segtri(const float* d_seg, const float* d_tri, uint32_t n, float* d_cls, double* d_dec,
                         cudaStream_t s) {
    if (!n) return;
    k_probe_segtri<<<(n + 127) / 128, 128, 0, s>>>(d_seg, d_tri, n, d_cls, d_dec);
    cuda_check(cudaGetLastError(), "k_probe_segtri");
}

void launch_popcount_rows(const uint32_t* d_bits, uint32_t words, uint32_t rows, uint32_t* d_out, cudaStream_t s) {
    if (!rows) return;
    k_popcount_rows<<<rows, 128, 0, s>>>(d_bits, words, rows, d_out);
    cuda_check(cudaGetLastError(), "k_popcount_rows");
}

__global__ void k_flags(const uint32_t* __restrict__ hit, const uint32_t* __restrict__ contain, uint32_t n,
                        uint8_t* __restrict__ flags) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[i] = (hit[i] ? 1 : 0) | (contain && contain[i] ? 2 : 0);
}

// ---------------------------------------------------------------- containment
// A pose whose meshes cross nowhere can still collide: a link inside an
// obstacle, or an obstacle inside a link.  The reference's ray tests cannot
// see that (they only follow surface crossings).  For every item of a pose
// not yet hit and every obstacle whose OBB overlaps the link's (the cull's
// SAT), a ray from one vertex of the link (of the obstacle) in a fixed
// direction is clipped beyond the obstacle's box (the link's OBB) and its
// crossings with that obstacle's triangles (the link's triangles) are
// counted: an odd count means the vertex, and with no surface crossing the
// whole mesh, is inside.  Both meshes are closed.
__device__ __forceinline__ f3 contain_dir() { return mk(0.48f, 0.6f, 0.64f); }

// Crossings of the segment p -> q with the triangles of one tree whose tag
// (third float4's w) equals `tag` (any tag when tag == kNone).
__device__ uint32_t count_crossings(const float4* __restrict__ nodes, const float4* __restrict__ prims, uint32_t root,
                                    f3 p, f3 q, uint32_t tag, uint32_t* err) {
    constexpr float kBoxTol = 2e-5f;
    if (root == kNone) return 0;
    const f3 d = q - p;
    const f3 inv = mk(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    uint32_t st[kStack];
    int sp = 0;
    st[sp++] = root;
    uint32_t n = 0;
    while (sp > 0) {
        const uint32_t ref = st[--sp];
        if (ref & kLeaf) {
            const float4* t = prims + 3ull * (ref & ~kLeaf);
            const float4 a = __ldg(t), b = __ldg(t + 1), c = __ldg(t + 2);
            if (tag != kNone && __float_as_uint(c.w) != tag) continue;
            int r = seg_tri_f32(p, q, f3of(a), f3of(b), f3of(c));
            if (r == 2) r = seg_tri_f64(d3of(p), d3of(q), d3of(f3of(a)), d3of(f3of(b)), d3of(f3of(c))) ? 1 : 0;
            n += (uint32_t) r;
            continue;
        }
        Box bl, br;
        uint32_t rl, rr;
        load_node(nodes, ref, bl, br, rl, rr);
        const bool hr = seg_box(p, inv, br, kBoxTol), hl = seg_box(p, inv, bl, kBoxTol);
        if (sp + 2 > kStack) {
            atomicOr(err, kErrStack);
            break;
        }
        if (hr) st[sp++] = rr;
        if (hl) st[sp++] = rl;
    }
    return n;
}

// Exit parameter of the ray p + t d from the box [lo, hi] (p inside it).
__device__ __forceinline__ float box_exit(f3 p, f3 d, float4 lo, float4 hi) {
    const float tx = d.x > 0 ? (hi.x - p.x) / d.x : (d.x < 0 ? (lo.x - p.x) / d.x : 3e38f);
    const float ty = d.y > 0 ? (hi.y - p.y) / d.y : (d.y < 0 ? (lo.y - p.y) / d.y : 3e38f);
    const float tz = d.z > 0 ? (hi.z - p.z) / d.z : (d.z < 0 ? (lo.z - p.z) / d.z : 3e38f);
    return fminf(tx, fminf(ty, tz));
}

__global__ void __launch_bounds__(128) k_contain(const RobotDev R, const SceneDev S, const DiscreteArgs A,
                                                 uint32_t* __restrict__ contain) {
    constexpr float kPad = 1e-4f;  // the segments run this far past the boxes that hold the meshes
    const uint32_t n_items = *A.n_items;
    const f3 dir = contain_dir();
    for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < n_items; it += gridDim.x * blockDim.x) {
        const uint32_t item = item_word(A, R.n_links, A.items[it]);
        const uint32_t pose = item / R.n_links, link = item - pose * R.n_links;
        if (pose >= A.n_poses) {
            atomicOr(A.err, kErrRange);
            continue;
        }
        if (ld_flag(A.pose_hit + pose) || ld_flag(contain + pose)) continue;
        float4 T[3];
        const float4* tp = A.T + ((size_t) pose * R.n_links + link) * 3;
        T[0] = tp[0]; T[1] = tp[1]; T[2] = tp[2];
        const ObbW ob = world_obb(R.obb[link], T);
        const float arad = sqrtf(dot(ob.h, ob.h)) + 2e-5f;
        const f3 lp = xf(T, f3of(R.link_point[link]));
        const float* lo = R.obb[link];
        const f3 oc = mk(lo[0], lo[1], lo[2]);
        const float lrad = sqrtf(lo[3] * lo[3] + lo[4] * lo[4] + lo[5] * lo[5]);
        bool inside = false;
        for (uint32_t o = 0; o < S.n_obs && !inside; ++o) {
            const float* B = S.obbs + 16ull * o;
            const f3 dc = mk(B[0], B[1], B[2]) - ob.c;
            const float rr = arad + B[15];
            if (dot(dc, dc) > rr * rr || !obb_overlap(ob, B)) continue;
            // (a) the link's vertex inside obstacle o
            const float4 blo = S.obs_box[2ull * o], bhi = S.obs_box[2ull * o + 1];
            if (lp.x >= blo.x - kPad && lp.x <= bhi.x + kPad && lp.y >= blo.y - kPad && lp.y <= bhi.y + kPad &&
                lp.z >= blo.z - kPad && lp.z <= bhi.z + kPad) {
                const float t = fmaxf(box_exit(lp, dir, blo, bhi), 0.f) + 10.f * kPad;
                const f3 q = lp + dir * t;
                if (count_crossings(S.tri_nodes, S.tri_prims, S.tri_root, lp, q, o, A.err) & 1u) inside = true;
            }
            // (b) obstacle o's vertex inside the link
            if (!inside) {
                const f3 op = xf_inv(T, f3of(S.obs_point[o]));
                const f3 r = op - oc;
                const float len = sqrtf(dot(r, r));
                if (len <= lrad + kPad) {
                    const f3 q = op + dir * (len + lrad + 10.f * kPad);
                    if (count_crossings(R.tri_nodes, R.tri_prims, R.tri_root[link], op, q, kNone, A.err) & 1u)
                        inside = true;
                }
            }
        }
        if (inside) atomicExch(contain + pose, 1u);
    }
}

void launch_contain(const RobotDev& R, const SceneDev& S, const DiscreteArgs& A, uint32_t* d_contain, cudaStream_t s) {
    static const uint32_t blocks = [] {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_contain, 128, 0);
        return (uint32_t) std::max(1, per_sm) * (uint32_t) device_sm_count();
    }();
    k_contain<<<blocks, 128, 0, s>>>(R, S, A, d_contain);
    cuda_check(cudaGetLastError(), "k_contain");
}

void launch_flags(const uint32_t* d_hit, uint32_t n, uint8_t* d_flags, cudaStream_t s, const uint32_t* d_contain) {
    if (!n) return;
    k_flags<<<(n + 255) / 256, 256, 0, s>>>(d_hit, d_contain, n, d_flags);
    cuda_check(cudaGetLastError(), "k_flags");
}

}  // namespace rtcd
