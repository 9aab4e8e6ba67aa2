// sweep.cu - continuous detectors: piecewise-linear (capsule) and quadratic
// B-spline swept spheres.
//
// Upstream (RTCD/Robot/batchCurveRobot.h:341-403, RTCD/Robot/sweptVolume.cu:
// 22-96, RTCD/CollisionDetector/CCCuda.cu:37-41): FK per waypoint, sphere
// centres per waypoint, (quadratic) control points C = W P, a full OptiX curve
// GAS rebuild per batch, then one RT-core ray per obstacle loop edge against
// the built-in ROUND_LINEAR / ROUND_QUADRATIC_BSPLINE intersectors.
//
// Here nothing is rebuilt per batch: the obstacle edges sit in a resident
// LBVH and each swept primitive (one sphere over one trajectory piece)
// queries it with its bounding box - the primitive-side traversal of the same
// predicate "some obstacle edge comes within r of the sphere path".  A unit is
// (piece, sphere); lanes pull units from a device counter, units of uneven
// trajectories share one launch, and a piece (or a trajectory) stops once it
// is flagged.  The exact tests run in FP32 and fall back to FP64 inside a
// narrow band around the radius: for the quadratic piece the FP64 step is a
// safeguarded Newton polish of the stationary points of the squared distance.
#include <cooperative_groups.h>

#include <algorithm>

#include "kernels.h"

namespace cg = cooperative_groups;

namespace rtcd {

// ---------------------------------------------------------------- FK + sphere centres
constexpr int kWpPerBlock = 32;

__global__ void __launch_bounds__(kWpPerBlock) k_fk_spheres(const RobotDev R, const float* __restrict__ q, uint32_t n_wp,
                                                           float4* __restrict__ centers) {
    __shared__ float sT[kWpPerBlock][kMaxLinks][12];
    uint32_t w = blockIdx.x * kWpPerBlock + threadIdx.x;
    if (w < n_wp) {
        float qq[kMaxDof];
        for (int k = 0; k < R.chain.dof; ++k) qq[k] = q[(size_t) w * R.chain.dof + k];
        fk_chain(R.chain, qq, sT[threadIdx.x]);
    }
    __syncthreads();
    uint32_t nw = min((uint32_t) kWpPerBlock, n_wp - blockIdx.x * kWpPerBlock);
    for (uint32_t idx = threadIdx.x; idx < nw * R.n_spheres; idx += kWpPerBlock) {
        uint32_t wl = idx / R.n_spheres, s = idx % R.n_spheres;
        const float* T = sT[wl][R.sphere_link[s]];
        float4 p = R.spheres[s];
        centers[((size_t) blockIdx.x * kWpPerBlock + wl) * R.n_spheres + s] =
            make_float4(T[0] * p.x + T[1] * p.y + T[2] * p.z + T[3], T[4] * p.x + T[5] * p.y + T[6] * p.z + T[7],
                        T[8] * p.x + T[9] * p.y + T[10] * p.z + T[11], p.w);
    }
}

void launch_fk_spheres(const RobotDev& R, const float* d_q, uint32_t n_wp, float4* d_centers, cudaStream_t s) {
    if (!n_wp) return;
    k_fk_spheres<<<(n_wp + kWpPerBlock - 1) / kWpPerBlock, kWpPerBlock, 0, s>>>(R, d_q, n_wp, d_centers);
    cuda_check(cudaGetLastError(), "k_fk_spheres");
}

// ---------------------------------------------------------------- quadratic fit
// One block per trajectory: C[k][s] = sum_t W_n[k][t] P[t][s]
// (upstream genCtrlPtsKern, RTCD/Robot/sweptVolume.cu:22-83).  W_n, the
// least-squares fit for n waypoints, comes from a table indexed by n.
__global__ void __launch_bounds__(256) k_fit(const float4* __restrict__ centers, const uint32_t* __restrict__ wp_off,
                                            const uint32_t* __restrict__ ctrl_off, const float* __restrict__ W,
                                            const uint32_t* __restrict__ W_off, uint32_t ns, float4* __restrict__ ctrl) {
    uint32_t tr = blockIdx.x;
    uint32_t w0 = wp_off[tr], nwp = wp_off[tr + 1] - w0;
    uint32_t c0 = ctrl_off[tr], nc = ctrl_off[tr + 1] - c0;
    const float* Wn = W + W_off[nwp];
    for (uint32_t idx = threadIdx.x; idx < nc * ns; idx += blockDim.x) {
        uint32_t k = idx / ns, s = idx % ns;
        float x = 0.f, y = 0.f, z = 0.f;
        const float* wr = Wn + (size_t) k * nwp;
        for (uint32_t t = 0; t < nwp; ++t) {
            float wt = __ldg(wr + t);
            float4 p = __ldg(centers + (size_t) (w0 + t) * ns + s);
            x = fmaf(wt, p.x, x);
            y = fmaf(wt, p.y, y);
            z = fmaf(wt, p.z, z);
        }
        float r = __ldg(centers + (size_t) w0 * ns + s).w;
        ctrl[(size_t) (c0 + k) * ns + s] = make_float4(x, y, z, r);
    }
}

void launch_fit(const float4* d_centers, const uint32_t* d_wp_off, const uint32_t* d_ctrl_off, const float* d_W,
                const uint32_t* d_W_off, uint32_t n_traj, uint32_t n_spheres, float4* d_ctrl, cudaStream_t s) {
    if (!n_traj) return;
    k_fit<<<n_traj, 256, 0, s>>>(d_centers, d_wp_off, d_ctrl_off, d_W, d_W_off, n_spheres, d_ctrl);
    cuda_check(cudaGetLastError(), "k_fit");
}

// ---------------------------------------------------------------- exact distances
template <class T>
struct V3 {
    T x, y, z;
};
template <class T>
__device__ __forceinline__ V3<T> vm(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T>
__device__ __forceinline__ V3<T> vsub(V3<T> a, V3<T> b) { return vm<T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T>
__device__ __forceinline__ V3<T> vadd(V3<T> a, V3<T> b) { return vm<T>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T>
__device__ __forceinline__ V3<T> vscale(V3<T> a, T s) { return vm<T>(a.x * s, a.y * s, a.z * s); }
template <class T>
__device__ __forceinline__ T vdot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T>
__device__ __forceinline__ T clamp01(T v) { return v < T(0) ? T(0) : (v > T(1) ? T(1) : v); }

template <class T>
__device__ __forceinline__ V3<T> v3cast(float4 v) { return vm<T>((T) v.x, (T) v.y, (T) v.z); }

// Squared distance between segments p1q1 and p2q2 (Ericson, Real-Time
// Collision Detection, 5.1.9).
template <class T>
__device__ T seg_seg2(V3<T> p1, V3<T> q1, V3<T> p2, V3<T> q2) {
    V3<T> d1 = vsub(q1, p1), d2 = vsub(q2, p2), r = vsub(p1, p2);
    T a = vdot(d1, d1), e = vdot(d2, d2), f = vdot(d2, r);
    T s, t;
    if (a <= T(0) && e <= T(0)) return vdot(r, r);
    if (a <= T(0)) {
        s = T(0);
        t = clamp01(f / e);
    } else {
        T c = vdot(d1, r);
        if (e <= T(0)) {
            t = T(0);
            s = clamp01(-c / a);
        } else {
            T b = vdot(d1, d2), den = a * e - b * b;
            s = den > T(0) ? clamp01((b * f - c * e) / den) : T(0);
            t = (b * s + f) / e;
            if (t < T(0)) {
                t = T(0);
                s = clamp01(-c / a);
            } else if (t > T(1)) {
                t = T(1);
                s = clamp01((b - c) / a);
            }
        }
    }
    V3<T> dd = vsub(vadd(p1, vscale(d1, s)), vadd(p2, vscale(d2, t)));
    return vdot(dd, dd);
}

// Real roots of a u^2 + b u + c (numerically stable form); returns the count.
template <class T>
__device__ __forceinline__ int quad_roots(T a, T b, T c, T* r) {
    if (a == T(0)) {
        if (b == T(0)) return 0;
        r[0] = -c / b;
        return 1;
    }
    T disc = b * b - T(4) * a * c;
    if (disc < T(0)) return 0;
    T sq = sqrt(disc);
    T qq = T(-0.5) * (b + (b >= T(0) ? sq : -sq));
    int n = 0;
    r[n++] = qq / a;
    if (qq != T(0)) r[n++] = c / qq;
    return n;
}

template <class T>
__device__ __forceinline__ T poly3(const T* c, T u) { return ((c[3] * u + c[2]) * u + c[1]) * u + c[0]; }

// Roots in [0, 1] of the cubic c[3] u^3 + ... + c[0]: the derivative's roots
// split [0, 1] into monotone brackets, each bracket with a sign change is
// solved by safeguarded Newton (falls back to bisection when a step leaves the
// bracket), at most `iters` steps per bracket.  The iteration stops once a
// step no longer moves u (or u is an exact root): a converged Newton point
// sits on the bracket's end, and bisecting on from there would throw the
// root away.
template <class T>
__device__ int cubic_roots01(const T* c, T* out, int iters) {
    T br[4];
    int nb = 0;
    br[nb++] = T(0);
    T cr[2];
    int ncr = quad_roots(T(3) * c[3], T(2) * c[2], c[1], cr);
    if (ncr == 2 && cr[0] > cr[1]) {
        T t = cr[0];
        cr[0] = cr[1];
        cr[1] = t;
    }
    for (int k = 0; k < ncr; ++k)
        if (cr[k] > T(0) && cr[k] < T(1)) br[nb++] = cr[k];
    br[nb++] = T(1);
    int n = 0;
    for (int k = 0; k + 1 < nb; ++k) {
        T lo = br[k], hi = br[k + 1];
        T flo = poly3(c, lo), fhi = poly3(c, hi);
        if (flo == T(0)) {
            out[n++] = lo;
            continue;
        }
        if ((flo > T(0)) == (fhi > T(0))) continue;
        T u = T(0.5) * (lo + hi);
        for (int it = 0; it < iters; ++it) {
            const T f = poly3(c, u);
            if (f == T(0)) break;
            if ((f > T(0)) == (flo > T(0))) lo = u; else hi = u;
            const T df = (T(3) * c[3] * u + T(2) * c[2]) * u + c[1];
            T nu = df != T(0) ? u - f / df : T(0.5) * (lo + hi);
            if (!(nu >= lo && nu <= hi)) nu = T(0.5) * (lo + hi);
            if (nu == u) break;
            u = nu;
        }
        out[n++] = u;
    }
    return n;
}

// Squared distance from the quadratic Bezier C(u) = A2 u^2 + A1 u + A0
// (coordinates relative to the segment start) to the segment [0, d].
template <class T>
__device__ __forceinline__ T g_at(V3<T> A2, V3<T> A1, V3<T> A0, V3<T> d, T dd, T u) {
    V3<T> w = vadd(vadd(vscale(A2, u * u), vscale(A1, u)), A0);
    T s = dd > T(0) ? clamp01(vdot(w, d) / dd) : T(0);
    V3<T> e = vsub(w, vscale(d, s));
    return vdot(e, e);
}

// Minimum over u in [0, 1] of the squared distance from the Bezier piece
// (B0, B1, B2) to the segment pq.  The distance is a piecewise quartic in u
// whose pieces switch where the closest segment point reaches an end (s = 0
// or 1); its minimum lies at u = 0, u = 1, a switch point (root of a
// quadratic) or a stationary point of one of the three quartics (root of a
// cubic).  All candidates are evaluated on the exact piecewise function.
template <class T>
__device__ T seg_quad2(V3<T> p, V3<T> q, V3<T> B0, V3<T> B1, V3<T> B2, int iters) {
    V3<T> A0 = vsub(B0, p);
    V3<T> A1 = vscale(vsub(B1, B0), T(2));
    V3<T> A2 = vadd(vsub(B0, vscale(B1, T(2))), B2);
    V3<T> d = vsub(q, p);
    T dd = vdot(d, d);
    T best = g_at(A2, A1, A0, d, dd, T(0));
    T g1 = g_at(A2, A1, A0, d, dd, T(1));
    if (g1 < best) best = g1;
    T cand[4];
    if (dd > T(0)) {
        T pa = vdot(A2, d), pb = vdot(A1, d), pc = vdot(A0, d);
        for (int k = 0; k < 2; ++k) {
            int n = quad_roots(pa, pb, pc - (k ? dd : T(0)), cand);
            for (int j = 0; j < n; ++j)
                if (cand[j] > T(0) && cand[j] < T(1)) {
                    T g = g_at(A2, A1, A0, d, dd, cand[j]);
                    if (g < best) best = g;
                }
        }
    }
    // stationary points: w.w' for the ends, w.w' - (w.d)(w'.d)/|d|^2 for the line
    T aa = vdot(A2, A2), ab = vdot(A2, A1), bb = vdot(A1, A1);
    for (int piece = 0; piece < 3; ++piece) {
        V3<T> C0 = piece == 1 ? vsub(A0, d) : A0;
        T c[4] = {vdot(A1, C0), bb + T(2) * vdot(A2, C0), T(3) * ab, T(2) * aa};
        if (piece == 2) {
            if (!(dd > T(0))) continue;
            T pa = vdot(A2, d), pb = vdot(A1, d), pc = vdot(A0, d);
            T inv = T(1) / dd;
            c[3] -= T(2) * pa * pa * inv;
            c[2] -= T(3) * pa * pb * inv;
            c[1] -= (pb * pb + T(2) * pa * pc) * inv;
            c[0] -= pb * pc * inv;
        }
        T roots[3];
        int n = cubic_roots01(c, roots, iters);
        for (int j = 0; j < n; ++j) {
            T g = g_at(A2, A1, A0, d, dd, roots[j]);
            if (g < best) best = g;
        }
    }
    return best;
}

// Out of line: the root finding keeps many registers live, the traversal
// loop should not pay for them.
__device__ __noinline__ float seg_quad_dist_f32(float4 ea, float4 eb, float4 P0, float4 P1, float4 P2) {
    return sqrtf(fmaxf(seg_quad2<float>(v3cast<float>(ea), v3cast<float>(eb), v3cast<float>(P0), v3cast<float>(P1),
                                        v3cast<float>(P2), 12),
                       0.f));
}

// FP64 decision for a pair whose FP32 distance lies within the band around r.
template <bool QUAD>
__device__ __noinline__ bool sweep_retest_f64(float4 ea, float4 eb, float4 P0, float4 P1, float4 P2, float r) {
    double dd2;
    if (!QUAD)
        dd2 = seg_seg2<double>(v3cast<double>(ea), v3cast<double>(eb), v3cast<double>(P0), v3cast<double>(P1));
    else
        dd2 = seg_quad2<double>(v3cast<double>(ea), v3cast<double>(eb), v3cast<double>(P0), v3cast<double>(P1),
                                v3cast<double>(P2), 48);
    return dd2 <= (double) r * (double) r;
}

// ---------------------------------------------------------------- traversal
__device__ __forceinline__ uint32_t ldflag(const uint32_t* p) { return __ldcg(p); }

// 1 / v, or a huge value of the same sign for v == 0 (a zero chord component:
// the slab test then keeps the box exactly when the origin lies in its slab).
__device__ __forceinline__ float chord_inv(float v) { return v != 0.0f ? 1.0f / v : copysignf(3.0e38f, v); }

// One unit of work: one sphere over one trajectory piece.  Linear: the
// capsule axis P0-P1.  Quadratic: the Bezier piece B0, B1, B2 (P0, P1, P2),
// or an end sphere (P0 = P1 = P2).
struct SweepUnit {
    float4 P0, P1, P2;
    float r;
    uint32_t traj, piece_g;
};

__device__ __forceinline__ void store_rec(SweepRec* r, const SweepUnit& U) {
    r->P0 = U.P0;
    r->P1 = U.P1;
    r->P2 = U.P2;
    r->r = U.r;
    r->traj = U.traj;
    r->piece_g = U.piece_g;
}

__device__ __forceinline__ void load_rec(const SweepRec* r, SweepUnit& U) {
    U.P0 = r->P0;
    U.P1 = r->P1;
    U.P2 = r->P2;
    U.r = r->r;
    U.traj = r->traj;
    U.piece_g = r->piece_g;
}

template <bool QUAD>
__device__ __forceinline__ bool load_unit(const SweepArgs& A, uint32_t u, SweepUnit& U) {
    U.piece_g = u / A.n_spheres;
    const uint32_t s = u - U.piece_g * A.n_spheres;
    U.traj = A.piece_traj[U.piece_g];
    if (U.traj >= A.n_traj) return false;
    const uint32_t piece = U.piece_g - A.traj_piece_off[U.traj];
    const uint32_t w0 = A.traj_wp_off[U.traj], nwp = A.traj_wp_off[U.traj + 1] - w0;
    if (!QUAD) {
        U.P0 = A.centers[(size_t) (w0 + piece) * A.n_spheres + s];
        U.P1 = A.centers[(size_t) (w0 + piece + 1) * A.n_spheres + s];
        U.P2 = U.P1;
    } else {
        const uint32_t c0 = A.traj_ctrl_off[U.traj], nc = A.traj_ctrl_off[U.traj + 1] - c0;
        if (piece + 2 < nc) {
            const float4 a = A.ctrl[(size_t) (c0 + piece) * A.n_spheres + s];
            const float4 b = A.ctrl[(size_t) (c0 + piece + 1) * A.n_spheres + s];
            const float4 c = A.ctrl[(size_t) (c0 + piece + 2) * A.n_spheres + s];
            U.P0 = make_float4(0.5f * (a.x + b.x), 0.5f * (a.y + b.y), 0.5f * (a.z + b.z), a.w);
            U.P1 = b;
            U.P2 = make_float4(0.5f * (b.x + c.x), 0.5f * (b.y + c.y), 0.5f * (b.z + c.z), a.w);
        } else {
            const uint32_t w = (piece + 2 == nc) ? w0 : w0 + nwp - 1;
            U.P0 = A.centers[(size_t) w * A.n_spheres + s];
            U.P1 = U.P0;
            U.P2 = U.P0;
        }
    }
    U.r = U.P0.w;
    return true;
}

// The node-box test of a unit.  The swept sphere lies inside the capsule of
// radius r + e around the chord P0-P2, e the chord deviation (0 for a linear
// piece; for the Bezier piece max |C(u) - chord(u)| = |B1 - (B0 + B2)/2| / 2,
// reached at u = 1/2); a box passes when the chord meets it grown by r + e.
// A curved piece (e >> r) fattens that capsule sideways, so the quadratic
// test also requires the box to meet the control points' box grown by r.
struct SweepCull {
    float co[3], cinv[3], fat;
    float blo[3], bhi[3];
};

template <bool QUAD>
__device__ __forceinline__ void make_cull(const SweepUnit& U, SweepCull& c) {
    float e = 0.f;
    if (QUAD) {
        const float dx = U.P1.x - 0.5f * (U.P0.x + U.P2.x), dy = U.P1.y - 0.5f * (U.P0.y + U.P2.y),
                    dz = U.P1.z - 0.5f * (U.P0.z + U.P2.z);
        e = 0.5f * sqrtf(dx * dx + dy * dy + dz * dz);
    }
    const float4 Pe = QUAD ? U.P2 : U.P1;
    c.co[0] = U.P0.x; c.co[1] = U.P0.y; c.co[2] = U.P0.z;
    c.cinv[0] = chord_inv(Pe.x - U.P0.x); c.cinv[1] = chord_inv(Pe.y - U.P0.y); c.cinv[2] = chord_inv(Pe.z - U.P0.z);
    c.fat = U.r + e + 2e-5f;
    if (QUAD) {
        const float pad = U.r + 2e-5f;
        c.blo[0] = fminf(U.P0.x, fminf(U.P1.x, U.P2.x)) - pad; c.bhi[0] = fmaxf(U.P0.x, fmaxf(U.P1.x, U.P2.x)) + pad;
        c.blo[1] = fminf(U.P0.y, fminf(U.P1.y, U.P2.y)) - pad; c.bhi[1] = fmaxf(U.P0.y, fmaxf(U.P1.y, U.P2.y)) + pad;
        c.blo[2] = fminf(U.P0.z, fminf(U.P1.z, U.P2.z)) - pad; c.bhi[2] = fmaxf(U.P0.z, fmaxf(U.P1.z, U.P2.z)) + pad;
    }
}

// t_enter: the chord parameter where it enters the grown box (visit order).
template <bool QUAD>
__device__ __forceinline__ bool cull_box(const SweepCull& c, const Box& b, float& t_enter) {
    const float t0x = (b.lo[0] - c.fat - c.co[0]) * c.cinv[0], t1x = (b.hi[0] + c.fat - c.co[0]) * c.cinv[0];
    const float t0y = (b.lo[1] - c.fat - c.co[1]) * c.cinv[1], t1y = (b.hi[1] + c.fat - c.co[1]) * c.cinv[1];
    const float t0z = (b.lo[2] - c.fat - c.co[2]) * c.cinv[2], t1z = (b.hi[2] + c.fat - c.co[2]) * c.cinv[2];
    t_enter = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), 0.0f));
    const float t_exit = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fminf(fmaxf(t0z, t1z), 1.0f));
    bool in = t_enter <= t_exit;
    if (QUAD) in = in && box_overlap(b, c.blo, c.bhi);
    return in;
}

constexpr size_t kSweepStagedMaxSmem = 96 * 1024;  // largest shared staging of one trajectory (per block)
constexpr float kSweepBand = 2e-6f;  // |d - r| below this (+ 1e-6 r) is re-tested in FP64

// FP32 distance from the segment pq to the unit's Bezier piece, bracketed.
// C(u) - chord(u) = 2u(1-u)(B1 - (B0+B2)/2): every point of the piece is
// within e of the chord B0-B2 and back, so the chord distance +- e brackets
// the exact distance; only the undecided middle needs roots.  certain_miss is
// set when the value returned (then a lower bound) exceeds r + tol; a value
// below r - tol is an upper bound (a certain hit); otherwise it is the root-
// found distance.
__device__ __forceinline__ float quad_dist_bracket(V3<float> p, V3<float> q, const SweepUnit& U, float r, float tol,
                                                   bool& certain_miss, unsigned long long& n_roots) {
    const V3<float> b0 = v3cast<float>(U.P0), b1 = v3cast<float>(U.P1), b2 = v3cast<float>(U.P2);
    const V3<float> dv = vsub(b1, vscale(vadd(b0, b2), 0.5f));
    const float e = 0.5f * sqrtf(vdot(dv, dv));
    const float dc = sqrtf(fmaxf(seg_seg2<float>(p, q, b0, b2), 0.f));
    if (dc - e > r + tol) {
        certain_miss = true;
        return dc - e;
    }
    if (dc + e < r - tol) return dc + e;
    // halve the piece twice more (de Casteljau: the chord deviation of a
    // half is a quarter), bracketing with the polyline through C(k/4)
    const float e2 = 0.0625f * e;  // deviation of a quarter piece from its chord
    float lo = 3.0e38f;
    V3<float> prev = b0;
    for (int k = 1; k <= 4; ++k) {
        const float u = 0.25f * (float) k;
        const V3<float> cu =
            vadd(vadd(vscale(b0, (1.f - u) * (1.f - u)), vscale(b1, 2.f * u * (1.f - u))), vscale(b2, u * u));
        lo = fminf(lo, seg_seg2<float>(p, q, prev, cu));
        prev = cu;
    }
    const float dq = sqrtf(fmaxf(lo, 0.f));
    if (dq - e2 > r + tol) {
        certain_miss = true;
        return dq - e2;
    }
    if (dq + e2 < r - tol) return dq + e2;
    ++n_roots;
    return seg_quad_dist_f32(make_float4(p.x, p.y, p.z, 0.f), make_float4(q.x, q.y, q.z, 0.f), U.P0, U.P1, U.P2);
}

// The exact leaf test: does obstacle edge `leaf` come within r of the unit's
// path?  FP32 with brackets; FP64 inside a narrow band around r.
template <bool QUAD>
__device__ __forceinline__ bool leaf_hit(const float4* __restrict__ ep, uint32_t leaf, const SweepUnit& U,
                                         unsigned long long* stats, unsigned long long& n_roots) {
    const float4* e = ep + 2ull * leaf;
    const float4 ea = __ldg(e), eb = __ldg(e + 1);
    const V3<float> p = v3cast<float>(ea), q = v3cast<float>(eb);
    const float r = U.r;
    float dist;
    bool decided = false;
    if (!QUAD)
        dist = sqrtf(fmaxf(seg_seg2<float>(p, q, v3cast<float>(U.P0), v3cast<float>(U.P1)), 0.f));
    else
        dist = quad_dist_bracket(p, q, U, r, kSweepBand + 1e-6f * r, decided, n_roots);
    bool hit = dist <= r;
    if (!decided && fabsf(dist - r) <= kSweepBand + 1e-6f * r) {
        atomicAdd(stats, 1ull);
        hit = sweep_retest_f64<QUAD>(ea, eb, U.P0, U.P1, U.P2, r);
    }
    return hit;
}

// ---- the reference's entering-ray semantics (RTCD_CHECK_SURFACE).
// The upstream casts each directed loop edge p -> q (RTCD/Meshes/mesh.h:
// 378-620) as a ray with tmin 0, tmax |q - p| (RTCD/CollisionDetector/
// CCCuda.cu:56-77) against OptiX's curve intersectors, which report a ray
// entering a curve primitive, not one starting inside it; the any-hit
// program counts every report (CCCuda.cu:37-41).  Per (edge, unit):
//     hit  <=>  p lies outside the unit's closed solid P  and  [p, q] meets P.
// Linear: P is the round-capped capsule (endcapFlags = 1, RTCD/Robot/
// batchCurveRobot.h:230).  Quadratic: the sphere-swept piece cut by flat
// caps, the planes through B0 and B2 normal to the end tangents B1 - B0 and
// B2 - B1 (B2 - B0 where one vanishes); the cap disks belong to P.
//
// FP32 decides when every margin clears the band: meeting is tested on the
// segment clipped to the caps grown by the band (a superset of the exact
// clip) for a certain miss and shrunk by it (a subset) for a certain hit;
// the start point is certainly inside (a certain miss) or certainly outside
// likewise.  Anything else is re-tested in FP64.

// Unit normals of the flat caps of a Bezier piece (zero: no cap).
template <class T>
__device__ __forceinline__ void quad_caps(V3<T> B0, V3<T> B1, V3<T> B2, V3<T>& n0, V3<T>& n1) {
    V3<T> t0 = vsub(B1, B0), t1 = vsub(B2, B1);
    const V3<T> ch = vsub(B2, B0);
    if (vdot(t0, t0) == T(0)) t0 = ch;
    if (vdot(t1, t1) == T(0)) t1 = ch;
    const T l0 = sqrt(vdot(t0, t0)), l1 = sqrt(vdot(t1, t1));
    n0 = l0 > T(0) ? vscale(t0, T(1) / l0) : vm<T>(T(0), T(0), T(0));
    n1 = l1 > T(0) ? vscale(t1, T(1) / l1) : vm<T>(T(0), T(0), T(0));
}

// The part of p + t (q - p), t in [0, 1], inside both caps grown by g
// (negative: shrunk): false when empty.
template <class T>
__device__ __forceinline__ bool cap_clip(V3<T> p, V3<T> q, V3<T> B0, V3<T> B2, V3<T> n0, V3<T> n1, T g, V3<T>& a,
                                         V3<T>& b) {
    const V3<T> d = vsub(q, p);
    T lo = T(0), hi = T(1);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const V3<T> n = k ? n1 : n0;
        if (vdot(n, n) == T(0)) continue;
        const T s = k ? vdot(vsub(B2, p), n) : vdot(vsub(p, B0), n);  // signed distance inside
        const T sl = k ? -vdot(d, n) : vdot(d, n);
        if (sl == T(0)) {
            if (s < -g) return false;
            continue;
        }
        const T t = (-g - s) / sl;
        if (sl > T(0)) lo = t > lo ? t : lo;
        else hi = t < hi ? t : hi;
    }
    if (lo > hi) return false;
    a = vadd(p, vscale(d, lo));
    b = vadd(p, vscale(d, hi));
    return true;
}

template <class T>
__device__ __forceinline__ bool cap_inside(V3<T> p, V3<T> B0, V3<T> B2, V3<T> n0, V3<T> n1, T g) {
    if (vdot(n0, n0) > T(0) && vdot(vsub(p, B0), n0) < -g) return false;
    if (vdot(n1, n1) > T(0) && vdot(vsub(B2, p), n1) < -g) return false;
    return true;
}

// FP64 decision of one (edge, unit) pair under the entering-ray semantics.
template <bool QUAD>
__device__ __noinline__ bool surface_retest_f64(float4 ea, float4 eb, float4 P0, float4 P1, float4 P2, float r) {
    const V3<double> p = v3cast<double>(ea), q = v3cast<double>(eb);
    const double rr = (double) r * (double) r;
    if (!QUAD) {
        const V3<double> a = v3cast<double>(P0), b = v3cast<double>(P1);
        return seg_seg2<double>(p, q, a, b) <= rr && seg_seg2<double>(p, p, a, b) > rr;
    }
    const V3<double> B0 = v3cast<double>(P0), B1 = v3cast<double>(P1), B2 = v3cast<double>(P2);
    V3<double> n0, n1, a, b;
    quad_caps<double>(B0, B1, B2, n0, n1);
    if (!cap_clip<double>(p, q, B0, B2, n0, n1, 0.0, a, b)) return false;
    if (seg_quad2<double>(a, b, B0, B1, B2, 48) > rr) return false;
    return !(cap_inside<double>(p, B0, B2, n0, n1, 0.0) && seg_quad2<double>(p, p, B0, B1, B2, 48) <= rr);
}

template <bool QUAD>
__device__ __forceinline__ bool leaf_hit_surface(const float4* __restrict__ ep, uint32_t leaf, const SweepUnit& U,
                                                 unsigned long long* stats, unsigned long long& n_roots) {
    const float4* e = ep + 2ull * leaf;
    const float4 ea = __ldg(e), eb = __ldg(e + 1);
    const V3<float> p = v3cast<float>(ea), q = v3cast<float>(eb);
    const float r = U.r, tol = kSweepBand + 1e-6f * r;
    if (!QUAD) {
        const V3<float> a = v3cast<float>(U.P0), b = v3cast<float>(U.P1);
        const float dseg = sqrtf(fmaxf(seg_seg2<float>(p, q, a, b), 0.f));
        if (dseg > r + tol) return false;
        const float dp = sqrtf(fmaxf(seg_seg2<float>(p, p, a, b), 0.f));
        if (dp < r - tol) return false;                     // starts inside: never enters
        if (dseg < r - tol && dp > r + tol) return true;    // a certain hit
    } else {
        const V3<float> B0 = v3cast<float>(U.P0), B1 = v3cast<float>(U.P1), B2 = v3cast<float>(U.P2);
        V3<float> n0, n1, a, b;
        quad_caps<float>(B0, B1, B2, n0, n1);
        if (!cap_clip<float>(p, q, B0, B2, n0, n1, kSweepBand, a, b)) return false;
        bool miss = false;
        const float dg = quad_dist_bracket(a, b, U, r, tol, miss, n_roots);
        if (miss || dg > r + tol) return false;
        bool pm = false;
        const float dp = quad_dist_bracket(p, p, U, r, tol, pm, n_roots);
        if (!pm && dp < r - tol && cap_inside<float>(p, B0, B2, n0, n1, -kSweepBand)) return false;  // inside
        const bool maybe_inside = !pm && dp <= r + tol && cap_inside<float>(p, B0, B2, n0, n1, kSweepBand);
        if (!maybe_inside) {
            bool sm = false;
            const bool clipped = cap_clip<float>(p, q, B0, B2, n0, n1, -kSweepBand, a, b);
            if (clipped && quad_dist_bracket(a, b, U, r, tol, sm, n_roots) < r - tol && !sm) return true;
        }
    }
    atomicAdd(stats, 1ull);
    return surface_retest_f64<QUAD>(ea, eb, U.P0, U.P1, U.P2, r);
}

// One lane's descent to its next leaf over the obstacle-edge tree (WIDE: the
// 4-wide copy, children pushed far to near; else the binary tree, the child
// met first along the chord visited first).  Returns the leaf, or kNone when
// the stack ran empty.  The nearest overlapping child of a node is carried
// to the next step in a register instead of being pushed and popped at once
// (the stack lives in local memory, so that round trip sat on every step's
// dependent chain); the visit order is the same.
template <bool QUAD, bool WIDE>
__device__ __forceinline__ uint32_t sweep_descend(const float4* __restrict__ en, uint32_t* st, int& sp, uint32_t& steps,
                                                  const SweepCull& c, unsigned long long& n_node, uint32_t* err,
                                                  uint32_t cap) {
    uint32_t leaf = kNone;
    uint32_t ref = kNone;  // the node to visit next, when not on the stack
    if (cap == 0) cap = 0xFFFFFFFFu;  // every call makes at least one visit
    for (uint32_t visits = 0;; ++visits) {
        if (ref == kNone) {
            if (sp <= 0) break;
            ref = st[--sp];
        }
        if (visits == cap) {  // hand the lane back; the stack holds the rest (the last push left room)
            st[sp++] = ref;
            break;
        }
        ++steps;
        if (ref & kLeaf) {
            leaf = ref & ~kLeaf;
            break;
        }
        if (WIDE) {
            const float4* rec = en + 2ull * kWide * ref;
            float4 ra[kWide], rb[kWide];
#pragma unroll
            for (int j = 0; j < kWide; ++j) {
                ra[j] = __ldg(rec + 2 * j);
                rb[j] = __ldg(rec + 2 * j + 1);
            }
            // key = entry parameter along the chord, 2 (past every hit's) for a miss
            float t[kWide];
            uint32_t cr[kWide];
#pragma unroll
            for (int j = 0; j < kWide; ++j) {
                cr[j] = __float_as_uint(rb[j].z);
                t[j] = 2.f;
                if (cr[j] != kNone) {
                    ++n_node;
                    Box bx;
                    bx.lo[0] = ra[j].x; bx.lo[1] = ra[j].y; bx.lo[2] = ra[j].z;
                    bx.hi[0] = ra[j].w; bx.hi[1] = rb[j].x; bx.hi[2] = rb[j].y;
                    float te;
                    if (cull_box<QUAD>(c, bx, te)) t[j] = te;
                }
            }
            // descending keys (a 4-input sorting network): misses first, then far to near
            auto cx = [&](int i, int k) {
                if (t[i] < t[k]) {
                    const float tt = t[i]; t[i] = t[k]; t[k] = tt;
                    const uint32_t rt = cr[i]; cr[i] = cr[k]; cr[k] = rt;
                }
            };
            cx(0, 1); cx(2, 3); cx(0, 2); cx(1, 3); cx(1, 2);
            ref = kNone;
            if (sp + kWide > kStack) {  // cannot happen: the wide form runs only on shallow enough trees
                atomicOr(err, kErrStack);
                sp = 0;
            } else {
#pragma unroll
                for (int j = 0; j < kWide - 1; ++j)
                    if (t[j] < 2.f) st[sp++] = cr[j];
                if (t[kWide - 1] < 2.f) ref = cr[kWide - 1];  // the nearest: visited next
            }
            continue;
        }
        Box bl, br;
        uint32_t rl, rr;
        load_node(en, ref, bl, br, rl, rr);
        n_node += 2;
        float tl, tr;
        bool hr = cull_box<QUAD>(c, br, tr), hl = cull_box<QUAD>(c, bl, tl);
        if (sp + 2 > kStack) {
            atomicOr(err, kErrStack);
            hr = hl = false;
            sp = 0;
        }
        // the child met first along the chord is visited first (next), the other stacked
        ref = kNone;
        if (hr && hl) {
            st[sp++] = tr < tl ? rl : rr;
            ref = tr < tl ? rr : rl;
        } else if (hr) {
            ref = rr;
        } else if (hl) {
            ref = rl;
        }
    }
    return leaf;
}

// Light pass: one lane per unit, "while-while" (Aila and Laine 2009): lanes
// without a unit take their next one, every lane descends to its next leaf,
// then the warp's leaf tests run together.  A unit still open after
// A.light_steps node and leaf visits is handed to the heavy pass (its hits
// so far are set as flags, which are idempotent; its counts are dropped and
// recounted there), so one lane never serialises a unit that meets thousands
// of nodes.
// The quadratic form is capped at 96 registers (5 blocks of 128 threads per
// SM), the linear one at 80 (6 blocks): the extra resident warps hide more
// load latency than the few spilled registers cost (measured on the
// 4,096-trajectory workloads; 6 blocks slowed the quadratic form).
// WIDE: the descent runs over the scene's 4-wide edge tree (a node's four
// child records loaded at once, the overlapping children pushed far to near
// so the nearest is visited first), half the dependent node loads of the
// binary tree; it needs a wide tree shallow enough for the lane stack.
template <bool QUAD, int BLOCK, bool WIDE, bool SURF>
__global__ void __launch_bounds__(BLOCK, QUAD ? 5 * 128 / BLOCK : 6 * 128 / BLOCK) k_sweep(const SceneDev S, const SweepArgs A) {
    const float4* __restrict__ en = WIDE ? S.edge_wide : S.edge_nodes;
    const float4* __restrict__ ep = S.edge_prims;
    const uint32_t root = WIDE ? S.edge_wide_root : S.edge_root;
    // the piece (trajectory without segment flags) this warp's lanes hit last: the lanes
    // on it stop at once (flags only; other decided units at their next 8-visit check)
    __shared__ uint32_t s_decided[BLOCK / 32];
    volatile uint32_t* decided = s_decided + (threadIdx.x >> 5);
    if ((threadIdx.x & 31) == 0) *decided = kNone;
    __syncwarp();
    uint32_t st[kStack];
    int sp = 0;
    bool busy = false;
    uint32_t steps = 0, checked = 0, u_hits = 0;
    SweepUnit U;
    SweepCull c;
    U.traj = U.piece_g = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t next = blockIdx.x * blockDim.x + threadIdx.x;  // neighbouring lanes: spheres of one piece
    unsigned long long n_acc = 0, n_skip = 0, n_leaf = 0, n_roots = 0, n_node = 0;
    const uint32_t budget = A.light_steps ? A.light_steps : 0xFFFFFFFFu;

    while (true) {
        while (!busy && next < A.total_units) {
            const uint32_t u = next;
            next += stride;
            if (!load_unit<QUAD>(A, u, U)) {
                atomicOr(A.err, kErrRange);
                continue;
            }
            if (A.want_pieces ? ldflag(A.piece_hit + U.piece_g) && !A.want_counts
                              : (!A.want_counts && ldflag(A.traj_hit + U.traj))) {
                ++n_skip;
                continue;
            }
            if (root == kNone) continue;
            make_cull<QUAD>(U, c);
            st[0] = root;
            sp = 1;
            busy = true;
            steps = 0;
            checked = 0;
            u_hits = 0;
            ++n_acc;
        }
        if (!busy) break;
        uint32_t leaf = kNone;
        // flags only: every 8 visits, drop a unit whose piece (or trajectory) another unit decided
        if (!A.want_counts && *decided == (A.want_pieces ? U.piece_g : U.traj)) sp = 0;
        if (!A.want_counts && steps >= checked + 8) {
            checked = steps;
            if (A.want_pieces ? ldflag(A.piece_hit + U.piece_g) : ldflag(A.traj_hit + U.traj)) sp = 0;
        }
        leaf = sweep_descend<QUAD, WIDE>(en, st, sp, steps, c, n_node, A.err, A.descend_cap);
        if (leaf != kNone) {
            ++n_leaf;
            if (SURF ? leaf_hit_surface<QUAD>(ep, leaf, U, A.stats, n_roots) : leaf_hit<QUAD>(ep, leaf, U, A.stats, n_roots)) {
                if (A.want_pieces) atomicExch(A.piece_hit + U.piece_g, 1u);
                if (A.want_counts) {
                    A.traj_hit[U.traj] = 1u;
                    ++u_hits;
                } else {
                    atomicExch(A.traj_hit + U.traj, 1u);
                    *decided = A.want_pieces ? U.piece_g : U.traj;
                    sp = 0;  // this unit is decided
                }
            }
        }
        if (sp > 0 && steps > budget) {
            const uint32_t slot = atomicAdd(A.heavy_count, 1u);
            if (slot < A.heavy_cap) {
                store_rec(A.heavy + slot, U);
                busy = false;
                continue;
            }
            steps = checked = 0;  // the heavy list is full: finish the unit here
        }
        if (sp == 0) {
            busy = false;
            if (u_hits) atomicAdd(A.counts + U.traj, u_hits);
        }
    }
    warp_count(A.stats + 1, n_acc);
    warp_count(A.stats + 2, n_skip);
    warp_count(A.stats + 4, n_leaf);
    warp_count(A.stats + 5, n_roots);
    warp_count(A.stats + 7, n_node);
}

// Staged light pass: one trajectory per block at a time.  The block takes a
// trajectory from A.work_counter, runs FK for its waypoints into shared
// memory (one thread per waypoint, link transforms [waypoint][link][12]) and,
// for the quadratic sweep, the least-squares fit there as well: the control
// point of sphere s is C_k = (sum_t W_n[k][t] T_t[link(s)]) p_s, so the fit
// runs once per (control point, link) on the 3x4 transforms instead of once
// per (control point, sphere) on the centres (upstream genCtrlPtsKern,
// RTCD/Robot/sweptVolume.cu:22-83, fits the sphere centres).  Lanes then take
// the trajectory's (piece, sphere) units from a shared counter and build each
// unit's centres from the staged transforms: no sphere centre or control
// point goes through global memory.  A hit sets the piece's (or the
// trajectory's) flag in shared memory, which every lane on it checks at
// every visit.  Same descent, leaf tests, light budget and heavy hand-off as
// k_sweep.
template <bool QUAD, int BLOCK, bool WIDE, bool SURF>
__global__ void __launch_bounds__(BLOCK, QUAD ? 5 * 128 / BLOCK : 6 * 128 / BLOCK)
    k_sweep_traj(const SceneDev S, const RobotDev R, const SweepArgs A) {
    extern __shared__ float4 s_dyn[];
    const uint32_t L = R.n_links, ns = R.n_spheres, L12 = L * 12;
    // one slot per trajectory of a group: T [max_wp][L][12] | C [max_nc][L][12] (quadratic) | piece
    // flags [max_pieces], each slot rounded to 16 bytes (the host sizes the same)
    const uint32_t c_at = A.max_wp * L12, f_at = c_at + (QUAD ? A.max_nc * L12 : 0u);
    const uint32_t slot_words = (f_at + A.max_pieces + 3u) & ~3u;
    float* s_slots = reinterpret_cast<float*>(s_dyn);
    __shared__ uint32_t s_tr0, s_ng, s_next;
    __shared__ uint32_t s_wp0[kSweepMaxGroup], s_nwp[kSweepMaxGroup], s_p0[kSweepMaxGroup];
    // prefixes over the group's valid trajectories: waypoints, units, fit outputs, pieces
    __shared__ uint32_t s_wb[kSweepMaxGroup + 1], s_ub[kSweepMaxGroup + 1], s_cb[kSweepMaxGroup + 1],
        s_pb[kSweepMaxGroup + 1];
    __shared__ volatile uint32_t s_hit[kSweepMaxGroup];
    const float4* __restrict__ en = WIDE ? S.edge_wide : S.edge_nodes;
    const float4* __restrict__ ep = S.edge_prims;
    const uint32_t root = WIDE ? S.edge_wide_root : S.edge_root;
    uint32_t st[kStack];
    unsigned long long n_acc = 0, n_skip = 0, n_leaf = 0, n_roots = 0, n_node = 0;
    const uint32_t budget = A.light_steps ? A.light_steps : 0xFFFFFFFFu;
    const int dof = R.chain.dof;
    const uint32_t group = max(1u, min(A.group, kSweepMaxGroup));
    // the group member g whose prefix range [b[g], b[g + 1]) holds i (i < b[ng])
    auto member = [](const uint32_t* b, uint32_t i) {
        uint32_t g = 0;
        while (i >= b[g + 1]) ++g;
        return g;
    };

    while (true) {
        __syncthreads();  // the previous group's shared state is no longer read
        if (threadIdx.x == 0) {
            const uint32_t t0 = atomicAdd(A.work_counter, group);
            const uint32_t ng = t0 < A.n_traj ? min(group, A.n_traj - t0) : 0u;
            uint32_t wb = 0, ub = 0, cb = 0, pb = 0;
            for (uint32_t g = 0; g < ng; ++g) {
                const uint32_t tr = t0 + g;
                const uint32_t w0 = A.traj_wp_off[tr], nwp = A.traj_wp_off[tr + 1] - w0;
                const uint32_t p0 = A.traj_piece_off[tr], np = A.traj_piece_off[tr + 1] - p0;
                const uint32_t nc = QUAD ? A.traj_ctrl_off[tr + 1] - A.traj_ctrl_off[tr] : 0u;
                const bool fits = nwp <= A.max_wp && np <= A.max_pieces && (!QUAD || nc <= A.max_nc);
                if (!fits) atomicOr(A.err, kErrRange);  // sized by the host: cannot happen
                s_wp0[g] = w0;
                s_nwp[g] = nwp;
                s_p0[g] = p0;
                s_wb[g] = wb;
                s_ub[g] = ub;
                s_cb[g] = cb;
                s_pb[g] = pb;
                s_hit[g] = 0;
                if (fits) {
                    wb += nwp;
                    ub += np * ns;
                    cb += nc * L12;
                    pb += np;
                }
            }
            s_wb[ng] = wb;
            s_ub[ng] = ub;
            s_cb[ng] = cb;
            s_pb[ng] = pb;
            s_tr0 = t0;
            s_ng = ng;
            s_next = 0;
        }
        __syncthreads();
        const uint32_t ng = s_ng;
        if (ng == 0) break;
        for (uint32_t i = threadIdx.x; i < s_wb[ng]; i += BLOCK) {
            const uint32_t g = member(s_wb, i), w = i - s_wb[g];
            float qq[kMaxDof];
            for (int k = 0; k < dof; ++k) qq[k] = __ldg(A.q + (size_t) (s_wp0[g] + w) * dof + k);
            fk_chain(R.chain, qq, reinterpret_cast<float(*)[12]>(s_slots + (size_t) g * slot_words + (size_t) w * L12));
        }
        for (uint32_t i = threadIdx.x; i < s_pb[ng]; i += BLOCK) {
            const uint32_t g = member(s_pb, i);
            reinterpret_cast<uint32_t*>(s_slots + (size_t) g * slot_words + f_at)[i - s_pb[g]] = 0;
        }
        __syncthreads();
        if (QUAD) {
            for (uint32_t i = threadIdx.x; i < s_cb[ng]; i += BLOCK) {
                const uint32_t g = member(s_cb, i), idx = i - s_cb[g];
                const uint32_t nwp = s_nwp[g], k = idx / L12, le = idx - k * L12;
                const float* wr = A.W + A.W_off[nwp] + (size_t) k * nwp;
                const float* sT = s_slots + (size_t) g * slot_words;
                float acc = 0.f;
                for (uint32_t t = 0; t < nwp; ++t) acc = fmaf(__ldg(wr + t), sT[(size_t) t * L12 + le], acc);
                s_slots[(size_t) g * slot_words + c_at + idx] = acc;
            }
            __syncthreads();
        }
        const uint32_t units = s_ub[ng];
        // world centre of sphere s under a staged 3x4 transform M
        auto at = [](const float* M, float4 p) {
            return make_float4(M[0] * p.x + M[1] * p.y + M[2] * p.z + M[3], M[4] * p.x + M[5] * p.y + M[6] * p.z + M[7],
                               M[8] * p.x + M[9] * p.y + M[10] * p.z + M[11], p.w);
        };
        int sp = 0;
        bool busy = false;
        uint32_t steps = 0, u_hits = 0, piece = 0, g = 0;
        SweepUnit U;
        SweepCull c;
        U.traj = s_tr0;
        U.piece_g = 0;
        while (true) {
            while (!busy) {
                const uint32_t u = atomicAdd(&s_next, 1u);
                if (u >= units) break;
                g = member(s_ub, u);
                const uint32_t local = u - s_ub[g];
                piece = local / ns;
                const uint32_t s = local - piece * ns;
                const volatile uint32_t* pf = reinterpret_cast<const volatile uint32_t*>(s_slots + (size_t) g * slot_words + f_at);
                if (!A.want_counts && (A.want_pieces ? pf[piece] : s_hit[g])) {
                    ++n_skip;
                    continue;
                }
                const float* sT = s_slots + (size_t) g * slot_words;
                const float4 sp4 = __ldg(R.spheres + s);
                const uint32_t link = __ldg(R.sphere_link + s);
                U.traj = s_tr0 + g;
                U.piece_g = s_p0[g] + piece;
                U.r = sp4.w;
                if constexpr (!QUAD) {
                    U.P0 = at(sT + (size_t) (piece * L + link) * 12, sp4);
                    U.P1 = at(sT + (size_t) ((piece + 1) * L + link) * 12, sp4);
                    U.P2 = U.P1;
                } else {
                    const uint32_t nc = (s_cb[g + 1] - s_cb[g]) / L12;
                    if (piece + 2 < nc) {
                        const float* sC = sT + c_at;
                        const float4 a = at(sC + (size_t) (piece * L + link) * 12, sp4);
                        const float4 b = at(sC + (size_t) ((piece + 1) * L + link) * 12, sp4);
                        const float4 cc = at(sC + (size_t) ((piece + 2) * L + link) * 12, sp4);
                        U.P0 = make_float4(0.5f * (a.x + b.x), 0.5f * (a.y + b.y), 0.5f * (a.z + b.z), sp4.w);
                        U.P1 = b;
                        U.P2 = make_float4(0.5f * (b.x + cc.x), 0.5f * (b.y + cc.y), 0.5f * (b.z + cc.z), sp4.w);
                    } else {  // the start / end sphere
                        const uint32_t w = (piece + 2 == nc) ? 0 : s_nwp[g] - 1;
                        U.P0 = at(sT + (size_t) (w * L + link) * 12, sp4);
                        U.P1 = U.P0;
                        U.P2 = U.P0;
                    }
                }
                if (root == kNone) continue;
                make_cull<QUAD>(U, c);
                st[0] = root;
                sp = 1;
                busy = true;
                steps = 0;
                u_hits = 0;
                ++n_acc;
            }
            if (!busy) break;
            volatile uint32_t* pf = reinterpret_cast<volatile uint32_t*>(s_slots + (size_t) g * slot_words + f_at);
            // flags only: drop the unit once its piece (or trajectory) is decided
            if (!A.want_counts && (A.want_pieces ? pf[piece] : s_hit[g])) sp = 0;
            const uint32_t leaf = sweep_descend<QUAD, WIDE>(en, st, sp, steps, c, n_node, A.err, A.descend_cap);
            if (leaf != kNone) {
                ++n_leaf;
                if (SURF ? leaf_hit_surface<QUAD>(ep, leaf, U, A.stats, n_roots)
                         : leaf_hit<QUAD>(ep, leaf, U, A.stats, n_roots)) {
                    if (A.want_pieces) {
                        pf[piece] = 1u;
                        atomicExch(A.piece_hit + U.piece_g, 1u);
                    }
                    if (A.want_counts) {
                        A.traj_hit[U.traj] = 1u;
                        ++u_hits;
                    } else {
                        if (!s_hit[g]) {
                            s_hit[g] = 1u;
                            atomicExch(A.traj_hit + U.traj, 1u);
                        }
                        sp = 0;  // this unit is decided
                    }
                }
            }
            if (sp > 0 && steps > budget) {
                const uint32_t slot = atomicAdd(A.heavy_count, 1u);
                if (slot < A.heavy_cap) {
                    store_rec(A.heavy + slot, U);
                    busy = false;
                    continue;
                }
                steps = 0;  // the heavy list is full: finish the unit here
            }
            if (sp == 0) {
                busy = false;
                if (u_hits) atomicAdd(A.counts + U.traj, u_hits);
            }
        }
    }
    warp_count(A.stats + 1, n_acc);
    warp_count(A.stats + 2, n_skip);
    warp_count(A.stats + 4, n_leaf);
    warp_count(A.stats + 5, n_roots);
    warp_count(A.stats + 7, n_node);
}

// Heavy pass: one warp per spilled unit.  The warp descends the obstacle-edge
// LBVH through a shared LIFO frontier (up to 32 nodes a step, survivors
// pushed), collects leaf survivors in a shared buffer and tests them 32 at a
// time, one leaf per lane.  The unit's serial depth drops from its node count
// to about its node count / 32 plus the tree depth.  WIDE: the frontier holds
// nodes of the scene's 4-wide edge tree instead, up to 8 a step with four
// lanes per node, each lane loading and testing one child record (half the
// levels of the binary tree; more boxes tested in all, which the reference's
// thin shelf boards do not repay: SweepArgs.heavy_wide chooses).
constexpr int kHeavyWarps = 4;
constexpr int kLeafBuf = 96;  // < 32 waiting + up to 64 added by one node step

// SPLIT = false: the heavy pass over the light pass's deferred units, each
// from the root.  A unit still open after A.heavy_steps frontier steps, once
// its frontier holds kSplitMinFront nodes or more, finishes its pending
// leaves, appends its open frontier nodes to A.split and stops (A.heavy_steps
// == 0: never), so the few units with very large traversals do not hold the
// pass while the other warps idle.  SPLIT = true: the split pass, one warp
// per (unit, node) pair of A.split, each descending that node's subtree to
// the end.  Every node is expanded exactly once either way, so flags and
// counts do not depend on where a unit split.
constexpr int kSplitMinFront = 4;
template <bool QUAD, bool SURF, bool SPLIT, bool WIDE>
__global__ void __launch_bounds__(kHeavyWarps * 32) k_sweep_heavy(const SceneDev S, const SweepArgs A) {
    __shared__ uint32_t s_front[kHeavyWarps][kFrontier];
    __shared__ uint32_t s_leaf[kHeavyWarps][kLeafBuf];
    const int lane = threadIdx.x & 31;
    uint32_t* fr = s_front[threadIdx.x >> 5];
    uint32_t* lf = s_leaf[threadIdx.x >> 5];
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t n_work = SPLIT ? min(*A.split_count, A.split_cap) : min(*A.heavy_count, A.heavy_cap);
    unsigned long long n_leaf = 0, n_roots = 0, n_node = 0;
    while (true) {
        uint32_t h = 0;
        if (lane == 0) h = atomicAdd(SPLIT ? A.split_work : A.heavy_work, 1u);
        h = __shfl_sync(0xffffffffu, h, 0);
        if (h >= n_work) break;
        uint32_t rec = h, start = WIDE ? S.edge_wide_root : S.edge_root;
        if (SPLIT) {
            const uint2 item = A.split[h];
            if (item.x == kNone) continue;  // a blanked slot of a reservation that did not fit
            rec = item.x;
            start = item.y;
        }
        SweepUnit U;
        load_rec(A.heavy + rec, U);
        SweepCull c;
        make_cull<QUAD>(U, c);
        if (lane == 0) fr[0] = start;
        __syncwarp();
        int sp = 1, nl = 0, step = 0;
        uint32_t hits = 0, warp_steps = 0;
        bool budgeted = !SPLIT && A.heavy_steps != 0, handing = false;
        while (true) {
            if (nl >= 32 || (sp == 0 && nl > 0) || (handing && nl > 0)) {  // leaf step
                const int take = min(nl, 32);
                nl -= take;
                const uint32_t leaf = lane < take ? lf[nl + lane] : kNone;
                __syncwarp();
                bool hit = false;
                if (leaf != kNone) {
                    ++n_leaf;
                    hit = SURF ? leaf_hit_surface<QUAD>(S.edge_prims, leaf, U, A.stats, n_roots)
                               : leaf_hit<QUAD>(S.edge_prims, leaf, U, A.stats, n_roots);
                }
                const uint32_t mh = __ballot_sync(0xffffffffu, hit);
                if (mh) {
                    if (lane == 0) {
                        if (A.want_pieces) atomicExch(A.piece_hit + U.piece_g, 1u);
                        if (A.want_counts) {
                            A.traj_hit[U.traj] = 1u;
                            hits += __popc(mh);
                        } else {
                            atomicExch(A.traj_hit + U.traj, 1u);
                        }
                    }
                    if (!A.want_counts) break;
                }
                continue;
            }
            if (sp == 0) break;
            if (handing) {  // no leaves pending: the open frontier goes to the split pass
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(A.split_count, (uint32_t) sp);
                base = __shfl_sync(0xffffffffu, base, 0);
                if ((uint64_t) base + (uint64_t) sp <= A.split_cap) {
                    for (int k = lane; k < sp; k += 32) A.split[base + k] = make_uint2(rec, fr[k]);
                    break;
                }
                // no room: this warp finishes the unit, and the reserved slots below the capacity
                // are blanked (the split pass reads every slot up to it)
                for (int k = lane; k < sp && (uint64_t) base + (uint64_t) k < A.split_cap; k += 32)
                    A.split[base + k] = make_uint2(kNone, kNone);
                handing = false;
                budgeted = false;
            }
            if (budgeted && ++warp_steps >= A.heavy_steps && sp >= kSplitMinFront) {
                handing = true;
                continue;
            }
            if (!A.want_counts && (++step & 7) == 0) {  // decided meanwhile by another unit?
                uint32_t dec = 0;
                if (lane == 0) dec = A.want_pieces ? ldflag(A.piece_hit + U.piece_g) : ldflag(A.traj_hit + U.traj);
                if (__shfl_sync(0xffffffffu, dec, 0)) break;
            }
            if constexpr (WIDE) {
                // up to 8 wide nodes a step, four lanes per node, one child record per lane
                const int take = min(sp, 32 / kWide);
                sp -= take;
                const int slot = lane / kWide, j = lane % kWide;
                const uint32_t ref = slot < take ? fr[sp + slot] : kNone;
                __syncwarp();
                bool hc = false;
                uint32_t rc = kNone;
                if (ref != kNone) {
                    if (ref & kLeaf) {  // a one-edge scene: the root itself is a leaf
                        if (j == 0) {
                            hc = true;
                            rc = ref;
                        }
                    } else {
                        const float4* r = S.edge_wide + 2ull * kWide * ref + 2 * j;
                        const float4 ra = __ldg(r), rb = __ldg(r + 1);
                        rc = __float_as_uint(rb.z);
                        if (rc != kNone) {  // an empty slot of a node with fewer than four children
                            ++n_node;
                            Box bx;
                            bx.lo[0] = ra.x; bx.lo[1] = ra.y; bx.lo[2] = ra.z;
                            bx.hi[0] = ra.w; bx.hi[1] = rb.x; bx.hi[2] = rb.y;
                            float t;
                            hc = cull_box<QUAD>(c, bx, t);
                        }
                    }
                }
                const bool pc = hc && !(rc & kLeaf), ec = hc && (rc & kLeaf);
                const uint32_t mpc = __ballot_sync(0xffffffffu, pc), mec = __ballot_sync(0xffffffffu, ec);
                const int npush = __popc(mpc);
                if (sp + npush > kFrontier) {  // cannot happen for trees within the depth limit
                    if (lane == 0) atomicOr(A.err, kErrStack);
                    break;
                }
                if (pc) fr[sp + __popc(mpc & lt)] = rc;
                sp += npush;
                if (ec) lf[nl + __popc(mec & lt)] = rc & ~kLeaf;
                nl += __popc(mec);
                __syncwarp();
                continue;
            }
            const int take = min(sp, 32);
            sp -= take;
            const uint32_t ref = lane < take ? fr[sp + lane] : kNone;
            __syncwarp();
            bool hl = false, hr = false;
            uint32_t rl = kNone, rr = kNone;
            if (ref != kNone) {
                if (ref & kLeaf) {  // a one-edge scene: the root itself is a leaf
                    hl = true;
                    rl = ref;
                } else {
                    Box bl, br;
                    float t;
                    load_node(S.edge_nodes, ref, bl, br, rl, rr);
                    n_node += 2;
                    hl = cull_box<QUAD>(c, bl, t);
                    hr = cull_box<QUAD>(c, br, t);
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
        if (lane == 0 && hits) atomicAdd(A.counts + U.traj, hits);
        __syncwarp();
    }
    warp_count(A.stats + 4, n_leaf);
    warp_count(A.stats + 5, n_roots);
    warp_count(A.stats + 7, n_node);
}

// Diagnostics of the sweeps' arithmetic: per (segment, piece) pair the FP32
// distance the light pass computes (linear: segment-segment; quadratic: the
// root-found distance to the Bezier piece) and the FP64 distance of the
// re-test, on pairs given in world coordinates (piece: B0 B1 B2, linear axis
// B0-B1).
template <bool QUAD>
__global__ void k_probe_sweep(const float* __restrict__ seg, const float* __restrict__ piece, uint32_t n,
                              float* __restrict__ d32, double* __restrict__ d64) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* e = seg + 6ull * i;
    const float* b = piece + 9ull * i;
    const float4 ea = make_float4(e[0], e[1], e[2], 0.f), eb = make_float4(e[3], e[4], e[5], 0.f);
    const float4 B0 = make_float4(b[0], b[1], b[2], 0.f), B1 = make_float4(b[3], b[4], b[5], 0.f),
                 B2 = make_float4(b[6], b[7], b[8], 0.f);
    if (QUAD) {
        d32[i] = seg_quad_dist_f32(ea, eb, B0, B1, B2);
        d64[i] = sqrt(seg_quad2<double>(v3cast<double>(ea), v3cast<double>(eb), v3cast<double>(B0),
                                        v3cast<double>(B1), v3cast<double>(B2), 48));
    } else {
        d32[i] = sqrtf(fmaxf(seg_seg2<float>(v3cast<float>(ea), v3cast<float>(eb), v3cast<float>(B0),
                                             v3cast<float>(B1)), 0.f));
        d64[i] = sqrt(seg_seg2<double>(v3cast<double>(ea), v3cast<double>(eb), v3cast<double>(B0),
                                       v3cast<double>(B1)));
    }
}

void launch_probe_sweep(bool quad, const float* d_seg, const float* d_piece, uint32_t n, float* d32, double* d64,
                        cudaStream_t s) {
    if (!n) return;
    if (quad) k_probe_sweep<true><<<(n + 127) / 128, 128, 0, s>>>(d_seg, d_piece, n, d32, d64);
    else k_probe_sweep<false><<<(n + 127) / 128, 128, 0, s>>>(d_seg, d_piece, n, d32, d64);
    cuda_check(cudaGetLastError(), "k_probe_sweep");
}

size_t sweep_staged_smem(bool quad, uint32_t n_links, uint32_t max_wp, uint32_t max_nc, uint32_t max_pieces) {
    const size_t bytes = 48ull * n_links * (max_wp + (quad ? max_nc : 0)) + 4ull * max_pieces;
    return bytes <= kSweepStagedMaxSmem ? ((bytes + 15) & ~size_t(15)) : 0;
}

template <bool QUAD>
static int sweep_per_sm(int threads) {
    int per_sm = 0;  // the wide and binary forms (and both semantics) share their register caps
    if (threads == 64)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep<QUAD, 64, true, false>, 64, 0);
    else if (threads == 256)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep<QUAD, 256, true, false>, 256, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep<QUAD, 128, true, false>, 128, 0);
    return std::max(1, per_sm);
}

uint32_t sweep_max_blocks_per_sm(bool quad, uint32_t threads) {
    return (uint32_t) (quad ? sweep_per_sm<true>((int) threads) : sweep_per_sm<false>((int) threads));
}

uint32_t sweep_persistent_blocks(bool quad) { return sweep_max_blocks_per_sm(quad, kTravThreads) * device_sm_count(); }

template <bool QUAD, bool SURF, bool WIDE>
static uint32_t heavy_blocks() {
    static uint32_t blocks = 0;
    if (!blocks) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_heavy<QUAD, SURF, false, WIDE>, kHeavyWarps * 32, 0);
        blocks = (uint32_t) std::max(1, per_sm) * device_sm_count();
    }
    return blocks;
}

// The staged light pass at BLOCK threads per block, `slot` bytes of shared
// memory per trajectory, on at most as many blocks as fit.  Trajectories per
// group (A.group, 0 = chosen here): about 1,024 (piece, sphere) units a
// group, within the slots that fit in the block's share of the SM at the
// occupancy one slot allows (and in kSweepStagedMaxSmem), leaving at least
// four groups per block, at most kSweepMaxGroup.
template <bool QUAD, int BLOCK, bool WIDE, bool SURF>
static void launch_staged(const SceneDev& S, const RobotDev& R, const SweepArgs& A, uint32_t blocks, size_t slot,
                          cudaStream_t s) {
    auto kern = k_sweep_traj<QUAD, BLOCK, WIDE, SURF>;
    static bool attr = false;
    if (!attr) {  // allow up to the largest staged size (set once, outside any capture: the first launch)
        cuda_check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) kSweepStagedMaxSmem),
                   "cudaFuncSetAttribute");
        attr = true;
    }
    const uint32_t sms = device_sm_count();
    int per_sm = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BLOCK, slot), "occupancy");
    blocks = std::min<uint32_t>(blocks, (uint32_t) std::max(1, per_sm) * sms);
    SweepArgs G = A;
    if (!G.group) {
        int dev = 0, sm_bytes = 0, reserved = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
        const long per_sm_used = (long) std::max<uint32_t>(1, (blocks + sms - 1) / sms);
        // the block's share of the SM's shared memory, less the per-block reserve and static arrays
        const long avail = (long) sm_bytes / per_sm_used - (long) reserved - 2048;
        const size_t share = std::min<size_t>(kSweepStagedMaxSmem, (size_t) std::max<long>(avail, (long) slot));
        const uint32_t by_smem = (uint32_t) std::max<size_t>(1, share / slot);
        const uint32_t by_work = std::max<uint32_t>(1, A.n_traj / (4 * std::max(1u, blocks)));
        // about 1,024 units a group: grouping pays for short trajectories (their FK and fit
        // phases and hand-over barriers are a large share), while a group of long ones only
        // lengthens the last group's tail (measured: linear 32-waypoint trajectories of 1,984
        // units are 5 % slower in pairs, quadratic 8-16-waypoint ones 8 % faster in threes)
        const uint64_t tu = std::max<uint64_t>(A.total_units, 1);
        const uint32_t by_units = (uint32_t) std::max<uint64_t>(1, (1024ull * A.n_traj + tu / 2) / tu);
        G.group = std::min(kSweepMaxGroup, std::min(by_smem, std::min(by_work, by_units)));
    }
    G.group = std::max(1u, std::min(G.group, kSweepMaxGroup));
    while (G.group > 1 && G.group * slot > kSweepStagedMaxSmem) --G.group;
    // the group's shared memory must not lower the occupancy one slot allows
    while (G.group > 1) {
        int per_sm_g = 0;
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_g, kern, BLOCK, G.group * slot), "occupancy");
        if ((uint32_t) std::max(1, per_sm_g) * sms >= blocks) break;
        --G.group;
    }
    const size_t smem = G.group * slot;
    const uint32_t groups = (A.n_traj + G.group - 1) / G.group;
    blocks = std::min<uint32_t>(blocks, std::max<uint32_t>(groups, 1));
    kern<<<blocks, BLOCK, smem, s>>>(S, R, G);
}

// The heavy pass over the light pass's deferred units, then (A.heavy_steps)
// the split pass over the frontier nodes the heavy pass handed on.
template <bool QUAD, bool SURF, bool WIDE>
static void launch_heavy(const SceneDev& S, const SweepArgs& H, uint32_t heavy_share, cudaStream_t s) {
    const uint32_t hb = std::max(1u, heavy_blocks<QUAD, SURF, WIDE>() * heavy_share / 100);
    k_sweep_heavy<QUAD, SURF, false, WIDE><<<hb, kHeavyWarps * 32, 0, s>>>(S, H);
    cuda_check(cudaGetLastError(), "k_sweep_heavy");
    if (H.heavy_steps) {
        k_sweep_heavy<QUAD, SURF, true, WIDE><<<hb, kHeavyWarps * 32, 0, s>>>(S, H);
        cuda_check(cudaGetLastError(), "k_sweep_heavy (split)");
    }
}

template <bool QUAD, bool SURF>
static void sweep_dispatch(const SceneDev& S, const RobotDev& R, const SweepArgs& A, uint32_t blocks, uint32_t threads,
                           uint32_t heavy_share, bool staged, cudaStream_t s, cudaEvent_t ev_light) {
    const bool wide = S.edge_wide_lane && !A.binary_tree;
    if (staged) {
        const size_t smem = sweep_staged_smem(QUAD, R.n_links, A.max_wp, A.max_nc, A.max_pieces);
        if (wide) {
            if (threads == 64) launch_staged<QUAD, 64, true, SURF>(S, R, A, blocks, smem, s);
            else if (threads == 256) launch_staged<QUAD, 256, true, SURF>(S, R, A, blocks, smem, s);
            else launch_staged<QUAD, 128, true, SURF>(S, R, A, blocks, smem, s);
        } else {
            if (threads == 64) launch_staged<QUAD, 64, false, SURF>(S, R, A, blocks, smem, s);
            else if (threads == 256) launch_staged<QUAD, 256, false, SURF>(S, R, A, blocks, smem, s);
            else launch_staged<QUAD, 128, false, SURF>(S, R, A, blocks, smem, s);
        }
    } else if (wide) {
        if (threads == 64)
            k_sweep<QUAD, 64, true, SURF><<<blocks, 64, 0, s>>>(S, A);
        else if (threads == 256)
            k_sweep<QUAD, 256, true, SURF><<<blocks, 256, 0, s>>>(S, A);
        else
            k_sweep<QUAD, 128, true, SURF><<<blocks, 128, 0, s>>>(S, A);
    } else {
        if (threads == 64)
            k_sweep<QUAD, 64, false, SURF><<<blocks, 64, 0, s>>>(S, A);
        else if (threads == 256)
            k_sweep<QUAD, 256, false, SURF><<<blocks, 256, 0, s>>>(S, A);
        else
            k_sweep<QUAD, 128, false, SURF><<<blocks, 128, 0, s>>>(S, A);
    }
    cuda_check(cudaGetLastError(), staged ? "k_sweep_traj" : "k_sweep");
    if (ev_light) cuda_check(cudaEventRecord(ev_light, s), "event");
    if (A.light_steps) {
        SweepArgs H = A;
        H.stats = A.stats + kStatBank;
        if (A.heavy_wide) launch_heavy<QUAD, SURF, true>(S, H, heavy_share, s);
        else launch_heavy<QUAD, SURF, false>(S, H, heavy_share, s);
    }
}

void launch_sweep(const SceneDev& S, const RobotDev& R, const SweepArgs& A, uint32_t blocks, uint32_t threads,
                  uint32_t heavy_share, bool staged, cudaStream_t s, cudaEvent_t ev_light) {
    if (A.quad) {
        if (A.surface) sweep_dispatch<true, true>(S, R, A, blocks, threads, heavy_share, staged, s, ev_light);
        else sweep_dispatch<true, false>(S, R, A, blocks, threads, heavy_share, staged, s, ev_light);
    } else {
        if (A.surface) sweep_dispatch<false, true>(S, R, A, blocks, threads, heavy_share, staged, s, ev_light);
        else sweep_dispatch<false, false>(S, R, A, blocks, threads, heavy_share, staged, s, ev_light);
    }
}

}  // namespace rtcd
