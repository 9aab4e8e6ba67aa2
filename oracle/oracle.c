/*
 * oracle.c - FP64 CPU restatement of the RTCollisionDetection query path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the correctness checker for the
 * CUDA detectors: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline load it.  The product library never links or calls it.
 *
 * What it restates (upstream file:line):
 *  - forward kinematics T_{i+1} = T_i * (cos q_i C_i + sin q_i S_i + O_i), base
 *    transform T_0 (RTCD/Robot/robot.cu:202-231, affine product :34-47) - here
 *    in double precision;
 *  - unique undirected mesh edges in first-seen orientation
 *    (RTCD/Meshes/mesh.h:200-216);
 *  - ObsToRobot: every obstacle edge is a segment [v0, v1] tested against
 *    every link triangle of every pose; the upstream any-hit program counts
 *    every (edge, link instance, triangle) hit (RTCD/CollisionDetector/
 *    CCCuda.cu:31-35, :56-77);
 *  - RobotToObs: every link edge, moved to the world by its link transform,
 *    is tested against the scene triangles; the upstream closest-hit path
 *    counts one per hitting edge (RTCD/CollisionDetector/CCRay.cu:74-116);
 *  - linear sweep: a sphere swept between consecutive waypoints is a capsule
 *    (round end caps, RTCD/Robot/batchCurveRobot.h:230), hit by an obstacle
 *    edge when their distance is <= r (solid semantics);
 *  - quadratic sweep: control points C = W P with W = pinv(B), B the uniform
 *    unclamped quadratic B-spline basis sampled at u = linspace(2, nC, nT)
 *    (RTCD/Robot/sweptVolume.cu:22-83, weight tables RTCD/data/weights/quad/
 *    normal/), segments of three consecutive control points
 *    (RTCD/Robot/batchCurveRobot.h:49-51); a segment is hit when an obstacle
 *    edge comes within r of the curve piece.  The start and end waypoint
 *    spheres, which the upstream test adds from a separate sphere check
 *    (RTCD/CollisionDetector/Test/testCollisionCheckerCurve.cpp:157-172), are
 *    optional extra pieces.
 *
 * The upstream OBB prefilter (RTCD/CollisionDetector/BBCollisionDetection.cu:
 * 4-37) is not applied: the oracle defines the truth the cull must preserve.
 * A canonical LBVH (30-bit Morton codes of float centroids, stable sort by
 * (code, index), Karras 2012 hierarchy, one primitive per leaf) accelerates the
 * queries without changing any result; its float arithmetic is spelled out so
 * the device builder can be compared with it bit for bit.
 *
 * epsilon band: a pose (segment, trajectory) is "in band" when no robust hit
 * exists and some primitive pair lies within eps of flipping: a hit whose
 * crossing point is within eps of the triangle boundary or whose segment
 * endpoint is within eps of the triangle plane, a miss within distance eps,
 * or a sweep distance within eps of the radius.  Flags must match the device
 * detectors on every pose outside the band.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned int u32;

/* ------------------------------------------------------------------ vectors */
typedef struct { double x, y, z; } d3;
static inline d3 v3(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static inline d3 sub(d3 a, d3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 add(d3 a, d3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 mul(d3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 cross(d3 a, d3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline double len(d3 a) { return sqrt(dot(a, a)); }
static inline double clamp01(double t) { return t < 0 ? 0 : (t > 1 ? 1 : t); }
static inline d3 fv(const float* p) { return v3(p[0], p[1], p[2]); }

/* affine 3x4 row-major */
static inline d3 xform(const double* T, d3 p) {
    return v3(T[0] * p.x + T[1] * p.y + T[2] * p.z + T[3], T[4] * p.x + T[5] * p.y + T[6] * p.z + T[7],
              T[8] * p.x + T[9] * p.y + T[10] * p.z + T[11]);
}
static inline d3 xform_inv(const double* T, d3 p) { /* rigid inverse: R^T (p - t) */
    d3 q = v3(p.x - T[3], p.y - T[7], p.z - T[11]);
    return v3(T[0] * q.x + T[4] * q.y + T[8] * q.z, T[1] * q.x + T[5] * q.y + T[9] * q.z,
              T[2] * q.x + T[6] * q.y + T[10] * q.z);
}

/* ---------------------------------------------------------------- kinematics */
/* T[(dof+1)*12] for one pose: link 0 = base, link i+1 = T_i * L_i(q_i). */
void orc_fk_pose(int dof, const float* cos_m, const float* sin_m, const float* one_m, const float* base,
                 const float* q, double* T) {
    for (int k = 0; k < 12; ++k) T[k] = base[k];
    for (int i = 0; i < dof; ++i) {
        double s = sin((double) q[i]), c = cos((double) q[i]);
        double L[12];
        for (int k = 0; k < 12; ++k)
            L[k] = c * cos_m[i * 12 + k] + s * sin_m[i * 12 + k] + one_m[i * 12 + k];
        const double* A = T + i * 12;
        double* R = T + (i + 1) * 12;
        for (int r = 0; r < 3; ++r) {
            for (int col = 0; col < 4; ++col) {
                double v = A[r * 4 + 0] * L[0 * 4 + col] + A[r * 4 + 1] * L[1 * 4 + col] + A[r * 4 + 2] * L[2 * 4 + col];
                if (col == 3) v += A[r * 4 + 3];
                R[r * 4 + col] = v;
            }
        }
    }
}

void orc_fk(int dof, const float* cos_m, const float* sin_m, const float* one_m, const float* base, const float* q,
            int n, double* T) {
    for (int p = 0; p < n; ++p) orc_fk_pose(dof, cos_m, sin_m, one_m, base, q + (size_t) p * dof, T + (size_t) p * (dof + 1) * 12);
}

/* -------------------------------------------------------------- mesh edges */
/* Unique undirected edges, first-seen orientation, triangles visited in order,
 * edges of a triangle in order (v0v1, v1v2, v2v0).  Returns the edge count;
 * `edges` must hold 3 * n_tris pairs. */
typedef struct { u32 a, b, id; int used; } edge_slot;

static uint64_t hash_pair(u32 a, u32 b) {
    uint64_t k = ((uint64_t) a << 32) | b;
    k ^= k >> 33; k *= 0xff51afd7ed558ccdULL; k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ULL; k ^= k >> 33;
    return k;
}

int orc_unique_edges(const u32* tris, int n_tris, u32* edges) {
    size_t cap = 1;
    while (cap < (size_t) n_tris * 6 + 16) cap <<= 1;
    edge_slot* tab = (edge_slot*) calloc(cap, sizeof(edge_slot));
    if (!tab) return -1;
    int ne = 0;
    for (int t = 0; t < n_tris; ++t) {
        for (int k = 0; k < 3; ++k) {
            u32 a = tris[t * 3 + k], b = tris[t * 3 + (k + 1) % 3];
            u32 lo = a < b ? a : b, hi = a < b ? b : a;
            size_t h = hash_pair(lo, hi) & (cap - 1);
            int found = 0;
            while (tab[h].used) {
                if (tab[h].a == lo && tab[h].b == hi) { found = 1; break; }
                h = (h + 1) & (cap - 1);
            }
            if (!found) {
                tab[h].used = 1; tab[h].a = lo; tab[h].b = hi;
                edges[2 * ne] = a; edges[2 * ne + 1] = b;
                ++ne;
            }
        }
    }
    free(tab);
    return ne;
}

/* Loop edges (RTCD/Meshes/mesh.h:378-620): directed edges chosen so that the
 * three edges of every triangle, taken in their directions, run around it as
 * a loop (v0->v1->v2->v0 or the reverse); an edge shared by two triangles that
 * need opposite directions is kept in both.  The continuous detectors cast
 * these instead of the unique edges: the curve intersectors report only a ray
 * entering the swept surface, and a triangle boundary that crosses a closed
 * surface crosses it inwards somewhere along the loop.
 *
 * The direction choice follows the upstream breadth-first walk exactly:
 * start at the first unprocessed triangle (index order); pop a triangle,
 * classify its three edges against the directed set (forward, backward, both,
 * undecided), complete the loop by the rules below, mark it processed and
 * queue its unprocessed neighbours (per undirected edge, triangles in
 * increasing index).  Rules, by the number of decided edges:
 *   3: not yet a loop -> the "rule breaker" gets its reverse added (equal
 *      forward/backward counts: the first edge not in both directions; fewer
 *      forward: the first forward edge; else the first backward edge);
 *   2: the two disagree (one forward, one backward) -> the first of them gets
 *      its reverse added and the undecided edge takes the opposite of that
 *      edge's direction; they agree -> the undecided edge takes the direction
 *      of the first edge decided one way only (forward when both are decided
 *      both ways: the upstream reads an unset variable there);
 *   1: the undecided edges take the decided edge's direction (an edge decided
 *      both ways counts as backward, as upstream);
 *   0: all three forward.
 * Output order: triangles in index order, per triangle its edges in order,
 * forward before backward, each directed edge at its first triangle.
 * Returns the count of directed edges written to `edges` (room for 6 *
 * n_tris pairs), or -1 when a triangle does not close a loop (the mesh is not
 * watertight: the upstream throws). */
typedef struct { uint64_t key; int used; } key_slot;
typedef struct { key_slot* tab; size_t cap; } key_set;

static uint64_t dkey(u32 a, u32 b) { return ((uint64_t) a << 32) | b; }
static size_t ks_find(const key_set* s, uint64_t k) {
    size_t h = hash_pair((u32) (k >> 32), (u32) k) & (s->cap - 1);
    while (s->tab[h].used && s->tab[h].key != k) h = (h + 1) & (s->cap - 1);
    return h;
}
static int ks_has(const key_set* s, u32 a, u32 b) { return s->tab[ks_find(s, dkey(a, b))].used == 1; }
static void ks_add(key_set* s, u32 a, u32 b) {
    size_t h = ks_find(s, dkey(a, b));
    s->tab[h].used = 1;
    s->tab[h].key = dkey(a, b);
}
static int ks_take(key_set* s, u32 a, u32 b) {  /* erase: the slot stays occupied (2) so probes pass it */
    size_t h = ks_find(s, dkey(a, b));
    if (s->tab[h].used != 1) return 0;
    s->tab[h].used = 2;
    return 1;
}

typedef struct { uint64_t key; int tri; } edge_tri;
static int edge_tri_cmp(const void* a, const void* b) {
    const edge_tri *x = (const edge_tri*) a, *y = (const edge_tri*) b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->tri - y->tri;
}

enum { E_UNDEF = 0, E_FWD = 1, E_BWD = 2, E_BOTH = 3 };

int orc_loop_edges(const u32* tris, int n_tris, u32* edges) {
    if (n_tris <= 0) return 0;
    key_set S;
    S.cap = 1;
    while (S.cap < (size_t) n_tris * 8 + 16) S.cap <<= 1;
    S.tab = (key_slot*) calloc(S.cap, sizeof(key_slot));
    /* undirected edge -> triangles, sorted by (edge, triangle) */
    edge_tri* et = (edge_tri*) malloc(sizeof(edge_tri) * 3 * (size_t) n_tris);
    unsigned char* done = (unsigned char*) calloc((size_t) n_tris, 1);
    size_t qcap = (size_t) n_tris * 4 + 16, qh = 0, qt = 0;
    int* queue = (int*) malloc(sizeof(int) * qcap);
    if (!S.tab || !et || !done || !queue) { free(S.tab); free(et); free(done); free(queue); return -1; }
    for (int t = 0; t < n_tris; ++t)
        for (int k = 0; k < 3; ++k) {
            u32 a = tris[t * 3 + k], b = tris[t * 3 + (k + 1) % 3];
            et[t * 3 + k].key = a < b ? dkey(a, b) : dkey(b, a);
            et[t * 3 + k].tri = t;
        }
    size_t n_et = 3 * (size_t) n_tris;
    qsort(et, n_et, sizeof(edge_tri), edge_tri_cmp);
    int next_start = 0;
    while (1) {
        while (next_start < n_tris && done[next_start]) ++next_start;
        if (next_start >= n_tris) break;
        qh = qt = 0;
        queue[qt++] = next_start;
        while (qh < qt) {
            int cur = queue[qh++];
            if (done[cur]) continue;
            u32 L[4] = {tris[cur * 3], tris[cur * 3 + 1], tris[cur * 3 + 2], tris[cur * 3]};
            int ty[3], fc = 0, bc = 0, nd = 0, und[3], nu = 0;
            for (int i = 0; i < 3; ++i) {
                int f = ks_has(&S, L[i], L[i + 1]), b = ks_has(&S, L[i + 1], L[i]);
                ty[i] = f && b ? E_BOTH : f ? E_FWD : b ? E_BWD : E_UNDEF;
                if (f) ++fc;
                if (b) ++bc;
                if (f || b) ++nd; else und[nu++] = i;
            }
            if (nd == 3) {
                if (!(fc == 3 || bc == 3)) {
                    int rb = -1;
                    for (int i = 0; i < 3 && rb < 0; ++i) {
                        if (fc == bc) { if (ty[i] != E_BOTH) rb = i; }
                        else if (fc < bc) { if (ty[i] == E_FWD) rb = i; }
                        else if (ty[i] == E_BWD) rb = i;
                    }
                    if (rb >= 0) {
                        if (ty[rb] == E_FWD) ks_add(&S, L[rb + 1], L[rb]);
                        else ks_add(&S, L[rb], L[rb + 1]);
                    }
                }
            } else if (nd == 2) {
                int k = und[0], dir = E_FWD;
                if (!(fc == 2 || bc == 2)) {
                    for (int i = 0; i < 3; ++i)
                        if (ty[i] == E_FWD || ty[i] == E_BWD) {
                            if (ty[i] == E_FWD) { ks_add(&S, L[i + 1], L[i]); dir = E_BWD; }
                            else { ks_add(&S, L[i], L[i + 1]); dir = E_FWD; }
                            break;
                        }
                } else {
                    for (int i = 0; i < 3; ++i)
                        if (ty[i] == E_FWD || ty[i] == E_BWD) { dir = ty[i]; break; }
                }
                if (dir == E_FWD) ks_add(&S, L[k], L[k + 1]);
                else ks_add(&S, L[k + 1], L[k]);
            } else if (nd == 1) {
                int dir = E_UNDEF;
                for (int i = 0; i < 3; ++i)
                    if (ty[i] != E_UNDEF) { dir = ty[i]; break; }
                for (int j = 0; j < nu; ++j) {
                    int k = und[j];
                    if (dir == E_FWD) ks_add(&S, L[k], L[k + 1]);
                    else ks_add(&S, L[k + 1], L[k]);
                }
            } else {
                for (int i = 0; i < 3; ++i) ks_add(&S, L[i], L[i + 1]);
            }
            done[cur] = 1;
            for (int i = 0; i < 3; ++i) {
                u32 a = L[i], b = L[i + 1];
                uint64_t key = a < b ? dkey(a, b) : dkey(b, a);
                /* first (edge, triangle) entry of this edge */
                size_t lo = 0, hi = n_et;
                while (lo < hi) { size_t m = (lo + hi) / 2; if (et[m].key < key) lo = m + 1; else hi = m; }
                for (size_t j = lo; j < n_et && et[j].key == key; ++j) {
                    int t = et[j].tri;
                    if (j > lo && et[j - 1].tri == t) continue;  /* a set holds each triangle once */
                    if (t != cur && !done[t]) {
                        if (qt == qcap) { qcap *= 2; queue = (int*) realloc(queue, sizeof(int) * qcap); }
                        queue[qt++] = t;
                    }
                }
            }
        }
    }
    /* every triangle must now be a loop */
    int ok = 1;
    for (int t = 0; t < n_tris && ok; ++t) {
        u32 L[4] = {tris[t * 3], tris[t * 3 + 1], tris[t * 3 + 2], tris[t * 3]};
        int fc = 0, bc = 0;
        for (int i = 0; i < 3; ++i) {
            int f = ks_has(&S, L[i], L[i + 1]), b = ks_has(&S, L[i + 1], L[i]);
            if (!f && !b) ok = 0;
            fc += f; bc += b;
        }
        if (!(fc == 3 || bc == 3)) ok = 0;
    }
    int n = 0;
    if (ok) {
        for (int t = 0; t < n_tris; ++t) {
            u32 L[4] = {tris[t * 3], tris[t * 3 + 1], tris[t * 3 + 2], tris[t * 3]};
            for (int i = 0; i < 3; ++i) {
                if (ks_take(&S, L[i], L[i + 1])) { edges[2 * n] = L[i]; edges[2 * n + 1] = L[i + 1]; ++n; }
                if (ks_take(&S, L[i + 1], L[i])) { edges[2 * n] = L[i + 1]; edges[2 * n + 1] = L[i]; ++n; }
            }
        }
    }
    free(S.tab); free(et); free(done); free(queue);
    return ok ? n : -1;
}

/* ------------------------------------------------------------ canonical LBVH */
static u32 expand_bits(u32 v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

static u32 quantize(float c, float lo, float ext) {
    float t = ext > 0.0f ? (c - lo) / ext : 0.0f;
    float v = t * 1024.0f;
    if (!(v >= 0.0f)) v = 0.0f;
    u32 q = (u32) floorf(v);
    return q > 1023u ? 1023u : q;
}

typedef struct { u32 code, idx; } key_t2;
static int key_cmp(const void* a, const void* b) {
    const key_t2* x = (const key_t2*) a; const key_t2* y = (const key_t2*) b;
    if (x->code != y->code) return x->code < y->code ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

static int delta(const u32* codes, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    u32 x = codes[i] ^ codes[j];
    if (x) return __builtin_clz(x);
    return 32 + __builtin_clz((u32) i ^ (u32) j);
}

/* BVH over n primitive boxes (plo/phi: n*3 floats).
 * Outputs: codes[n] (sorted), perm[n] (sorted position -> primitive),
 * child[2*(n-1)] (>=0 internal node, <0 leaf ~sorted position),
 * node_lo/node_hi[(n-1)*3] internal node boxes.  Returns 0 on success. */
int orc_lbvh_build(const float* plo, const float* phi, int n, u32* codes_out, u32* perm, int* child, float* node_lo,
                   float* node_hi) {
    if (n <= 0) return 0;
    float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    float* cen = (float*) malloc(sizeof(float) * 3 * (size_t) n);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            float c = 0.5f * (plo[i * 3 + k] + phi[i * 3 + k]);
            cen[i * 3 + k] = c;
            if (c < clo[k]) clo[k] = c;
            if (c > chi[k]) chi[k] = c;
        }
    float ext[3] = {chi[0] - clo[0], chi[1] - clo[1], chi[2] - clo[2]};
    key_t2* keys = (key_t2*) malloc(sizeof(key_t2) * (size_t) n);
    for (int i = 0; i < n; ++i) {
        u32 qx = quantize(cen[i * 3 + 0], clo[0], ext[0]);
        u32 qy = quantize(cen[i * 3 + 1], clo[1], ext[1]);
        u32 qz = quantize(cen[i * 3 + 2], clo[2], ext[2]);
        keys[i].code = (expand_bits(qx) << 2) | (expand_bits(qy) << 1) | expand_bits(qz);
        keys[i].idx = (u32) i;
    }
    qsort(keys, (size_t) n, sizeof(key_t2), key_cmp);
    u32* codes = codes_out;
    for (int i = 0; i < n; ++i) { codes[i] = keys[i].code; perm[i] = keys[i].idx; }
    free(keys);
    free(cen);
    if (n == 1) return 0;
    int* parent = (int*) malloc(sizeof(int) * (size_t) (2 * n));  /* internal 0..n-2, leaves n-1+s */
    for (int i = 0; i < n - 1; ++i) {
        int d = (delta(codes, n, i, i + 1) - delta(codes, n, i, i - 1)) >= 0 ? 1 : -1;
        int dmin = delta(codes, n, i, i - d);
        int lmax = 2;
        while (delta(codes, n, i, i + lmax * d) > dmin) lmax *= 2;
        int l = 0;
        for (int t = lmax / 2; t >= 1; t /= 2)
            if (delta(codes, n, i, i + (l + t) * d) > dmin) l += t;
        int j = i + l * d;
        int dnode = delta(codes, n, i, j);
        int s = 0;
        for (int div = 2;; div *= 2) {
            int t = (l + div - 1) / div;
            if (delta(codes, n, i, i + (s + t) * d) > dnode) s += t;
            if (t <= 1) break;
        }
        int g = i + s * d + (d < 0 ? -1 : 0);
        int lo = i < j ? i : j, hi = i < j ? j : i;
        int left = (lo == g) ? ~g : g;
        int right = (hi == g + 1) ? ~(g + 1) : g + 1;
        child[2 * i] = left;
        child[2 * i + 1] = right;
        parent[left >= 0 ? left : (n - 1 + ~left)] = i;
        parent[right >= 0 ? right : (n - 1 + ~right)] = i;
    }
    /* bottom-up boxes: post-order over the tree with an explicit stack */
    int* stack = (int*) malloc(sizeof(int) * (size_t) (2 * n + 4));
    char* done = (char*) calloc((size_t) n, 1);
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        int nd = stack[sp - 1];
        int ready = 1;
        for (int c = 0; c < 2; ++c) {
            int ch = child[2 * nd + c];
            if (ch >= 0 && !done[ch]) { stack[sp++] = ch; ready = 0; }
        }
        if (!ready) continue;
        --sp;
        for (int k = 0; k < 3; ++k) { node_lo[nd * 3 + k] = INFINITY; node_hi[nd * 3 + k] = -INFINITY; }
        for (int c = 0; c < 2; ++c) {
            int ch = child[2 * nd + c];
            const float *lo, *hi;
            if (ch >= 0) { lo = node_lo + ch * 3; hi = node_hi + ch * 3; }
            else { u32 pr = perm[~ch]; lo = plo + pr * 3; hi = phi + pr * 3; }
            for (int k = 0; k < 3; ++k) {
                if (lo[k] < node_lo[nd * 3 + k]) node_lo[nd * 3 + k] = lo[k];
                if (hi[k] > node_hi[nd * 3 + k]) node_hi[nd * 3 + k] = hi[k];
            }
        }
        done[nd] = 1;
    }
    free(done);
    free(stack);
    free(parent);
    return 0;
}

/* a BVH with its primitive boxes, for queries */
typedef struct {
    int n;
    float *plo, *phi;
    u32 *codes, *perm;
    int* child;
    float *nlo, *nhi;
} bvh_t;

static void bvh_free(bvh_t* b) {
    free(b->plo); free(b->phi); free(b->codes); free(b->perm); free(b->child); free(b->nlo); free(b->nhi);
    memset(b, 0, sizeof(*b));
}

static void bvh_make(bvh_t* b, int n, float* plo, float* phi) {
    b->n = n; b->plo = plo; b->phi = phi;
    b->codes = (u32*) malloc(sizeof(u32) * (size_t) (n > 0 ? n : 1));
    b->perm = (u32*) malloc(sizeof(u32) * (size_t) (n > 0 ? n : 1));
    b->child = (int*) malloc(sizeof(int) * (size_t) (2 * (n > 1 ? n : 1)));
    b->nlo = (float*) malloc(sizeof(float) * 3 * (size_t) (n > 1 ? n : 1));
    b->nhi = (float*) malloc(sizeof(float) * 3 * (size_t) (n > 1 ? n : 1));
    orc_lbvh_build(plo, phi, n, b->codes, b->perm, b->child, b->nlo, b->nhi);
}

static int box_hit(const float* lo, const float* hi, const double* qlo, const double* qhi) {
    return !(qlo[0] > hi[0] || qhi[0] < lo[0] || qlo[1] > hi[1] || qhi[1] < lo[1] || qlo[2] > hi[2] || qhi[2] < lo[2]);
}

/* visits every primitive whose box overlaps [qlo, qhi]; returns #nodes tested */
typedef int (*visit_fn)(void* ctx, u32 prim);  /* nonzero return stops the query */

static uint64_t bvh_query(const bvh_t* b, const double* qlo, const double* qhi, visit_fn fn, void* ctx) {
    if (b->n <= 0) return 0;
    uint64_t tests = 0;
    if (b->n == 1) {
        ++tests;
        if (box_hit(b->plo, b->phi, qlo, qhi)) fn(ctx, b->perm[0]);
        return tests;
    }
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        int nd = stack[--sp];
        for (int c = 0; c < 2; ++c) {
            int ch = b->child[2 * nd + c];
            ++tests;
            if (ch >= 0) {
                if (box_hit(b->nlo + ch * 3, b->nhi + ch * 3, qlo, qhi)) stack[sp++] = ch;
            } else {
                u32 pr = b->perm[~ch];
                if (box_hit(b->plo + pr * 3, b->phi + pr * 3, qlo, qhi))
                    if (fn(ctx, pr)) return tests;
            }
        }
    }
    return tests;
}

/* ----------------------------------------------------------- distances */
static double pt_seg2(d3 p, d3 a, d3 b) {
    d3 ab = sub(b, a);
    double L = dot(ab, ab);
    double t = L > 0 ? clamp01(dot(sub(p, a), ab) / L) : 0.0;
    d3 c = add(a, mul(ab, t));
    d3 d = sub(p, c);
    return dot(d, d);
}

/* squared distance between segments p1q1 and p2q2 (Ericson, RTCD 5.1.9) */
static double seg_seg2(d3 p1, d3 q1, d3 p2, d3 q2) {
    d3 d1 = sub(q1, p1), d2 = sub(q2, p2), r = sub(p1, p2);
    double a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    double s, t;
    if (a <= 1e-300 && e <= 1e-300) return dot(r, r);
    if (a <= 1e-300) { s = 0; t = clamp01(f / e); }
    else {
        double c = dot(d1, r);
        if (e <= 1e-300) { t = 0; s = clamp01(-c / a); }
        else {
            double b = dot(d1, d2), den = a * e - b * b;
            s = den > 0 ? clamp01((b * f - c * e) / den) : 0.0;
            t = (b * s + f) / e;
            if (t < 0) { t = 0; s = clamp01(-c / a); }
            else if (t > 1) { t = 1; s = clamp01((b - c) / a); }
        }
    }
    d3 c1 = add(p1, mul(d1, s)), c2 = add(p2, mul(d2, t));
    d3 d = sub(c1, c2);
    return dot(d, d);
}

/* squared distance from p to triangle abc (Ericson 5.1.5), degenerate-safe */
static double pt_tri2(d3 p, d3 a, d3 b, d3 c) {
    d3 ab = sub(b, a), ac = sub(c, a);
    d3 n = cross(ab, ac);
    double nn = dot(n, n);
    double scale = dot(ab, ab) * dot(ac, ac);
    if (!(nn > 1e-24 * scale) || nn <= 0) {
        double d = pt_seg2(p, a, b), e = pt_seg2(p, b, c), f = pt_seg2(p, c, a);
        return d < e ? (d < f ? d : f) : (e < f ? e : f);
    }
    d3 ap = sub(p, a);
    double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0 && d2 <= 0) return dot(ap, ap);
    d3 bp = sub(p, b);
    double d3_ = dot(ab, bp), d4 = dot(ac, bp);
    if (d3_ >= 0 && d4 <= d3_) return dot(bp, bp);
    double vc = d1 * d4 - d3_ * d2;
    if (vc <= 0 && d1 >= 0 && d3_ <= 0) { double v = d1 / (d1 - d3_); d3 q = sub(p, add(a, mul(ab, v))); return dot(q, q); }
    d3 cp = sub(p, c);
    double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0 && d5 <= d6) return dot(cp, cp);
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) { double w = d2 / (d2 - d6); d3 q = sub(p, add(a, mul(ac, w))); return dot(q, q); }
    double va = d3_ * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3_) >= 0 && (d5 - d6) >= 0) {
        double w = (d4 - d3_) / ((d4 - d3_) + (d5 - d6));
        d3 q = sub(p, add(b, mul(sub(c, b), w)));
        return dot(q, q);
    }
    double dn = 1.0 / (va + vb + vc);
    double v = vb * dn, w = vc * dn;
    d3 q = sub(p, add(a, add(mul(ab, v), mul(ac, w))));
    return dot(q, q);
}

/*
 * Segment pq vs triangle abc.  Returns 1 when the closed segment properly
 * crosses the triangle (through its plane, crossing point inside the closed
 * triangle) or touches it; *m receives the robustness margin of a hit (the
 * smallest of: endpoint distances to the plane, in-plane distance of the
 * crossing point to the three edge lines) or the distance of a miss.
 */
static int seg_tri(d3 p, d3 q, d3 a, d3 b, d3 c, double* m) {
    d3 n = cross(sub(b, a), sub(c, a));
    double nl = len(n);
    if (nl > 0) {
        double dp = dot(n, sub(p, a)) / nl, dq = dot(n, sub(q, a)) / nl;
        if ((dp > 0 && dq < 0) || (dp < 0 && dq > 0) || (dp == 0) != (dq == 0)) {
            double t = dp / (dp - dq);
            d3 x = add(p, mul(sub(q, p), t));
            d3 nu = mul(n, 1.0 / nl);
            /* signed in-plane distances of x to the three edge lines (positive inside) */
            d3 e0 = sub(b, a), e1 = sub(c, b), e2 = sub(a, c);
            double l0 = len(e0), l1 = len(e1), l2 = len(e2);
            if (l0 > 0 && l1 > 0 && l2 > 0) {
                double s0 = dot(cross(e0, sub(x, a)), nu) / l0;
                double s1 = dot(cross(e1, sub(x, b)), nu) / l1;
                double s2 = dot(cross(e2, sub(x, c)), nu) / l2;
                if (s0 >= 0 && s1 >= 0 && s2 >= 0) {
                    double mm = fabs(dp);
                    if (fabs(dq) < mm) mm = fabs(dq);
                    if (s0 < mm) mm = s0;
                    if (s1 < mm) mm = s1;
                    if (s2 < mm) mm = s2;
                    *m = mm;
                    return 1;
                }
            }
        }
    }
    /* no proper crossing: distance from the boundary features */
    double d = pt_tri2(p, a, b, c), t;
    if ((t = pt_tri2(q, a, b, c)) < d) d = t;
    if ((t = seg_seg2(p, q, a, b)) < d) d = t;
    if ((t = seg_seg2(p, q, b, c)) < d) d = t;
    if ((t = seg_seg2(p, q, c, a)) < d) d = t;
    d = sqrt(d);
    if (d <= 1e-12) { *m = 0.0; return 1; }  /* touching (to rounding): a hit with zero margin */
    *m = d;
    return 0;
}

/* --------------------------------------------------------------- thread pool */
typedef struct {
    int n;
    int next;
    pthread_mutex_t mu;
    void (*work)(void* ctx, int i, void* scratch);
    void* ctx;
    size_t scratch_bytes;
} pool_t;

static void* pool_main(void* arg) {
    pool_t* p = (pool_t*) arg;
    void* scratch = p->scratch_bytes ? malloc(p->scratch_bytes) : NULL;
    for (;;) {
        pthread_mutex_lock(&p->mu);
        int i = p->next++;
        pthread_mutex_unlock(&p->mu);
        if (i >= p->n) break;
        p->work(p->ctx, i, scratch);
    }
    free(scratch);
    return NULL;
}

static void run_pool(int n, int threads, void (*work)(void*, int, void*), void* ctx, size_t scratch_bytes) {
    pool_t p;
    p.n = n; p.next = 0; p.work = work; p.ctx = ctx; p.scratch_bytes = scratch_bytes;
    pthread_mutex_init(&p.mu, NULL);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    for (int t = 0; t < threads; ++t) pthread_create(&th[t], NULL, pool_main, &p);
    for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&p.mu);
}

/* ---------------------------------------------------------------- robot/scene */
typedef struct {
    int dof;
    const float *cos_mask, *sin_mask, *one_mask, *base_tf;
    int n_links;
    const float* link_verts;
    const u32 *link_vert_off, *link_tris, *link_tri_off, *link_edges, *link_edge_off;
    int skip_base;
    int n_spheres;
    const float *sphere_centers, *sphere_radii;
    const u32* sphere_links;
} orc_robot;

typedef struct {
    int n_verts;
    const float* verts;
    int n_tris;
    const u32* tris;
    int n_edges;
    const u32* edges;
} orc_scene;

typedef struct {
    uint64_t node_tests;  /* BVH child-box tests */
    uint64_t prim_tests;  /* exact primitive tests */
} orc_work;

static void tri_boxes(const float* verts, const u32* tris, int n, float** lo, float** hi) {
    *lo = (float*) malloc(sizeof(float) * 3 * (size_t) (n ? n : 1));
    *hi = (float*) malloc(sizeof(float) * 3 * (size_t) (n ? n : 1));
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            float a = verts[tris[i * 3] * 3 + k], b = verts[tris[i * 3 + 1] * 3 + k], c = verts[tris[i * 3 + 2] * 3 + k];
            (*lo)[i * 3 + k] = fminf(a, fminf(b, c));
            (*hi)[i * 3 + k] = fmaxf(a, fmaxf(b, c));
        }
}

static void edge_boxes(const float* verts, const u32* edges, int n, float** lo, float** hi) {
    *lo = (float*) malloc(sizeof(float) * 3 * (size_t) (n ? n : 1));
    *hi = (float*) malloc(sizeof(float) * 3 * (size_t) (n ? n : 1));
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            float a = verts[edges[i * 2] * 3 + k], b = verts[edges[i * 2 + 1] * 3 + k];
            (*lo)[i * 3 + k] = fminf(a, b);
            (*hi)[i * 3 + k] = fmaxf(a, b);
        }
}

/* ------------------------------------------------------------ discrete check */
enum { ORC_OBS_TO_ROBOT = 0, ORC_ROBOT_TO_OBS = 1 };

typedef struct {
    int kind;
    const orc_robot* R;
    const orc_scene* S;
    const float* q;
    double eps;
    bvh_t scene_tri, scene_edge;
    bvh_t* link_tri;
    unsigned char *hit, *band, *marg;
    u32* count;
    orc_work* work;  /* per pose, optional */
    int early;       /* stop a pose at its first hit (flags only) */
} disc_ctx;

typedef struct {
    /* query-local state */
    d3 p, q;        /* segment, in the frame of the target triangles */
    const float* tv; const u32* tt; /* target triangle verts / indices */
    const double* T;  /* transform from target-local to world, or NULL */
    double eps;
    int any_hit, robust, marginal;
    u32 hits;
    uint64_t prim_tests;
} seg_query;

static int visit_tri(void* vctx, u32 t) {
    seg_query* s = (seg_query*) vctx;
    const u32* ix = s->tt + (size_t) t * 3;
    d3 a = fv(s->tv + ix[0] * 3), b = fv(s->tv + ix[1] * 3), c = fv(s->tv + ix[2] * 3);
    if (s->T) { a = xform(s->T, a); b = xform(s->T, b); c = xform(s->T, c); }
    double m;
    ++s->prim_tests;
    int h = seg_tri(s->p, s->q, a, b, c, &m);
    if (h) {
        s->any_hit = 1;
        s->hits++;
        if (m > s->eps) s->robust = 1; else s->marginal = 1;
    } else if (m <= s->eps) {
        s->marginal = 1;
    }
    return 0;
}

typedef struct {
    u32* ids;
    u32 n;
} edge_list;

static int collect_prim(void* vctx, u32 prim) {
    edge_list* l = (edge_list*) vctx;
    l->ids[l->n++] = prim;
    return 0;
}

static void disc_pose(void* vctx, int pose, void* scratch) {
    disc_ctx* C = (disc_ctx*) vctx;
    const orc_robot* R = C->R;
    const orc_scene* S = C->S;
    double T[9 * 12];
    double* Tp = (C->R->dof + 1) * 12 <= 9 * 12 ? T : (double*) malloc(sizeof(double) * (size_t) (R->dof + 1) * 12);
    orc_fk_pose(R->dof, R->cos_mask, R->sin_mask, R->one_mask, R->base_tf, C->q + (size_t) pose * R->dof, Tp);
    int any = 0, robust = 0, marginal = 0;
    u32 count = 0;
    uint64_t ntests = 0, ptests = 0;
    double eps = C->eps;
    for (int l = R->skip_base ? 1 : 0; l < R->n_links; ++l) {
        const double* TL = Tp + l * 12;
        const float* lv = R->link_verts + (size_t) R->link_vert_off[l] * 3;
        if (C->kind == ORC_ROBOT_TO_OBS) {
            /* every link edge, moved to the world, against the scene triangles */
            u32 e0 = R->link_edge_off[l], e1 = R->link_edge_off[l + 1];
            for (u32 e = e0; e < e1; ++e) {
                seg_query s;
                memset(&s, 0, sizeof(s));
                s.p = xform(TL, fv(lv + R->link_edges[e * 2] * 3));
                s.q = xform(TL, fv(lv + R->link_edges[e * 2 + 1] * 3));
                s.tv = S->verts; s.tt = S->tris; s.T = NULL; s.eps = eps;
                double qlo[3] = {fmin(s.p.x, s.q.x) - eps, fmin(s.p.y, s.q.y) - eps, fmin(s.p.z, s.q.z) - eps};
                double qhi[3] = {fmax(s.p.x, s.q.x) + eps, fmax(s.p.y, s.q.y) + eps, fmax(s.p.z, s.q.z) + eps};
                ntests += bvh_query(&C->scene_tri, qlo, qhi, visit_tri, &s);
                ptests += s.prim_tests;
                if (s.any_hit) { any = 1; ++count; }
                robust |= s.robust; marginal |= s.marginal;
                if (C->early && any) goto done;
            }
        } else {
            /* every obstacle edge, moved into the link frame, against the link triangles;
             * only edges whose boxes reach the link's world box can hit (pure acceleration) */
            const u32* lt = R->link_tris + (size_t) R->link_tri_off[l] * 3;
            double wlo[3] = {INFINITY, INFINITY, INFINITY}, whi[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (u32 v = R->link_vert_off[l]; v < R->link_vert_off[l + 1]; ++v) {
                d3 w = xform(TL, fv(R->link_verts + (size_t) v * 3));
                double c[3] = {w.x, w.y, w.z};
                for (int k = 0; k < 3; ++k) { wlo[k] = fmin(wlo[k], c[k] - eps); whi[k] = fmax(whi[k], c[k] + eps); }
            }
            edge_list cand = {(u32*) scratch, 0};
            ntests += bvh_query(&C->scene_edge, wlo, whi, collect_prim, &cand);
            for (u32 ci = 0; ci < cand.n; ++ci) {
                u32 e = cand.ids[ci];
                d3 pw = fv(S->verts + S->edges[e * 2] * 3), qw = fv(S->verts + S->edges[e * 2 + 1] * 3);
                seg_query s;
                memset(&s, 0, sizeof(s));
                s.p = xform_inv(TL, pw);
                s.q = xform_inv(TL, qw);
                s.tv = lv; s.tt = lt; s.T = NULL; s.eps = eps;
                double qlo[3] = {fmin(s.p.x, s.q.x) - eps, fmin(s.p.y, s.q.y) - eps, fmin(s.p.z, s.q.z) - eps};
                double qhi[3] = {fmax(s.p.x, s.q.x) + eps, fmax(s.p.y, s.q.y) + eps, fmax(s.p.z, s.q.z) + eps};
                ntests += bvh_query(&C->link_tri[l], qlo, qhi, visit_tri, &s);
                ptests += s.prim_tests;
                if (s.any_hit) { any = 1; count += s.hits; }
                robust |= s.robust; marginal |= s.marginal;
                if (C->early && any) goto done;
            }
        }
    }
done:
    if (Tp != T) free(Tp);
    C->hit[pose] = (unsigned char) any;
    if (C->count) C->count[pose] = count;
    if (C->band) C->band[pose] = (unsigned char) (!robust && marginal);
    if (C->marg) C->marg[pose] = (unsigned char) marginal;
    if (C->work) { C->work[pose].node_tests = ntests; C->work[pose].prim_tests = ptests; }
}

/* A prepared discrete query: the acceleration structures are built once so
 * repeated runs (the timed CPU baseline) measure the queries alone. */
void* orc_discrete_prepare(int kind, const orc_robot* R, const orc_scene* S) {
    disc_ctx* C = (disc_ctx*) calloc(1, sizeof(disc_ctx));
    C->kind = kind; C->R = R; C->S = S;
    float *lo, *hi;
    if (kind == ORC_ROBOT_TO_OBS) {
        tri_boxes(S->verts, S->tris, S->n_tris, &lo, &hi);
        bvh_make(&C->scene_tri, S->n_tris, lo, hi);
    } else {
        edge_boxes(S->verts, S->edges, S->n_edges, &lo, &hi);
        bvh_make(&C->scene_edge, S->n_edges, lo, hi);
        C->link_tri = (bvh_t*) calloc((size_t) R->n_links, sizeof(bvh_t));
        for (int l = 0; l < R->n_links; ++l) {
            int nt = (int) (R->link_tri_off[l + 1] - R->link_tri_off[l]);
            tri_boxes(R->link_verts + (size_t) R->link_vert_off[l] * 3, R->link_tris + (size_t) R->link_tri_off[l] * 3, nt,
                      &lo, &hi);
            bvh_make(&C->link_tri[l], nt, lo, hi);
        }
    }
    return C;
}

void orc_discrete_free(void* h) {
    disc_ctx* C = (disc_ctx*) h;
    if (!C) return;
    if (C->kind == ORC_ROBOT_TO_OBS) bvh_free(&C->scene_tri);
    else {
        bvh_free(&C->scene_edge);
        for (int l = 0; l < C->R->n_links; ++l) bvh_free(&C->link_tri[l]);
        free(C->link_tri);
    }
    free(C);
}

/* early != 0: flags only, each pose stops at its first hit (count/band/marg
 * are then partial and must not be used). */
int orc_discrete_run(void* h, const float* q, int n, double eps, int threads, int early, unsigned char* hit, u32* count,
                     unsigned char* band, unsigned char* marg, orc_work* work) {
    disc_ctx* C = (disc_ctx*) h;
    C->q = q; C->eps = eps; C->early = early;
    C->hit = hit; C->count = count; C->band = band; C->marg = marg; C->work = work;
    run_pool(n, threads, disc_pose, C, sizeof(u32) * (size_t) (C->S->n_edges + 1));
    return 0;
}

int orc_discrete(int kind, const orc_robot* R, const orc_scene* S, const float* q, int n, double eps, int threads,
                 unsigned char* hit, u32* count, unsigned char* band, unsigned char* marg, orc_work* work) {
    void* h = orc_discrete_prepare(kind, R, S);
    orc_discrete_run(h, q, n, eps, threads, 0, hit, count, band, marg, work);
    orc_discrete_free(h);
    return 0;
}

/* ------------------------------------------------------------- containment
 * No upstream counterpart: the reference's rays follow surface crossings only,
 * so a link wholly inside an obstacle (or an obstacle inside a link) is never
 * seen.  For a pose with no surface crossing (skip[pose] == 0), every checked
 * link l and obstacle o: (a) the link's first vertex inside o, or (b) o's
 * first vertex (first vertex of its first triangle) inside the link, decided
 * by the parity of the crossings of the segment from the point along
 * (0.48, 0.6, 0.64) to beyond the other mesh's box, with that mesh's
 * triangles (closed segment vs closed triangle).  A crossing within eps of
 * flipping puts the pose in band.  Both meshes must be closed.
 */
typedef struct {
    const orc_robot* R;
    const orc_scene* S;
    const u32* ooff;
    int n_obs;
    const float* q;
    double eps;
    const unsigned char* skip;
    unsigned char *contain, *band;
    bvh_t scene_tri;
    bvh_t* link_tri;
    u32* tri_obs;
    double* obox;  /* [o][6] lo, hi */
    double* lbox;  /* [l][6] link-frame lo, hi */
} cont_ctx;

typedef struct {
    d3 p, q;
    const float* tv; const u32* tt;
    const u32* tag; u32 want;  /* count only triangles with tag[t] == want (tag NULL: all) */
    double eps;
    u32 crossings;
    int marginal;
} ray_query;

static int visit_cross(void* vctx, u32 t) {
    ray_query* r = (ray_query*) vctx;
    if (r->tag && r->tag[t] != r->want) return 0;
    d3 a = fv(r->tv + r->tt[t * 3] * 3), b = fv(r->tv + r->tt[t * 3 + 1] * 3), c = fv(r->tv + r->tt[t * 3 + 2] * 3);
    double m;
    int h = seg_tri(r->p, r->q, a, b, c, &m);
    if (h) r->crossings++;
    if (m <= r->eps) r->marginal = 1;
    return 0;
}

/* exit parameter of p + t d from the box [lo, hi] */
static double box_exit_d(d3 p, d3 d, const double* lo, const double* hi) {
    double pc[3] = {p.x, p.y, p.z}, dc[3] = {d.x, d.y, d.z}, t = INFINITY;
    for (int k = 0; k < 3; ++k) {
        double tk = dc[k] > 0 ? (hi[k] - pc[k]) / dc[k] : (dc[k] < 0 ? (lo[k] - pc[k]) / dc[k] : INFINITY);
        if (tk < t) t = tk;
    }
    return t < 0 ? 0 : t;
}

static int in_box(d3 p, const double* b, double pad) {
    return p.x >= b[0] - pad && p.x <= b[3] + pad && p.y >= b[1] - pad && p.y <= b[4] + pad && p.z >= b[2] - pad &&
           p.z <= b[5] + pad;
}

/* crossings parity of the ray from p (direction dir) through a mesh held in box b */
static int ray_parity(const bvh_t* bvh, d3 p, const double* b, const float* tv, const u32* tt, const u32* tag, u32 want,
                      double eps, int* marginal) {
    const d3 dir = v3(0.48, 0.6, 0.64);
    double t = box_exit_d(p, dir, b, b + 3) + 1e-2;
    ray_query r;
    memset(&r, 0, sizeof(r));
    r.p = p; r.q = add(p, mul(dir, t)); r.tv = tv; r.tt = tt; r.tag = tag; r.want = want; r.eps = eps;
    double qlo[3] = {fmin(r.p.x, r.q.x) - eps, fmin(r.p.y, r.q.y) - eps, fmin(r.p.z, r.q.z) - eps};
    double qhi[3] = {fmax(r.p.x, r.q.x) + eps, fmax(r.p.y, r.q.y) + eps, fmax(r.p.z, r.q.z) + eps};
    bvh_query(bvh, qlo, qhi, visit_cross, &r);
    if (r.marginal) *marginal = 1;
    return (int) (r.crossings & 1u);
}

static void cont_pose(void* vctx, int pose, void* scratch) {
    (void) scratch;
    cont_ctx* C = (cont_ctx*) vctx;
    const orc_robot* R = C->R;
    const orc_scene* S = C->S;
    C->contain[pose] = 0;
    if (C->band) C->band[pose] = 0;
    if (C->skip && C->skip[pose]) return;
    double T[9 * 12];
    double* Tp = (R->dof + 1) * 12 <= 9 * 12 ? T : (double*) malloc(sizeof(double) * (size_t) (R->dof + 1) * 12);
    orc_fk_pose(R->dof, R->cos_mask, R->sin_mask, R->one_mask, R->base_tf, C->q + (size_t) pose * R->dof, Tp);
    int inside = 0, marginal = 0;
    for (int l = R->skip_base ? 1 : 0; l < R->n_links && !inside; ++l) {
        if (R->link_vert_off[l + 1] == R->link_vert_off[l]) continue;
        const double* TL = Tp + l * 12;
        const float* lv = R->link_verts + (size_t) R->link_vert_off[l] * 3;
        const u32* lt = R->link_tris + (size_t) R->link_tri_off[l] * 3;
        d3 p = xform(TL, fv(lv));
        for (int o = 0; o < C->n_obs && !inside; ++o) {
            const double* ob = C->obox + 6 * o;
            if (in_box(p, ob, 1e-4) &&
                ray_parity(&C->scene_tri, p, ob, S->verts, S->tris, C->tri_obs, (u32) o, C->eps, &marginal))
                inside = 1;
            if (inside || C->ooff[o + 1] == C->ooff[o]) continue;
            d3 qo = xform_inv(TL, fv(S->verts + S->tris[(size_t) C->ooff[o] * 3] * 3));
            const double* lb = C->lbox + 6 * l;
            if (in_box(qo, lb, 1e-4) && ray_parity(&C->link_tri[l], qo, lb, lv, lt, NULL, 0, C->eps, &marginal))
                inside = 1;
        }
    }
    if (Tp != T) free(Tp);
    C->contain[pose] = (unsigned char) inside;
    if (C->band) C->band[pose] = (unsigned char) marginal;
}

int orc_containment(const orc_robot* R, const orc_scene* S, const u32* obstacle_tri_off, int n_obs, const float* q,
                    int n, double eps, int threads, const unsigned char* skip, unsigned char* contain,
                    unsigned char* band) {
    cont_ctx C;
    memset(&C, 0, sizeof(C));
    C.R = R; C.S = S; C.ooff = obstacle_tri_off; C.n_obs = n_obs; C.q = q; C.eps = eps; C.skip = skip;
    C.contain = contain; C.band = band;
    float *lo, *hi;
    tri_boxes(S->verts, S->tris, S->n_tris, &lo, &hi);
    bvh_make(&C.scene_tri, S->n_tris, lo, hi);
    C.tri_obs = (u32*) malloc(sizeof(u32) * (size_t) (S->n_tris ? S->n_tris : 1));
    C.obox = (double*) malloc(sizeof(double) * 6 * (size_t) (n_obs ? n_obs : 1));
    for (int o = 0; o < n_obs; ++o) {
        double* b = C.obox + 6 * o;
        b[0] = b[1] = b[2] = INFINITY; b[3] = b[4] = b[5] = -INFINITY;
        for (u32 t = obstacle_tri_off[o]; t < obstacle_tri_off[o + 1]; ++t) {
            C.tri_obs[t] = (u32) o;
            for (int k = 0; k < 3; ++k)
                for (int a = 0; a < 3; ++a) {
                    double v = S->verts[S->tris[t * 3 + k] * 3 + a];
                    if (v < b[a]) b[a] = v;
                    if (v > b[3 + a]) b[3 + a] = v;
                }
        }
    }
    C.link_tri = (bvh_t*) calloc((size_t) R->n_links, sizeof(bvh_t));
    C.lbox = (double*) malloc(sizeof(double) * 6 * (size_t) R->n_links);
    for (int l = 0; l < R->n_links; ++l) {
        int nt = (int) (R->link_tri_off[l + 1] - R->link_tri_off[l]);
        const float* lv = R->link_verts + (size_t) R->link_vert_off[l] * 3;
        tri_boxes(lv, R->link_tris + (size_t) R->link_tri_off[l] * 3, nt, &lo, &hi);
        bvh_make(&C.link_tri[l], nt, lo, hi);
        double* b = C.lbox + 6 * l;
        b[0] = b[1] = b[2] = INFINITY; b[3] = b[4] = b[5] = -INFINITY;
        for (u32 v = 0; v < R->link_vert_off[l + 1] - R->link_vert_off[l]; ++v)
            for (int a = 0; a < 3; ++a) {
                double x = lv[v * 3 + a];
                if (x < b[a]) b[a] = x;
                if (x > b[3 + a]) b[3 + a] = x;
            }
    }
    run_pool(n, threads, cont_pose, &C, 16);
    bvh_free(&C.scene_tri);
    for (int l = 0; l < R->n_links; ++l) bvh_free(&C.link_tri[l]);
    free(C.link_tri); free(C.lbox); free(C.obox); free(C.tri_obs);
    return 0;
}

/* ------------------------------------------------------------- sweep checks */
typedef struct {
    d3 a, b;        /* capsule axis (linear) */
    d3 B0, B1, B2;  /* quadratic Bezier piece */
    int quad;
    int surface;    /* reference semantics: a directed edge hits when it enters the piece (below) */
    d3 n0, n1;      /* quadratic, surface: unit normals of the flat end caps (zero: no cap) */
    double r, eps;
    const float* sv; const u32* se;  /* scene verts / edges */
    int any_hit, robust, marginal;
    u32 hits;
    uint64_t prim_tests;
} sweep_query;

/* classify d (distance) against radius r with band eps */
static void classify(sweep_query* s, double d) {
    if (d <= s->r) { s->any_hit = 1; s->hits++; if (d < s->r - s->eps) s->robust = 1; else s->marginal = 1; }
    else if (d <= s->r + s->eps) s->marginal = 1;
}

/* distance from segment pq to quadratic Bezier (B0,B1,B2) by branch and bound:
 * the convex hull (triangle) of a piece's control points bounds it from below,
 * its end points from above.  Stops once the distance is certainly below
 * hit_below or a piece is certainly beyond miss_above, or the bracket is
 * tighter than 1e-12 m. */
static double seg_quad_dist(d3 p, d3 q, d3 B0, d3 B1, d3 B2, double hit_below, double miss_above) {
    typedef struct { d3 a, b, c; double lb; int depth; } piece;
    piece st[256];
    int sp = 0;
    double ub = sqrt(seg_seg2(p, q, B0, B0));
    double t = sqrt(seg_seg2(p, q, B2, B2));
    if (t < ub) ub = t;
    double m;
    double lb0 = seg_tri(p, q, B0, B1, B2, &m) ? 0.0 : m;
    st[sp].a = B0; st[sp].b = B1; st[sp].c = B2; st[sp].lb = lb0; st[sp].depth = 0; ++sp;
    while (sp) {
        piece pc = st[--sp];
        if (pc.lb >= ub) continue;
        if (ub < hit_below) return ub;               /* decided: robust hit */
        if (pc.lb > miss_above) continue;            /* cannot reach the band: a certain miss */
        if (ub - pc.lb < 1e-12 || pc.depth > 48) continue;
        /* de Casteljau split at 1/2 */
        d3 ab = mul(add(pc.a, pc.b), 0.5), bc = mul(add(pc.b, pc.c), 0.5), mid = mul(add(ab, bc), 0.5);
        double dm = sqrt(seg_seg2(p, q, mid, mid));
        if (dm < ub) ub = dm;
        piece L = {pc.a, ab, mid, 0, pc.depth + 1}, Rr = {mid, bc, pc.c, 0, pc.depth + 1};
        L.lb = seg_tri(p, q, L.a, L.b, L.c, &m) ? 0.0 : m;
        Rr.lb = seg_tri(p, q, Rr.a, Rr.b, Rr.c, &m) ? 0.0 : m;
        if (Rr.lb < ub) st[sp++] = Rr;
        if (L.lb < ub) st[sp++] = L;
    }
    return ub;
}

/* ---- surface (reference) semantics of the sweeps.
 * The upstream casts each directed loop edge p -> q as a ray (tmin 0, tmax
 * |q - p|, RTCD/CollisionDetector/CCCuda.cu:56-77) against OptiX's built-in
 * curve intersectors and counts every reported intersection in its any-hit
 * program (CCCuda.cu:37-41).  Those intersectors report a ray entering a
 * curve primitive from outside, not a ray that starts inside it; that is why
 * the curve scenes cast loop edges (RTCD/Meshes/mesh.h:378-620).  Per (edge,
 * primitive) the predicate is therefore
 *     hit  <=>  p lies outside the primitive's closed solid P  and  [p, q] meets P.
 * Linear primitive: the capsule of radius r around the axis, round caps
 * (endcapFlags = 1, RTCD/Robot/batchCurveRobot.h:230).  Quadratic primitive:
 * the sphere-swept piece u in [0, 1] cut by flat caps, the planes through its
 * ends normal to its end tangents (B1 - B0 at u = 0, B2 - B1 at u = 1; B2 - B0
 * where one of those vanishes); the upstream comment on the quadratic curves'
 * flat caps is RTCD/CollisionDetector/Test/testCollisionCheckerCurve.cpp:
 * 157-162.  The cap disks belong to the solid (closed flat caps).  Quadratic
 * pieces carry no start/end spheres in these semantics.
 *
 * Band: the pair is marginal when the decision changes with the radius and
 * the cap planes moved by eps either way:
 *   robust hit  = meets(r - eps, caps - eps) and not inside(p; r + eps, caps + eps)
 *   robust miss = not meets(r + eps, caps + eps) or inside(p; r - eps, caps - eps). */
static void quad_caps(d3 B0, d3 B1, d3 B2, d3* n0, d3* n1) {
    d3 t0 = sub(B1, B0), t1 = sub(B2, B1), ch = sub(B2, B0);
    if (dot(t0, t0) == 0.0) t0 = ch;
    if (dot(t1, t1) == 0.0) t1 = ch;
    double l0 = len(t0), l1 = len(t1);
    *n0 = l0 > 0 ? mul(t0, 1.0 / l0) : v3(0, 0, 0);
    *n1 = l1 > 0 ? mul(t1, 1.0 / l1) : v3(0, 0, 0);
}

/* the parameter range [t0, t1] of p + t (q - p), t in [0, 1], inside both cap
 * half-spaces grown by g (negative g: shrunk); 0 when empty */
static int cap_clip(const sweep_query* s, d3 p, d3 q, double g, double* t0, double* t1) {
    d3 d = sub(q, p);
    double lo = 0.0, hi = 1.0;
    for (int k = 0; k < 2; ++k) {
        /* signed distance inside: (x - B0).n0 at the start cap, (B2 - x).n1 at the end cap */
        double a = k == 0 ? dot(sub(p, s->B0), s->n0) : dot(sub(s->B2, p), s->n1);
        double b = k == 0 ? dot(d, s->n0) : -dot(d, s->n1);
        if (k == 0 ? dot(s->n0, s->n0) == 0.0 : dot(s->n1, s->n1) == 0.0) continue;
        /* a + b t >= -g */
        if (b == 0.0) { if (a < -g) return 0; continue; }
        double t = (-g - a) / b;
        if (b > 0) { if (t > lo) lo = t; }
        else if (t < hi) hi = t;
    }
    if (lo > hi) return 0;
    *t0 = lo; *t1 = hi;
    return 1;
}

static int cap_inside(const sweep_query* s, d3 p, double g) {
    if (dot(s->n0, s->n0) > 0 && dot(sub(p, s->B0), s->n0) < -g) return 0;
    if (dot(s->n1, s->n1) > 0 && dot(sub(s->B2, p), s->n1) < -g) return 0;
    return 1;
}

/* distance from the part of [p, q] inside the caps grown by g to the piece;
 * INFINITY when that part is empty */
static double quad_clipped_dist(const sweep_query* s, d3 p, d3 q, double g, double hit_below, double miss_above) {
    double t0, t1;
    if (!cap_clip(s, p, q, g, &t0, &t1)) return INFINITY;
    d3 d = sub(q, p);
    return seg_quad_dist(add(p, mul(d, t0)), add(p, mul(d, t1)), s->B0, s->B1, s->B2, hit_below, miss_above);
}

static void visit_surface(sweep_query* s, d3 p, d3 q) {
    const double r = s->r, e = s->eps;
    int hit, rob_hit, rob_miss;
    if (!s->quad) {
        double dseg = sqrt(seg_seg2(p, q, s->a, s->b));
        double dp = sqrt(pt_seg2(p, s->a, s->b));
        hit = dseg <= r && dp > r;
        rob_hit = dseg <= r - e && dp > r + e;
        rob_miss = dseg > r + e || dp < r - e;
    } else {
        /* the grown cut first: most pairs are certain misses there */
        double dg = quad_clipped_dist(s, p, q, e, r - e, r + e);
        if (dg > r + e) return;  /* robust miss */
        /* every value below is compared only with r - e, r and r + e: the
         * branch and bound may stop once it is certainly below r - e or above
         * r + e, and is exact (to 1e-12 m) in between */
        double dp = seg_quad_dist(p, p, s->B0, s->B1, s->B2, r - e, r + e);
        double d0 = quad_clipped_dist(s, p, q, 0.0, r - e, r + e);
        double ds = quad_clipped_dist(s, p, q, -e, r - e, r + e);
        int in0 = cap_inside(s, p, 0.0) && dp <= r;
        int in_g = cap_inside(s, p, e) && dp <= r + e;
        int in_s = cap_inside(s, p, -e) && dp <= r - e;
        hit = d0 <= r && !in0;
        rob_hit = ds <= r - e && !in_g;
        rob_miss = dg > r + e || in_s;
    }
    if (hit) {
        s->any_hit = 1;
        s->hits++;
        if (rob_hit) s->robust = 1; else s->marginal = 1;
    } else if (!rob_miss) {
        s->marginal = 1;
    }
}

static int visit_edge(void* vctx, u32 e) {
    sweep_query* s = (sweep_query*) vctx;
    d3 p = fv(s->sv + s->se[e * 2] * 3), q = fv(s->sv + s->se[e * 2 + 1] * 3);
    ++s->prim_tests;
    if (s->surface) {
        visit_surface(s, p, q);
        return 0;
    }
    double d;
    if (!s->quad) d = sqrt(seg_seg2(p, q, s->a, s->b));
    else d = seg_quad_dist(p, q, s->B0, s->B1, s->B2, s->r - s->eps, s->r + s->eps);
    classify(s, d);
    return 0;
}

typedef struct {
    const orc_robot* R;
    const orc_scene* S;
    const float* q;
    const u32* traj_off;
    int quad, endpoints, surface;
    double eps;
    bvh_t scene_edge;
    unsigned char *traj_hit, *traj_band, *seg_hit, *seg_band, *traj_marg;
    u32* traj_count;
    const u32* seg_off;  /* per-trajectory offsets into seg_hit / seg_band */
    orc_work* work;
} sweep_ctx;

/* W = pinv(B) = (B^T B)^{-1} B^T for the nt x nc uniform quadratic B-spline basis */
static int fit_weights(int nc, int nt, double* W /* nc*nt */) {
    double* B = (double*) calloc((size_t) nt * nc, sizeof(double));
    for (int t = 0; t < nt; ++t) {
        double x = nt > 1 ? 2.0 + (double) (nc - 2) * t / (nt - 1) : 2.0;
        int seg = (int) floor(x) - 2;
        if (seg > nc - 3) seg = nc - 3;
        if (seg < 0) seg = 0;
        double s = x - (seg + 2);
        B[t * nc + seg] += 0.5 * (1 - s) * (1 - s);
        B[t * nc + seg + 1] += 0.5 + s - s * s;
        B[t * nc + seg + 2] += 0.5 * s * s;
    }
    /* G = B^T B (nc x nc), Cholesky, solve G W = B^T */
    double* G = (double*) calloc((size_t) nc * nc, sizeof(double));
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) {
            double acc = 0;
            for (int t = 0; t < nt; ++t) acc += B[t * nc + i] * B[t * nc + j];
            G[i * nc + j] = acc;
        }
    for (int j = 0; j < nc; ++j) {
        double d = G[j * nc + j];
        for (int k = 0; k < j; ++k) d -= G[j * nc + k] * G[j * nc + k];
        if (d <= 0) { free(B); free(G); return -1; }
        d = sqrt(d);
        G[j * nc + j] = d;
        for (int i = j + 1; i < nc; ++i) {
            double v = G[i * nc + j];
            for (int k = 0; k < j; ++k) v -= G[i * nc + k] * G[j * nc + k];
            G[i * nc + j] = v / d;
        }
    }
    double* y = (double*) malloc(sizeof(double) * (size_t) nc);  /* any number of control points */
    for (int t = 0; t < nt; ++t) {
        for (int i = 0; i < nc; ++i) {  /* L y = b */
            double v = B[t * nc + i];
            for (int k = 0; k < i; ++k) v -= G[i * nc + k] * y[k];
            y[i] = v / G[i * nc + i];
        }
        for (int i = nc - 1; i >= 0; --i) {  /* L^T x = y */
            double v = y[i];
            for (int k = i + 1; k < nc; ++k) v -= G[k * nc + i] * y[k];
            y[i] = v / G[i * nc + i];
        }
        for (int i = 0; i < nc; ++i) W[i * nt + t] = y[i];
    }
    free(y);
    free(B);
    free(G);
    return 0;
}

int orc_fit_weights(int nc, int nt, double* W) { return (nc < 3 || nc > 256 || nt < nc) ? -1 : fit_weights(nc, nt, W); }

int orc_quad_ctrl_count(int n_wp) { int c = (n_wp + 1) / 2; return c < 3 ? 3 : c; }

static void sweep_traj(void* vctx, int tr, void* scratch) {
    (void) scratch;
    sweep_ctx* C = (sweep_ctx*) vctx;
    const orc_robot* R = C->R;
    int nwp = (int) (C->traj_off[tr + 1] - C->traj_off[tr]);
    int ns = R->n_spheres;
    int nl = R->dof + 1;
    double* T = (double*) malloc(sizeof(double) * (size_t) nl * 12);
    d3* cen = (d3*) malloc(sizeof(d3) * (size_t) nwp * ns);   /* [wp][sphere] */
    for (int w = 0; w < nwp; ++w) {
        orc_fk_pose(R->dof, R->cos_mask, R->sin_mask, R->one_mask, R->base_tf, C->q + (size_t) (C->traj_off[tr] + w) * R->dof, T);
        for (int s = 0; s < ns; ++s) cen[w * ns + s] = xform(T + R->sphere_links[s] * 12, fv(R->sphere_centers + s * 3));
    }
    int trob = 0, trmarg = 0, trhit = 0;
    u32 trcount = 0;
    uint64_t ntests = 0, ptests = 0;
    unsigned char* seg_hit = C->seg_hit ? C->seg_hit + C->seg_off[tr] : NULL;
    unsigned char* seg_band = C->seg_band ? C->seg_band + C->seg_off[tr] : NULL;
    if (!C->quad) {
        for (int g = 0; g + 1 < nwp; ++g) {
            int srob = 0, smarg = 0, shit = 0;
            for (int s = 0; s < ns; ++s) {
                sweep_query Q;
                memset(&Q, 0, sizeof(Q));
                Q.a = cen[g * ns + s]; Q.b = cen[(g + 1) * ns + s]; Q.r = R->sphere_radii[s]; Q.eps = C->eps;
                Q.surface = C->surface;
                Q.sv = C->S->verts; Q.se = C->S->edges;
                double pad = Q.r + C->eps;
                double qlo[3] = {fmin(Q.a.x, Q.b.x) - pad, fmin(Q.a.y, Q.b.y) - pad, fmin(Q.a.z, Q.b.z) - pad};
                double qhi[3] = {fmax(Q.a.x, Q.b.x) + pad, fmax(Q.a.y, Q.b.y) + pad, fmax(Q.a.z, Q.b.z) + pad};
                ntests += bvh_query(&C->scene_edge, qlo, qhi, visit_edge, &Q);
                ptests += Q.prim_tests;
                shit |= Q.any_hit; srob |= Q.robust; smarg |= Q.marginal;
                trcount += Q.hits;
            }
            if (seg_hit) seg_hit[g] = (unsigned char) shit;
            if (seg_band) seg_band[g] = (unsigned char) (!srob && smarg);
            trhit |= shit; trob |= srob; trmarg |= smarg;
        }
    } else {
        int nc = orc_quad_ctrl_count(nwp);
        double* W = (double*) malloc(sizeof(double) * (size_t) nc * nwp);
        d3* ctrl = (d3*) malloc(sizeof(d3) * (size_t) nc * ns);
        if (nwp < 3 || fit_weights(nc, nwp, W)) {
            /* too short to fit: flag as hit-and-band so it cannot pass silently */
            C->traj_hit[tr] = 1;
            if (C->traj_band) C->traj_band[tr] = 1;
            free(W); free(ctrl); free(T); free(cen);
            return;
        }
        for (int k = 0; k < nc; ++k)
            for (int s = 0; s < ns; ++s) {
                d3 acc = v3(0, 0, 0);
                for (int w = 0; w < nwp; ++w) acc = add(acc, mul(cen[w * ns + s], W[k * nwp + w]));
                ctrl[k * ns + s] = acc;
            }
        int npieces = nc - 2 + (C->endpoints && !C->surface ? 2 : 0);
        for (int g = 0; g < npieces; ++g) {
            int srob = 0, smarg = 0, shit = 0;
            for (int s = 0; s < ns; ++s) {
                sweep_query Q;
                memset(&Q, 0, sizeof(Q));
                Q.quad = 1; Q.r = R->sphere_radii[s]; Q.eps = C->eps; Q.sv = C->S->verts; Q.se = C->S->edges;
                Q.surface = C->surface;
                if (g < nc - 2) {
                    d3 P0 = ctrl[g * ns + s], P1 = ctrl[(g + 1) * ns + s], P2 = ctrl[(g + 2) * ns + s];
                    Q.B0 = mul(add(P0, P1), 0.5); Q.B1 = P1; Q.B2 = mul(add(P1, P2), 0.5);
                    if (Q.surface) quad_caps(Q.B0, Q.B1, Q.B2, &Q.n0, &Q.n1);
                } else {
                    d3 c = cen[(g == nc - 2 ? 0 : nwp - 1) * ns + s];
                    Q.B0 = c; Q.B1 = c; Q.B2 = c;
                }
                double pad = Q.r + C->eps;
                double qlo[3] = {fmin(Q.B0.x, fmin(Q.B1.x, Q.B2.x)) - pad, fmin(Q.B0.y, fmin(Q.B1.y, Q.B2.y)) - pad,
                                 fmin(Q.B0.z, fmin(Q.B1.z, Q.B2.z)) - pad};
                double qhi[3] = {fmax(Q.B0.x, fmax(Q.B1.x, Q.B2.x)) + pad, fmax(Q.B0.y, fmax(Q.B1.y, Q.B2.y)) + pad,
                                 fmax(Q.B0.z, fmax(Q.B1.z, Q.B2.z)) + pad};
                ntests += bvh_query(&C->scene_edge, qlo, qhi, visit_edge, &Q);
                ptests += Q.prim_tests;
                shit |= Q.any_hit; srob |= Q.robust; smarg |= Q.marginal;
                trcount += Q.hits;
            }
            if (seg_hit) seg_hit[g] = (unsigned char) shit;
            if (seg_band) seg_band[g] = (unsigned char) (!srob && smarg);
            trhit |= shit; trob |= srob; trmarg |= smarg;
        }
        free(W);
        free(ctrl);
    }
    C->traj_hit[tr] = (unsigned char) trhit;
    if (C->traj_band) C->traj_band[tr] = (unsigned char) (!trob && trmarg);
    if (C->traj_marg) C->traj_marg[tr] = (unsigned char) trmarg;
    if (C->traj_count) C->traj_count[tr] = trcount;
    if (C->work) { C->work[tr].node_tests = ntests; C->work[tr].prim_tests = ptests; }
    free(T);
    free(cen);
}

/* quad = 0: piecewise-linear capsules, seg_off[t] = sum of (nwp - 1);
 * quad = 1: quadratic pieces, seg_off[t] = sum of (nc - 2 + 2 * endpoints).
 * surface = 0: solid semantics (an edge within r of the sphere path), S's
 * edges the unique edges; surface = 1: the reference's entering-ray
 * semantics (visit_surface), S's edges the directed loop edges, no end
 * spheres. */
int orc_sweep(int quad, int endpoints, int surface, const orc_robot* R, const orc_scene* S, const float* q, const u32* traj_off,
              int n_traj, double eps, int threads, unsigned char* traj_hit, unsigned char* traj_band,
              unsigned char* traj_marg, u32* traj_count, const u32* seg_off, unsigned char* seg_hit,
              unsigned char* seg_band, orc_work* work) {
    sweep_ctx C;
    memset(&C, 0, sizeof(C));
    C.R = R; C.S = S; C.q = q; C.traj_off = traj_off; C.quad = quad; C.endpoints = endpoints; C.eps = eps;
    C.surface = surface;
    C.traj_hit = traj_hit; C.traj_band = traj_band; C.seg_hit = seg_hit; C.seg_band = seg_band; C.seg_off = seg_off;
    C.traj_marg = traj_marg; C.traj_count = traj_count;
    C.work = work;
    float *lo, *hi;
    edge_boxes(S->verts, S->edges, S->n_edges, &lo, &hi);
    bvh_make(&C.scene_edge, S->n_edges, lo, hi);
    run_pool(n_traj, threads, sweep_traj, &C, 0);
    bvh_free(&C.scene_edge);
    return 0;
}

/* ---------------------------------------------------------- small exports */
int orc_seg_tri(const double* p, const double* q, const double* a, const double* b, const double* c, double* m) {
    return seg_tri(v3(p[0], p[1], p[2]), v3(q[0], q[1], q[2]), v3(a[0], a[1], a[2]), v3(b[0], b[1], b[2]),
                   v3(c[0], c[1], c[2]), m);
}
double orc_seg_seg(const double* p1, const double* q1, const double* p2, const double* q2) {
    return sqrt(seg_seg2(v3(p1[0], p1[1], p1[2]), v3(q1[0], q1[1], q1[2]), v3(p2[0], p2[1], p2[2]), v3(q2[0], q2[1], q2[2])));
}
/* one (directed edge p -> q, primitive) pair under the surface semantics:
 * quad = 0: capsule b0-b1; quad = 1: flat-capped piece (b0, b1, b2).
 * *hit = the upstream decision, *band = 1 when it lies in the eps band. */
void orc_surface_pair(int quad, const double* p, const double* q, const double* b0, const double* b1,
                      const double* b2, double r, double eps, int* hit, int* band) {
    sweep_query Q;
    memset(&Q, 0, sizeof(Q));
    Q.quad = quad; Q.surface = 1; Q.r = r; Q.eps = eps;
    if (!quad) {
        Q.a = v3(b0[0], b0[1], b0[2]); Q.b = v3(b1[0], b1[1], b1[2]);
    } else {
        Q.B0 = v3(b0[0], b0[1], b0[2]); Q.B1 = v3(b1[0], b1[1], b1[2]); Q.B2 = v3(b2[0], b2[1], b2[2]);
        quad_caps(Q.B0, Q.B1, Q.B2, &Q.n0, &Q.n1);
    }
    visit_surface(&Q, v3(p[0], p[1], p[2]), v3(q[0], q[1], q[2]));
    *hit = Q.any_hit;
    *band = !Q.robust && Q.marginal;
}

double orc_seg_quad(const double* p, const double* q, const double* b0, const double* b1, const double* b2) {
    return seg_quad_dist(v3(p[0], p[1], p[2]), v3(q[0], q[1], q[2]), v3(b0[0], b0[1], b0[2]), v3(b1[0], b1[1], b1[2]),
                         v3(b2[0], b2[1], b2[2]), -INFINITY, INFINITY);
}
