// kernels.h - device-side views and launchers of the query kernels.
#pragma once
#include "engine.h"

namespace rtcd {

// Robot resident on the device (passed by value to the kernels).
struct RobotDev {
    Chain chain;
    uint32_t n_links;
    uint32_t first_link;            // 1 when the base link is skipped
    float obb[kMaxLinks][16];       // local OBB: centre(3), half(3), axes x/y/z (9), pad
    const float4* tri_nodes;        // link triangle LBVHs (link frames)
    const float4* tri_prims;        // 3 float4 per triangle
    uint32_t tri_root[kMaxLinks];
    const float4* edge_nodes;       // link edge LBVHs (link frames)
    const float4* edge_prims;       // 2 float4 per edge; w of the first = global edge id
    uint32_t edge_root[kMaxLinks];
    uint32_t n_edges_total;
    float4 link_point[kMaxLinks];   // one vertex of each link mesh (link frame)
    const float4* spheres;          // local centre xyz, radius w
    const uint32_t* sphere_link;
    uint32_t n_spheres;
};

// Scene resident on the device.
struct SceneDev {
    const float4* tri_nodes;
    const float4* tri_prims;
    uint32_t tri_root;
    uint32_t n_tris;
    const float4* edge_nodes;
    const float4* edge_prims;
    uint32_t edge_root;
    uint32_t n_edges;
    const float* obbs;  // 16 floats per obstacle: centre(3), half(3), axes(9), bounding radius
    const float4* obs_box;    // [obstacle][2]: exact box of its vertices (lo, hi)
    const float4* obs_point;  // [obstacle]: one of its vertices
    uint32_t n_obs;           // scene triangles carry their obstacle in the third float4's w
    const float4* tri_wide;   // 4-wide copies of the two trees (8 float4 per node), same leaf references
    uint32_t tri_wide_root;   // 0, or the binary root when that is kNone or a leaf
    const float4* edge_wide;
    uint32_t edge_wide_root;
    uint32_t wide_front;      // frontier entries a warp needs over either wide tree
    const float4* tri_cut;    // top cuts of the wide trees: child records (2 float4 each)
    const float4* edge_cut;
    uint32_t n_tri_cut, n_edge_cut;
    uint32_t edge_wide_lane;  // nonzero when a lane stack of kStack entries holds a wide edge-tree descent
    uint32_t n_tri_wide, n_edge_wide;  // nodes of the two wide trees
};

struct DiscreteArgs {
    const float4* T;           // [pose][link][3] link transforms
    const uint32_t* items;     // compacted (pose * n_links + link); NULL = all links >= first_link
    uint32_t link_major;       // items hold (link order slot) * n_poses + pose instead (see item_word)
    const uint32_t* n_items;   // device count of items
    uint32_t n_poses;
    uint32_t* pose_hit;        // [pose] nonzero when colliding
    uint32_t* counts;          // [pose] upstream counts (ObsToRobot) or NULL
    uint32_t* edge_bits;       // [pose][edge_words] RobotToObs hit-edge bitset or NULL
    uint32_t edge_words;
    uint32_t* work_counter;    // zeroed before launch
    uint32_t* err;
    unsigned long long* stats; // [0] fp64 re-tests
    int want_counts;
};

constexpr int kFkThreads = 128;
constexpr int kTravThreads = 128;

// Wavefront form of the discrete traversal: stage A (one warp per item)
// emits (item position, scene primitive) candidates, stage B (one lane per
// candidate) runs the link-side descent.  Items whose candidates do not fit
// the buffer are flagged and re-run by the fused kernel.
struct WaveArgs {
    DiscreteArgs d;
    uint32_t top_nodes;        // fused form: wide-tree nodes (from the root) each block stages in shared memory
    uint2* cand;               // (item word pose * n_links + link, scene primitive)
    uint32_t* cand_count;      // zeroed before stage A; may exceed cand_cap
    uint32_t cand_cap;
    uint8_t* item_overflow;    // [item word] set when its candidates overflowed; zeroed before stage A
    uint32_t* overflow_items;  // compacted overflowed items (item words, for the fused kernel)
    uint32_t* overflow_count;  // zeroed before stage A
    uint32_t chunk;            // stage B: consecutive candidates (lanes) or 32-candidate groups (packets) per worker
    uint32_t item_steps;       // fused forms: stage-B steps an item runs in its warp before deferring the rest
    uint32_t light_steps;      // stage B visits before a candidate moves to the heavy pass; 0 = no heavy pass
    uint2* heavy;              // [heavy_cap] candidates (item word, primitive) handed to the heavy pass
    uint32_t heavy_cap;
    uint32_t* heavy_count;     // appended (may exceed heavy_cap: those stayed in the light pass); zeroed
    uint32_t* heavy_work;      // heavy-pass work counter; zeroed
    uint2* sub;                // [2][sub_cap] (item word, wide node): crowded items' frontiers, then the split pieces
    uint32_t sub_cap;
    uint32_t* sub_count;       // [4] zeroed: frontier nodes appended, their work counter, pieces appended, their work
                               // counter (appends may exceed sub_cap: those items went to the fallback)
};

constexpr int kStageAWarps = 4;
constexpr int kFrontier = 32 * (kStack + 2);  // bound of a 32-wide LIFO frontier over a tree of depth <= kStack - 2

void launch_stage_a(bool robot_to_obs, const RobotDev& R, const SceneDev& S, const WaveArgs& W, uint32_t blocks,
                    cudaStream_t s);
// Stage B's light pass (32-candidate packets, or one lane per candidate) on
// `blocks` x `threads`, then (when W.light_steps) its heavy pass on
// heavy_share percent of the full persistent grid.
void launch_stage_b(bool robot_to_obs, const RobotDev& R, const SceneDev& S, const WaveArgs& W, uint32_t blocks,
                    uint32_t threads, uint32_t heavy_share, bool packets, cudaStream_t s);
// The heavy pass alone (after a light pass that spilled into W.heavy).
void launch_stage_b_heavy(bool robot_to_obs, const RobotDev& R, const SceneDev& S, const WaveArgs& W,
                          uint32_t heavy_share, cudaStream_t s);
// Stages A and B fused in one warp per item (stage_b_form 3; 4 with packet
// descents of the link tree); spilled candidates go to W.cand / W.heavy.
void launch_stage_ab(bool robot_to_obs, bool packets, const RobotDev& R, const SceneDev& S, const WaveArgs& W,
                     uint32_t blocks, cudaStream_t s);
uint32_t stage_ab_blocks(bool robot_to_obs, bool packets, const SceneDev& S);
// The subtree pass over the frontiers crowded items handed over (after the
// fused kernel, before the one-lane pass over the candidates), on share
// percent of its full persistent grid.
void launch_subtree(bool robot_to_obs, const RobotDev& R, const SceneDev& S, const WaveArgs& W, uint32_t share,
                    cudaStream_t s);
uint32_t stage_a_blocks(bool robot_to_obs);
uint32_t stage_b_blocks(bool robot_to_obs);
uint32_t stage_b_max_blocks_per_sm(bool robot_to_obs, uint32_t threads);  // threads: 64, 128 or 256

void launch_fk_poses(const Chain& ch, const float* d_q, uint32_t n, float4* d_T, cudaStream_t s);
// link_major: the mask (and so the compacted items) in link order, every pose's
// last link before any pose's next-to-last one (item_word decodes it).
void launch_cull(const RobotDev& R, const SceneDev& S, const float4* d_T, uint32_t n, uint8_t* d_mask, bool link_major,
                 unsigned long long* d_stats, cudaStream_t s);
void launch_all_items(const RobotDev& R, uint32_t n, uint32_t* d_items, uint32_t* d_count, cudaStream_t s);
void launch_discrete(bool robot_to_obs, const RobotDev& R, const SceneDev& S, const DiscreteArgs& A, uint32_t blocks,
                     cudaStream_t s);
void launch_popcount_rows(const uint32_t* d_bits, uint32_t words, uint32_t rows, uint32_t* d_out, cudaStream_t s);
// flags[i] = (hit[i] != 0) | 2 * (contain[i] != 0); contain may be NULL.
void launch_flags(const uint32_t* d_hit, uint32_t n, uint8_t* d_flags, cudaStream_t s,
                  const uint32_t* d_contain = nullptr);
// Containment of the items' poses not yet hit (sets contain[pose] = 1).
void launch_contain(const RobotDev& R, const SceneDev& S, const DiscreteArgs& A, uint32_t* d_contain, cudaStream_t s);
uint32_t discrete_persistent_blocks(bool robot_to_obs);

// ---- sweeps
// A sweep unit handed to the heavy pass: its geometry (linear: capsule axis
// P0-P1; quadratic: Bezier piece P0 P1 P2, or an end sphere), radius, owner.
struct SweepRec {
    float4 P0, P1, P2;
    float r;
    uint32_t traj, piece_g, pad;
};

struct SweepArgs {
    const float4* centers;     // [waypoint][sphere] world centre xyz, radius w
    const float4* ctrl;        // [control point][sphere] (quadratic) or NULL
    const uint32_t* traj_piece_off;  // [n_traj + 1] prefix of pieces
    const uint32_t* traj_wp_off;     // [n_traj + 1] waypoint offsets
    const uint32_t* traj_ctrl_off;   // [n_traj + 1] control point offsets (quadratic)
    const uint32_t* piece_traj;      // [pieces] owning trajectory of each piece
    uint32_t n_traj;
    uint32_t n_spheres;
    uint32_t total_units;      // pieces * spheres
    int quad;
    int endpoints;
    int surface;               // entering-ray semantics over the loop edges (leaf_hit_surface)
    uint32_t* traj_hit;        // [n_traj]
    uint32_t* piece_hit;       // [pieces] or NULL
    uint32_t* counts;          // [n_traj] or NULL
    uint32_t* work_counter;
    uint32_t* err;
    unsigned long long* stats;
    int want_counts;
    int want_pieces;
    uint32_t light_steps;      // visits before a unit moves to the heavy pass; 0 = no heavy pass
    uint32_t descend_cap;      // light pass: visits a lane makes per descent before the warp's lanes
                               // without work take new units (its descent resumes after); 0 = until a leaf
    int binary_tree;           // light pass on the binary edge tree (else the 4-wide one where the scene allows)
    SweepRec* heavy;           // [heavy_cap] units handed to the heavy pass
    uint32_t heavy_cap;
    uint32_t* heavy_count;     // units appended (may exceed heavy_cap: those stayed in the light pass)
    uint32_t* heavy_work;      // heavy-pass work counter
    uint32_t heavy_steps;      // frontier steps a heavy unit takes before its open frontier goes to the split
                               // pass (0: never)
    int heavy_wide;            // heavy and split passes on the 4-wide edge tree (else the binary one)
    uint2* split;              // [split_cap] (heavy record, edge-tree node) pairs for the split pass
    uint32_t split_cap;
    uint32_t* split_count;     // pairs appended (past split_cap: the unit was finished by its warp)
    uint32_t* split_work;      // split-pass work counter
    // the staged light pass (k_sweep_traj): a block takes `group` consecutive trajectories at a time
    // from work_counter, runs their FK (and quadratic fit) into shared memory and their units from there
    const float* q;            // [waypoint][dof] joint values
    const float* W;            // quadratic fit tables, W_off[n] = the table of n waypoints
    const uint32_t* W_off;
    uint32_t max_wp, max_nc, max_pieces;  // largest trajectory of the batch (shared-memory sizing)
    uint32_t group;            // staged: trajectories per claim, 0 = chosen at launch (1..kSweepMaxGroup)
};
constexpr uint32_t kSweepMaxGroup = 8;

void launch_fk_spheres(const RobotDev& R, const float* d_q, uint32_t n_wp, float4* d_centers, cudaStream_t s);
void launch_fit(const float4* d_centers, const uint32_t* d_wp_off, const uint32_t* d_ctrl_off, const float* d_W,
                const uint32_t* d_W_off, uint32_t n_traj, uint32_t n_spheres, float4* d_ctrl, cudaStream_t s);
// The light pass on `blocks` blocks of `threads`, then (when A.light_steps)
// the heavy pass on heavy_share percent of its full persistent grid.
// ev_light (optional) is recorded between the two passes.  The heavy pass
// counts into the second stats bank (A.stats + kStatBank).  staged: the
// light pass stages each trajectory's FK (and fit) in shared memory
// (k_sweep_traj) instead of reading A.centers / A.ctrl.
void launch_sweep(const SceneDev& S, const RobotDev& R, const SweepArgs& A, uint32_t blocks, uint32_t threads,
                  uint32_t heavy_share, bool staged, cudaStream_t s, cudaEvent_t ev_light = nullptr);
// Shared memory of the staged light pass for a batch; 0 when it does not fit (the caller then
// computes the centres and control points in global memory and runs the unstaged light pass).
size_t sweep_staged_smem(bool quad, uint32_t n_links, uint32_t max_wp, uint32_t max_nc, uint32_t max_pieces);
uint32_t sweep_persistent_blocks(bool quad);
uint32_t sweep_max_blocks_per_sm(bool quad, uint32_t threads);  // threads: 64, 128 or 256

// diagnostics of the exact tests (discrete.cu, sweep.cu)
void launch_probe_segtri(const float* d_seg, const float* d_tri, uint32_t n, float* d_cls, double* d_dec,
                         cudaStream_t s);
void launch_probe_sweep(bool quad, const float* d_seg, const float* d_piece, uint32_t n, float* d32, double* d64,
                        cudaStream_t s);

// planner side (planner.cu)
constexpr uint32_t kKnnMaxK = 32;
constexpr uint32_t kKnnMaxDim = 16;
void launch_knn(const float* pts, uint32_t n, uint32_t dim, const float* w2_dev, uint32_t k, const uint8_t* mask,
                uint32_t* idx, float* dist, cudaStream_t s);
void launch_interp_edges(const float* nodes, uint32_t n_nodes, uint32_t dof, const uint32_t* edges, uint32_t n_edges,
                         uint32_t n_wp, float* q, uint32_t* err, cudaStream_t s);
void launch_or_rows(const uint8_t* pose_flags, uint32_t n_edges, uint32_t n_wp, uint8_t* flags, cudaStream_t s);

}  // namespace rtcd
