/*
 * rtcd.h - C ABI of the B200 batched collision-query engine.
 *
 * The upstream RTCollisionDetection exposes a header-only C++ template API
 * (RTCD::CollisionDetector<NSTREAM, LinkType>, RTCD/CollisionDetector/
 * CollisionDetector.h:18-157) driven as
 *     construct -> setupScene -> setupOptix -> setupRobot -> buildSBT ->
 *     per query: robot->prepareUpdateData(poses, n); setNCheck(n); check();
 *                downloadResult(result)
 * (RTCD/Demo/DemoCollisionDetectorDisc.cpp:56-76).  This ABI carries the same
 * objects - a robot, a resident scene, a detector of one of the four kinds -
 * as opaque handles with plain pointers and sizes, so any language with a C
 * FFI can bind it.  include/rtcd/CollisionDetector.hpp re-creates the upstream
 * method names on top of it.
 *
 * Conventions
 *  - Every call returns an rtcd_status; no exception crosses the ABI.
 *    rtcd_last_error() returns the calling thread's last message.
 *  - Outputs are caller-owned.  Handles own all device memory they allocate.
 *  - A handle may be used from several threads; calls on one detector are
 *    serialised by the detector.
 *  - Units: metres, radians.  Transforms are 3x4 row-major [R | t].
 */
#ifndef RTCD_H
#define RTCD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RTCD_ABI_VERSION 1

#if defined(__GNUC__)
#define RTCD_API __attribute__((visibility("default")))
#else
#define RTCD_API
#endif

typedef enum {
    RTCD_OK = 0,
    RTCD_ERR_INVALID_ARGUMENT = 1,
    RTCD_ERR_CUDA = 2,
    RTCD_ERR_OUT_OF_MEMORY = 3,
    RTCD_ERR_DEVICE_TIMEOUT = 4, /* a bounded device-side wait ran out */
    RTCD_ERR_CAPACITY = 5,       /* a structure exceeded a compiled limit */
    RTCD_ERR_INTERNAL = 6
} rtcd_status;

/* The four detectors (upstream LinkType, RTCD/Meshes/meshTypes.h:37-48). */
typedef enum {
    RTCD_OBS_TO_ROBOT = 0, /* LinkType::MESH: obstacle edges vs link triangles */
    RTCD_ROBOT_TO_OBS = 1, /* LinkType::RAY_ONLINE: link edges vs scene triangles */
    RTCD_LINEAR_SWEEP = 2, /* LinkType::LINEAR_CURVE: obstacle edges vs swept capsules */
    RTCD_QUAD_SWEEP = 3    /* LinkType::QUADRATIC_CURVE: obstacle edges vs quadratic B-spline sweeps */
} rtcd_detector_kind;

/* rtcd_check flags */
#define RTCD_CHECK_COUNTS (1u << 0)        /* also produce the upstream hit counts (no early exit) */
#define RTCD_CHECK_HOST_BUFFERS (1u << 1)  /* q, traj offsets and outputs are host memory; a q in page-locked
                                              memory (cudaHostAlloc, cudaHostRegister) is uploaded by DMA
                                              directly, pageable memory is copied into the detector's pinned
                                              staging first */
#define RTCD_CHECK_NO_CULL (1u << 2)       /* skip the OBB prefilter of the discrete detectors (every item goes to
                                              the traversal, whose first step rejects the far ones: up to 9 % faster at
                                              a few thousand poses, slower at tens of thousands) */
#define RTCD_CHECK_PLAIN (1u << 3)         /* discrete: the upstream check() shape - frames of frame_size poses over
                                              plain_streams streams, one host thread per stream, a host round trip
                                              per frame (the culled item count) and a wait after every group of
                                              plain_streams frames; synchronous */
#define RTCD_CHECK_NO_ENDPOINTS (1u << 4)  /* quadratic: do not add the start/end waypoint spheres */
#define RTCD_CHECK_TIMING (1u << 5)        /* record device events around the stages (rtcd_last_stats) */
#define RTCD_CHECK_FUSED (1u << 6)         /* discrete: one fused traversal kernel instead of the two-stage wavefront */
#define RTCD_CHECK_CONTAINMENT (1u << 8)   /* discrete: also flag poses with no surface crossing where a link lies
                                              inside an obstacle or an obstacle inside a link (ray parity);
                                              such poses get flag value 2, surface crossings 1 */
#define RTCD_CHECK_TWO_WAY (1u << 9)       /* discrete: run both directions (ObsToRobot and RobotToObs) in one check
                                              over the same FK, cull and items: flags are the union, counts the
                                              sum of the two upstream counts */
#define RTCD_CHECK_SURFACE (1u << 10)       /* sweeps: the reference's semantics instead of the solid ones.  The scene's
                                              directed loop edges (RTCD/Meshes/mesh.h:378-620) are cast, and an edge
                                              hits a swept piece only when it starts outside the piece and reaches it
                                              (the curve intersectors report entering rays only, CCCuda.cu:37-41);
                                              linear pieces are round-capped capsules, quadratic pieces are cut by
                                              flat caps normal to their end tangents and carry no start/end spheres.
                                              The first such check on a scene builds its loop-edge tree (once,
                                              synchronously): make it before any stream capture */
#define RTCD_CHECK_GRAPH (1u << 7)         /* replay the launch sequence as a CUDA graph (captured on the first call
                                              with these pointers, sizes, flags and - for sweeps - trajectory
                                              offsets; any other call on the detector retires it).  With
                                              RTCD_CHECK_HOST_BUFFERS the graph holds the upload from the
                                              detector's pinned staging (from a page-locked q itself, whose
                                              address then joins the replay key), the kernels and the download
                                              back to the staging;
                                              only the copies between the caller's arrays and the staging run
                                              outside it, and the call returns with the results in place */

typedef struct rtcd_ctx rtcd_ctx;
typedef struct rtcd_robot rtcd_robot;
typedef struct rtcd_scene rtcd_scene;
typedef struct rtcd_detector rtcd_detector;

/* Serial-chain robot (upstream robotConfig + robot<DOF>, RTCD/Robot/robotConfig.h:14-38,
 * RTCD/Robot/robot.h:91-124).  Link i (0 = fixed base) has transform
 * T_0 = base_tf, T_{i+1} = T_i * (cos q_i C_i + sin q_i S_i + O_i). */
typedef struct {
    uint32_t dof;                      /* joints; the robot has dof + 1 links */
    const float* base_tf;              /* 12 */
    const float* cos_mask;             /* dof * 12 */
    const float* sin_mask;             /* dof * 12 */
    const float* one_mask;             /* dof * 12 */
    const float* link_verts;           /* link-local xyz */
    const uint32_t* link_vert_offsets; /* dof + 2 */
    const uint32_t* link_tris;         /* per-link vertex indices */
    const uint32_t* link_tri_offsets;  /* dof + 2 */
    const uint32_t* link_edges;        /* optional; NULL: unique edges are extracted */
    const uint32_t* link_edge_offsets; /* dof + 2 when link_edges is given */
    const float* link_obbs;            /* optional 15 floats per link (centre, half sizes, x/y/z axes); NULL: PCA fit */
    uint32_t n_spheres;                /* sphere model used by the sweep detectors */
    const float* sphere_centers;       /* link-local xyz */
    const float* sphere_radii;
    const uint32_t* sphere_links;
    int32_t skip_base;                 /* nonzero: link 0 is never checked (upstream SKIP_BASE) */
} rtcd_robot_desc;

typedef struct {
    uint32_t frame_size;             /* poses per frame of the plain path; 0 = 1024 (the upstream benchmark's
                                        batchSize, RTCD/Benchmark/Discrete/benchmarkUtils.h:16) */
    uint32_t traverse_threads;       /* threads per block of the traversal kernel: 64, 128 or 256; 0 = 128 */
    uint32_t traverse_blocks_per_sm; /* resident traversal blocks per SM; 0 = as many as fit */
    int32_t stream_priority;         /* priority of the detector's own stream (CUDA convention: lower = higher) */
    uint32_t residency_percent;      /* share of each SM its persistent kernels may hold (room for other
                                        launches to run alongside); 0 = 100 */
    uint32_t light_steps;            /* node + leaf visits one lane spends on a unit of traversal work (a
                                        discrete (link item, scene primitive) candidate, a sweep (piece,
                                        sphere) unit) before a whole warp takes it over; 0 = 32 (16 for
                                        the sweeps), 0xFFFFFFFF = never */
    uint32_t stage_b_form;           /* discrete stage B: 1 = one lane per candidate, 2 = 32-candidate packets
                                        that share each link-BVH node load, 3 = stages A and B fused in one
                                        warp per item (an item stops generating candidates once its pose
                                        is hit), 4 = 3 with packet descents of the link tree; 0 = 3 (the
                                        autotuner tries all four).  Sweeps: 1 = the light pass's lanes descend
                                        the binary edge tree, any other value the 4-wide one (when the
                                        scene's is shallow enough for a lane stack; the autotuner tries
                                        both) */
    uint32_t stage_b_chunk;          /* discrete stage B: consecutive candidates one lane takes in order (lanes
                                        form) or 32-candidate groups one warp takes (packets), so a pose's
                                        candidates spread over few workers that stop at its first hit; for
                                        the fused forms, the stage-B steps (32 candidates each) an item runs
                                        in its warp before its further candidates go to a one-lane pass over
                                        the whole GPU; 0 = 64 lanes / 4 packets / 8 steps; at most 4096 */
    uint32_t plain_streams;          /* streams of the plain path, each driven by its own host thread; frames go to
                                        them round-robin and the call waits for every group of plain_streams
                                        frames (upstream NSTREAM = 4 and its thread pool,
                                        RTCD/CollisionDetector/CollisionDetector.h:396-433); 0 = 4, at most 16 */
    uint32_t top_nodes_shared;       /* discrete fused form: wide scene-tree nodes (breadth-first from the root: its
                                        top levels) each block copies to shared memory and its descents read
                                        there; 0 = none, at most 256 (the autotuner tries 0 and 85, the first
                                        four levels) */
    uint32_t sweep_unstaged;         /* sweeps: 0 = the light pass stages each trajectory's FK (and quadratic fit)
                                        in shared memory when the batch's longest trajectory fits and the batch
                                        has at least four trajectories per resident block; 1 = sphere centres
                                        and control points always go through global memory (separate FK and
                                        fit kernels) */
    uint32_t sweep_group;            /* sweeps, staged light pass: trajectories a block stages and works through
                                        together (one FK and fit phase and one hand-over barrier per group
                                        instead of per trajectory); 0 = about 1,024 (piece, sphere) units a
                                        group (short trajectories are grouped, long ones staged one at a
                                        time), within the block's share of the SM's shared memory and at
                                        least four groups per resident block (at most 8); 1 = one at a time */
    uint32_t sweep_heavy_steps;      /* sweeps: frontier steps (each expands up to 32 edge-tree nodes) a heavy-pass
                                        unit runs before the nodes still open on its frontier (once there are
                                        four or more) go, one per warp, to a split pass, so a few units with
                                        very large traversals do not hold the pass while the rest of the GPU
                                        idles; 0 = 32, 0xFFFFFFFF = never */
    uint32_t sweep_descend_cap;      /* sweeps, light pass: node visits a lane makes in one descent before the
                                        warp's lanes without work take new units (the descent then resumes
                                        where it stopped), so a lane that finished a short unit does not wait
                                        out a long one; 0 = 3, 0xFFFFFFFF = every descent runs to its next
                                        leaf (the autotuner tries 2, 3, 4 and 6) */
    uint32_t sweep_heavy_wide;       /* sweeps: 1 = the heavy and split passes expand the scene's 4-wide edge tree,
                                        four lanes per node (half the levels; faster where many units reach
                                        the heavy pass near dense geometry), 0 = the binary tree, one lane
                                        per node (fewer boxes tested: faster on thin geometry); the
                                        autotuner tries both */
} rtcd_config;

/* Replaces the OptiX context + streams of createContextStream
 * (RTCD/Utils/Test/cudaCtxUtils.h:63-74). */
RTCD_API rtcd_status rtcd_context_create(int device, rtcd_ctx** out);
RTCD_API rtcd_status rtcd_context_destroy(rtcd_ctx* ctx);

/* Robot input at run time.  The reference generates a header of joint masks
 * from a URDF offline (scripts/URDFParser/urdfParserUtils.py:527-605 ->
 * RTCD/Robot/models/panda.h) and loads link meshes with tinyobjloader
 * (RTCD/Meshes/mesh.h:311-360); these two calls do both inside the library.
 *
 * rtcd_urdf_chain_parse reads URDF text (len bytes) describing a serial chain
 * from its root link: every revolute (or continuous) joint adds a link and its
 * masks L(q) = cos q C + sin q S + O = origin * Rot(axis, q) (values within
 * 1e-5 of 0 or +-1 set to them, as the reference does); fixed joints fold
 * into the next joint's origin (links they attach are not separate links:
 * merge their meshes beforehand, as the reference's parser does); the base
 * transform is the identity.  Branching chains, prismatic joints and more
 * than RTCD_URDF_MAX_LINKS links are rejected. */
#define RTCD_URDF_MAX_LINKS 16
#define RTCD_URDF_NAME 128
typedef struct {
    uint32_t dof;
    uint32_t n_links;                                  /* dof + 1: the root, then each joint's child */
    float base_tf[12];
    float cos_mask[(RTCD_URDF_MAX_LINKS - 1) * 12];   /* dof * 12 used, as rtcd_robot_desc wants them */
    float sin_mask[(RTCD_URDF_MAX_LINKS - 1) * 12];
    float one_mask[(RTCD_URDF_MAX_LINKS - 1) * 12];
    float lower[RTCD_URDF_MAX_LINKS - 1];
    float upper[RTCD_URDF_MAX_LINKS - 1];
    char link_name[RTCD_URDF_MAX_LINKS][RTCD_URDF_NAME];
    char link_mesh[RTCD_URDF_MAX_LINKS][2 * RTCD_URDF_NAME]; /* the link's visual mesh file name, "" if none */
} rtcd_urdf_chain;
RTCD_API rtcd_status rtcd_urdf_chain_parse(const char* urdf, size_t len, rtcd_urdf_chain* out);

/* Loads an OBJ mesh: vertices deduplicated by exact float position (first
 * occurrence wins, faces in file order), polygons fan-triangulated, only
 * vertices that faces use.  Call with NULL outputs to learn the sizes. */
RTCD_API rtcd_status rtcd_obj_load(const char* path, float* verts_out, uint32_t max_verts, uint32_t* n_verts,
                                   uint32_t* tris_out, uint32_t max_tris, uint32_t* n_tris);

/* Directed loop edges of a triangle mesh (upstream meshModel::loadOBJ,
 * RTCD/Meshes/mesh.h:378-620): every triangle's edges, in the directions
 * kept, run around it as a loop; an edge two neighbouring triangles need in
 * opposite directions is kept in both.  The directions follow the upstream
 * breadth-first walk over the triangles in index order.  edges_out receives
 * (from, to) vertex pairs, at most max_edges of them; call with NULL to learn
 * the count.  Host only (no GPU). */
RTCD_API rtcd_status rtcd_loop_edges(const uint32_t* tris, uint32_t n_tris, uint32_t* edges_out, uint32_t max_edges,
                                     uint32_t* n_edges);

/* Replaces robot<DOF>(robotConfig) and the link GAS builds
 * (RTCD/Robot/robot.h:91-124, RTCD/Robot/batchIASRobot.h:310-365): uploads
 * the chain and builds one triangle and one edge LBVH per link. */
RTCD_API rtcd_status rtcd_robot_create(rtcd_ctx* ctx, const rtcd_robot_desc* desc, rtcd_robot** out);
RTCD_API rtcd_status rtcd_robot_destroy(rtcd_robot* robot);

/* Replaces scene::addObstacle / uploadToDevice / wrapScene
 * (RTCD/CollisionScenes/scene.h:60-147): obstacle i owns triangles
 * [obstacle_tri_offsets[i], obstacle_tri_offsets[i+1]).  Builds the resident
 * triangle and edge LBVHs, the unique obstacle edges and one PCA OBB per
 * obstacle (RTCD/CollisionScenes/obstacle.h:186-219). */
RTCD_API rtcd_status rtcd_scene_create(rtcd_ctx* ctx, const float* verts, uint32_t n_verts, const uint32_t* tris,
                              uint32_t n_tris, const uint32_t* obstacle_tri_offsets, uint32_t n_obstacles,
                              rtcd_scene** out);
RTCD_API rtcd_status rtcd_scene_destroy(rtcd_scene* scene);
RTCD_API rtcd_status rtcd_scene_info(const rtcd_scene* scene, uint32_t* n_tris, uint32_t* n_edges, uint32_t* n_obstacles);

/* Replaces CollisionDetector(ctx, streams, robot, scene) + setupScene +
 * setupRobot + buildSBT (RTCD/CollisionDetector/CollisionDetector.h:166-305,
 * :777-835).  config may be NULL. */
RTCD_API rtcd_status rtcd_detector_create(rtcd_ctx* ctx, rtcd_detector_kind kind, rtcd_robot* robot, rtcd_scene* scene,
                                 const rtcd_config* config, rtcd_detector** out);
RTCD_API rtcd_status rtcd_detector_destroy(rtcd_detector* det);

/*
 * Replaces prepareUpdateData + setNCheck + check + downloadResult
 * (RTCD/CollisionDetector/CCRobotWrapper.h:39-70,
 *  RTCD/CollisionDetector/CollisionDetector.h:354-471, :62).
 *
 * Discrete kinds: q is float[n][dof]; flags_out[i] = 1 when pose i collides.
 * Sweep kinds:    q is float[traj_offsets[n]][dof] waypoints; trajectory i
 *                 owns rows [traj_offsets[i], traj_offsets[i+1]);
 *                 flags_out[i] = 1 when trajectory i collides.  traj_offsets
 *                 is always host memory.  seg_flags_out (optional) receives
 *                 one flag per segment, laid out as rtcd_segment_offsets()
 *                 describes.
 * counts_out (optional, with RTCD_CHECK_COUNTS) receives the upstream hit
 * counts: ObsToRobot - intersecting (obstacle edge, link, link triangle)
 * triples; RobotToObs - link edges with at least one hit; sweeps -
 * intersecting (obstacle edge, sphere segment) pairs.
 *
 * Without RTCD_CHECK_HOST_BUFFERS, q and the outputs are device pointers and
 * the call is asynchronous on `stream` (a cudaStream_t; NULL = the
 * detector's stream).  With it, the call copies through pinned staging
 * buffers and returns after the results are in the host buffers.
 */
RTCD_API rtcd_status rtcd_check(rtcd_detector* det, const float* q, const uint32_t* traj_offsets, uint32_t n,
                       uint8_t* flags_out, uint8_t* seg_flags_out, uint32_t* counts_out, uint32_t flags,
                       void* stream);

/* Waits for the detector's work and reports device-side errors
 * (upstream final CUDA_SYNC_CHECK, CollisionDetector.h:470). */
RTCD_API rtcd_status rtcd_sync(rtcd_detector* det, void* stream);

/* Autotuner: runs the given device-resident batch (q_dev; traj_offsets on the
 * host for sweeps) with every traversal launch shape - 64, 128 and 256
 * threads per block, each at a quarter, half and all of the blocks per SM
 * that fit; then light-pass budgets (light_steps) of the default, 16, 32 and
 * 64 visits; then, for the discrete kinds, the four stage B forms at chunk
 * lengths from 1 to 256 candidates and the shared-memory top levels, for the
 * sweeps the binary and the 4-wide edge tree, staged or unstaged centres and
 * grouped or single trajectories; then the launch shapes again - rounds of
 * this coordinate descent until one changes nothing (at most three; sweeps
 * are timed with segment flags on)
 * - times each candidate's whole check replayed as a CUDA graph with device
 * events, after a write of twice the L2 size when free memory allows (median
 * of three replays after a warm-up run; the three fastest candidates are
 * timed again over nine), keeps the fastest configuration in the detector
 * and writes it to best_out and its time to best_ms (both optional).  The
 * call allocates its flag buffers and that flush buffer for its duration.
 * The upstream picks its batch size per experiment by hand
 * (CollisionDetector.h:365-394). */
RTCD_API rtcd_status rtcd_detector_autotune(rtcd_detector* det, const float* q_dev, const uint32_t* traj_offsets,
                                            uint32_t n, void* stream, rtcd_config* best_out, float* best_ms);

/* Segments per trajectory for the sweep kinds: linear n_wp - 1; quadratic
 * max(3, ceil(n_wp/2)) - 2 (+2 start/end spheres unless RTCD_CHECK_NO_ENDPOINTS
 * or RTCD_CHECK_SURFACE).
 * offsets_out (n + 1 entries, host) is the exclusive prefix sum. */
RTCD_API rtcd_status rtcd_segment_offsets(rtcd_detector_kind kind, const uint32_t* traj_offsets, uint32_t n, uint32_t flags,
                                 uint32_t* offsets_out);

/* Host-side least-squares quadratic B-spline fit: W_out (n_ctrl x n_wp,
 * row-major) = pinv(B), B[t][k] the uniform unclamped quadratic basis on knots
 * 0..n_ctrl+2 sampled at u = linspace(2, n_ctrl, n_wp).  Replaces loading the
 * shipped tables RTCD/data/weights/quad/normal/{nC}_{nT}.txt
 * (RTCD/Robot/batchCurveRobot.h:560-605); the quadratic detector fits with
 * n_ctrl = max(3, ceil(n_wp/2)).  Needs no GPU. */
RTCD_API rtcd_status rtcd_quad_fit_weights(uint32_t n_ctrl, uint32_t n_wp, float* W_out);

/* Statistics of the last completed check: items after the cull, etc. */
typedef struct {
    uint64_t work_items;   /* (pose, link) items or sweep units processed */
    uint64_t culled_items; /* items the OBB prefilter removed */
    uint64_t fp64_retests; /* candidates re-tested in FP64 */
    float ms_prepare;      /* with RTCD_CHECK_TIMING: FK / sphere centres / fit */
    float ms_cull;         /* OBB prefilter + compaction (discrete) */
    float ms_traverse;     /* the traversal kernel */
    float ms_total;        /* whole check on the device */
    uint64_t candidates;   /* discrete: (item, scene primitive) candidates of the scene stage;
                              quadratic sweep: pairs that needed the root finding */
    uint64_t exact_tests;  /* primitive-pair tests run in FP32 */
    uint64_t skipped;      /* candidates dropped because their pose (trajectory) was already decided */
    uint64_t node_tests;   /* BVH child-box tests of the traversal kernels */
    float ms_first_pass;   /* with RTCD_CHECK_TIMING: the first traversal kernel alone (discrete: the fused or
                              stage-A kernel of the first direction; sweeps: the light pass) */
    uint32_t path_flags;         /* bit 0: the sweep light pass staged its trajectories in shared memory */
    uint64_t first_node_tests;   /* node_tests of that first kernel (the rest: the passes after it) */
    uint64_t first_exact_tests;  /* exact_tests of that first kernel */
    uint64_t cull_sphere_tests;  /* discrete: bounding-sphere tests of the OBB cull */
    uint64_t cull_sat_tests;     /* discrete: 15-axis SATs the cull evaluated (after the sphere reject, up to each
                                    item's first overlap) */
    uint64_t deferred;           /* work the light pass handed to the heavy pass: sweep (piece, sphere) units,
                                    discrete (item, primitive) candidates */
} rtcd_stats;
RTCD_API rtcd_status rtcd_last_stats(rtcd_detector* det, rtcd_stats* out);

/* ---- serving: continuous batching over resident scenes ----
 *
 * The upstream detector serves one caller at a time: check() splits a query
 * into frames of BATCHSIZE over NSTREAM streams with a thread pool
 * (CollisionDetector.h:354-471, threadPool.h:10-92).  A server instead takes
 * requests of any size from any thread as they arrive, merges queued requests
 * for the same detector into one launch, runs up to `slots` launches
 * concurrently (one stream and one workspace each), and admits a launch only
 * while the bytes of the launches in flight stay within a memory budget.
 * Each request's result equals what rtcd_check returns for it alone. */
typedef struct rtcd_server rtcd_server;

typedef struct {
    uint32_t slots;              /* launches in flight at once; 0 = 4 */
    uint32_t max_batch_units;    /* poses / trajectory waypoints merged into one launch; 0 = 65536 */
    uint64_t memory_budget;      /* bytes the in-flight launches may hold; 0 = half the free device memory */
    uint32_t fast_slots;         /* slots reserved for small requests, on high-priority streams; 0 = 1 when slots > 1 */
    uint32_t fast_max_units;     /* a request is small up to this many units; 0 = 4096 */
    uint32_t bulk_share;         /* percent of each SM's traversal residency the other slots may take; 0 = 50 */
    uint32_t reserved[1];
} rtcd_server_config;

typedef struct {
    uint64_t submitted, completed, failed;
    uint64_t units_completed;   /* poses + trajectories */
    uint64_t batches;           /* launches */
    uint64_t inflight_bytes_peak;
    uint32_t queue_depth;       /* requests waiting for a slot */
    uint32_t reserved0;
    double p50_ms, p99_ms, mean_ms, max_ms; /* submit -> result ready, over completed requests */
    double queue_p50_ms, queue_p99_ms;      /* submit -> its launch started */
    double run_p99_ms;                      /* launch started -> result ready */
    uint64_t workspace_grows;   /* device or pinned workspace re-allocations inside launches (each can
                                 * synchronise the device, stalling every slot) */
    double grow_ms;             /* host time those re-allocations took */
    double run_max_ms;          /* the longest launch ... */
    uint32_t run_max_kind;      /* ... its detector kind (rtcd_detector_kind) */
    uint32_t run_max_units;     /* ... its poses or trajectory waypoints */
    uint32_t run_max_grows;     /* ... re-allocations inside it */
    uint32_t run_max_slot;      /* ... the slot that ran it (fast slots first) */
    double run_max_at_s;        /* ... when it started, seconds after the last stats reset */
} rtcd_server_stats;

#define RTCD_WAIT_FOREVER (-1)

RTCD_API rtcd_status rtcd_server_create(rtcd_ctx* ctx, const rtcd_server_config* config, rtcd_server** out);
/* Creates every slot's workspace for `det` and sizes it for launches of up to
 * max_units units (0 = the server's max_batch_units), so serving never
 * allocates (an allocation would synchronise the device).  Sweep detectors are
 * prepared for trajectories of up to 128 waypoints, in both sweep semantics
 * (this builds the scene's loop-edge trees).  Optional; rtcd_server_stats
 * counts the re-allocations serving still made. */
RTCD_API rtcd_status rtcd_server_prepare(rtcd_server* server, rtcd_detector* det, uint32_t max_units);
/* Finishes every accepted request, then stops the workers. */
RTCD_API rtcd_status rtcd_server_destroy(rtcd_server* server);
/* Copies the inputs (host memory, as rtcd_check with RTCD_CHECK_HOST_BUFFERS)
 * and returns a ticket at once.  `flags` may carry RTCD_CHECK_COUNTS,
 * RTCD_CHECK_NO_ENDPOINTS and RTCD_CHECK_SURFACE. */
RTCD_API rtcd_status rtcd_server_submit(rtcd_server* server, rtcd_detector* det, const float* q,
                                        const uint32_t* traj_offsets, uint32_t n, uint32_t flags, uint64_t* ticket);
/* Waits up to timeout_ms (RTCD_WAIT_FOREVER: no limit) for the ticket; on
 * completion copies the outputs (any may be NULL), releases the ticket and
 * reports the request's latency.  RTCD_ERR_DEVICE_TIMEOUT when the wait ran
 * out (the ticket stays valid).  When several threads wait on one ticket, the
 * first to find it complete collects it; the others return
 * RTCD_ERR_INVALID_ARGUMENT ("collected by another waiter"). */
RTCD_API rtcd_status rtcd_server_wait(rtcd_server* server, uint64_t ticket, int32_t timeout_ms, uint8_t* flags_out,
                                      uint8_t* seg_flags_out, uint32_t* counts_out, double* latency_ms);
RTCD_API rtcd_status rtcd_server_get_stats(rtcd_server* server, rtcd_server_stats* out);
RTCD_API rtcd_status rtcd_server_reset_stats(rtcd_server* server);

/* ---- planner side: roadmap samples, neighbour edges, batched edge checks ----
 *
 * The reference's planner tooling samples the configuration space with a
 * Halton sequence (RTCD/Planner/sampler/sampler.h:11-82), links samples to
 * their K weighted nearest neighbours on the GPU (RTCD/Planner/KNN/knn.h,
 * knnCUDA.cu) and checks each edge as a straight line of evenly spaced
 * configurations (RTCD/Utils/Test/poseUtils.h:115-141). */

/* Host only: n samples of dimension dim, sample i, coordinate d =
 * halton(i, prime[d + skip]) * (upper[d] - lower[d]) + lower[d], with the
 * reference's float arithmetic; out is n x dim row-major. */
RTCD_API rtcd_status rtcd_halton_samples(uint32_t n, uint32_t dim, uint32_t skip, const float* lower,
                                         const float* upper, float* out);
/* For every point (device, n x dim, dim <= 16) its k (<= 32) nearest others
 * by the weighted distance sqrt(sum_d (w_d (a_d - b_d))^2) (weights on the
 * host, NULL = 1); points with mask_dev[i] != 0 (optional) take no part.
 * idx_dev / dist_dev: n x k, nearest first, ties to the lower index; rows
 * with fewer than k candidates end with index 0xFFFFFFFF, distance FLT_MAX. */
RTCD_API rtcd_status rtcd_knn(rtcd_ctx* ctx, const float* points_dev, uint32_t n, uint32_t dim, const float* weights,
                              uint32_t k, const uint8_t* mask_dev, uint32_t* idx_dev, float* dist_dev, void* stream);
/* Checks n_edges straight-line edges between configurations: nodes_dev
 * (device, n_nodes x dof), edges_dev (device, n_edges x 2 node indices).
 * Each edge becomes n_wp evenly spaced configurations a + (b - a)/(n_wp-1) i,
 * built on the device; sweep detectors check them as one trajectory each,
 * discrete detectors check every configuration.  flags_dev[e] != 0 when the
 * edge collides.  flags may carry RTCD_CHECK_NO_ENDPOINTS (sweeps),
 * RTCD_CHECK_TWO_WAY and RTCD_CHECK_CONTAINMENT (discrete). */
RTCD_API rtcd_status rtcd_check_edges(rtcd_detector* det, const float* nodes_dev, uint32_t n_nodes,
                                      const uint32_t* edges_dev, uint32_t n_edges, uint32_t n_wp, uint8_t* flags_dev,
                                      uint32_t flags, void* stream);

/* ---- building blocks, exposed for callers that compose their own pipelines ---- */

/* Batched forward kinematics (upstream batchFkineAdj, RTCD/Robot/robot.cu:202-241;
 * declared in RTCD/Robot/robot.cuh:10-46).  q_dev: float[n][dof] on the device;
 * T_dev: float[n][dof+1][12] on the device, link transforms 3x4 row-major.
 * Asynchronous on `stream` (NULL = the context stream). */
RTCD_API rtcd_status rtcd_robot_fk(rtcd_robot* robot, const float* q_dev, uint32_t n, float* T_dev, void* stream);

/* Exclusive scan of n uint32 (upstream exclusiveScan,
 * RTCD/Utils/cuda/cudaAlgorithms.cuh:33-114).  Device pointers; in != out;
 * total_dev (optional) receives the sum.  Asynchronous on `stream`. */
RTCD_API rtcd_status rtcd_exclusive_scan_u32(rtcd_ctx* ctx, const uint32_t* in_dev, uint32_t* out_dev, uint32_t n,
                                             uint32_t* total_dev, void* stream);

/* Stable compaction of the indices of nonzero bytes (upstream streamCompact /
 * compactCpy, RTCD/Utils/cuda/streamCompact.inl:12-89).  Device pointers;
 * count_dev receives how many.  Asynchronous on `stream`. */
RTCD_API rtcd_status rtcd_select_flags_u8(rtcd_ctx* ctx, const uint8_t* mask_dev, uint32_t n, uint32_t* idx_dev,
                                          uint32_t* count_dev, void* stream);

/* Diagnostics of the exact tests' arithmetic, on n pairs given in world
 * coordinates (device arrays, asynchronous on `stream`).  test 0:
 * segment-triangle - a: n x 6 floats (p, q), b: n x 9 (triangle a, b, c);
 * f32_out[i] = the FP32 filter's class (0 certain miss, 1 certain hit, 2 too
 * close to call: re-tested in FP64), f64_out[i] = the FP64 re-test's decision
 * (0 / 1).  test 1: segment vs capsule axis - b: n x 9 (axis B0 B1, 3 floats
 * unused); test 2: segment vs quadratic Bezier piece - b: n x 9 (B0 B1 B2);
 * f32_out = the distance the light pass computes in FP32, f64_out = the FP64
 * re-test's distance.  No counterpart in the reference (its intersectors are
 * closed). */
RTCD_API rtcd_status rtcd_exact_test_probe(rtcd_ctx* ctx, int test, const float* a_dev, const float* b_dev, uint32_t n,
                                           float* f32_out_dev, double* f64_out_dev, void* stream);

/* Self-test of the failure detection of the bounded device waits.  No
 * counterpart in the reference (its device code has no bounded waits).  Runs
 * the compaction of n (1 to 1,048,576) zero flags with the tile counter
 * seeded so that no block takes tile 0: tile 0's look-back word is never
 * published, every other tile's look-back waits on it, and each wait gives up
 * after spin_limit (1 to 65,536) polls, sets the device error word and lets
 * its block finish.  Returns RTCD_ERR_DEVICE_TIMEOUT when the waits ran out
 * as designed (the context stays usable), RTCD_ERR_INTERNAL if they did not.
 * Synchronous on the context stream. */
RTCD_API rtcd_status rtcd_selftest_lookback_timeout(rtcd_ctx* ctx, uint32_t n, uint32_t spin_limit);

/* rtcd_select_flags_u8 for callers that cannot allocate device memory when
 * they query: a control loop with a hard deadline cannot afford cudaMalloc /
 * cudaFree (they may synchronise the device and take unbounded time), and a
 * process whose device memory belongs to another owner may not allocate at
 * all.  No counterpart in the reference.  The look-back scratch lives in a
 * fixed 131 KB device array inside this library, so the call allocates
 * nothing; that array is held on every GPU that loads the library until the
 * process exits.  Limit: n <= 33,554,432 flags (RTCD_ERR_CAPACITY beyond).
 * Every call looks up the array's device address on the current device
 * (cudaGetSymbolAddress), so the call stays valid after cudaDeviceReset; the
 * first call on a device may also load the library's device code there, so
 * make that first call before any stream capture.  All calls share the one array, and it keeps the
 * previous call's contents (each call first clears the words it uses); two
 * calls that overlap on the GPU would race on it, so the library serialises
 * them: each call takes a process-wide lock and returns only after its work
 * has finished.  `stream` is a cudaStream_t (NULL = the legacy default
 * stream); on return idx_dev / count_dev hold the result. */
RTCD_API rtcd_status rtcd_select_flags_u8_noalloc(const uint8_t* mask_dev, uint32_t n, uint32_t* idx_dev,
                                                  uint32_t* count_dev, void* stream);

/* Canonical LBVH over n boxes (replaces optixAccelBuild, RTCD/Meshes/mesh.h:725-740).
 * Host arrays: lo/hi float[n][3] in; codes_out[n] (sorted Morton codes),
 * perm_out[n] (sorted position -> box), child_out[2(n-1)] (bit 31 set = leaf
 * with sorted position, else internal node), node_lo/node_hi float[n-1][3]
 * out (any output may be NULL).  *depth_out: longest root-leaf path.
 * Synchronous. */
RTCD_API rtcd_status rtcd_lbvh_build(rtcd_ctx* ctx, const float* lo, const float* hi, uint32_t n, uint32_t* codes_out,
                                     uint32_t* perm_out, uint32_t* child_out, float* node_lo, float* node_hi,
                                     uint32_t* depth_out);

/* Thread-local message of the last failing call (empty when none). */
RTCD_API rtcd_status rtcd_last_error(char* buf, size_t n);
RTCD_API int rtcd_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* RTCD_H */
