/*
 * behavert_b200.h -- C-ABI of the B200-native BehaveRT per-step agent pipeline.
 *
 * One shared library (libbehavert_b200.so) exports these functions.  The
 * signatures use plain C types only (no CUDA or torch types): pointers, sizes
 * and status codes.  Every function returns an int status (BRT_OK == 0) and
 * never exits the process; brt_last_error() returns a message for the last
 * failing call made on the calling thread.
 *
 * Reference interfaces replaced (paths are inside the BehaveRT project):
 *   - The plugin functionalities of the mixin engine
 *       EnvGrid3DPlugIn::reorderSimData        PlugIns/EnvGrid3D/include/EnvGrid3DPlugIn.h:293-415
 *       Proximity3DPlugIn::computeNeighborhoods PlugIns/Proximity3D/include/Proximity3DPlugIn.h:261-308
 *       OpenSteerWrapperPlugIn::{resetSteerForce, computeSeparations,
 *         computeAlignments, computeCohesions, computeSeekingsWorldCenter,
 *         applySteeringForces}                   PlugIns/OpenSteerWrapper/include/OpenSteerWrapperPlugIn.h:288-424
 *       BehaviorClusteringPlugIn::steerForClustering
 *                                                PlugIns/BehaviorClustering/include/BehaviorClusteringPlugIn.h:740-822
 *   - The feature arrays (DeviceArrayWrapper<T>, Core/include/DeviceArrayWrapper.h:58-192):
 *       position / forward / smoothAccel (float4), featuresVector (float x F),
 *       similarityStats (float4), agentHash (uint2), cellStart (uint),
 *       neighList (uint, stride maxNeighbors+1).
 *   - The parameter structs hBody3DParams, hEnvGrid3DParams, hProximity3DParams,
 *       hOpenSteerWrapperParams, hBehaviorClusteringParams (field names kept).
 *   - BehaveRT::RadixSort(KeyValuePair*, KeyValuePair*, elements, bits)
 *       PlugIns/EnvGrid3D/radixsort.cu:50-80
 *
 * Layout conventions
 *   - All per-agent arrays handed across this boundary are in AGENT-ID order,
 *     like the reference's id-ordered features after applySteeringForces
 *     (OpenSteerWrapper_kernel.cu:324-331).  float4 arrays are 4 floats per
 *     agent; features are featuresCount floats per agent.
 *   - Sorted-order outputs (hash pairs, cell ranges, neighbour lists, steering
 *     forces) use SORTED SLOTS, exactly like the reference's getHash(),
 *     getCellStart() and neighList.
 *   - `where` selects host (BRT_MEM_HOST) or device (BRT_MEM_DEVICE) pointers.
 *
 * Threading: one engine per host thread.  Work is enqueued on the engine's own
 * CUDA stream; host-buffer getters synchronise that stream.
 */
#ifndef BEHAVERT_B200_H
#define BEHAVERT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BRT_ABI_VERSION 1

/* status codes */
#define BRT_OK            0
#define BRT_ERR_CUDA      1  /* a CUDA runtime call failed                     */
#define BRT_ERR_CONFIG    2  /* invalid parameters (grid < 3 cells, M > 128 ...) */
#define BRT_ERR_CAPACITY  3  /* a size limit was exceeded                      */
#define BRT_ERR_TIMEOUT   4  /* a bounded device spin-wait gave up             */
#define BRT_ERR_ARG       5  /* null pointer / bad argument                    */
#define BRT_ERR_STATE     6  /* call order violated (e.g. lists not computed)  */
#define BRT_ERR_NODEVICE  7  /* no CUDA device                                 */

#define BRT_MEM_HOST   0
#define BRT_MEM_DEVICE 1

#define BRT_MAX_NEIGHBORS   128  /* Proximity3d_MAX_NEIGHBORS, Proximity3D_kernel.cuh:37        */
#define BRT_MAX_FEATUREDIM   32  /* BehaviorClustering_MAX_FEATUREDIM, BehaviorClustering_kernel.cuh:39 */
#define BRT_MAX_OBSTACLES    64  /* per flock                                                     */

/*
 * Parameters of one flock (one independent simulation).  Field names follow
 * the reference's host parameter structs; the world is the periodic cube
 * [0, worldSize)^3 split into gridSize^3 cells of side cellSize
 * (worldSize == gridSize * cellSize, gridSize >= 3).
 */
/* SchoolingParams (PlugIns/Schooling/include/Schooling_kernel.cuh:36-56),
   the schooling member of brt_params below. */
typedef struct brt_schooling_params {
    int32_t  mode;                 /* 0 flocking law, 1 animateSchool, 2 split path */
    float    theta;                /* cos of the maximum turning angle     */
    float    delta;                /* accepted, unused (as in the reference) */
    float    r_r;                  /* repulsion radius                     */
    float    r_p;                  /* attraction / orientation radius      */
    float    eta;                  /* cos of the blind-angle limit         */
    float    w_a;                  /* attraction weight                    */
    float    w_o;                  /* orientation weight                   */
    float    s;                    /* constant speed                       */
    float    randomDeviationWeight;
    uint32_t seed;                 /* random-stream seed                   */
} brt_schooling_params;

typedef struct brt_params {
    /* Body3DParams (PlugIns/Body/include/body3d_kernel.cuh:39-58) */
    uint32_t numBodies;
    float    commonRadius;
    int32_t  use2DProjection;

    /* EnvGrid3DParams (PlugIns/EnvGrid3D/include/envgrid3d_kernel.cuh:38-65),
       periodic cube instead of the reference's padded clamped box */
    float    worldSize;
    float    cellSize;
    uint32_t maxBodiesPerCell;     /* 0 = unbounded (per-cell scan cap)      */
    int32_t  disableSorting;       /* accepted for drop-in, must be 0        */

    /* Proximity3DParams (PlugIns/Proximity3D/include/Proximity3D_kernel.cuh:40-73) */
    uint32_t maxNeighbors;         /* 1..BRT_MAX_NEIGHBORS                   */
    int32_t  useKnn;               /* replace-farthest when the list is full */
    float    commonSearchRadius;

    /* OpenSteerWrapperParams (PlugIns/OpenSteerWrapper/include/OpenSteerWrapper_kernel.cuh:36-55) */
    float    commonMaxSpeed;
    float    commonMaxForce;
    float    commonMass;
    float    commonSensingMinRadius;
    float    separationParams[3];  /* weight, radius, cosMaxAngle            */
    float    cohesionParams[3];
    float    alignmentParams[3];

    /* BehaviorClusteringParams (PlugIns/BehaviorClustering/include/BehaviorClustering_kernel.cuh:41-60) */
    uint32_t featuresCount;        /* 0..BRT_MAX_FEATUREDIM                  */
    float    clusteringForceParams[3];          /* .x = weight               */
    float    alignmentClusteringForceParams[3]; /* .x = weight               */
    float    similarityStatsParams[3];          /* avg rate, min/max rate, memory */
    float    avgSimilarityController;
    /* Feature relaxation toward the similarity-weighted neighbour mean
       (rate per step; 0 disables).  No reference counterpart. */
    float    featureRelaxRate;

    /* Static sphere obstacles on the EnvGrid3D grid (no reference counterpart;
       nearest analogue moveAwayFromTarget_kernel, OpenSteerWrapper_kernel.cu:185-212) */
    uint32_t numObstacles;         /* 0..BRT_MAX_OBSTACLES                    */
    float    obstacleAvoidanceWeight;
    float    obstacles[BRT_MAX_OBSTACLES][4]; /* centre xyz, radius            */

    /* SchoolingParams (PlugIns/Schooling/include/Schooling_kernel.cuh:36-56).
       mode selects the steering law of the flock:
         0  flocking (OpenSteerWrapper separation / alignment / cohesion)
         1  Schooling_animateSchool (Schooling_kernel.cu:226-318): repulsion
            within r_r, else attraction + orientation within r_p; turn limited
            to theta; constant speed s, step s * forward * 0.1
         2  the split path calcRepulsion -> calcAttractionOrientation ->
            calcMovement (Schooling_kernel.cu:64-221): as 1 but with the blind
            angle eta in the attraction/orientation zone, a random deviation of
            weight randomDeviationWeight, and step s * forward * 0.2.
       The reference draws the deviation from a time-seeded Mersenne Twister;
       here it is a counter-based generator (splitmix64 of seed, step, agent
       id), so runs are reproducible.  All flocks of one engine use the same
       family (mode 0, or modes 1/2). */
    brt_schooling_params schooling;
} brt_params;

/* Fills *p with the reference defaults used by the flocking demo and the
   unspecified constants fixed by this library (commonMass 1, sensing min
   radius 0, cosMaxAngle -2, unbounded maxBodiesPerCell, clustering steering
   off). */
int brt_params_default(brt_params* p);

typedef struct brt_engine brt_engine;

/* ---- library ---------------------------------------------------------- */
const char* brt_version(void);
const char* brt_error_string(int status);
const char* brt_last_error(void);
int brt_device_count(int* count);

/* ---- engine lifetime (CommonResources + plugin install chain,
        Core/src/CommonResources.cpp:49-92, Core/src/SimEnginePlugIn.cpp:45-56).
   A single engine may hold many flocks; agent ids of flock f are
   [sum_{g<f} numBodies_g, sum_{g<=f} numBodies_g). ---------------------- */
int brt_engine_create(const brt_params* flocks, uint32_t num_flocks, int device, brt_engine** out);
int brt_engine_destroy(brt_engine* e);
int brt_engine_num_agents(const brt_engine* e, uint32_t* num_agents);
int brt_engine_num_cells(const brt_engine* e, uint32_t* num_cells);
/* Replace the parameters of one flock; geometry fields (numBodies,
   worldSize, cellSize, maxNeighbors, featuresCount) must not change. */
int brt_engine_set_params(brt_engine* e, uint32_t flock, const brt_params* p);
/* Tuning options (the reference's DeviceInterface BlockDim / commonBlockDim
   knobs, Core/src/CommonResources.cpp:78-82, generalised):
     "sort_digit_bits"  4..9  radix digit width of the onesweep passes (default 8;
                              at most 4 passes, so narrow digits on wide keys widen)
     "incremental_sort" 0/1   derive a fused step's sorted order from the
                              previous step's when few agents changed cell
                              (default 1); the device falls back to the full
                              radix sort after a state change, when more
                              than one agent in 8 moved, or when a cell
                              received more than 32 movers.  The order is
                              the same either way.
     "two_pass"         0/1   build each neighbour list before steering even
                              when the single-pass kernel applies (default 0)
     "block_size"       32..256, multiple of 32: threads per block of the
                              single-pass flock kernel (default 64)
     "scan_variant"     0..7  neighbour-scan loop: 0 four candidates in flight
                              with exact cell culling (skipped for a step whose
                              state holds a NaN position or one outside the
                              world), 1 two in flight with the same culling,
                              2 four without culling, 3 one at a time,
                              4 warp-cooperative (a warp tests 32 candidates of
                              a home cell's neighbourhood per step, the first
                              96 held in registers), 5 as 4, with further
                              96-candidate windows while 8 or more of a home
                              cell's agents still need neighbours (default),
                              6 a persistent work queue over (flock, row
                              segment) tiles: each block stages a tile's
                              neighbour cells in shared memory once and every
                              thread scans its agent's 27 cells from there
                              (dense tiles that do not fit take scan 5),
                              7 as 4, with each home cell's candidates first
                              tested against the bounding box of the cell's
                              agents and only the survivors voted on
     "phase2_variant"   0..2  list walk: 0 one neighbour at a time, 1 two at a
                              time (per-agent scans 0..3 only), 2 (default)
                              two walks, geometry then feature sums (with
                              scan_variant 4, 5 or 7 and features; otherwise as 0)
     "wide_registers"   0/1   the flock kernel built for 128 registers a thread
                              (2 resident 256-thread blocks per SM) instead of 64
     "registers"        128, 64, 48 or 40: the flock kernel's register budget
                              a thread (64 default; 48 and 40 trade spills for
                              resident warps and apply to scan_variant 4, 5, 7)
     "adjoint_graphs"   0/1   capture the adjoint forward/backward as graphs (default 1)
     "adjoint_export"   0/1   keep the frozen lists and branch flags (brt_adjoint_get_tape)
     "random_step"      uint32 the step counter of the Schooling random stream
                              (every hash pass adds 1 before the move reads it)
     "lookback_spin_limit" 0..2^31-1: polls of an unpublished predecessor
                              before a look-back wait (onesweep passes, the
                              re-sort's cell scan) gives up (default 2^21,
                              about a second); the step then reports
                              BRT_ERR_TIMEOUT at the next sync or getter
     "lookback_stall_tile" -1 or a tile index: that tile's look-back polls as
                              if its predecessor never published (a status
                              word that nothing sets), so tests can make the
                              bounded wait run out; -1 (default) in normal use
   None of these changes results (the two look-back options only when no wait
   runs out); unknown keys return BRT_ERR_ARG. */
int brt_engine_set_option(brt_engine* e, const char* key, int64_t value);
/* Autotuner: times the sort digit width, then the flock kernel's block size
   and scan loop, then its list walk, on the engine's own state (graphs of
   `steps` steps, each trial started from the same snapshot), keeps the
   fastest, and leaves the state as it found it.  report (optional) receives
   a JSON object with the choice and every trial's ms per step. */
int brt_engine_autotune(brt_engine* e, float elapsedTime, uint32_t steps, char* report, size_t report_len);
/* The engine's CUDA stream (a cudaStream_t), for callers that enqueue their
   own work around the engine's. */
int brt_engine_stream(brt_engine* e, void** stream);
int brt_sync(brt_engine* e);

/* ---- feature arrays (DeviceArrayWrapper::copyArrayToDevice /
        copyArrayFromDevice, Core/include/DeviceArrayWrapper.h:345-386) ---- */
/* Any pointer may be NULL to leave that feature unchanged / not read.
   pos4.w is ignored on input (the reference keeps w = 1); fwd4.w = speed.
   After a call reported a failed device check (BRT_ERR_TIMEOUT, or
   BRT_ERR_STATE from the device error word) the engine state is undefined;
   brt_set_state then also restores the identity slot order, and registered
   arrays must be set again. */
int brt_set_state(brt_engine* e, const float* pos4, const float* fwd4,
                  const float* acc4, const float* features, int where);
int brt_get_state(brt_engine* e, float* pos4, float* fwd4,
                  float* acc4, float* features, int where);
/* On-disk snapshot of the engine state, for resuming a run.  No reference
   counterpart (the reference keeps no resumable state; its reset() and
   dataset loaders start runs).  Little-endian binary: magic "BRTSNAP1",
   uint32 version (1), agents, features per agent, flocks, the Schooling
   random-stream step, 3 reserved words; then, in agent-id order, float4
   position, forward, smoothed acceleration and similarityStats arrays and
   the float feature array.  brt_load_snapshot returns BRT_ERR_CONFIG when
   the agent, feature or flock counts differ from the engine's. */
int brt_save_snapshot(brt_engine* e, const char* path);
int brt_load_snapshot(brt_engine* e, const char* path);
/* similarityStats (float4 per agent: min, avg, max, unused) of BehaviorClustering */
int brt_set_similarity_stats(brt_engine* e, const float* stats4, int where);
int brt_get_similarity_stats(brt_engine* e, float* stats4, int where);

/* ---- the fused per-step pipeline ------------------------------------------
   hash -> onesweep sort -> reorder + cell ranges -> fused neighbour search +
   steering + integration + clustering update, nsteps times.  nsteps > 1 runs
   a CUDA graph of the whole loop.  Replaces the BehaveRT_Flocking update
   sequence, Samples/OpensteerDemo/plugins/BehaveRT_Flocking.cpp:177-199. */
int brt_step(brt_engine* e, float elapsedTime, uint32_t nsteps);
/* Capture and instantiate the CUDA graph that brt_step(e, elapsedTime,
   nsteps > 1) launches, without running it (so a timed loop excludes capture). */
int brt_step_prepare(brt_engine* e, float elapsedTime, uint32_t nsteps);
/* Per-stage CUDA-event timing of single-step brt_step calls (not graphs):
   when enabled, events are recorded on the engine stream after the hash,
   sort, reorder and fused stages of every step.  brt_engine_stage_times
   synchronises and returns the accumulated milliseconds per stage
   (ms[0] hash, ms[1] all sort passes, ms[2] reorder + cell ranges, ms[3]
   fused pass; with the incremental re-sort ms[0] also holds its mark kernel
   and ms[1] its cell-scan and place kernels), the number of timed steps and
   the kernel launches per step. */
int brt_engine_stage_timing(brt_engine* e, int enable);
int brt_engine_stage_times(brt_engine* e, double* ms4, uint64_t* steps, uint32_t* launches_per_step);

/* ---- stage-wise functionalities (same names and order as the reference) -- */
int brt_reorder_sim_data(brt_engine* e);              /* EnvGrid3DPlugIn.h:293-415          */
int brt_compute_neighborhoods(brt_engine* e);         /* Proximity3DPlugIn.h:261-308        */
int brt_reset_steer_force(brt_engine* e);             /* OpenSteerWrapperPlugIn.h:421-424   */
int brt_compute_separations(brt_engine* e);           /* OpenSteerWrapperPlugIn.h:288-302   */
int brt_compute_alignments(brt_engine* e);            /* OpenSteerWrapperPlugIn.h:326-344   */
int brt_compute_cohesions(brt_engine* e);             /* OpenSteerWrapperPlugIn.h:350-366   */
int brt_steer_for_clustering(brt_engine* e);          /* BehaviorClusteringPlugIn.h:740-822 */
int brt_compute_seekings_world_center(brt_engine* e); /* OpenSteerWrapperPlugIn.h:380-393   */
/* steerAndSlowToAvoidNeighbors (OpenSteerWrapperPlugIn.h:309-322, kernel
   OpenSteerWrapper_kernel.cu:110-154): adds the weighted separation force,
   times (n - 16) * 0.5 above 16 listed neighbours, and scales each agent's
   speed by 0.9 / 1.02 when that force points against / along its heading
   (the speed the next stages and brt_apply_steering_forces see). */
int brt_steer_and_slow_to_avoid_neighbors(brt_engine* e);
/* steerForMoveAwayBaseTarget (OpenSteerWrapperPlugIn.h:428-440, kernel
   OpenSteerWrapper_kernel.cu:185-212): adds (w * (p - base)) / |p - base|, and
   nothing beyond twice the radius, to every agent's steering force.
   base3 = avoidBase; params3 = avoidBaseParams (steering weight w,
   acceleration factor, radius), NULL or w = 0 for the reference's defaults
   (500, 500, 1000).  As in the reference: the direct offset (no periodic
   image), the smoothed acceleration left unchanged (the kernel's own write
   of it is overwritten), and 0/0 for an agent exactly at the base point. */
int brt_steer_for_move_away_base_target(brt_engine* e, const float* base3, const float* params3);
int brt_apply_steering_forces(brt_engine* e, float elapsedTime); /* OpenSteerWrapperPlugIn.h:400-418 */
/* SchoolingPlugIn functionalities (engines whose flocks have schooling.mode
   1 or 2), after brt_compute_neighborhoods; the first two write the steering
   force (brt_get_steer_force), the last two the new state. */
int brt_school_repulsion(brt_engine* e);              /* calcRepulsion, SchoolingPlugIn.h:236-248             */
int brt_school_attraction_orientation(brt_engine* e); /* calcAttractionOrientation, SchoolingPlugIn.h:252-264 */
int brt_school_movement(brt_engine* e);               /* calcMovement, SchoolingPlugIn.h:268-299              */
int brt_school_animate(brt_engine* e);                /* animateSchool, SchoolingPlugIn.h:219-232             */

/* ---- BehaviorClustering analytics over the current neighbour lists
        (after brt_compute_neighborhoods, or a brt_step with record_lists) ----
   brt_compute_cluster_membership: local label propagation
   (BehaviorClusteringPlugIn::computeClusterMembership,
   BehaviorClusteringPlugIn.h:828-871): every agent's label starts as its
   sorted slot, then `iterations` Jacobi sweeps (the reference uses
   iterationLP = 10) replace it by the minimum over the agent and its listed
   neighbours.
   brt_analyze_cluster_hit_rate (analyzeClusterHitRate, :885-894): among the
   listed neighbours closer than same_cluster_max_radius (reference 1.5), the
   fraction sharing the agent's label and the mean of their labels (-1 with
   none).
   brt_get_cluster_membership: float4 per agent id (label, hit rate, mean
   neighbour label, 0), the reference's float3 clusterMembership feature. */
int brt_compute_cluster_membership(brt_engine* e, uint32_t iterations);
int brt_analyze_cluster_hit_rate(brt_engine* e, float same_cluster_max_radius);
int brt_get_cluster_membership(brt_engine* e, float* membership4, int where);

/* ---- getters of the intermediate features --------------------------------- */
/* Sorted (cell hash, agent id) pairs as uint2, like getHash() after
   reorderSimData (EnvGrid3DPlugIn.h:101-105).  keys/ids may be NULL. */
int brt_get_hash(brt_engine* e, uint32_t* keys, uint32_t* ids, int where);
/* cellStart / cellEnd per global cell; 0xFFFFFFFF for empty cells
   (Proximity3D_kernel.cu:54-84 writes cellStart only). */
int brt_get_cell_ranges(brt_engine* e, uint32_t* cell_start, uint32_t* cell_end, int where);
/* Neighbour lists of the last computeNeighborhoods (or of the last fused step
   when brt_engine_record_lists is on): numAgents * (maxNeighbors+1) uint32,
   [count, slot_0, ..., slot_{count-1}, unused...] per sorted slot
   (Proximity3D_kernel.cu:117-124).  Flocks with different maxNeighbors use
   the engine-wide maximum as stride. */
int brt_get_neighbor_lists(brt_engine* e, uint32_t* lists, int where);
int brt_neighbor_list_stride(const brt_engine* e, uint32_t* stride);
/* Steering force accumulated by the stage-wise calls, per sorted slot (float4). */
int brt_get_steer_force(brt_engine* e, float* steer4, int where);
/* Make brt_step also write the neighbour lists of every step (off by default:
   the timed pipeline does not materialise them). */
int brt_engine_record_lists(brt_engine* e, int enable);
/* Device error word: nonzero after a bounded spin gave up or a capacity check
   fired inside a kernel; cleared by this call. */
int brt_engine_check_device_error(brt_engine* e, uint32_t* word);

/* ---- plugin extension: per-agent arrays and user kernels -------------------
   A reference plugin keeps per-agent features in the device data repository
   (DataInfo table, devicedata.cuh:51-70, through DeviceArrayWrapper,
   DeviceArrayWrapper.h:74-168) and launches its own kernels over them with
   DeviceInterface::kernelCall (Core/DeviceInterface.cu:380-458).

   brt_engine_add_array registers a per-agent array of bytes_per_agent bytes
   (a multiple of 4, at most 1024; at most BRT_MAX_USER_ARRAYS arrays),
   zero-filled.  The engine permutes it with the agents at every reorder, as
   the reference reorders registered features, so slot i always belongs to
   agent user_agent_id[i] of brt_arrays.  brt_engine_array_set / _get copy it
   from / to agent-id order.

   brt_engine_get_arrays fills a view of the engine's device arrays (borrowed:
   valid until the engine is destroyed or its parameters change).
   brt_engine_launch calls fn(user_data, stream, &view) on the calling thread;
   fn enqueues its kernels on `stream`, the engine's stream, so they run in
   order with the engine's stages (the before / after hooks of kernelCall are
   the code around its launches).  The state arrays are in the engine's slot
   order (agent_id maps slot to agent); the sorted_* arrays, steer4 and
   neighbor_lists are those of the current step, valid after
   brt_reorder_sim_data / brt_compute_neighborhoods, and the state arrays and
   the registered arrays share the sorted order once a step completes.  In an
   engine with features, sorted_pos4's w holds each agent's feature norm
   (the state's pos4 keeps w = 1).  Kernels may change any value of the
   state arrays but must not move agents between slots or rewrite agent_id:
   the next step's incremental re-sort starts from the current slot order. */
#define BRT_MAX_USER_ARRAYS 8
typedef struct brt_arrays {
  uint32_t num_agents, num_cells, features_stride, list_stride;
  float* pos4; float* forward4; float* smooth_accel4; float* features;
  const uint32_t* agent_id;
  float* sorted_pos4; float* sorted_forward4; float* sorted_smooth_accel4; float* sorted_features;
  const uint32_t* sorted_agent_id;
  float* steer4;
  const uint32_t* neighbor_lists;  /* [n, slot...] per sorted slot, stride list_stride */
  const uint32_t* cell_start; const uint32_t* cell_end;
  uint32_t num_user;
  uint32_t user_bytes[BRT_MAX_USER_ARRAYS];
  void* user[BRT_MAX_USER_ARRAYS];
  const uint32_t* user_agent_id;
} brt_arrays;
typedef void (*brt_launch_fn)(void* user_data, void* stream, const brt_arrays* arrays);
int brt_engine_add_array(brt_engine* e, uint32_t bytes_per_agent, uint32_t* array_id);
int brt_engine_array_set(brt_engine* e, uint32_t array_id, const void* src, int where);
int brt_engine_array_get(brt_engine* e, uint32_t array_id, void* dst, int where);
int brt_engine_get_arrays(brt_engine* e, brt_arrays* out);
int brt_engine_launch(brt_engine* e, brt_launch_fn fn, void* user_data);

/* ---- differentiable rollout ---------------------------------------------------
   No counterpart in the reference (BehaveRT has no differentiation).
   Neighbour sets and branch decisions (inBoidNeighborhood memberships, the
   adjustRawSteeringForce low-speed and deviation-limit branches, the two
   truncateLength clips) are frozen per step; the gradient is that of the FP32
   forward through those fixed choices.  Supported: flocking, static sphere
   obstacles and integration; kNN lists, use2DProjection, feature clustering
   steering and maxNeighbors > 32 return BRT_ERR_CONFIG.

   brt_adjoint_forward runs nsteps fused steps from the current state,
   checkpointing the state every checkpoint_every steps, and evaluates
       loss_f = (1 / n_f) sum_{i in flock f} |minimum image(p_i(T) - target_i)|^2
   in FP64 (target_pos4: float4 per agent in agent-id order).  loss_per_flock
   (nflocks doubles, may be NULL) follows `where`.  The engine is left at the
   final state.

   brt_adjoint_backward propagates the adjoint of
       sum_f loss_scale[f] * loss_f  (+ <g*_T, final state> for the optional
       id-ordered adjoints gpos4_T / gfwd4_T (xyz forward, w speed) / gacc4_T)
   back through the taped forward, recomputing hash, sort and neighbour lists
   of each checkpoint segment.  loss_scale: host array of nflocks doubles or
   NULL for 1.  Outputs (float4 per agent, agent-id order, each may be NULL):
   grad_pos4 = dL/dposition(0), grad_fwd4 = dL/dforward(0) (w = dL/dspeed),
   grad_vel4 = dL/dvelocity(0) with velocity = forward * speed,
   grad_acc4 = dL/dsmoothed acceleration(0); grad_weights = dL/d(separation,
   alignment, cohesion weight) per flock (nflocks x 3 doubles, reduced in
   FP64).  The engine is left at the forward's final state. */
int brt_adjoint_forward(brt_engine* e, float elapsedTime, uint32_t nsteps, uint32_t checkpoint_every,
                        const float* target_pos4, int where, double* loss_per_flock);
int brt_adjoint_backward(brt_engine* e, const double* loss_scale,
                         const float* gpos4_T, const float* gfwd4_T, const float* gacc4_T, int where_in,
                         float* grad_pos4, float* grad_fwd4, float* grad_vel4, float* grad_acc4,
                         double* grad_weights, int where_out);
/* With option "adjoint_export" set before brt_adjoint_forward, the backward
   also writes, for every step t and agent id, the frozen neighbour list
   (count, then neighbour agent ids; stride brt_neighbor_list_stride) and
   four flag words: branch bits (1 low-speed adjust, 2 deviation limited,
   4 force clipped, 8 velocity clipped) and the separation, alignment and
   cohesion membership masks over list positions.  Sizes: nsteps * N *
   stride and nsteps * N * 4 uint32. */
int brt_adjoint_get_tape(brt_engine* e, uint32_t* lists_by_id, uint32_t* flags_by_id, int where);
/* With option "adjoint_export", also the input state of every step t as the
   backward recomputed it (float4 per agent id: position, forward with speed
   in w, smoothed acceleration; nsteps * N each, any pointer may be NULL).
   An FP64 reverse linearised at these FP32 states separates the adjoint's
   own rounding from the FP32 forward's.  No reference counterpart. */
int brt_adjoint_get_tape_states(brt_engine* e, float* pos4, float* fwd4, float* acc4, int where);
/* Per-flock steering weights (separationParams[0], alignmentParams[0],
   cohesionParams[0]; nflocks x 3 floats).  Setting them does not invalidate
   captured step graphs (the kernels read them from device memory). */
int brt_set_steering_weights(brt_engine* e, const float* weights3, int where);
int brt_get_steering_weights(brt_engine* e, float* weights3, int where);

/* ---- standalone key/value radix sort (BehaveRT::RadixSort replacement) ----
   Stable LSD onesweep sort with decoupled look-back of `n` (key, value) pairs
   (uint2: key in .x, value in .y) on the low `bits` bits of the key.
   pairs_in is not modified; the result goes to pairs_out.  `scratch` is
   device memory of at least brt_radix_sort_scratch_bytes(n, bits) bytes;
   `stream` is a cudaStream_t (NULL = default stream). */
size_t brt_radix_sort_scratch_bytes(uint32_t n, uint32_t bits);
int brt_radix_sort_pairs(const uint32_t* pairs_in, uint32_t* pairs_out, uint32_t n,
                         uint32_t bits, void* scratch, size_t scratch_bytes, void* stream);

/* ---- the same sort without any allocation ------------------------------------
   No counterpart in the reference.  For callers that cannot call cudaMalloc:
   frame loops and engine plugins that must not stall the device (cudaFree
   synchronises it), code running under another framework's caching allocator
   that owns all device memory, and hosts that fix their GPU memory budget at
   start-up.  The scratch is one static device array inside this library
   (about 10 MiB on every GPU that loads it, held until the process exits), so:
     - n is limited to brt_radix_sort_noalloc_max_pairs() (1,048,576) pairs;
       larger n returns BRT_ERR_CAPACITY;
     - every call looks up the array's device address on the current device
       (cudaGetSymbolAddress, which allocates nothing), so a device reset or a
       re-created primary context never leaves it a stale address;
     - every call clears the parts of the array that must start at zero, but
       all calls share the array: calls that overlap on the GPU (other
       streams, other host threads) race and must be serialised by the caller;
     - it allocates nothing: no cudaMalloc, cudaFree or allocating library call.
   Results are identical to brt_radix_sort_pairs.  Before it returns, the call
   copies the device error word to the host and synchronises `stream`, so the
   host waits for the sort to finish; for the same reason it cannot be called
   while `stream` is being captured into a CUDA graph (the capture would be
   invalidated): use brt_radix_sort_pairs with caller-owned scratch there. */
size_t brt_radix_sort_noalloc_max_pairs(void);
int brt_radix_sort_pairs_noalloc(const uint32_t* pairs_in, uint32_t* pairs_out, uint32_t n,
                                 uint32_t bits, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BEHAVERT_B200_H */
