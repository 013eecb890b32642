/*
 * fastrrt_b200.h -- C ABI of the B200 FastRRT planner (libfastrrt_b200.so).
 *
 * Part 1 keeps the reference's planner ABI (out0/FastRRT src/python_bind.cpp)
 * name for name, so the reference's ctypes layer binds it unchanged.  The
 * one difference is the frame argument of set_plan_data: the reference takes
 * a driveless SearchFrame*, this library takes a handle from
 * fastrrt_frame_create*().  Errors never cross the ABI as C++ exceptions;
 * calls that fail return NULL / false / a negative status and leave a message
 * for fastrrt_last_error().
 *
 * Part 2 adds frame handles and deterministic seeding; part 3 the
 * per-candidate kernels (kinematic expansion, Hermite connection, footprint)
 * used for bit-exact parity and microbenchmarks; part 4 the batched planner
 * that plans many instances in one CUDA graph per iteration; part 5 the
 * served planner.
 */
#ifndef FASTRRT_B200_H
#define FASTRRT_B200_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- part 1: the reference planner ABI --------------------------------- */

/* replaces fastrrt_initialize (src/python_bind.cpp:7-30).  class_costs[0] is
 * the class count followed by the costs; like the reference, the frame's own
 * class costs are what the planner uses. */
void *fastrrt_initialize(int width, int height, float perceptionWidthSize_m,
                         float perceptionHeightSize_m, float maxSteeringAngle_deg,
                         float vehicleLength, int lowerBound_x, int lowerBound_z,
                         int upperBound_x, int upperBound_z, float *classCosts,
                         float max_curvature);
/* replaces fastrrt_destroy (src/python_bind.cpp:32-36) */
void fastrrt_destroy(void *ptr);
/* replaces set_plan_data (src/python_bind.cpp:38-64); `frame` is a handle
 * from fastrrt_frame_create*() */
void set_plan_data(void *ptr, void *frame, int start_x, int start_z, float start_heading_rad,
                   int goal_x, int goal_z, float goal_heading_rad, float velocity_m_s,
                   int min_dist_x, int min_dist_z, int timeout_ms, float maxPathSize,
                   float distToGoalTolerance, float headingErrorTolerance_rad);
/* replaces goal_reached (src/python_bind.cpp:66-70) */
bool goal_reached(void *ptr);
/* The planner's goal direct connections (processDirectGoalConnection) follow
 * the frame's preprocessing flags from the next set_plan_data on: the
 * distance channel when isDistanceToGoalProcessed, the safe-zone skip when
 * isSafeZoneChecked.  Off by default, as the reference's FastRRT passes false
 * for both (fastrrt.cpp:79 -> graph_direct_goal_connection.cu:222, the
 * frame's flags commented out there).  0 or -1. */
int fastrrt_set_frame_preprocessing(void *ptr, int use);
/* replaces search_init (src/python_bind.cpp:72-76) */
void search_init(void *ptr, bool copyIntrinsicCostsFromFrame);
/* replaces loop (src/python_bind.cpp:77-81) */
bool loop(void *ptr, bool smartExpansion);
/* replaces path_optimize (src/python_bind.cpp:83-87) */
bool path_optimize(void *ptr);
/* replaces export_graph_nodes (src/python_bind.cpp:89-108): [n, x, z, type, ...] */
int *export_graph_nodes(void *ptr);
/* replaces release_export_graph_nodes (src/python_bind.cpp:109-112) */
void release_export_graph_nodes(int *ptr);
/* replace compute_apf_repulsion / compute_apf_attraction
 * (src/python_cuda_graph_bind.cpp:41-54 -> CudaGraph::computeRepulsiveFieldAPF /
 * computeAttractiveFieldAPF, src/cuda/apf.cu:123-154) on the planner's
 * intrinsic costs, for the planner's frame size (set_plan_data first).
 * Repulsion: every obstacle cell outside the ego box is set to 100 kr / 2,
 * then every cell outside it adds kr / 2 (1/p - 1/radius)^2 for each obstacle
 * with a free 4-neighbour at distance p <= radius, in the obstacles' row-major
 * order (the reference adds them with float atomics in an arbitrary order, its
 * sets racing with them).  Attraction: every free cell loses ka / 2 times its
 * squared distance to the goal.  The plan's remaining deferred goal direct
 * connections are evaluated first with the costs they were set up with.
 * 0 or -1. */
int fastrrt_apf_repulsion(void *ptr, void *frame, float kr, int radius);
int fastrrt_apf_attraction(void *ptr, void *frame, float ka, int goal_x, int goal_z);
/* replaces get_intrinsic_costs (src/python_cuda_graph_bind.cpp:56-72): the
 * width*height intrinsic costs into out; returns the count or -1 */
int fastrrt_intrinsic_costs(void *ptr, float *out);
/* CudaGraph::checkGraphIsConsistent (src/graph_check_dag_consistency.cpp:33-76)
 * on the planner's graph, on the device: every node's parent chain ends at a
 * root within count(NODE) + 4 hops, no node is its own parent, and every
 * parent is a NODE, COLLISION or CONNECT_TO_GOAL cell.  1 consistent, 0 not,
 * -1 error.  (The reference exposes it to its unit tests only.) */
int fastrrt_check_graph_consistent(void *ptr);
/* The path validator of the batched planner on a given path
 * [x0, z0, h0, x1, ...] of n waypoints against the planner's frame, graph
 * and plan data: it starts at the start cell and reaches the goal within
 * the distance and heading tolerances, every waypoint lies in the frame, is
 * a graph cell whose parent is the previous waypoint, repeats no cell,
 * turns within the curvature bound and has a feasible footprint outside the
 * ego box.  1 valid, 0 not, -1 error.  No counterpart in the reference (its
 * tests check paths by hand). */
int fastrrt_validate_path(void *ptr, const float *xyh, int n);
/* replace get_planned_path / interpolate_planned_path (src/python_bind.cpp:138-150):
 * [n, x0, z0, heading0, ...] */
float *get_planned_path(void *ptr);
float *interpolate_planned_path(void *ptr);
/* replaces release_planned_path_data (src/python_bind.cpp:152-155) */
void release_planned_path_data(float *ptr);
/* replaces interpolate_planned_path_p (src/python_bind.cpp:157-171) */
float *interpolate_planned_path_p(void *ptr, float *p, int size);
/* replaces ideal_curve (src/python_bind.cpp:173-180) */
float *ideal_curve(void *ptr, int goal_x, int goal_z, float goal_heading_rad);
/* replaces compute_region_debug_performance (src/python_bind.cpp:182-186) */
void compute_region_debug_performance(void *ptr);
/* replace save_current_graph_state / load_graph_state (src/python_bind.cpp:188-198);
 * text dump, one line per cell: "px pz type childcount heading cost intrinsic direct" */
void save_current_graph_state(void *ptr, const char *filename);
void load_graph_state(void *ptr, const char *filename);

/* ---- part 2: frames, seeding, errors ------------------------------------ */

/* last error message of the calling thread ("" when none) */
const char *fastrrt_last_error(void);
/* a BEV frame: W*H class ids (uint8), class costs (cost < 0 = obstacle),
 * optional W*H traversability bits (NULL = none) */
void *fastrrt_frame_create(int width, int height, const uint8_t *class_ids,
                           const float *class_costs, int n_classes, const int32_t *trav_bits);
/* the reference SearchFrame layout: W*H float3 (class id, distance, bits) */
void *fastrrt_frame_create_f3(int width, int height, const float *xyz, const float *class_costs,
                              int n_classes);
void fastrrt_frame_destroy(void *frame);
/* SearchFrame preprocessing on the device, in place of the driveless
 * SearchFrame's processDistanceToGoal / processSafeDistanceZone (not in the
 * reference tree; their outputs are read at graph_direct_goal_connection.cu:
 * 28-36 and 124-135).  The distance channel gets every cell's distance to
 * (goal_x, goal_z), sqrtf(dx * dx + dz * dz) as checkDirectConnectionToGoal
 * computes it, and the frame counts as isDistanceToGoalProcessed.  The safe
 * zone sets traversability bit 0x100 on every cell whose footprint of half
 * extents (min_dist / 2) holds no obstacle at any heading, and the frame
 * counts as isSafeZoneChecked.  0 or -1. */
int fastrrt_frame_process_distance_to_goal(void *frame, int goal_x, int goal_z);
int fastrrt_frame_process_safe_zone(void *frame, int min_dist_x, int min_dist_z);
/* the frame's isSafeZoneChecked / isDistanceToGoalProcessed flags */
int fastrrt_frame_flags(void *frame, int *safe_zone_checked, int *distance_to_goal_processed);
/* host copies of the distance and traversability channels (W*H each, NULL
 * to skip one; zeros when the frame has none) */
int fastrrt_frame_channels(void *frame, float *distance, int32_t *traversability);
/* expansion RNG seed (default: wall-clock milliseconds, like the reference) */
int fastrrt_set_seed(void *ptr, uint64_t seed);
/* footprint probes of the reference algorithm run so far (instrumentation) */
int fastrrt_probe_count(void *ptr, uint64_t *probes);
/* loop() calls and expansion passes run since search_init */
int fastrrt_loop_count(void *ptr);

/* ---- part 3: per-candidate kernels -------------------------------------- */

/* A footprint/kinematics context over one frame: the planner's parameters
 * (min distances are halved like CudaGraph::setSearchParams, graph.cu:306-314)
 * and a node grid whose heading/cost per cell the candidates start from
 * (NULL = zeros). */
void *fastrrt_candidates_create(void *frame, int min_dist_x, int min_dist_z, int lowerBound_x,
                                int lowerBound_z, int upperBound_x, int upperBound_z,
                                double max_steering_rad, double lr_m, const float *heading_grid,
                                const float *cost_grid);
void fastrrt_candidates_destroy(void *ctx);
/* check_kinematic_new_path (src/cuda/kinematics.cu:123-231) for n candidates;
 * out4 = (end x, end z, cost, heading) or (-1, -1, 0, 0).  Host buffers. */
int fastrrt_candidates_kinematic(void *ctx, int n, const int32_t *sx, const int32_t *sz,
                                 const float *steer, const float *length, float velocity_m_s,
                                 float *out4, uint64_t *probes);
/* same with device pointers on `stream` (cudaStream_t, NULL = default) */
int fastrrt_candidates_kinematic_device(void *ctx, int n, const int32_t *sx, const int32_t *sz,
                                        const float *steer, const float *length,
                                        float velocity_m_s, float *out4, uint64_t *probes,
                                        void *stream);
/* checkDirectConnectionToGoal (src/cuda/graph_direct_goal_connection.cu:16-167);
 * out = cost or -1.  safe_zone_checked: bit 0 isSafeZoneChecked (skip the
 * footprints when the start cell has traversability bit 0x100), bit 1
 * isDistanceToGoalProcessed (the distance from the frame's distance
 * channel).  Host buffers. */
int fastrrt_candidates_hermite(void *ctx, int n, const int32_t *x, const int32_t *z,
                               const float *local_heading, const int32_t *goal_x,
                               const int32_t *goal_z, const float *goal_heading,
                               float max_curvature, int safe_zone_checked, float *out,
                               uint64_t *probes);
int fastrrt_candidates_hermite_device(void *ctx, int n, const int32_t *x, const int32_t *z,
                                      const float *local_heading, const int32_t *goal_x,
                                      const int32_t *goal_z, const float *goal_heading,
                                      float max_curvature, int safe_zone_checked, float *out,
                                      uint64_t *probes, void *stream);
/* No counterpart in the reference.  The kinematic candidate check of
 * fastrrt_candidates_kinematic_device() for callers that cannot allocate
 * device memory: a real-time loop whose memory is reserved up front, a
 * process whose memory-pool policy forbids new device allocations, code that
 * must not enter the driver's allocator while other work runs.  It calls no
 * cudaMalloc / cudaFree: its working memory (instance record and frame masks,
 * about 390 KB) is one static device array that every GPU loading this
 * library keeps until the process exits.  Every pointer is device memory:
 * the frame's width*height class ids, its n_classes costs (cost < 0 =
 * obstacle), the width*height heading and cost grids the candidates start
 * from, the n candidates and out4 (n float4); *probes, when given, is added
 * to.  Frames larger than 1024 x 1024 cells are rejected with an error; a
 * candidate whose start cell lies outside the frame gets the rejected row
 * (-1, -1, 0, 0) and the call returns an error.  The first call on a device
 * looks up the array's address on that device and keeps it, so the entry
 * point must not be used on a device after cudaDeviceReset.  The call runs
 * on `stream` (NULL = default), copies its small error flags back and
 * synchronises that stream before it returns, so it must not be called while
 * `stream` is being captured into a CUDA graph.  Calls share the array:
 * calls from this library's callers are serialised by a lock, but work that
 * overlaps on the GPU from another route (e.g. the same library loaded twice
 * in one process) would race. */
int fastrrt_candidates_kinematic_noalloc(int width, int height, const uint8_t *class_ids,
                                         const float *class_costs, int n_classes,
                                         const float *heading_grid, const float *cost_grid,
                                         int min_dist_x, int min_dist_z, int lowerBound_x,
                                         int lowerBound_z, int upperBound_x, int upperBound_z,
                                         double max_steering_rad, double lr_m, int n,
                                         const int32_t *sx, const int32_t *sz, const float *steer,
                                         const float *length, float velocity_m_s, float *out4,
                                         uint64_t *probes, void *stream);
/* Test hooks of the bounded waits, no counterpart in the reference.  The
 * per-candidate kernels stage the frame masks in shared memory with a bulk
 * copy and wait for it at most `rounds` mbarrier polls (default 4194304);
 * a block that gives up counts a timeout, lets its copy finish (a second
 * bounded wait) and reads the global masks, with the same results.
 * fastrrt_debug_stage_timeouts returns the count since its last call and
 * resets it.  0 or -1. */
int fastrrt_debug_set_stage_wait_limit(int64_t rounds);
int fastrrt_debug_stage_timeouts(uint64_t *count);
/* __computeFeasibleForAngle (src/cuda/path_feasible.cu:18-78). Host buffers. */
int fastrrt_candidates_feasible(void *ctx, int n, const int32_t *x, const int32_t *z,
                                const float *angle, int32_t *out, uint64_t *probes);

/* ---- part 4: batched planner -------------------------------------------- */

/* One planning request: FastRRT(ego) + set_plan_data + search_init + loop
 * until goal, as a batch slot.  No counterpart in the reference (it plans one
 * instance per CudaGraph). */
typedef struct {
    int width, height;
    const uint8_t *class_ids;  /* host, width*height */
    const float *class_costs;
    int n_classes;
    float perception_w_m, perception_h_m;
    float max_steering_deg;
    float vehicle_length_m;
    float max_curvature;       /* < 0: derived (graph.cu:297-303) */
    int lb_x, lb_z, ub_x, ub_z;
    int start_x, start_z;
    float start_heading;
    int goal_x, goal_z;
    float goal_heading;
    float velocity_m_s;
    int min_dist_x, min_dist_z;
    float max_path_size;
    float dist_to_goal_tol;
    float heading_tol_rad;
    uint64_t seed;
    int smart;
    int max_iterations;        /* 0 = unlimited */
    int class_ids_on_device;   /* class_ids points to device memory */
    int timeout_ms;            /* > 0: the request fails this long after it starts
                                  planning (device clock); 0 = the call's timeout */
} fastrrt_request;

void *fastrrt_batch_create(int n_slots, int max_width, int max_height);
/* A batched planner whose slots take device memory by their frame's size:
 * one arena of budget_bytes (allocated here) from which a slot gets its
 * storage (node grid, frame copy, masks, scratch: fastrrt_slot_bytes of its
 * frame) when a request is admitted, and to which it returns the storage when
 * the slot is released or, in fastrrt_batch_serve, harvested.  Admission
 * fails with a "budget exhausted" error when the arena has no room;
 * fastrrt_batch_serve then keeps the request (and those after it) waiting
 * until finished requests free memory.  No counterpart in the reference
 * (one CudaGraph of fixed size per planner, src/cuda/graph.cu:249-280). */
void *fastrrt_batch_create_budget(int max_slots, int max_width, int max_height, uint64_t budget_bytes);
/* device memory of one slot's storage for a width x height frame */
uint64_t fastrrt_slot_bytes(int width, int height);
/* the arena's budget, the bytes slots hold now and the most they held (a
 * batch created without a budget reports its preallocated arena for all) */
int fastrrt_batch_memory(void *batch, uint64_t *budget, uint64_t *used, uint64_t *peak);
void fastrrt_batch_destroy(void *batch);
/* loads a request into a slot (frame upload, masks, goal precompute, start) */
int fastrrt_batch_admit(void *batch, int slot, const fastrrt_request *req, int timeout_ms);
/* loads n requests into slots 0..n-1 in one pass */
int fastrrt_batch_admit_many(void *batch, int n, const fastrrt_request *reqs, int timeout_ms);
/* runs iterations until every admitted slot is done or `max_launches` graph
 * launches ran; returns the number of launches */
int fastrrt_batch_run(void *batch, int max_launches, int check_every);
/* one graph launch (no host synchronisation) */
int fastrrt_batch_step(void *batch);
/* done flags, goal flags and loop counts of all slots (host arrays of n_slots) */
int fastrrt_batch_status(void *batch, int32_t *done, int32_t *goal, int32_t *loops);
/* extracts and validates the paths of the n listed slots; valid[k] = path
 * passed the validator, length[k] = coarse path length in cells */
int fastrrt_batch_collect(void *batch, int n, const int32_t *slots, int32_t *valid,
                          float *length, int32_t *path_n);
/* copies the last collected path of list entry k: up to cap (x, z, heading) */
int fastrrt_batch_path(void *batch, int k, float *xyh, int cap);
/* interpolate (src/interpolation.cpp:112-135) of the paths of the last
 * collected list, on the device: interpolateHermiteCurve between consecutive
 * waypoints with the reference's float arithmetic (cells from round(), the
 * heading of the curve's tangent), at most `cap` points per path; and the
 * curve-quality metrics of each interpolated curve as the reference's
 * tests/python_dataset/curve_quality.py computes them (length, jerk of the
 * windowed direction, tangential discontinuity of the windowed heading above
 * 15 degrees from the start heading; jerk NaN and discontinuity -1 where its
 * arithmetic is undefined: fewer than 3 points or a window beyond the
 * curve).  length / jerk / tan_disc get one value per path (NULL to skip);
 * returns the number of paths or -1.  No counterpart in the reference ABI
 * (its interpolation runs on the host, interpolate_planned_path). */
int fastrrt_batch_interpolate(void *batch, int cap, float *length, float *jerk, int32_t *tan_disc);
/* the k-th interpolated path of the last fastrrt_batch_interpolate:
 * [x, z, heading] * m into xyh (at most cap points); returns m */
int fastrrt_batch_interpolated_path(void *batch, int k, float *xyh, int cap);
/* deactivates a slot; in a batch with a memory budget its storage returns to
 * the arena */
int fastrrt_batch_release(void *batch, int slot);
/* device time of the last fastrrt_batch_run, milliseconds */
float fastrrt_batch_last_ms(void *batch);
/* one batched planning pass: admits reqs into slots 0..n-1, loops until all
 * are done (at most max_launches graph launches), extracts and validates the
 * paths.  valid / length / latency_ms are per request (latency = admission
 * + the request's own loop time, device clock); *device_ms = the pass on the
 * device clock.  Returns the number of validated plans. */
int fastrrt_batch_plan(void *batch, int n, const fastrrt_request *reqs, int max_launches,
                       int check_every, int32_t *valid, float *length, float *latency_ms,
                       float *device_ms);
/* Served planning with continuous batching.  Request k arrives arrival_ms[k]
 * milliseconds after the call starts (NULL: all at once; non-decreasing). It
 * is admitted as soon as it has arrived and a slot is free, is planned in the
 * same graph launches as whatever else is in flight, and its slot is refilled
 * as soon as it finishes: goal reached, loop cap, or timeout_ms after it
 * started planning (device clock; a request's own timeout_ms wins).  Per
 * request (any output may be NULL): valid, coarse path length, latency from
 * arrival and from admission to finish (ms: the device clock's finish in
 * host time), loops run, and result_ms, the latency from arrival to the
 * moment its validated path was on the host (the harvest of its slot, every
 * check_every launches).  *wall_ms = the whole call on the host clock,
 * *device_ms = the same span between CUDA events on the planner's stream.
 * Returns the number of validated plans. */
int fastrrt_batch_serve(void *batch, int n, const fastrrt_request *reqs, const double *arrival_ms,
                        int timeout_ms, int check_every, int32_t *valid, float *length,
                        float *latency_ms, float *service_ms, int32_t *loops, double *wall_ms,
                        float *device_ms, float *result_ms);
/* launch shape of the iteration: blocks per SM of the sweep kernels (1..64,
 * default 8) and of the persistent expansion kernel (1..8, default 2); the
 * autotuner (fastrrt_b200/autotune.py) picks them */
int fastrrt_batch_set_launch(void *batch, int sweep_blocks_per_sm, int work_blocks_per_sm);
/* kernel timing mode (1 = on): iterations launch kernels one by one between
 * CUDA events instead of replaying the CUDA graph */
int fastrrt_batch_profile(void *batch, int on);
/* per-kernel device time (ms) and launch counts since profiling was turned
 * on: fastrrt_kernel_count() entries, the last one the admission-time reset
 * of the goal direct connections (which the iterations evaluate on demand) */
int fastrrt_batch_kernel_times(void *batch, double *ms, int64_t *launches);
int fastrrt_kernel_count(void);
/* footprint probes of the reference algorithm, summed over the slots of the
 * last admission: expansion, goal-connection search, goal direct-connection
 * evaluation */
int fastrrt_batch_probes(void *batch, uint64_t *expand, uint64_t *goal, uint64_t *precompute);
const char *fastrrt_kernel_name(int k);
/* inspection, no counterpart in the reference (whose eager pass fills these
 * arrays at set_plan_data, graph_direct_goal_connection.cu:169-227): the
 * goal direct connections of `slot`'s cells as evaluated so far, W x H each
 * (host arrays): flag 0 / 1, or 255 for a cell not evaluated yet; the cost
 * and heading of connected cells */
int fastrrt_batch_direct_connections(void *batch, int slot, uint8_t *flag, float *cost,
                                     float *heading);

/* ---- part 5: the learned expansion proposal ------------------------------
 * No counterpart in the reference.  A BF16 MLP (1030 -> 256 -> 256 -> 128,
 * ReLU, FP32 accumulation, tcgen05 tensor-core GEMMs) that proposes the
 * (steering, length) bin of an expansion from a 32 x 32 obstacle patch around
 * the parent (its heading frame, 2 px stride), the goal in that frame, the
 * distance to the goal, sin / cos of the heading and the steering limit.
 * Weights: w1 256 x 1040 (inputs 1030..1039 are padding), b1 256, w2
 * 256 x 256, b2 256, w3 128 x 256, b3 128; all f32 on the host. */
void *fastrrt_mlp_create(uint64_t seed, int max_batch);
void fastrrt_mlp_destroy(void *mlp);
int fastrrt_mlp_get_weights(void *mlp, float *w1, float *b1, float *w2, float *b2, float *w3,
                            float *b3);
int fastrrt_mlp_set_weights(void *mlp, const float *w1, const float *b1, const float *w2,
                            const float *b2, const float *w3, const float *b3);
/* logits (n x 128) of n host feature rows of 1030 floats */
int fastrrt_mlp_forward(void *mlp, int n, const float *X, float *logits);
/* mean cross-entropy gradients of a host batch (labels in 0..127) */
int fastrrt_mlp_gradients(void *mlp, int n, const float *X, const int32_t *labels, float *gw1,
                          float *gb1, float *gw2, float *gb2, float *gw3, float *gb3, float *loss);
/* Planner side.  With a network attached, each iteration lists up to cap
 * expansion candidates, computes their features and logits, and with
 * probability mix samples the (steering, length) of a candidate from the
 * network's softmax (the value uniform inside the bin); otherwise, and for
 * candidates beyond cap, the uniform draw of the reference.  The
 * kinematic and collision checks decide every expansion as before.
 * mlp == NULL detaches. */
int fastrrt_batch_set_proposal(void *batch, void *mlp, float mix, int cap);
/* After fastrrt_batch_collect / fastrrt_batch_plan: training rows of the
 * valid paths of that list, one per expansion on a path (features of the
 * parent, label = the bin of the draw that made the child), written at rows
 * offset.. of the device arrays X_bf16 (rows of 1040 bf16) and labels (int32),
 * at most cap rows in all.  Returns the rows written. */
int fastrrt_batch_log_paths(void *batch, void *X_bf16, int32_t *labels, int offset, int cap);
/* The same for every accepted expansion of the solved requests of that list:
 * one row per node of the final graph but the start (features of its parent,
 * label = the bin of the draw that made it), in no particular order. */
int fastrrt_batch_log_nodes(void *batch, void *X_bf16, int32_t *labels, int offset, int cap);
/* Adam training on a device dataset: X_bf16 n x 1040 bf16 rows, labels n
 * int32 (device pointers); *last_loss = mean loss of the last batch */
int fastrrt_mlp_train(void *mlp, const void *X_bf16, const int32_t *labels, int n, int epochs,
                      int batch, float lr, uint64_t seed, float *last_loss);
/* The network's GEMM on device buffers (synchronous on `stream`, NULL = the
 * default stream): C (M x N) = epilogue(sum_k A(m, k) B(k, n)), bf16 operands,
 * f32 accumulation in TMEM.  A(m, k) = A[m * lda + k], or A[k * lda + m] with
 * transA; B(k, n) = B[n * ldb + k] (out x in weights), or B[k * ldb + n] with
 * transB.  Epilogue: + bias[n] (f32, optional), ReLU when relu, times
 * (mask[m * ldm + n] > 0) when mask (bf16, optional); the result goes to Cf
 * (f32) or Cb (bf16), exactly one of them, rows ldc apart.  M is capped by
 * *dM when dM (device int) is given.  A and B start on 16 bytes with lda,
 * ldb multiples of 8.  split_ws (device, split_floats floats, optional): a
 * raw f32 product of few output tiles and a long K is split over K into
 * partial sums there and reduced in a fixed order. */
int fastrrt_gemm_bf16(int M, int N, int K, const void *A, int lda, int transA, const void *B, int ldb,
                      int transB, const float *bias, int relu, const void *mask, int ldm, float *Cf, void *Cb,
                      int ldc, const int *dM, float *split_ws, uint64_t split_floats, void *stream);

#ifdef __cplusplus
}
#endif
#endif
