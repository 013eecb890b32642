/*
 * fastrrt_oracle.h -- CPU restatement of the FastRRT planning hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker used by tests/,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py.  No product
 * code path links, imports or calls it.
 *
 * Every function restates the behaviour of the reference (out0/FastRRT)
 * function cited beside it (file:line within that project).  The reference
 * depends on the un-vendored `driveless` library; the facts this oracle
 * assumes about it (truncating TO_INT, double PI/HALF_PI/TO_DEG constants,
 * class id in the frame's first channel, zero-initialised node grid, frame
 * footprint equal to the planner's) are pinned only where the reference's
 * own unit tests pin them.
 *
 * Two arithmetic modes exist (orc_set_fp_mode):
 *   ORC_FP_HOST   : every float/double operation rounded separately, and
 *                   float->int conversions as the host CPU does them.  This
 *                   is what the reference's `__device__ __host__` functions
 *                   compute when compiled for the host.
 *   ORC_FP_DEVICE : the multiply-add steps that the CUDA compiler contracts
 *                   into fused multiply-adds are fused here too, and
 *                   float->int conversions saturate with NaN -> 0 as the GPU
 *                   conversion instruction does.  Transcendentals still come
 *                   from the host libm, so this mode is close to, not
 *                   identical with, the GPU.
 */
#ifndef FASTRRT_ORACLE_H
#define FASTRRT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* node types (include/graph.h:31-36) */
#define ORC_NULL 0
#define ORC_NODE 1
#define ORC_TEMP 2
#define ORC_PROCESSING 3
#define ORC_COLLISION 4
#define ORC_CONNECT_TO_GOAL 5

#define ORC_FP_HOST 0
#define ORC_FP_DEVICE 1

typedef struct { float x, y, z, w; } orc_f4;

/* BEV frame: the reference's SearchFrame stores float3 per pixel
 * (class id, distance to goal, traversability bits).  The class id is held
 * as uint8 here; `trav` is the third channel (NULL = all zero), `dist` the
 * second (NULL = none). */
typedef struct {
    int W, H;
    const uint8_t *cls;
    const float *class_costs;
    int n_classes;
    const int32_t *trav;
    const float *dist;
} orc_frame;

/* flag bits of orc_direct_connection's `safe_zone_checked` argument: the
 * reference's isSafeZoneChecked and isDistanceToGoalProcessed
 * (graph_direct_goal_connection.cu:16) */
#define ORC_SAFE_ZONE_CHECKED 1
#define ORC_DISTANCE_PROCESSED 2

/* search-space parameters (graph.cu:306-314, FRAME_PARAM_*) */
typedef struct {
    int W, H;
    int mdx, mdz;            /* half footprint = TO_INT(min_dist / 2) */
    int lbx, lbz, ubx, ubz;  /* ego box, skipped by the footprint probe */
} orc_search;

/* physical parameters (graph.cu:286-304, PHYSICAL_PARAMS_*) */
typedef struct {
    double rate_w, inv_rate_w, rate_h, inv_rate_h;
    double max_steer_rad, max_steer_deg, lr, max_curvature;
} orc_physical;

/* node grid: the reference's int4 graph + float4 graphData + float3 goal
 * direct-connection frames (graph.h:45-48), held as separate arrays */
typedef struct {
    int W, H;
    int32_t *px, *pz, *type, *child;
    float *heading, *cost, *intrinsic, *direct;
    float *gd_flag, *gd_heading, *gd_cost;
    float og_x, og_z, og_h;
    int goal_reached, node_collision;
    int density_w, density_h, density_size;
    uint32_t *region_count;
    orc_search sp;
    orc_physical pp;
    int has_pp;
} orc_graph;

typedef struct {
    int start_x, start_z; float start_heading;
    int goal_x, goal_z; float goal_heading;
    float velocity;
    float max_path_size;
    float dist_tol;
    float heading_tol;
    uint64_t seed;
} orc_plan_params;

typedef struct {
    orc_graph *g;
    const orc_frame *f;
    orc_plan_params pp;
    int last_expanded;
    uint32_t iter;            /* RNG counter: number of expansions done */
    int smart;
    int has_plan;
    long long probes;         /* footprint probes executed (reference early exit):
                                 expansion and path optimisation */
    long long probes_goal;    /* ... of the goal-connection search */
    long long probes_pre;     /* ... of the goal direct-connection precompute */
} orc_planner;

/* ---- arithmetic mode ---------------------------------------------------- */
void orc_set_fp_mode(int mode);
int orc_get_fp_mode(void);

/* ---- RNG: Philox4x32-10 (Salmon et al., SC'11), counter = (pos, iter) ---- */
void orc_philox4x32(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                    uint32_t k0, uint32_t k1, uint32_t out[4]);
float orc_u01(uint32_t r);
void orc_draw_expansion(uint64_t seed, uint32_t pos, uint32_t iter,
                        float max_steer, float max_path, float *steer, float *len);

/* ---- parameters ------------------------------------------------------- */
void orc_physical_params(orc_physical *pp, int W, int H, float pw_m, float ph_m,
                         double max_steer_rad, float vehicle_len, float max_curvature);
void orc_search_params(orc_search *sp, int W, int H, int min_dist_x, int min_dist_z,
                       int lbx, int lbz, int ubx, int ubz);

/* ---- per-candidate functions ------------------------------------------- */
int orc_feasible(const orc_frame *f, const orc_search *sp, int x, int z,
                 float angle, long long *probes);
orc_f4 orc_kinematic_path(const orc_graph *g, const orc_frame *f, int sx, int sz,
                          float steering, float path_size, float velocity,
                          long long *probes, int *steps);
/* the pose after `steps` integration steps, in FP64 and in FP32 */
void orc_kinematic_f64_pose(const orc_graph *g, int sx, int sz, float steering,
                            float velocity, int steps, double out_pose[3]);
void orc_kinematic_f32_pose(const orc_graph *g, int sx, int sz, float steering,
                            float velocity, int steps, double out_pose[3]);
float orc_direct_connection(const orc_graph *g, const orc_frame *f, const orc_search *sp,
                            float max_curvature, int x, int z, float local_heading,
                            int goal_x, int goal_z, float goal_heading,
                            int safe_zone_checked, long long *probes);
float orc_hermite_test(const orc_graph *g, const orc_frame *f, const float *frame_dist,
                       int x, int z, int goal_x, int goal_z, float goal_heading,
                       int compute_distance, float max_curvature, long long *probes);
double orc_compute_heading(int x1, int z1, int x2, int z2);
int orc_kinematic_connection(const orc_graph *g, const orc_frame *f, int sx, int sz,
                             int ex, int ez, float velocity, double *final_heading,
                             double *path_cost);
float orc_max_curvature_default(float max_steer_rad, float vehicle_len);

/* ---- node grid -------------------------------------------------------- */
orc_graph *orc_graph_new(int W, int H);
void orc_graph_free(orc_graph *g);
void orc_graph_set_coordinate_start(orc_graph *g, int x, int z, float heading);
void orc_graph_add(orc_graph *g, int x, int z, float heading, int ppx, int ppz, float cost);
void orc_graph_add_temporary(orc_graph *g, int x, int z, float heading, int ppx, int ppz, float cost);
void orc_graph_remove(orc_graph *g, int x, int z);
void orc_graph_clear(orc_graph *g);
uint32_t orc_graph_count(const orc_graph *g, int type);
uint32_t orc_graph_count_all(const orc_graph *g);
void orc_graph_set_collision(orc_graph *g, int x, int z, int npx, int npz, float heading, float cost);
void orc_graph_get_parent(const orc_graph *g, int x, int z, int *ppx, int *ppz);
void orc_graph_solve_collisions(orc_graph *g);
void orc_graph_accept(orc_graph *g);
void orc_graph_density(orc_graph *g);
int orc_graph_check_goal_reached(orc_graph *g, const orc_frame *f, int gx, int gz,
                                 float gh, float tol, float max_err);
int orc_graph_find_best_node(const orc_graph *g, const orc_frame *f, float heading,
                             float radius, int x, int z, float max_err, int *bx, int *bz);
int orc_graph_is_consistent(const orc_graph *g);
void orc_graph_process_direct_goal(orc_graph *g, const orc_frame *f, const orc_search *fsp,
                                   int goal_x, int goal_z, float goal_heading,
                                   float max_curvature, long long *probes);
/* best node->precomputed cell connection; returns 1 when found and fills
 * parent (x, z, heading, seg cost) and child (x, z, heading, total) */
int orc_graph_best_goal_connection(orc_graph *g, const orc_frame *f, float radius,
                                   int safe_zone_checked, orc_f4 out[2], long long *probes);
/* one expansion pass (uniform or density-gated) with snapshot semantics and
 * lowest-cell-index-wins conflicts; returns the number of candidates run */
int orc_graph_expand(orc_graph *g, const orc_frame *f, uint64_t seed, uint32_t iter,
                     float max_path, float velocity, int smart, int frontier,
                     int force_expand, long long *probes);

/* ---- planner (fastrrt.cpp:35-232) --------------------------------------- */
orc_planner *orc_planner_new(int W, int H, float pw_m, float ph_m, float max_steer_deg,
                             float vehicle_len, int lbx, int lbz, int ubx, int ubz,
                             float max_curvature);
void orc_planner_free(orc_planner *p);
void orc_planner_set_plan_data(orc_planner *p, const orc_frame *f, const orc_plan_params *pp,
                               int min_dist_x, int min_dist_z);
void orc_planner_search_init(orc_planner *p);
int orc_planner_loop(orc_planner *p, int smart);
int orc_planner_goal_reached(orc_planner *p);
/* coarse path; writes up to cap waypoints (x, z, heading) and returns the count */
int orc_planner_path(orc_planner *p, float *xyh, int cap);
int orc_planner_optimize(orc_planner *p);
int orc_interpolate(const float *xyh, int n, int W, int H, float *out, int cap);
/* run search_init + loop until goal or max_iter; returns 1 on success */
int orc_plan(orc_planner *p, int smart, int max_iter, int *iters);
/* path validator: DAG, per-waypoint footprint, curvature bound, goal tolerance */
int orc_validate_path(orc_planner *p, const float *xyh, int n);
/* the same checks without the graph's own (DAG, parent links): for paths
 * produced elsewhere, e.g. by the GPU planner */
int orc_validate_waypoints(orc_planner *p, const float *xyh, int n);

/* batch helpers (OpenMP over candidates) */
void orc_kinematic_batch(const orc_graph *g, const orc_frame *f, int n, const int32_t *sx,
                         const int32_t *sz, const float *steer, const float *len, float velocity,
                         float *out4, long long *probes, int32_t *steps);
void orc_feasible_batch(const orc_frame *f, const orc_search *sp, int n, const int32_t *x,
                        const int32_t *z, const float *a, int32_t *out, long long *probes);
void orc_direct_batch(const orc_graph *g, const orc_frame *f, const orc_search *sp, float maxc,
                      int n, const int32_t *x, const int32_t *z, const float *lh,
                      const int32_t *gx, const int32_t *gz, const float *gh, int safe,
                      float *out, long long *probes);

/* CPU baseline: plans `n` instances with OpenMP (one planner per thread) */
int orc_plan_batch(int n, int W, int H, const uint8_t *cls, const float *class_costs,
                   int n_classes, const int32_t *start_goal, const uint64_t *seeds,
                   float pw_m, float ph_m, float max_steer_deg, float vehicle_len,
                   int min_dist_x, int min_dist_z, float velocity, float max_path,
                   float dist_tol, float heading_tol, int timeout_ms, int max_iter,
                   int smart, int threads, int32_t *ok, int32_t *iters, float *path_cost,
                   double *ms);

#ifdef __cplusplus
}
#endif
#endif
