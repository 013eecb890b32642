/*
 * fastrrt_oracle.c -- CPU restatement of the FastRRT planning hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see fastrrt_oracle.h).  Compiled with
 * -ffp-contract=off so that ORC_FP_HOST rounds every operation separately.
 * Reference citations are file:line within out0/FastRRT.
 */
#include "fastrrt_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* driveless constants (assumed double precision; not in the reference tree) */
#define ORC_PI 3.14159265358979323846
#define ORC_HALF_PI (ORC_PI / 2.0)
#define ORC_TO_DEG (180.0 / ORC_PI)
/* math_constants.h values used by compute_path_heading (kinematics.cu:75-93) */
#define ORC_CUDART_PI 3.1415926535897931e+0
#define ORC_CUDART_PIO2_HI 1.5707963267948966e+0

#define ORC_BIG_COST 99999999999LL
#define ORC_REGION 128

static int g_fp_mode = ORC_FP_HOST;

void orc_set_fp_mode(int mode) { g_fp_mode = mode; }
int orc_get_fp_mode(void) { return g_fp_mode; }

/* float -> int with the reference's TO_INT (truncation).  The GPU conversion
 * saturates and maps NaN to 0; x86 returns INT_MIN for both. */
static inline int toi_f(float v)
{
    if (v != v)
        return g_fp_mode == ORC_FP_DEVICE ? 0 : INT32_MIN;
    if (v >= 2147483648.0f)
        return g_fp_mode == ORC_FP_DEVICE ? INT32_MAX : INT32_MIN;
    if (v < -2147483648.0f)
        return INT32_MIN;
    return (int)v;
}

static inline int toi_d(double v)
{
    if (v != v)
        return g_fp_mode == ORC_FP_DEVICE ? 0 : INT32_MIN;
    if (v >= 2147483648.0)
        return g_fp_mode == ORC_FP_DEVICE ? INT32_MAX : INT32_MIN;
    if (v <= -2147483649.0)
        return INT32_MIN;
    return (int)v;
}

/* x + a*b as the device build computes `x += a * b` (one fused rounding) */
static inline float madd_f(float a, float b, float x)
{
    return g_fp_mode == ORC_FP_DEVICE ? fmaf(a, b, x) : x + a * b;
}

/* ------------------------------------------------------------------------ */
/* RNG                                                                      */
/* ------------------------------------------------------------------------ */

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
 * easy as 1, 2, 3", SC 2011).  The reference seeds one cuRAND XORWOW state
 * per cell from the wall clock (random_number_gen.cu:5-45), which is not
 * reproducible; this counter-based generator draws the same two uniforms
 * per expansion (steering, then length) from (seed, cell, iteration). */
void orc_philox4x32(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                    uint32_t k0, uint32_t k1, uint32_t out[4])
{
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* uniform in (0, 1] like curand_uniform: ((r >> 8) + 1) * 2^-24, exact */
float orc_u01(uint32_t r) { return (float)((r >> 8) + 1u) * (1.0f / 16777216.0f); }

#define ORC_RNG_TAG 0x46525254u /* "FRRT" */

void orc_draw_expansion(uint64_t seed, uint32_t pos, uint32_t iter,
                        float max_steer, float max_path, float *steer, float *len)
{
    uint32_t r[4];
    orc_philox4x32(pos, iter, ORC_RNG_TAG, 0u, (uint32_t)seed, (uint32_t)(seed >> 32), r);
    float u0 = orc_u01(r[0]);
    float u1 = orc_u01(r[1]);
    /* generateRandomNeg (random_number_gen.cu:18-20) */
    *steer = (2.0f * u0 - 1.0f) * max_steer;
    /* generateRandom(state, pos, 5.0, maxPathSize) (random_number_gen.cu:14-16,
     * graph_expansion.cu:177-180) */
    float l = max_path * u1;
    *len = l > 5.0f ? l : 5.0f;
}

/* ------------------------------------------------------------------------ */
/* parameters                                                               */
/* ------------------------------------------------------------------------ */

/* CudaGraph::setPhysicalParams (graph.cu:286-304), including the
 * sqrtf(4 + t) curvature formula (t, not t squared). */
void orc_physical_params(orc_physical *pp, int W, int H, float pw_m, float ph_m,
                         double max_steer_rad, float vehicle_len, float max_curvature)
{
    pp->rate_w = W / pw_m;
    pp->inv_rate_w = pw_m / W;
    pp->rate_h = H / ph_m;
    pp->inv_rate_h = ph_m / H;
    pp->max_steer_rad = max_steer_rad;
    pp->max_steer_deg = max_steer_rad * ORC_TO_DEG;
    pp->lr = vehicle_len / 2;
    const float t = tanf((float)max_steer_rad);
    if (max_curvature < 0)
        pp->max_curvature = 2 * t / (0.5 * vehicle_len * sqrtf(4 + t));
    else
        pp->max_curvature = max_curvature;
}

float orc_max_curvature_default(float max_steer_rad, float vehicle_len)
{
    const float t = tanf(max_steer_rad);
    return (float)(2 * t / (0.5 * vehicle_len * sqrtf(4 + t)));
}

/* CudaGraph::setSearchParams (graph.cu:306-314): min distances are halved */
void orc_search_params(orc_search *sp, int W, int H, int min_dist_x, int min_dist_z,
                       int lbx, int lbz, int ubx, int ubz)
{
    sp->W = W;
    sp->H = H;
    sp->mdx = toi_f((float)min_dist_x / 2);
    sp->mdz = toi_f((float)min_dist_z / 2);
    sp->lbx = lbx;
    sp->lbz = lbz;
    sp->ubx = ubx;
    sp->ubz = ubz;
}

/* ------------------------------------------------------------------------ */
/* footprint                                                                */
/* ------------------------------------------------------------------------ */

/* __computeFeasibleForAngle (path_feasible.cu:18-78).  isAllAngleFeasible
 * (path_feasible.cu:13-16) reads `TO_INT(frame.z) & 256 > 0`, which C
 * precedence parses as `& (256 > 0)`, i.e. bit 0; kept as written. */
int orc_feasible(const orc_frame *f, const orc_search *sp, int x, int z,
                 float angle, long long *probes)
{
    const int W = sp->W, H = sp->H;
    const long pos = (long)z * W + x;
    if (f->trav && (f->trav[pos] & 1))
        return 1;

    const float c = cosf(angle);
    const float s = sinf(angle);
    long long n = 0;
    int ok = 1;
    for (int i = -sp->mdz; i <= sp->mdz && ok; i++) {
        const float fi = (float)i;
        for (int j = -sp->mdx; j <= sp->mdx; j++) {
            const float fj = (float)j;
            int xl, zl;
            if (g_fp_mode == ORC_FP_DEVICE) {
                xl = toi_f(fmaf(fj, c, -(fi * s)) + (float)x);
                zl = toi_f(fmaf(fj, s, fi * c) + (float)z);
            } else {
                xl = toi_f(fj * c - fi * s + (float)x);
                zl = toi_f(fj * s + fi * c + (float)z);
            }
            n++;
            if (xl < 0 || xl >= W)
                continue;
            if (zl < 0 || zl >= H)
                continue;
            if (xl >= sp->lbx && xl <= sp->ubx && zl >= sp->ubz && zl <= sp->lbz)
                continue;
            const int cls = f->cls[(long)zl * W + xl];
            if (f->class_costs[cls] < 0) {
                ok = 0;
                break;
            }
        }
    }
    if (probes)
        *probes += n;
    return ok;
}

/* ------------------------------------------------------------------------ */
/* kinematics                                                               */
/* ------------------------------------------------------------------------ */

static inline float intrinsic_at(const orc_graph *g, int x, int z)
{
    return g->intrinsic[(long)z * g->W + x];
}

/* check_kinematic_new_path (kinematics.cu:123-231).  Pixel-unit pose
 * (convert_waypoint_to_map_pose, kinematics.cu:54-59), beta = atanf(steer/2)
 * with the constant 2, heading increment ds*cos(beta)*steer/(2*lr) with lr in
 * metres, one cost unit per new cell, footprint check at each new cell. */
orc_f4 orc_kinematic_path(const orc_graph *g, const orc_frame *f, int sx, int sz,
                          float steering, float path_size, float velocity,
                          long long *probes, int *steps)
{
    orc_f4 fail = {-1.0f, -1.0f, 0.0f, 0.0f};
    if (steps)
        *steps = 0;
    if (!g->has_pp)
        return fail;
    const double maxSteering = g->pp.max_steer_rad;
    const double lr = g->pp.lr;
    const int W = g->sp.W, H = g->sp.H;

    float x = g->og_z - (float)sz;
    float y = (float)sx - g->og_x;

    if (steering > maxSteering)
        steering = (float)maxSteering;
    else if (steering < -maxSteering)
        steering = (float)(-maxSteering);

    const float steer = tanf(steering);
    const float dt = 0.1f;
    const float ds = velocity * dt;
    const float beta = atanf(steer / 2);
    const float hif = (float)((double)(ds * cosf(beta) * steer) / (2 * lr));

    const int maxSize = toi_f(path_size) + 1;
    int size = 0;
    int last_x = sx, last_z = sz;
    const long startPos = (long)sz * W + sx;
    float heading = g->heading[startPos];
    float nodeCost = g->cost[startPos];
    int loop_count = 0;
    const int loop_max = toi_f((float)(100 * maxSize) / dt);
    int nsteps = 0;

    while (size < maxSize) {
        if (loop_count++ > loop_max)
            break;
        x = madd_f(ds, cosf(heading + beta), x);
        y = madd_f(ds, sinf(heading + beta), y);
        heading += hif;
        nsteps++;
        /* convert_map_pose_to_waypoint (kinematics.cu:25-46), in double */
        const int lpx = toi_d((double)g->og_x + (double)y);
        const int lpz = toi_d((double)g->og_z - (double)x);
        if (lpx == last_x && lpz == last_z)
            continue;
        if (lpx < 0 || lpx >= W)
            break;
        if (lpz < 0 || lpz >= H)
            break;
        size += 1;
        nodeCost += intrinsic_at(g, lpx, lpz) + 1;
        if (!orc_feasible(f, &g->sp, lpx, lpz, heading, probes)) {
            if (steps)
                *steps = nsteps;
            return fail;
        }
        last_x = lpx;
        last_z = lpz;
    }
    if (steps)
        *steps = nsteps;
    if (size < 1)
        return fail;
    orc_f4 r = {(float)last_x, (float)last_z, nodeCost, heading};
    return r;
}

/* FP64 shadow of the same integration, for pose-error reporting */
void orc_kinematic_f64_pose(const orc_graph *g, int sx, int sz, float steering,
                            float velocity, int steps, double out_pose[3])
{
    const double maxSteering = g->pp.max_steer_rad, lr = g->pp.lr;
    double st = steering;
    if (st > maxSteering)
        st = maxSteering;
    else if (st < -maxSteering)
        st = -maxSteering;
    double x = (double)g->og_z - sz, y = (double)sx - g->og_x;
    const double steer = tan(st), ds = (double)velocity * 0.1;
    const double beta = atan(steer / 2), hif = ds * cos(beta) * steer / (2 * lr);
    double heading = g->heading[(long)sz * g->W + sx];
    for (int k = 0; k < steps; k++) {
        x += ds * cos(heading + beta);
        y += ds * sin(heading + beta);
        heading += hif;
    }
    out_pose[0] = x;
    out_pose[1] = y;
    out_pose[2] = heading;
}

/* the FP32 pose after `steps` steps (same arithmetic as orc_kinematic_path) */
void orc_kinematic_f32_pose(const orc_graph *g, int sx, int sz, float steering,
                            float velocity, int steps, double out_pose[3])
{
    const double maxSteering = g->pp.max_steer_rad, lr = g->pp.lr;
    float x = g->og_z - (float)sz, y = (float)sx - g->og_x;
    if (steering > maxSteering)
        steering = (float)maxSteering;
    else if (steering < -maxSteering)
        steering = (float)(-maxSteering);
    const float steer = tanf(steering), dt = 0.1f, ds = velocity * dt;
    const float beta = atanf(steer / 2);
    const float hif = (float)((double)(ds * cosf(beta) * steer) / (2 * lr));
    float heading = g->heading[(long)sz * g->W + sx];
    for (int k = 0; k < steps; k++) {
        x = madd_f(ds, cosf(heading + beta), x);
        y = madd_f(ds, sinf(heading + beta), y);
        heading += hif;
    }
    out_pose[0] = x;
    out_pose[1] = y;
    out_pose[2] = heading;
}

/* compute_path_heading (kinematics.cu:75-93) */
static double path_heading(double p1x, double p1y, double p2x, double p2y)
{
    double dy = p2y - p1y, dx = p2x - p1x;
    if (dy >= 0 && dx > 0)
        return atan(dy / dx);
    else if (dy >= 0 && dx < 0)
        return ORC_CUDART_PI - atan(dy / fabs(dx));
    else if (dy < 0 && dx > 0)
        return -atan(fabs(dy) / dx);
    else if (dy < 0 && dx < 0)
        return atan(dy / dx) - ORC_CUDART_PI;
    else if (dx == 0 && dy > 0)
        return ORC_CUDART_PIO2_HI;
    else if (dx == 0 && dy < 0)
        return -ORC_CUDART_PIO2_HI;
    return 0.0;
}

static double clipd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* check_kinematic_connection_start_end (kinematics.cu:233-306) */
int orc_kinematic_connection(const orc_graph *g, const orc_frame *f, int sx, int sz,
                             int ex, int ez, float velocity, double *final_heading,
                             double *path_cost)
{
    double ddx = ex - sx, ddz = ez - sz;
    double distance = sqrt(ddx * ddx + ddz * ddz);
    const double lr = g->pp.lr, maxSteering = g->pp.max_steer_rad;
    const int W = g->sp.W;
    double smx = g->og_z - (float)sz, smy = (float)sx - g->og_x;
    double emx = g->og_z - (float)ez, emy = (float)ex - g->og_x;
    double dt = 0.1;
    double heading = g->heading[(long)sz * W + sx];
    double ph = path_heading(smx, smy, emx, emy);
    double steering = clipd(ph - heading, -maxSteering, maxSteering);
    double ds = velocity * dt;
    int total_steps = toi_d(distance / ds);
    double nx = smx, ny = smy;
    int lx = sx, lz = sz;
    double bestEndDist = distance;
    *final_heading = 0;
    *path_cost = 0;
    float curr_cost = 0;
    for (int i = 0; i < total_steps; i++) {
        double steer = tan(steering);
        double beta = atan(steer / lr);
        nx += ds * cos(heading + beta);
        ny += ds * sin(heading + beta);
        heading += ds * cos(beta) * steer / (2 * lr);
        ph = path_heading(nx, ny, emx, emy);
        steering = clipd(ph - heading, -maxSteering, maxSteering);
        double dx2 = emx - nx, dy2 = emy - ny;
        double dist = sqrt(dx2 * dx2 + dy2 * dy2);
        int npx = toi_d((double)g->og_x + ny);
        int npz = toi_d((double)g->og_z - nx);
        if (npx == lx && npz == lz)
            continue;
        curr_cost += intrinsic_at(g, npx, npz) + 1;
        if (bestEndDist < dist) {
            *final_heading = heading;
            *path_cost = curr_cost;
            return bestEndDist <= 2;
        }
        if (!orc_feasible(f, &g->sp, lx, lz, (float)heading, NULL))
            return 0;
        lx = npx;
        lz = npz;
        bestEndDist = dist;
    }
    return 1;
}

/* ------------------------------------------------------------------------ */
/* Hermite connections                                                      */
/* ------------------------------------------------------------------------ */

/* computeHeading (graph.cu:219-234): atan2f on doubles narrowed to float */
double orc_compute_heading(int x1, int z1, int x2, int z2)
{
    double dz = z2 - z1, dx = x2 - x1;
    if (dx == 0 && dz == 0)
        return 0;
    double v1 = 0;
    if (dz != 0)
        v1 = atan2f((float)-dz, (float)dx);
    else
        v1 = atan2f(0.0f, (float)dx);
    return ORC_HALF_PI - v1;
}

/* checkDirectConnectionToGoal (graph_direct_goal_connection.cu:16-167),
 * with isDistanceToGoalProcessed = false (the only value FastRRT passes).
 * Double Hermite basis, curvature |x'z''-z'x''|/(x'^2+z'^2)^1.5, footprint at
 * each new cell, success requires `last_x == goal_x || last_z == goal_z`.
 * The safe-zone test reads the traversability bits of the START cell. */
float orc_direct_connection(const orc_graph *g, const orc_frame *f, const orc_search *sp,
                            float max_curvature, int x, int z, float local_heading,
                            int goal_x, int goal_z, float goal_heading,
                            int safe_zone_checked, long long *probes)
{
    const int W = sp->W, H = sp->H;
    const long pos = (long)z * W + x;
    const int dxi = goal_x - x, dzi = goal_z - z;
    /* isDistanceToGoalProcessed: the frame's distance channel
     * (graph_direct_goal_connection.cu:28-36) */
    const float distance = ((safe_zone_checked & ORC_DISTANCE_PROCESSED) && f->dist)
                               ? f->dist[pos]
                               : sqrtf((float)(dxi * dxi + dzi * dzi));
    const int numPoints = toi_f(distance);
    const float a1 = (float)(local_heading - ORC_HALF_PI);
    const float a2 = (float)(goal_heading - ORC_HALF_PI);
    const float t1x = distance * cosf(a1), t1y = distance * sinf(a1);
    const float t2x = distance * cosf(a2), t2y = distance * sinf(a2);
    int last_x = -1, last_z = -1;
    float nodeCost = g->cost[(long)z * g->W + x];
    const int trav = f->trav ? f->trav[pos] : 0;

    for (int i = 0; i < numPoints; ++i) {
        double t = (0.0 + i) / (numPoints - 1);
        double t2 = t * t, t3 = t2 * t;
        double h00 = 2 * t3 - 3 * t2 + 1;
        double h10 = t3 - 2 * t2 + t;
        double h01 = -2 * t3 + 3 * t2;
        double h11 = t3 - t2;
        double px = h00 * x + h10 * t1x + h01 * goal_x + h11 * t2x;
        double pz = h00 * z + h10 * t1y + h01 * goal_z + h11 * t2y;
        if (px < 0 || px >= W)
            continue;
        if (pz < 0 || pz >= H)
            continue;
        int cx = toi_d(px), cz = toi_d(pz);
        if (cx == last_x && cz == last_z)
            continue;
        if (cx < 0 || cx >= W)
            continue;
        if (cz < 0 || cz >= H)
            continue;
        nodeCost += intrinsic_at(g, cx, cz) + 1;
        double t00 = 6 * t2 - 6 * t;
        double t10 = 3 * t2 - 4 * t + 1;
        double t01 = -6 * t2 + 6 * t;
        double t11 = 3 * t2 - 2 * t;
        double ddx = t00 * x + t10 * t1x + t01 * goal_x + t11 * t2x;
        double ddz = t00 * z + t10 * t1y + t01 * goal_z + t11 * t2y;
        float heading = (float)(atan2f((float)ddz, (float)ddx) + ORC_HALF_PI);
        double d00 = 12 * t - 6;
        double d10 = 6 * t - 4;
        double d01 = -12 * t + 6;
        double d11 = 6 * t - 2;
        double dd2x = d00 * x + d10 * t1x + d01 * goal_x + d11 * t2x;
        double dd2z = d00 * z + d10 * t1y + d01 * goal_z + d11 * t2y;
        if (max_curvature > 0) {
            float k = (float)(fabs(ddx * dd2z - ddz * dd2x) / pow(ddx * ddx + ddz * ddz, 1.5));
            if (k > max_curvature)
                return -1;
        }
        last_x = cx;
        last_z = cz;
        if ((safe_zone_checked & ORC_SAFE_ZONE_CHECKED) && (trav & 0x100))
            continue;
        if (!orc_feasible(f, sp, last_x, last_z, heading, probes))
            return -1;
    }
    if (numPoints <= 0)
        return -1;
    if (last_x != goal_x && last_z != goal_z)
        return -1;
    return nodeCost;
}

/* cudaHermite (graph_hermite_connection.cu:13-141) behind the test-only
 * canConnectToGoal API: distance from the frame's distance channel unless
 * compute_distance, curvature divided by pow(v, 3 / 2) == pow(v, 1)
 * (integer division, :105), start cell counted as visited. */
float orc_hermite_test(const orc_graph *g, const orc_frame *f, const float *frame_dist,
                       int x, int z, int goal_x, int goal_z, float goal_heading,
                       int compute_distance, float max_curvature, long long *probes)
{
    const int W = g->sp.W, H = g->sp.H;
    const long pos = (long)z * W + x;
    float distance = frame_dist ? frame_dist[pos] : 0.0f;
    if (compute_distance) {
        const float dx = (float)(goal_x - x), dz = (float)(goal_z - z);
        distance = sqrtf(dx * dx + dz * dz);
    }
    const int numPoints = toi_f(distance);
    const float lh = g->heading[pos];
    const float a1 = (float)(lh - ORC_PI / 2);
    const float a2 = (float)(goal_heading - ORC_PI / 2);
    const float t1x = distance * cosf(a1), t1y = distance * sinf(a1);
    const float t2x = distance * cosf(a2), t2y = distance * sinf(a2);
    int last_x = x, last_z = z;
    float nodeCost = g->cost[pos];
    for (int i = 0; i < numPoints; ++i) {
        double t = (0.0 + i) / (numPoints - 1);
        double t2 = t * t, t3 = t2 * t;
        double h00 = 2 * t3 - 3 * t2 + 1, h10 = t3 - 2 * t2 + t;
        double h01 = -2 * t3 + 3 * t2, h11 = t3 - t2;
        double px = h00 * x + h10 * t1x + h01 * goal_x + h11 * t2x;
        double pz = h00 * z + h10 * t1y + h01 * goal_z + h11 * t2y;
        if (px < 0 || px >= W || pz < 0 || pz >= H)
            continue;
        int cx = toi_d(px), cz = toi_d(pz);
        if (cx == last_x && cz == last_z)
            continue;
        if (cx < 0 || cx >= W || cz < 0 || cz >= H)
            continue;
        nodeCost += intrinsic_at(g, cx, cz) + 1;
        double t00 = 6 * t2 - 6 * t, t10 = 3 * t2 - 4 * t + 1;
        double t01 = -6 * t2 + 6 * t, t11 = 3 * t2 - 2 * t;
        double ddx = t00 * x + t10 * t1x + t01 * goal_x + t11 * t2x;
        double ddz = t00 * z + t10 * t1y + t01 * goal_z + t11 * t2y;
        float heading = (float)(atan2f((float)ddz, (float)ddx) + ORC_HALF_PI);
        double d00 = 12 * t - 6, d10 = 6 * t - 4, d01 = -12 * t + 6, d11 = 6 * t - 2;
        double dd2x = d00 * x + d10 * t1x + d01 * goal_x + d11 * t2x;
        double dd2z = d00 * z + d10 * t1y + d01 * goal_z + d11 * t2y;
        if (max_curvature > 0) {
            float k = (float)(fabs(ddx * dd2z - ddz * dd2x) / pow(ddx * ddx + ddz * ddz, 1));
            if (k > max_curvature)
                return -2;
        }
        last_x = cx;
        last_z = cz;
        if (!orc_feasible(f, &g->sp, last_x, last_z, heading, probes))
            return -1;
    }
    if (numPoints <= 0)
        return -1;
    return nodeCost;
}

/* ------------------------------------------------------------------------ */
/* node grid                                                                */
/* ------------------------------------------------------------------------ */

orc_graph *orc_graph_new(int W, int H)
{
    orc_graph *g = (orc_graph *)calloc(1, sizeof(orc_graph));
    const size_t n = (size_t)W * H;
    g->W = W;
    g->H = H;
    g->px = (int32_t *)calloc(n, 4);
    g->pz = (int32_t *)calloc(n, 4);
    g->type = (int32_t *)calloc(n, 4);
    g->child = (int32_t *)calloc(n, 4);
    g->heading = (float *)calloc(n, 4);
    g->cost = (float *)calloc(n, 4);
    g->intrinsic = (float *)calloc(n, 4);
    g->direct = (float *)calloc(n, 4);
    g->gd_flag = (float *)calloc(n, 4);
    g->gd_heading = (float *)calloc(n, 4);
    g->gd_cost = (float *)calloc(n, 4);
    /* __initializeRegionDensity (graph_expansion_search_zones.cu:80-104) */
    g->density_w = W / ORC_REGION + 1;
    g->density_h = H / ORC_REGION + 1;
    g->density_size = g->density_w * g->density_h;
    g->region_count = (uint32_t *)calloc((size_t)g->density_size, 4);
    g->sp.W = W;
    g->sp.H = H;
    g->sp.lbx = g->sp.lbz = g->sp.ubx = g->sp.ubz = -1;
    /* default coordinate origin: frame centre (graph.cu:279) */
    orc_graph_set_coordinate_start(g, W / 2, H / 2, 0.0f);
    return g;
}

void orc_graph_free(orc_graph *g)
{
    if (!g)
        return;
    free(g->px); free(g->pz); free(g->type); free(g->child);
    free(g->heading); free(g->cost); free(g->intrinsic); free(g->direct);
    free(g->gd_flag); free(g->gd_heading); free(g->gd_cost);
    free(g->region_count);
    free(g);
}

void orc_graph_set_coordinate_start(orc_graph *g, int x, int z, float heading)
{
    g->og_x = (float)x;
    g->og_z = (float)z;
    g->og_h = heading;
}

static inline int in_limits(const orc_graph *g, int x, int z)
{
    return x >= 0 && x < g->W && z >= 0 && z < g->H;
}

/* set(..., override = true) (graph.cu:14-72) */
static void set_cell(orc_graph *g, long pos, float heading, int ppx, int ppz, float cost, int type)
{
    g->type[pos] = type;
    g->px[pos] = ppx;
    g->pz[pos] = ppz;
    g->heading[pos] = heading;
    g->cost[pos] = cost;
}

/* CudaGraph::add (graph.cu:364-374) */
void orc_graph_add(orc_graph *g, int x, int z, float heading, int ppx, int ppz, float cost)
{
    if (!in_limits(g, x, z))
        return;
    const long pos = (long)z * g->W + x;
    if (ppx != -1 && ppz != -1 && in_limits(g, ppx, ppz))
        g->child[(long)ppz * g->W + ppx]++;
    set_cell(g, pos, heading, ppx, ppz, cost, ORC_NODE);
}

/* CudaGraph::addTemporary (graph.cu:375-381) */
void orc_graph_add_temporary(orc_graph *g, int x, int z, float heading, int ppx, int ppz, float cost)
{
    if (!in_limits(g, x, z))
        return;
    set_cell(g, (long)z * g->W + x, heading, ppx, ppz, cost, ORC_TEMP);
}

/* CudaGraph::remove (graph.cu:393-398) */
void orc_graph_remove(orc_graph *g, int x, int z)
{
    if (!in_limits(g, x, z))
        return;
    g->type[(long)z * g->W + x] = ORC_NULL;
}

/* CudaGraph::clear (graph.cu:400-427): only the type is reset */
void orc_graph_clear(orc_graph *g)
{
    const long n = (long)g->W * g->H;
    for (long i = 0; i < n; i++)
        g->type[i] = ORC_NULL;
    g->goal_reached = 0;
    g->node_collision = 0;
}

/* count / countAll (graph_list.cu:7-60) */
uint32_t orc_graph_count(const orc_graph *g, int type)
{
    const long n = (long)g->W * g->H;
    uint32_t c = 0;
    for (long i = 0; i < n; i++)
        c += g->type[i] == type;
    return c;
}

uint32_t orc_graph_count_all(const orc_graph *g)
{
    const long n = (long)g->W * g->H;
    uint32_t c = 0;
    for (long i = 0; i < n; i++)
        c += g->type[i] != ORC_NULL;
    return c;
}

/* CudaGraph::setCollision (graph.cu:553-563) + setCollisionCuda (:74-94) */
void orc_graph_set_collision(orc_graph *g, int x, int z, int npx, int npz, float heading, float cost)
{
    const long pos = (long)z * g->W + x;
    const int cpx = g->px[pos], cpz = g->pz[pos];
    if (g->type[pos] != ORC_NODE)
        return;
    g->type[pos] = ORC_COLLISION;
    g->px[pos] = npx;
    g->pz[pos] = npz;
    g->heading[pos] = heading;
    g->cost[pos] = cost;
    if (in_limits(g, cpx, cpz))
        g->child[(long)cpz * g->W + cpx]--;
}

/* CudaGraph::getParent (graph.cu:446-453) */
void orc_graph_get_parent(const orc_graph *g, int x, int z, int *ppx, int *ppz)
{
    if (!in_limits(g, x, z) || g->type[(long)z * g->W + x] == ORC_NULL) {
        *ppx = -1;
        *ppz = -1;
        return;
    }
    const long pos = (long)z * g->W + x;
    *ppx = g->px[pos];
    *ppz = g->pz[pos];
}

/* solveCollisions (graph_collision.cu:32-125).  The erase walk is bounded by
 * numNodes + 4 hops; on exhaustion the post-decremented counter is -1, so the
 * `i == 0` cyclic-reference branch never runs and the node is kept.  Parents
 * outside the grid (user-built graphs only) end the walk like the root. */
void orc_graph_solve_collisions(orc_graph *g)
{
    const int numNodes = (int)orc_graph_count(g, ORC_NODE);
    if (numNodes <= 2)
        return;
    const long n = (long)g->W * g->H;
    for (long pos = 0; pos < n; pos++) {
        if (g->type[pos] == ORC_NULL)
            continue;
        long curr = pos;
        int i = numNodes + 4;
        while (i-- > 0) {
            const int ppx = g->px[curr], ppz = g->pz[curr];
            if (ppx == -1 && ppz == -1)
                break;
            if (!in_limits(g, ppx, ppz))
                break;
            const long next = (long)ppz * g->W + ppx;
            const int tn = g->type[next];
            if (tn == ORC_COLLISION || tn == ORC_NULL) {
                g->type[pos] = ORC_NULL;
                break;
            }
            curr = next;
        }
    }
    for (long pos = 0; pos < n; pos++) {
        if (g->type[pos] != ORC_COLLISION)
            continue;
        g->type[pos] = ORC_NODE;
        g->child[pos] = 0;
        const int ppx = g->px[pos], ppz = g->pz[pos];
        if (in_limits(g, ppx, ppz))
            g->child[(long)ppz * g->W + ppx]++;
    }
    g->node_collision = 0;
}

/* acceptDerivedNodes (graph_expansion.cu:36-82) */
void orc_graph_accept(orc_graph *g)
{
    const long n = (long)g->W * g->H;
    for (long i = 0; i < n; i++)
        if (g->type[i] == ORC_TEMP)
            g->type[i] = ORC_NODE;
}

/* computeGraphRegionDensity (graph_expansion_search_zones.cu:42-66,111-159) */
void orc_graph_density(orc_graph *g)
{
    for (int i = 0; i < g->density_size; i++)
        g->region_count[i] = 0;
    for (int z = 0; z < g->H; z++)
        for (int x = 0; x < g->W; x++) {
            const int t = g->type[(long)z * g->W + x];
            if (t == ORC_NULL || t == ORC_PROCESSING)
                continue;
            g->region_count[(z / ORC_REGION) * g->density_w + x / ORC_REGION]++;
        }
}

/* checkGoalReached (graph_best_node.cu:181-250); the flag is sticky until clear */
int orc_graph_check_goal_reached(orc_graph *g, const orc_frame *f, int gx, int gz,
                                 float gh, float tol, float max_err)
{
    (void)f;
    if (g->goal_reached)
        return 1;
    for (int z = 0; z < g->H; z++)
        for (int x = 0; x < g->W; x++) {
            const long pos = (long)z * g->W + x;
            if (g->type[pos] != ORC_NODE)
                continue;
            const double dx = gx - x, dz = gz - z;
            if (sqrt(dx * dx + dz * dz) > tol)
                continue;
            if (fabsf(g->heading[pos] - gh) <= max_err)
                g->goal_reached = 1;
        }
    return g->goal_reached;
}

/* findBestNode (graph_best_node.cu:15-178): cost floor(dist + 3*deg(heading)
 * + cost) with the ABSOLUTE heading; ties go to the highest cell index (the
 * last writer of the reference's second pass when it runs sequentially). */
int orc_graph_find_best_node(const orc_graph *g, const orc_frame *f, float heading,
                             float radius, int tx, int tz, float max_err, int *bx, int *bz)
{
    long long best = ORC_BIG_COST;
    long bpos = -1;
    for (int z = 0; z < g->H; z++)
        for (int x = 0; x < g->W; x++) {
            const long pos = (long)z * g->W + x;
            if (g->type[pos] != ORC_NODE)
                continue;
            const int dx = tx - x, dz = tz - z;
            const float dist = sqrtf((float)(dx * dx + dz * dz));
            if (dist > radius)
                continue;
            const float h = g->heading[pos];
            if (fabsf(h - heading) > max_err)
                continue;
            if (!orc_feasible(f, &g->sp, x, z, h, NULL))
                continue;
            const double v = (double)(1 * dist) + 3 * ORC_TO_DEG * (double)h + (double)(1 * g->cost[pos]);
            const long long c = (long long)floorf((float)v);
            if (c <= best) {
                if (c < best || pos > bpos) {
                    best = c;
                    bpos = pos;
                }
            }
        }
    if (best >= ORC_BIG_COST || bpos < 0) {
        *bx = -1;
        *bz = -1;
        return 0;
    }
    *bx = (int)(bpos % g->W);
    *bz = (int)(bpos / g->W);
    return 1;
}

/* checkGraphIsConsistent (graph_check_dag_consistency.cpp:33-76) */
int orc_graph_is_consistent(const orc_graph *g)
{
    const int maxLoop = (int)orc_graph_count(g, ORC_NODE) + 4;
    for (int z = 0; z < g->H; z++)
        for (int x = 0; x < g->W; x++) {
            if (g->type[(long)z * g->W + x] == ORC_NULL)
                continue;
            int cx = x, cz = z;
            int i = maxLoop;
            while (i-- > 0) {
                int ppx, ppz;
                orc_graph_get_parent(g, cx, cz, &ppx, &ppz);
                if (ppx == cx && ppz == cz)
                    return 0;
                if (ppx == -1)
                    break;
                int pt = in_limits(g, ppx, ppz) ? g->type[(long)ppz * g->W + ppx] : -1;
                if (pt != ORC_NODE && pt != ORC_COLLISION && pt != ORC_CONNECT_TO_GOAL)
                    return 0;
                cx = ppx;
                cz = ppz;
            }
            if (i <= 0)
                return 0;
        }
    return 1;
}

/* processDirectGoalConnection (graph_direct_goal_connection.cu:169-227):
 * per cell, Hermite from the cell (heading pointing at the goal) to the goal.
 * Only the flag is reset for cells that do not connect. */
void orc_graph_process_direct_goal(orc_graph *g, const orc_frame *f, const orc_search *fsp,
                                   int goal_x, int goal_z, float goal_heading,
                                   float max_curvature, long long *probes)
{
    if (max_curvature < 0)
        max_curvature = (float)g->pp.max_curvature;
    long long total = 0;
    /* cells are independent; rows run in parallel when this is the outermost
     * parallel region (inside orc_plan_batch's per-plan threads it is serial) */
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : total)
#endif
    for (int z = 0; z < g->H; z++) {
        long long pr = 0;
        for (int x = 0; x < g->W; x++) {
            const long pos = (long)z * g->W + x;
            g->gd_flag[pos] = 0;
            const float lh = (float)orc_compute_heading(x, z, goal_x, goal_z);
            const float c = orc_direct_connection(g, f, fsp, max_curvature, x, z, lh,
                                                  goal_x, goal_z, goal_heading, 0, &pr);
            if (c < 0)
                continue;
            g->gd_flag[pos] = 1.0f;
            g->gd_heading[pos] = lh;
            g->gd_cost[pos] = c;
        }
        total += pr;
    }
    if (probes)
        *probes += total;
}

/* findBestGoalDirectConnection (graph_check_goal_reached.cu:17-188).  The
 * window is [z - r, z + r) x [x - r, x + r) with the reference's float/int
 * conversions.  Minimum of floor(100 * total); ties go to the highest node
 * index, then to the last window cell in scan order (the last writer of the
 * second pass when it runs sequentially). */
int orc_graph_best_goal_connection(orc_graph *g, const orc_frame *f, float radius,
                                   int safe_zone_checked, orc_f4 out[2], long long *probes)
{
    long long best = ORC_BIG_COST;
    const float maxc = (float)g->pp.max_curvature;
    int found = 0;
    for (int z = 0; z < g->H; z++)
        for (int x = 0; x < g->W; x++) {
            const long pos = (long)z * g->W + x;
            if (g->type[pos] != ORC_NODE)
                continue;
            const float heading = g->heading[pos];
            for (int zp = toi_f((float)z - radius); (float)zp < (float)z + radius; zp++)
                for (int xp = toi_f((float)x - radius); (float)xp < (float)x + radius; xp++) {
                    if (zp < 0 || zp >= g->H || xp < 0 || xp >= g->W)
                        continue;
                    const long cell = (long)zp * g->W + xp;
                    if (!(g->gd_flag[cell] > 0))
                        continue;
                    const float lih = g->gd_heading[cell];
                    const float c = orc_direct_connection(g, f, &g->sp, maxc, x, z, heading, xp, zp,
                                                          lih, safe_zone_checked, probes);
                    if (c < 0)
                        continue;
                    const float total = c + g->gd_cost[cell];
                    const long long lc = (long long)floorf(100 * total);
                    if (lc <= best) {
                        best = lc;
                        found = 1;
                        out[0].x = (float)x; out[0].y = (float)z; out[0].z = heading; out[0].w = c;
                        out[1].x = (float)xp; out[1].y = (float)zp; out[1].z = lih; out[1].w = total;
                    }
                }
        }
    return found && best < ORC_BIG_COST;
}

/* one expansion pass: __CUDA_random_node_expansion (graph_expansion.cu:148-183)
 * or __CUDA_smart_node_expansion (graph_expansion_search_zones.cu:161-194),
 * each calling expand_node (graph_expansion.cu:103-145).  All candidates read
 * the grid as it was before the pass; a target cell claimed by several
 * candidates goes to the lowest expanding-cell index. */
int orc_graph_expand(orc_graph *g, const orc_frame *f, uint64_t seed, uint32_t iter,
                     float max_path, float velocity, int smart, int frontier,
                     int force_expand, long long *probes)
{
    const long n = (long)g->W * g->H;
    const float max_steer = (float)g->pp.max_steer_rad;
    long *cpos = (long *)malloc(sizeof(long) * (size_t)n);
    long *cend = (long *)malloc(sizeof(long) * (size_t)n);
    float *ch = (float *)malloc(sizeof(float) * (size_t)n);
    float *cc = (float *)malloc(sizeof(float) * (size_t)n);
    int nc = 0;
    g->node_collision = 0;
    for (long pos = 0; pos < n; pos++) {
        if (g->type[pos] != ORC_NODE)
            continue;
        const int z = (int)(pos / g->W), x = (int)(pos - (long)z * g->W);
        if (smart) {
            if (!force_expand) {
                int can;
                if (frontier)
                    can = g->child[pos] == 0;
                else
                    can = g->region_count[(z / ORC_REGION) * g->density_w + x / ORC_REGION] <= 0.5 * ORC_REGION;
                if (!can)
                    continue;
            }
        } else if (frontier && g->child[pos] > 0) {
            continue;
        }
        float steer, len;
        orc_draw_expansion(seed, (uint32_t)pos, iter, max_steer, max_path, &steer, &len);
        orc_f4 e = orc_kinematic_path(g, f, x, z, steer, len, velocity, probes, NULL);
        long end = -1;
        if (!(e.x < 0 || e.y < 0)) {
            const int ex = toi_f(e.x), ez = toi_f(e.y);
            if (!((float)ex == g->og_x && (float)ez == g->og_z)) {
                const long ep = (long)ez * g->W + ex;
                if (ep != pos)
                    end = ep;
            }
        }
        cpos[nc] = pos;
        cend[nc] = end;
        ch[nc] = e.w;
        cc[nc] = e.z;
        nc++;
    }
    unsigned char *claimed = (unsigned char *)calloc((size_t)n, 1);
    for (int k = 0; k < nc; k++) {
        const long end = cend[k], pos = cpos[k];
        if (end < 0 || claimed[end])
            continue;
        claimed[end] = 1;
        const int z = (int)(pos / g->W), x = (int)(pos - (long)z * g->W);
        if (g->type[end] == ORC_NULL) {
            g->child[pos]++;
            set_cell(g, end, ch[k], x, z, cc[k], ORC_TEMP);
        } else if (g->type[end] == ORC_NODE) {
            set_cell(g, end, ch[k], x, z, cc[k], ORC_COLLISION);
            g->node_collision = 1;
            g->child[pos]--;
        }
    }
    free(claimed);
    free(cpos);
    free(cend);
    free(ch);
    free(cc);
    return nc;
}

/* ------------------------------------------------------------------------ */
/* planner                                                                  */
/* ------------------------------------------------------------------------ */

/* FastRRT::FastRRT (fastrrt.cpp:35-45); heading tolerance default 10 deg */
orc_planner *orc_planner_new(int W, int H, float pw_m, float ph_m, float max_steer_deg,
                             float vehicle_len, int lbx, int lbz, int ubx, int ubz,
                             float max_curvature)
{
    orc_planner *p = (orc_planner *)calloc(1, sizeof(orc_planner));
    p->g = orc_graph_new(W, H);
    orc_physical_params(&p->g->pp, W, H, pw_m, ph_m, max_steer_deg * ORC_PI / 180.0,
                        vehicle_len, max_curvature);
    p->g->has_pp = 1;
    p->g->sp.lbx = lbx;
    p->g->sp.lbz = lbz;
    p->g->sp.ubx = ubx;
    p->g->sp.ubz = ubz;
    p->pp.heading_tol = (float)(10.0 * ORC_PI / 180.0);
    return p;
}

void orc_planner_free(orc_planner *p)
{
    if (!p)
        return;
    orc_graph_free(p->g);
    free(p);
}

/* FastRRT::setPlanData (fastrrt.cpp:64-81): search params, then the
 * direct-goal precompute with max curvature 0.8.  The frame's own footprint
 * parameters are taken equal to the planner's. */
void orc_planner_set_plan_data(orc_planner *p, const orc_frame *f, const orc_plan_params *pp,
                               int min_dist_x, int min_dist_z)
{
    p->f = f;
    p->pp = *pp;
    p->has_plan = 1;
    orc_graph *g = p->g;
    orc_search_params(&g->sp, g->W, g->H, min_dist_x, min_dist_z, g->sp.lbx, g->sp.lbz,
                      g->sp.ubx, g->sp.ubz);
    orc_graph_process_direct_goal(g, f, &g->sp, pp->goal_x, pp->goal_z, pp->goal_heading,
                                  0.8f, &p->probes_pre);
}

/* FastRRT::search_init (fastrrt.cpp:85-98) */
void orc_planner_search_init(orc_planner *p)
{
    orc_graph_clear(p->g);
    orc_graph_add(p->g, p->pp.start_x, p->pp.start_z, p->pp.start_heading, -1, -1, 0);
    p->last_expanded = 0;
}

int orc_planner_goal_reached(orc_planner *p)
{
    return orc_graph_check_goal_reached(p->g, p->f, p->pp.goal_x, p->pp.goal_z,
                                        p->pp.goal_heading, p->pp.dist_tol, p->pp.heading_tol);
}

/* FastRRT::loop (fastrrt.cpp:108-181); the caller handles the timeout */
int orc_planner_loop(orc_planner *p, int smart)
{
    orc_graph *g = p->g;
    const int frontier = p->last_expanded >= 100;
    if (smart) {
        orc_graph_expand(g, p->f, p->pp.seed, p->iter, p->pp.max_path_size, p->pp.velocity, 1,
                         frontier, p->last_expanded == 0, &p->probes);
        orc_graph_density(g);
    } else {
        orc_graph_expand(g, p->f, p->pp.seed, p->iter, p->pp.max_path_size, p->pp.velocity, 0,
                         frontier, 0, &p->probes);
    }
    p->iter++;
    if (g->node_collision)
        orc_graph_solve_collisions(g);

    p->last_expanded = (int)orc_graph_count(g, ORC_TEMP);
    if (p->last_expanded == 0 && orc_graph_count_all(g) == 0) {
        orc_graph_add(g, p->pp.start_x, p->pp.start_z, p->pp.start_heading, -1, -1, 0);
        return 1;
    }
    orc_graph_accept(g);

    orc_f4 bc[2];
    if (orc_graph_best_goal_connection(g, p->f, p->pp.dist_tol, 1, bc, &p->probes_goal)) {
        const int ppx = toi_f(bc[0].x), ppz = toi_f(bc[0].y);
        const float base = in_limits(g, ppx, ppz) ? g->cost[(long)ppz * g->W + ppx] : -1.0f;
        orc_graph_add(g, toi_f(bc[1].x), toi_f(bc[1].y), bc[1].z, ppx, ppz, bc[0].w + base);
        const int cx = toi_f(bc[1].x), cz = toi_f(bc[1].y);
        const float child_cost = bc[1].z + base;
        orc_graph_add(g, p->pp.goal_x, p->pp.goal_z, p->pp.goal_heading, cx, cz, child_cost);
    }
    if (orc_planner_goal_reached(p))
        return 0;
    return 1;
}

/* FastRRT::getPlannedPath (fastrrt.cpp:204-232) */
int orc_planner_path(orc_planner *p, float *xyh, int cap)
{
    if (!p->has_plan)
        return 0;
    if (!orc_planner_goal_reached(p))
        return 0;
    int bx, bz;
    orc_graph_find_best_node(p->g, p->f, p->pp.goal_heading, p->pp.dist_tol, p->pp.goal_x,
                             p->pp.goal_z, p->pp.heading_tol, &bx, &bz);
    int n = 0;
    long i = 0;
    while (bx != -1 && bz != -1) {
        if (n < cap) {
            xyh[3 * n] = (float)bx;
            xyh[3 * n + 1] = (float)bz;
            xyh[3 * n + 2] = p->g->heading[(long)bz * p->g->W + bx];
        }
        n++;
        int ppx, ppz;
        orc_graph_get_parent(p->g, bx, bz, &ppx, &ppz);
        bx = ppx;
        bz = ppz;
        if (i++ >= 1000000)
            return 0;
    }
    if (n > cap)
        n = cap;
    for (int a = 0, b = n - 1; a < b; a++, b--)
        for (int k = 0; k < 3; k++) {
            float t = xyh[3 * a + k];
            xyh[3 * a + k] = xyh[3 * b + k];
            xyh[3 * b + k] = t;
        }
    return n;
}

/* FastRRT::path_optimize (fastrrt.cpp:183-196) + optimizePathLoop
 * (graph_optimization.cu:25-56, 76-195) */
int orc_planner_optimize(orc_planner *p)
{
    orc_graph *g = p->g;
    const int cap = 1 << 16;
    float *xyh = (float *)malloc(sizeof(float) * 3 * cap);
    int n = orc_planner_path(p, xyh, cap);
    orc_f4 *path = (orc_f4 *)malloc(sizeof(orc_f4) * (size_t)(n > 0 ? n : 1));
    orc_f4 *pd = (orc_f4 *)calloc((size_t)(n > 0 ? n : 1), sizeof(orc_f4));
    for (int i = 0; i < n; i++) {
        path[i].x = xyh[3 * i];
        path[i].y = xyh[3 * i + 1];
        path[i].z = xyh[3 * i + 2];
        const int x = (int)path[i].x, z = (int)path[i].y;
        path[i].w = in_limits(g, x, z) ? g->cost[(long)z * g->W + x] : -1.0f;
    }
    free(xyh);
    const float maxc = (float)g->pp.max_curvature;
    for (int i = 0; i < n - 2; i++) {
        pd[i].x = 0;
        const int x = toi_f(path[i].x), z = toi_f(path[i].y);
        for (int j = i + 2; j < n; j++) {
            const float cur = path[j].w;
            const float nc = orc_direct_connection(g, p->f, &g->sp, maxc, x, z, path[i].z,
                                                   toi_f(path[j].x), toi_f(path[j].y), path[j].z,
                                                   1, &p->probes);
            if (nc > 0 && nc < cur) {
                pd[i].x = 1;
                pd[i].y = (float)j;
                pd[i].z = nc;
                pd[i].w = cur - nc;
            }
        }
    }
    float maxGain = -1;
    int mg = -1;
    for (int i = 0; i < n - 2; i++) {
        if (pd[i].x == 0.0f)
            continue;
        if (maxGain < pd[i].w) {
            maxGain = pd[i].w;
            mg = i;
        }
    }
    if (mg < 0) {
        free(path);
        free(pd);
        return 0;
    }
    const int next_pos = toi_f(pd[mg].y);
    if (next_pos > mg + 1) {
        path[next_pos].w = pd[mg].z;
        const int rm = next_pos - mg - 1;
        for (int i = mg + 1; i + rm < n; ++i)
            path[i] = path[i + rm];
        n -= rm;
    }
    orc_graph_clear(g);
    int ppx = toi_f(path[0].x), ppz = toi_f(path[0].y);
    orc_graph_add(g, ppx, ppz, path[0].z, -1, -1, path[0].w);
    for (int i = 1; i < n; i++) {
        orc_graph_add(g, toi_f(path[i].x), toi_f(path[i].y), path[i].z, ppx, ppz, path[i].w);
        ppx = toi_f(path[i].x);
        ppz = toi_f(path[i].y);
    }
    free(path);
    free(pd);
    return 1;
}

/* interpolateHermiteCurve + interpolate (interpolation.cpp:36-135), host
 * float arithmetic, round() to cells */
int orc_interpolate(const float *xyh, int n, int W, int H, float *out, int cap)
{
    if (n < 2)
        return 0;
    int m = 0;
    for (int s = 1; s < n; s++) {
        const int p1x = (int)xyh[3 * (s - 1)], p1z = (int)xyh[3 * (s - 1) + 1];
        const float p1h = xyh[3 * (s - 1) + 2];
        const int p2x = (int)xyh[3 * s], p2z = (int)xyh[3 * s + 1];
        const float p2h = xyh[3 * s + 2];
        const double ddx = p2x - p1x, ddz = p2z - p1z;
        const int numPoints = toi_d(sqrt(ddx * ddx + ddz * ddz));
        const float dx = (float)(p2x - p1x), dz = (float)(p2z - p1z);
        const float d = sqrtf(dx * dx + dz * dz);
        const float a1 = (float)(p1h - ORC_PI / 2), a2 = (float)(p2h - ORC_PI / 2);
        const float t1x = d * cosf(a1), t1y = d * sinf(a1);
        const float t2x = d * cosf(a2), t2y = d * sinf(a2);
        int lx = -1, lz = -1;
        for (int i = 0; i < numPoints; ++i) {
            const float t = (float)i / (float)(numPoints - 1);
            const float t2 = t * t, t3 = t2 * t;
            const float h00 = 2 * t3 - 3 * t2 + 1, h10 = t3 - 2 * t2 + t;
            const float h01 = -2 * t3 + 3 * t2, h11 = t3 - t2;
            const float x = h00 * p1x + h10 * t1x + h01 * p2x + h11 * t2x;
            const float z = h00 * p1z + h10 * t1y + h01 * p2z + h11 * t2y;
            if (x < 0 || x >= W)
                continue;
            if (z < 0 || z >= H)
                continue;
            const int cx = (int)roundf(x), cz = (int)roundf(z);
            if (cx == lx && cz == lz)
                continue;
            if (cx < 0 || cx >= W || cz < 0 || cz >= H)
                continue;
            const float t00 = 6 * t2 - 6 * t, t10 = 3 * t2 - 4 * t + 1;
            const float t01 = -6 * t2 + 6 * t, t11 = 3 * t2 - 2 * t;
            const float ddx2 = t00 * p1x + t10 * t1x + t01 * p2x + t11 * t2x;
            const float ddz2 = t00 * p1z + t10 * t1y + t01 * p2z + t11 * t2y;
            const float heading = (float)(atan2f(ddz2, ddx2) + ORC_HALF_PI);
            if (m < cap) {
                out[3 * m] = (float)cx;
                out[3 * m + 1] = (float)cz;
                out[3 * m + 2] = heading;
            }
            m++;
            lx = cx;
            lz = cz;
        }
    }
    return m < cap ? m : cap;
}

/* search_init + loop until the goal is reached, loop() returns false or
 * max_iter loops ran (README.md:50-52 usage) */
int orc_plan(orc_planner *p, int smart, int max_iter, int *iters)
{
    orc_planner_search_init(p);
    int it = 0;
    while (!orc_planner_goal_reached(p) && it < max_iter) {
        it++;
        if (!orc_planner_loop(p, smart))
            break;
    }
    if (iters)
        *iters = it;
    return orc_planner_goal_reached(p);
}

static float wrap_pi(float a)
{
    const float tp = (float)(2 * ORC_PI);
    while (a > ORC_PI)
        a -= tp;
    while (a < -ORC_PI)
        a += tp;
    return a;
}

/* Path validator.  A coarse path passes when (1) it has >= 2 distinct
 * in-grid waypoints starting at the start cell, (2) the node grid is a DAG
 * (graph_check_dag_consistency.cpp:33-76) and consecutive waypoints are
 * parent links, (3) every waypoint outside the ego box passes the footprint
 * check at its heading (checkStateFeasible, path_feasible.cu:80-117), (4)
 * every segment turns by at most (pi/2) * kappa * chord + 1e-3 rad, kappa the
 * largest curvature the planner admits (bicycle model at full steering, the
 * goal-connection and direct-goal Hermite limits), and (5) the last waypoint
 * is within the goal tolerance in distance and heading. */
/* Path checks that need only the frame and the planner's parameters: start
 * cell, cells in the frame, footprint feasible outside the ego box, no
 * repeated cell, heading change per chord within the curvature bound, goal
 * within the distance and heading tolerances.  with_graph adds the graph's
 * own checks: the graph is a DAG and each waypoint's parent is the one before. */
static int validate_waypoints(orc_planner *p, const float *xyh, int n, int with_graph)
{
    const orc_graph *g = p->g;
    if (n < 2)
        return 0;
    if ((int)xyh[0] != p->pp.start_x || (int)xyh[1] != p->pp.start_z)
        return 0;
    if (with_graph && !orc_graph_is_consistent(g))
        return 0;
    const double ms = g->pp.max_steer_rad;
    const double steer = tan(ms), beta = atan(steer / 2);
    double kappa = cos(beta) * steer / (2 * g->pp.lr);
    if (g->pp.max_curvature > kappa)
        kappa = g->pp.max_curvature;
    if (0.8 > kappa)
        kappa = 0.8;
    for (int i = 0; i < n; i++) {
        const int x = (int)xyh[3 * i], z = (int)xyh[3 * i + 1];
        const float h = xyh[3 * i + 2];
        if (!in_limits(g, x, z))
            return 0;
        const int in_ego = x >= g->sp.lbx && x <= g->sp.ubx && z >= g->sp.ubz && z <= g->sp.lbz;
        if (!in_ego && !orc_feasible(p->f, &g->sp, x, z, h, NULL))
            return 0;
        if (i > 0) {
            const int px = (int)xyh[3 * (i - 1)], pz = (int)xyh[3 * (i - 1) + 1];
            if (px == x && pz == z)
                return 0;
            if (with_graph) {
                int ppx, ppz;
                orc_graph_get_parent(g, x, z, &ppx, &ppz);
                if (ppx != px || ppz != pz)
                    return 0;
            }
            const double chord = sqrt((double)(x - px) * (x - px) + (double)(z - pz) * (z - pz));
            const float dh = wrap_pi(h - xyh[3 * (i - 1) + 2]);
            if (fabs(dh) > (ORC_PI / 2) * kappa * chord + 1e-3)
                return 0;
        }
    }
    const int lx = (int)xyh[3 * (n - 1)], lz = (int)xyh[3 * (n - 1) + 1];
    const double gdx = lx - p->pp.goal_x, gdz = lz - p->pp.goal_z;
    if (sqrt(gdx * gdx + gdz * gdz) > p->pp.dist_tol)
        return 0;
    if (fabsf(xyh[3 * (n - 1) + 2] - p->pp.goal_heading) > p->pp.heading_tol)
        return 0;
    return 1;
}

int orc_validate_path(orc_planner *p, const float *xyh, int n)
{
    return validate_waypoints(p, xyh, n, 1);
}

int orc_validate_waypoints(orc_planner *p, const float *xyh, int n)
{
    return validate_waypoints(p, xyh, n, 0);
}

void orc_kinematic_batch(const orc_graph *g, const orc_frame *f, int n, const int32_t *sx,
                         const int32_t *sz, const float *steer, const float *len, float velocity,
                         float *out4, long long *probes, int32_t *steps)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = 0; i < n; i++) {
        long long pr = 0;
        int st = 0;
        orc_f4 r = orc_kinematic_path(g, f, sx[i], sz[i], steer[i], len[i], velocity, &pr, &st);
        out4[4 * i] = r.x;
        out4[4 * i + 1] = r.y;
        out4[4 * i + 2] = r.z;
        out4[4 * i + 3] = r.w;
        if (probes)
            probes[i] = pr;
        if (steps)
            steps[i] = st;
    }
}

void orc_feasible_batch(const orc_frame *f, const orc_search *sp, int n, const int32_t *x,
                        const int32_t *z, const float *a, int32_t *out, long long *probes)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = 0; i < n; i++) {
        long long pr = 0;
        out[i] = orc_feasible(f, sp, x[i], z[i], a[i], &pr);
        if (probes)
            probes[i] = pr;
    }
}

void orc_direct_batch(const orc_graph *g, const orc_frame *f, const orc_search *sp, float maxc,
                      int n, const int32_t *x, const int32_t *z, const float *lh,
                      const int32_t *gx, const int32_t *gz, const float *gh, int safe,
                      float *out, long long *probes)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int i = 0; i < n; i++) {
        long long pr = 0;
        out[i] = orc_direct_connection(g, f, sp, maxc, x[i], z[i], lh[i], gx[i], gz[i], gh[i],
                                       safe, &pr);
        if (probes)
            probes[i] = pr;
    }
}

static double now_ms(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

int orc_plan_batch(int n, int W, int H, const uint8_t *cls, const float *class_costs,
                   int n_classes, const int32_t *start_goal, const uint64_t *seeds,
                   float pw_m, float ph_m, float max_steer_deg, float vehicle_len,
                   int min_dist_x, int min_dist_z, float velocity, float max_path,
                   float dist_tol, float heading_tol, int timeout_ms, int max_iter,
                   int smart, int threads, int32_t *ok, int32_t *iters, float *path_cost,
                   double *ms)
{
#ifdef _OPENMP
    if (threads > 0)
        omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int k = 0; k < n; k++) {
        const double t0 = now_ms();
        orc_frame f;
        f.W = W;
        f.H = H;
        f.cls = cls + (size_t)k * W * H;
        f.class_costs = class_costs;
        f.n_classes = n_classes;
        f.trav = NULL;
        f.dist = NULL;
        orc_planner *p = orc_planner_new(W, H, pw_m, ph_m, max_steer_deg, vehicle_len,
                                         -1, -1, -1, -1, -1.0f);
        orc_plan_params pp;
        const int32_t *sg = start_goal + 6 * k;
        pp.start_x = sg[0];
        pp.start_z = sg[1];
        pp.start_heading = (float)sg[2] * 1e-6f;
        pp.goal_x = sg[3];
        pp.goal_z = sg[4];
        pp.goal_heading = (float)sg[5] * 1e-6f;
        pp.velocity = velocity;
        pp.max_path_size = max_path;
        pp.dist_tol = dist_tol;
        pp.heading_tol = heading_tol;
        pp.seed = seeds[k];
        orc_planner_set_plan_data(p, &f, &pp, min_dist_x, min_dist_z);
        orc_planner_search_init(p);
        int it = 0;
        while (!orc_planner_goal_reached(p) && (max_iter <= 0 || it < max_iter)) {
            if (timeout_ms > 0 && now_ms() - t0 > timeout_ms)
                break;
            it++;
            if (!orc_planner_loop(p, smart))
                break;
        }
        int good = 0;
        float len = 0;
        if (orc_planner_goal_reached(p)) {
            float *xyh = (float *)malloc(sizeof(float) * 3 * 4096);
            const int m = orc_planner_path(p, xyh, 4096);
            good = orc_validate_path(p, xyh, m);
            for (int i = 1; i < m; i++) {
                const float dx = xyh[3 * i] - xyh[3 * i - 3], dz = xyh[3 * i + 1] - xyh[3 * i - 2];
                len += sqrtf(dx * dx + dz * dz);
            }
            free(xyh);
        }
        ok[k] = good;
        iters[k] = it;
        path_cost[k] = len;
        ms[k] = now_ms() - t0;
        orc_planner_free(p);
    }
    return 0;
}
