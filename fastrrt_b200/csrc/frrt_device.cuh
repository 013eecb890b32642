// frrt_device.cuh -- device functions of the B200 FastRRT planner.
//
// The per-candidate arithmetic (kinematic integration, footprint probe
// coordinates, Hermite samples) is written with the same expression shapes
// and types as the reference so that the CUDA compiler produces the same
// roundings and fused multiply-adds; the feasibility booleans, cell indices
// and parent links are therefore bit-identical to the reference kernels.
// Everything around that arithmetic is organised for the GPU: warp-wide
// cooperative footprint probes, bit-packed frames, a conservative "clear"
// shortcut that answers most footprint checks with one bit lookup, and a
// counter-based RNG.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "frrt_common.cuh"

namespace frrt {

// driveless constants (double precision, as the reference headers use them)
constexpr double kPi = 3.14159265358979323846;
constexpr double kHalfPi = kPi / 2.0;
constexpr double kToDeg = 180.0 / kPi;

// ---------------------------------------------------------------------------
// RNG: Philox4x32-10 (Salmon et al., "Parallel random numbers: as easy as
// 1, 2, 3", SC 2011).  Counter (cell, iteration, tag, 0), key = seed.
// ---------------------------------------------------------------------------
constexpr uint32_t kRngTag = 0x46525254u;

__host__ __device__ inline void philox4x32(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                           uint32_t k0, uint32_t k1, uint32_t out[4])
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// uniform in (0, 1] with 24 random bits (exact in float)
__host__ __device__ inline float u01(uint32_t r) { return (float)((r >> 8) + 1u) * (1.0f / 16777216.0f); }

// steering U(-max, max] then length max(5, max_path * U) -- generateRandomNeg /
// generateRandom (random_number_gen.cu:14-20) as called by the expansion
// kernels (graph_expansion.cu:174-180)
__device__ inline void draw_expansion(unsigned long long seed, uint32_t pos, uint32_t iter,
                                      float max_steer, float max_path, float &steer, float &len)
{
    uint32_t r[4];
    philox4x32(pos, iter, kRngTag, 0u, (uint32_t)seed, (uint32_t)(seed >> 32), r);
    const float u0 = u01(r[0]);
    const float u1 = u01(r[1]);
    steer = (2.0f * u0 - 1.0f) * max_steer;
    len = fmaxf(5.0f, max_path * u1);
}

// ---------------------------------------------------------------------------
// frame access
// ---------------------------------------------------------------------------
// Programmatic dependent launch: a kernel of the iteration graph waits for
// the kernel before it (completion and memory visibility) before it reads
// anything, then lets the kernel after it be scheduled, so that kernel's
// launch overlaps this one's run instead of following its end.  Without a
// programmatic predecessor the wait returns at once.
__device__ __forceinline__ void griddep_wait()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ bool bit_xz(const uint32_t *m, int rw, int x, int z)
{
    return (m[(long)z * rw + (x >> 5)] >> (x & 31)) & 1u;
}

// what a footprint probe needs; the mask pointers may be shared or global memory
struct Foot {
    int W, H;
    int mdx, mdz;
    int lbx, lbz, ubx, ubz;
    int rw;
    const uint32_t *blocked;
    const uint32_t *clear;
    const int32_t *trav;
    const uint16_t *sat;   // obstacle counts, summed-area table mod 2^16, or nullptr
};

__device__ __forceinline__ Foot foot_of(const Inst &I, const uint32_t *blocked, const uint32_t *clear)
{
    Foot f;
    f.W = I.W; f.H = I.H; f.mdx = I.mdx; f.mdz = I.mdz;
    f.lbx = I.lbx; f.lbz = I.lbz; f.ubx = I.ubx; f.ubz = I.ubz;
    f.rw = I.mask_rw;
    f.blocked = blocked; f.clear = clear; f.trav = I.trav;
    // a box count is exact mod 2^16 only while the box holds fewer cells
    f.sat = (I.mdx + I.mdz <= 120) ? I.sat : nullptr;
    return f;
}



__device__ __forceinline__ unsigned full_probes(const Foot &f)
{
    return (unsigned)((2 * f.mdx + 1) * (2 * f.mdz + 1));
}

// No obstacle in the box [x0, x1] x [z0, z1] (clipped to the frame), from the
// summed-area table: S[z][x] = obstacles in [0, x) x [0, z), (W+1) columns.
__device__ __forceinline__ bool box_clear(const Foot &f, int x0, int z0, int x1, int z1)
{
    x0 = max(x0, 0);
    z0 = max(z0, 0);
    x1 = min(x1, f.W - 1);
    z1 = min(z1, f.H - 1);
    if (x0 > x1 || z0 > z1)
        return true;
    const long w = f.W + 1;
    const uint16_t a = f.sat[(z1 + 1) * w + x1 + 1], b = f.sat[(long)z0 * w + x1 + 1];
    const uint16_t c = f.sat[(z1 + 1) * w + x0], d = f.sat[(long)z0 * w + x0];
    return (uint16_t)(a - b - c + d) == 0;
}

// The footprint at heading direction (|cos|, |sin|) = (ac, as) probes only
// cells within its axis-aligned bounding box: offsets j c - i s and j s + i c
// with |j| <= mdx, |i| <= mdz are at most e = mdx ac + mdz as (resp.
// mdx as + mdz ac) away, so the truncated cells lie within ceil(e + 1e-3)
// (the slack covers the rounding of the reference's cosf / sinf and float
// arithmetic).  An empty box means every probe misses, so the footprint is
// feasible and the reference runs all its probes.
__device__ __forceinline__ bool box_feasible(const Foot &f, int x, int z, float ac, float as,
                                             unsigned long long &probes)
{
    if (!f.sat || !(ac <= 1.5f) || !(as <= 1.5f))
        return false;
    const int ex = (int)ceilf(f.mdx * ac + f.mdz * as + 1e-3f);
    const int ez = (int)ceilf(f.mdx * as + f.mdz * ac + 1e-3f);
    if (!box_clear(f, x - ex, z - ez, x + ex, z + ez))
        return false;
    probes += full_probes(f);
    return true;
}

// 1: feasible without probing (isAllAngleFeasible quirk or clear shortcut),
// 0: the footprint has to be probed.  `probes` gets the reference's count.
__device__ __forceinline__ int quick_feasible(const Foot &f, int x, int z, unsigned long long &probes)
{
    const long pos = (long)z * f.W + x;
    // both words are loaded before either is tested: one memory round trip
    const int tv = f.trav ? f.trav[pos] : 0;
    const bool clear = bit_xz(f.clear, f.rw, x, z);
    // isAllAngleFeasible (path_feasible.cu:13-16): `TO_INT(z) & 256 > 0` == bit 0
    if (tv & 1)
        return 1;
    // no obstacle within the Chebyshev radius that bounds every probe
    if (clear) {
        probes += full_probes(f);
        return 1;
    }
    return 0;
}

// the probe loop of __computeFeasibleForAngle (path_feasible.cu:18-78), one
// lane, reference order
__device__ inline bool probe_scalar(const Foot &f, int x, int z, float angle, unsigned long long &probes)
{
    const float c = cosf(angle);
    const float s = sinf(angle);
    for (int i = -f.mdz; i <= f.mdz; i++)
        for (int j = -f.mdx; j <= f.mdx; j++) {
            probes++;
            const int xl = (int)(j * c - i * s + x);
            const int zl = (int)(j * s + i * c + z);
            if (xl < 0 || xl >= f.W)
                continue;
            if (zl < 0 || zl >= f.H)
                continue;
            if (xl >= f.lbx && xl <= f.ubx && zl >= f.ubz && zl <= f.lbz)
                continue;
            if (bit_xz(f.blocked, f.rw, xl, zl))
                return false;
        }
    return true;
}

__device__ inline bool feasible_scalar(const Foot &f, int x, int z, float angle, unsigned long long &probes)
{
    if (quick_feasible(f, x, z, probes))
        return true;
    return probe_scalar(f, x, z, angle, probes);
}

// The same probe loop, all 32 lanes of a warp on one (x, z, angle): lane k
// of batch b evaluates probe b*32+k in the reference's i-major order, and the
// first blocked probe of the first batch that has one is the reference's
// early exit, so the returned count is the reference's probe count.
__device__ inline bool probe_warp(const Foot &f, int x, int z, float angle, int lane, unsigned &count)
{
    const float c = cosf(angle);
    const float s = sinf(angle);
    const int wdt = 2 * f.mdx + 1;
    const int total = wdt * (2 * f.mdz + 1);
    const int q = 32 / wdt, r = 32 % wdt;
    int ii = lane / wdt, jj = lane % wdt;
    for (int base = 0; base < total; base += 32) {
        bool hit = false;
        if (base + lane < total) {
            const int i = ii - f.mdz;
            const int j = jj - f.mdx;
            const int xl = (int)(j * c - i * s + x);
            const int zl = (int)(j * s + i * c + z);
            if (xl >= 0 && xl < f.W && zl >= 0 && zl < f.H &&
                !(xl >= f.lbx && xl <= f.ubx && zl >= f.ubz && zl <= f.lbz))
                hit = bit_xz(f.blocked, f.rw, xl, zl);
        }
        const unsigned m = __ballot_sync(kFull, hit);
        if (m) {
            count = (unsigned)(base + __ffs(m));
            return false;
        }
        ii += q;
        jj += r;
        if (jj >= wdt) {
            jj -= wdt;
            ii++;
        }
    }
    count = (unsigned)total;
    return true;
}

// A cheaper exact test than the full probe loop, for footprints that turn
// out feasible.  Every probe (j, i) of the footprint at (x, z) with direction
// (c, s) lies in the rectangle |u| <= mdx, |v| <= mdz, with u = X' c + Z' s,
// v = -X' s + Z' c relative to the cell.  A probe lands in frame row zr when
// Z' is in [zr - z, zr - z + 1) (row 0 also takes Z' in (-1, 0): truncation
// toward zero), and over that strip each constraint bounds X' by an interval
// whose ends move linearly, so their hulls bound every probe of the row; the
// probe's column is the truncation of x + X'.  Lane k tests rows z0 + k,
// z0 + k + 32, ...; 1e-3 of slack covers the rounding of the reference's
// float probe arithmetic.  No obstacle bit in any interval means no probe can
// hit.
__device__ inline bool rows_clear_warp(const Foot &f, int x, int z, float c, float s, int lane)
{
    const float ac = fabsf(c), as = fabsf(s);
    const float ez = f.mdx * as + f.mdz * ac;
    const int z0 = max(0, (int)floorf(z - ez) - 1);
    const int z1 = min(f.H - 1, (int)floorf(z + ez) + 1);
    const bool use1 = ac > 1e-6f, use2 = as > 1e-6f;
    const float ic = use1 ? 1.0f / c : 0.0f, is = use2 ? 1.0f / s : 0.0f;
    const float h1 = f.mdx * fabsf(ic), h2 = f.mdz * fabsf(is);
    const float sic = s * ic, cis = c * is;
    bool hit = false;
    for (int zr = z0 + lane; zr <= z1 && !hit; zr += 32) {
        const float za = (float)(zr - z) - (zr == 0 ? 1.001f : 0.001f);
        const float zb = (float)(zr - z + 1) + 0.001f;
        float lo = -1e30f, hi = 1e30f;
        if (use1) {  // X' = (+-mdx - Z' s) / c
            const float pa = -za * sic, pb = -zb * sic;
            lo = fmaxf(lo, fminf(pa, pb) - h1);
            hi = fminf(hi, fmaxf(pa, pb) + h1);
        }
        if (use2) {  // X' = (Z' c +- mdz) / s
            const float qa = za * cis, qb = zb * cis;
            lo = fmaxf(lo, fminf(qa, qb) - h2);
            hi = fminf(hi, fmaxf(qa, qb) + h2);
        }
        if (!(lo <= hi))
            continue;
        const int xa = max(0, (int)floorf(x + lo - 1e-3f));
        const int xb = min(f.W - 1, (int)(x + hi + 1e-3f));
        if (xa > xb)
            continue;
        const uint32_t *row = f.blocked + (long)zr * f.rw;
        for (int q = xa >> 5; q <= (xb >> 5); q++) {
            const int b0 = max(xa - q * 32, 0), b1 = min(xb - q * 32, 31);
            const uint32_t mask =
                (b1 - b0 == 31) ? 0xffffffffu : (((1u << (b1 - b0 + 1)) - 1u) << b0);
            if (row[q] & mask) {
                hit = true;
                break;
            }
        }
    }
    return !__any_sync(kFull, hit);
}

// ---------------------------------------------------------------------------
// per-candidate checks, one candidate per warp
// ---------------------------------------------------------------------------

// sample stride of the first pass of the direct goal connections (0: none);
// a build-time knob for measurement
#ifndef FRRT_COARSE_STRIDE
#define FRRT_COARSE_STRIDE 16
#endif
constexpr int kCoarseStride = FRRT_COARSE_STRIDE;

// The start pose and constants of one check_kinematic_new_path candidate
// (kinematics.cu:123-231); kin_warp integrates it.
struct KinTask {
    float x, y, heading, beta, ds, hif, nodeCost, velocity;
    int maxSize, loop_max;
    float og_x, og_z;
    int W, H;
    const float *intrinsic;

    __device__ void init(const Inst &I, int sx, int sz, float steeringAngle, float pathSize,
                         float velocity_m_s, float start_heading, float start_cost)
    {
        const double maxSteering = I.max_steer;
        const double lr = I.lr;
        W = I.W;
        H = I.H;
        og_x = I.og_x;
        og_z = I.og_z;
        intrinsic = I.intrinsic;
        // convert_waypoint_to_map_pose (kinematics.cu:54-59)
        x = og_z - sz;
        y = sx - og_x;
        if (steeringAngle > maxSteering)
            steeringAngle = maxSteering;
        else if (steeringAngle < -maxSteering)
            steeringAngle = -maxSteering;
        const float steer = tanf(steeringAngle);
        const float dt = 0.1;
        velocity = velocity_m_s;
        ds = velocity_m_s * dt;
        beta = atanf(steer / 2);
        hif = ds * cosf(beta) * steer / (2 * lr);
        maxSize = (int)(pathSize) + 1;
        heading = start_heading;
        nodeCost = start_cost;
        loop_max = (100 * maxSize) / dt;
    }

};

// The reference's curvature, (float)(num / pow(s2, 1.5)).  Only samples
// within 1e-6 of the limit reach it, so it stays out of line: the curve
// loops keep their code small (their warps stall on instruction fetch).
static __device__ __noinline__ float curv_pow(double num, double s2)
{
    return num / pow(s2, 1.5);
}

// The constants of one checkDirectConnectionToGoal curve
// (graph_direct_goal_connection.cu:16-167, isDistanceToGoalProcessed =
// false) and the reference's per-sample arithmetic; curve_warp walks it.
struct HermTask {
    int x, z, goal_x, goal_z, numPoints, W, H, trav;
    float distance, t1x, t1y, t2x, t2y, nodeCost, max_curvature;
    int safe;
    const float *intrinsic;
    double inv_span;           // RN(1 / (numPoints - 1))
    double kap_hi2, kap_lo2;   // (max_curvature (1 +- 1e-6))^2

    __device__ void init(const Inst &I, const Foot &f, float max_curv, int x_, int z_,
                         float local_heading, int gx, int gz, float goal_heading, int safe_zone,
                         float start_cost, const float *dist_channel = nullptr)
    {
        W = f.W;
        H = f.H;
        x = x_;
        z = z_;
        goal_x = gx;
        goal_z = gz;
        max_curvature = max_curv;
        intrinsic = I.intrinsic;
        const long pos = (long)z * W + x;
        const int dx = goal_x - x;
        const int dz = goal_z - z;
        // isDistanceToGoalProcessed: the frame's distance channel
        distance = dist_channel ? dist_channel[pos] : sqrtf(dx * dx + dz * dz);
        numPoints = (int)(distance);
        const float a1 = local_heading - kHalfPi;
        const float a2 = goal_heading - kHalfPi;
        t1x = distance * cosf(a1);
        t1y = distance * sinf(a1);
        t2x = distance * cosf(a2);
        t2y = distance * sinf(a2);
        nodeCost = start_cost;
        trav = f.trav ? f.trav[pos] : 0;
        inv_span = 1.0 / (double)(numPoints - 1);
        const double khi = (double)max_curvature * (1.0 + 1e-6);
        const double klo = (double)max_curvature * (1.0 - 1e-6);
        kap_hi2 = khi * khi;
        kap_lo2 = klo * klo;
        safe = safe_zone;
    }

    // the reference's evaluation of the curve at t: position, first and
    // second derivative, in its order of operations
    __device__ __forceinline__ void ref_pos(double t, double &px, double &pz) const
    {
        const double t2 = t * t;
        const double t3 = t2 * t;
        const double h00 = 2 * t3 - 3 * t2 + 1;
        const double h10 = t3 - 2 * t2 + t;
        const double h01 = -2 * t3 + 3 * t2;
        const double h11 = t3 - t2;
        px = h00 * x + h10 * t1x + h01 * goal_x + h11 * t2x;
        pz = h00 * z + h10 * t1y + h01 * goal_z + h11 * t2y;
    }
    __device__ __forceinline__ void ref_deriv(double t, double &ddx, double &ddz, double &dd2x,
                                              double &dd2z) const
    {
        const double t2 = t * t;
        const double t00 = 6 * t2 - 6 * t;
        const double t10 = 3 * t2 - 4 * t + 1;
        const double t01 = -6 * t2 + 6 * t;
        const double t11 = 3 * t2 - 2 * t;
        ddx = t00 * x + t10 * t1x + t01 * goal_x + t11 * t2x;
        ddz = t00 * z + t10 * t1y + t01 * goal_z + t11 * t2y;
        const double d00 = 12 * t - 6;
        const double d10 = 6 * t - 4;
        const double d01 = -12 * t + 6;
        const double d11 = 6 * t - 2;
        dd2x = d00 * x + d10 * t1x + d01 * goal_x + d11 * t2x;
        dd2z = d00 * z + d10 * t1y + d01 * goal_z + d11 * t2y;
    }
    // The reference tests (float)(num / pow(s2, 1.5)) > limit.  Outside a
    // 1e-6 relative band around the limit (hi2 / lo2: the band's squared
    // ends) the answer follows from num^2 against limit^2 s2^3 (products
    // rounded to ~1e-15); pow only decides cases inside the band.  s2 == 0:
    // num > 0 is over (num / 0 = inf), num == 0 falls through to the
    // reference's own 0 / 0.
    __device__ __forceinline__ bool ref_over(double ddx, double ddz, double dd2x, double dd2z,
                                             double hi2, double lo2) const
    {
        const double s2 = ddx * ddx + ddz * ddz;
        const double num = fabs(ddx * dd2z - ddz * dd2x);
        const double n2 = num * num;
        const double s6 = s2 * s2 * s2;
        if (n2 > hi2 * s6)
            return true;
        if (n2 < lo2 * s6)
            return false;
        return curv_pow(num, s2) > max_curvature;
    }
    // t = i / (numPoints - 1), correctly rounded, without a division per
    // sample: with y = RN(1/b), q = RN(a y) and the exact remainder
    // r = a - q b, RN(q + r y) is RN(a/b) (Markstein 1990); checked
    // exhaustively for 0 <= a <= b <= 16384 against IEEE division
    // (tests/sample_t_check.c), which covers every frame up to 4096 x 4096
    __device__ __forceinline__ double sample_t(int k) const
    {
        const double span = (double)(numPoints - 1);
        const double ak = (double)k;
        const double q = __dmul_rn(ak, inv_span);
        return __fma_rn(__fma_rn(-q, span, ak), inv_span, q);
    }

};

// The full footprint test of one cell by the whole warp (all lanes pass the
// same arguments): the row-interval test clears most feasible footprints,
// the probe loop in the reference's order decides the rest.  `cnt` gets the
// reference's probe count.
__device__ inline bool footprint_warp(const Foot &f, int x, int z, float angle, int lane, unsigned &cnt)
{
    if (rows_clear_warp(f, x, z, cosf(angle), sinf(angle), lane)) {
        cnt = full_probes(f);  // feasible: the reference runs all its probes
        return true;
    }
    return probe_warp(f, x, z, angle, lane, cnt);
}
// footprint_warp out of line, for loops where the full test is rare (the
// goal curves: most samples are decided by the clear bit or the summed-area
// box): a smaller loop body fetches fewer instructions; the call costs
// registers, so the expansion and goal-search loops keep it inline.
static __device__ __noinline__ unsigned long long footprint_warp_out(Foot f, int x, int z, float angle, int lane)
{
    unsigned cnt = 0;
    const bool ok = footprint_warp(f, x, z, angle, lane, cnt);
    return ((unsigned long long)(ok ? 1u : 0u) << 32) | cnt;
}
template <bool kOut>
__device__ __forceinline__ bool footprint_call(const Foot &f, int x, int z, float angle, int lane, unsigned &cnt)
{
    if (!kOut)
        return footprint_warp(f, x, z, angle, lane, cnt);
    const unsigned long long r = footprint_warp_out(f, x, z, angle, lane);
    cnt = (unsigned)r;
    return (r >> 32) != 0;
}

// Result of one kinematic candidate (check_kinematic_new_path).
struct KinResult {
    int ok;            // 1: a feasible end cell
    int last_x, last_z;
    float cost, heading;
};

// check_kinematic_new_path (kinematics.cu:123-231) of one candidate,
// evaluated by the whole warp: lane k takes integration step base + k.
//
// The pose chains are the reference's, in its order and roundings: the
// heading before step s is the start heading plus s serial float adds of the
// increment, and x, y advance by one fused multiply-add per step (the
// contraction the compiler applies to the reference's `x += ds * cosf(..)`).
// Those adds run as one serial chain per warp (32 steps, a shuffle each);
// the cosines and sines, the cell of each step and its tests run across the
// lanes.  Every step either stays in the last cell, leaves the frame (the
// loop ends after the step) or enters a new cell, so the last cell before
// step s is the cell of step s - 1.  The loop also ends before the step that
// would exceed its iteration bound or follow the maxSize-th new cell.  New
// cells before the first stop are checked (clear bit, summed-area box, then
// the warp's probe loop in step order); the first infeasible one rejects the
// candidate.  The cost adds (intrinsic + 1) of each new cell in step order.
// `probes` gets the reference's exact probe count.  Every argument is the
// same in all lanes, and so is the result.
__device__ inline KinResult kin_warp(const Inst &I, const Foot &f, int sx, int sz, float steer, float len,
                                     float velocity, float start_heading, float start_cost, int lane,
                                     unsigned long long &probes)
{
    KinTask k;
    k.init(I, sx, sz, steer, len, velocity, start_heading, start_cost);
    const unsigned lower = (1u << lane) - 1u;
    float x = k.x, y = k.y, hd = k.heading, cost = k.nodeCost;
    int last_x = sx, last_z = sz, size = 0;
    KinResult r;
    for (int base = 0;; base += 32) {
        // headings before (hb) and after (ha) this lane's step
        float hb = hd, ha = hd;
        {
            float h = hd;
#pragma unroll
            for (int q = 0; q < 32; q++) {
                if (q == lane)
                    hb = h;
                h = h + k.hif;
                if (q == lane)
                    ha = h;
            }
        }
        const float c = cosf(hb + k.beta), s = sinf(hb + k.beta);
        float px = x, py = y;  // pose after this lane's step
        {
            float xa = x, ya = y;
#pragma unroll
            for (int q = 0; q < 32; q++) {
                xa = __fmaf_rn(k.ds, __shfl_sync(kFull, c, q), xa);
                ya = __fmaf_rn(k.ds, __shfl_sync(kFull, s, q), ya);
                if (q == lane) {
                    px = xa;
                    py = ya;
                }
            }
        }
        // convert_map_pose_to_waypoint (kinematics.cu:25-46)
        const double2 coord = {px, py};
        const int lpx = (int)(k.og_x + coord.y);
        const int lpz = (int)(k.og_z - coord.x);
        const int ux = __shfl_up_sync(kFull, lpx, 1), uz = __shfl_up_sync(kFull, lpz, 1);
        const int prev_x = lane ? ux : last_x, prev_z = lane ? uz : last_z;
        const bool moved = !(lpx == prev_x && lpz == prev_z);
        const bool oob = moved && (lpx < 0 || lpx >= k.W || lpz < 0 || lpz >= k.H);
        const bool fresh = moved && !oob;
        const unsigned nm = __ballot_sync(kFull, fresh);
        // the first step that does not run, and the first that leaves the frame
        const int step = base + lane;
        const unsigned over_m = __ballot_sync(kFull, step > k.loop_max || size + __popc(nm & lower) >= k.maxSize);
        const int e_stop = over_m ? __ffs(over_m) - 1 : 32;
        const unsigned oob_m = __ballot_sync(kFull, oob) & (e_stop < 32 ? ((1u << e_stop) - 1u) : kFull);
        const int end = oob_m ? __ffs(oob_m) : e_stop;  // steps of this chunk that run
        // the loop ends in this chunk (a step that leaves the frame may be the
        // chunk's last, with all 32 steps run)
        const bool stopped = oob_m != 0 || e_stop < 32;
        const unsigned run_m = end >= 32 ? kFull : ((1u << end) - 1u);
        const bool check = fresh && ((run_m >> lane) & 1u);
        // footprint of each new cell: shortcuts per lane, then the warp's
        // probe loop for the rest in step order up to the first failure
        unsigned long long pl = 0;
        float v = 0.0f;
        bool hard = false;
        if (check) {
            v = (k.intrinsic ? k.intrinsic[(long)lpz * k.W + lpx] : 0.0f) + 1;
            if (!quick_feasible(f, lpx, lpz, pl)) {
                bool box = false;
                if (f.sat) {
                    float sn, cs;
                    sincosf(ha, &sn, &cs);
                    box = box_feasible(f, lpx, lpz, fabsf(cs), fabsf(sn), pl);
                }
                hard = !box;
            }
        }
        unsigned hm = __ballot_sync(kFull, hard);
        int ff = 32;
        unsigned fcnt = 0;
        while (hm) {
            const int leader = __ffs(hm) - 1;
            hm &= hm - 1;
            unsigned cnt = 0;
            const bool ok = footprint_warp(f, __shfl_sync(kFull, lpx, leader), __shfl_sync(kFull, lpz, leader),
                                           __shfl_sync(kFull, ha, leader), lane, cnt);
            if (!ok) {
                ff = leader;
                fcnt = cnt;
                break;
            }
            if (lane == leader)
                pl += cnt;
        }
        if (lane < ff)
            probes += pl;
        if (ff < 32 && lane == 0)
            probes += fcnt;
        // costs in step order, up to and including a failing cell
        unsigned cm = __ballot_sync(kFull, check) & (ff < 32 ? ((2u << ff) - 1u) : kFull);
        while (cm) {
            const int q = __ffs(cm) - 1;
            cm &= cm - 1;
            cost += __shfl_sync(kFull, v, q);
        }
        if (ff < 32) {
            r.ok = 0;
            r.last_x = last_x;
            r.last_z = last_z;
            r.cost = cost;
            r.heading = __shfl_sync(kFull, ha, ff);
            return r;
        }
        const unsigned done_m = nm & run_m;
        size += __popc(done_m);
        if (done_m) {
            const int q = 31 - __clz(done_m);
            last_x = __shfl_sync(kFull, lpx, q);
            last_z = __shfl_sync(kFull, lpz, q);
        }
        if (stopped) {
            r.ok = size >= 1;
            r.last_x = last_x;
            r.last_z = last_z;
            r.cost = cost;
            r.heading = end > 0 ? __shfl_sync(kFull, ha, end - 1) : hd;
            return r;
        }
        hd = __shfl_sync(kFull, ha, 31);
        x = __shfl_sync(kFull, px, 31);
        y = __shfl_sync(kFull, py, 31);
    }
}

// checkDirectConnectionToGoal (graph_direct_goal_connection.cu:16-167) of
// one curve, evaluated by the whole warp: lane k takes sample base + k, with
// the same arithmetic as HermTask.
//
// The reference walks the samples in order and tests a sample when it and
// its cell lie in the frame and the cell differs from the last tested cell.
// Every such sample either repeats that cell or becomes it, so the last
// tested cell before sample i is the cell of the nearest earlier sample in
// the frame: a ballot and a shuffle, with the last chunk's cell carried over.
// A tested sample fails on curvature, else on its footprint; the reference's
// answer is "no connection" at the first failure, so any failure decides it.
// A chunk with a curvature failure ends the walk before its footprints are
// tested.  Otherwise lanes that need the full probe loop are probed by the
// whole warp one after another in sample order, so the first footprint
// failure found is the reference's; `probes` gets the reference's count for
// the chunks walked up to that failure (at most the reference's count for
// the curve, equal to it for a connected curve).  The connection cost is the start cost plus (intrinsic + 1) of
// every tested sample, added in sample order (one lane's term after
// another), so the float sum rounds as the reference's.
//
// `coarse` >= 2 first tests every coarse-th sample whose predecessor lies in
// the frame and in another cell: such a sample is one the reference tests,
// so a failure there is the reference's answer whatever comes before it (a
// curve rejected there adds nothing to `probes`); a curve the pass clears is
// walked in order.  Every argument is the same in all lanes, and so is the
// result: the reference's return value (the cost, or -1 for no connection;
// callers treat any negative value as none, as the reference's do).
// `dist_channel` (isDistanceToGoalProcessed) takes the curve's distance from
// the frame's distance channel at the start cell instead of computing it.
// `kOut` calls the full footprint test out of line (footprint_warp_out).
template <bool kOut = false>
__device__ inline float curve_warp(const Inst &I, const Foot &f, float max_curv, int x, int z,
                                   float local_heading, int gx, int gz, float goal_heading, int safe,
                                   float start_cost, int coarse, int lane, unsigned long long &probes,
                                   const float *dist_channel = nullptr)
{
    HermTask h;
    h.init(I, f, max_curv, x, z, local_heading, gx, gz, goal_heading, safe, start_cost, dist_channel);
    const int np = h.numPoints;
    const bool skip_foot = safe && (h.trav & 0x100);
    const unsigned lower = (1u << lane) - 1u;
    if (coarse >= 2) {
        for (int base = coarse - 1; base < np; base += 32 * coarse) {
            const int i = base + lane * coarse;
            bool test = false;
            int cx = 0, cz = 0;
            double t = 0.0;
            if (i < np) {
                t = h.sample_t(i);
                double px, pz, qx, qz;
                h.ref_pos(t, px, pz);
                h.ref_pos(h.sample_t(i - 1), qx, qz);
                if (!(px < 0 || px >= h.W || pz < 0 || pz >= h.H) &&
                    !(qx < 0 || qx >= h.W || qz < 0 || qz >= h.H)) {
                    cx = (int)(px);
                    cz = (int)(pz);
                    const int ax = (int)(qx), az = (int)(qz);
                    // both cells inside the frame (see the walk below)
                    test = cx >= 0 && cx < h.W && cz >= 0 && cz < h.H && ax >= 0 && ax < h.W && az >= 0 &&
                           az < h.H && !(cx == ax && cz == az);
                }
            }
            bool over = false, hard = false;
            float ang = 0.0f;
            if (test) {
                double ddx, ddz, dd2x, dd2z;
                h.ref_deriv(t, ddx, ddz, dd2x, dd2z);
                over = max_curv > 0 && h.ref_over(ddx, ddz, dd2x, dd2z, h.kap_hi2, h.kap_lo2);
                unsigned long long uncounted = 0;
                if (!over && !skip_foot && !quick_feasible(f, cx, cz, uncounted)) {
                    const double s2 = ddx * ddx + ddz * ddz;
                    bool box = false;
                    if (f.sat && s2 > 0.0) {
                        const float inv = rsqrtf((float)s2);
                        box = box_feasible(f, cx, cz, fabsf((float)ddz) * inv, fabsf((float)ddx) * inv,
                                           uncounted);
                    }
                    if (!box) {
                        hard = true;
                        ang = atan2f(ddz, ddx) + kHalfPi;
                    }
                }
            }
            if (__any_sync(kFull, over))
                return -1.0f;
            unsigned hm = __ballot_sync(kFull, hard);
            while (hm) {
                const int leader = __ffs(hm) - 1;
                hm &= hm - 1;
                unsigned cnt = 0;
                if (!footprint_call<kOut>(f, __shfl_sync(kFull, cx, leader), __shfl_sync(kFull, cz, leader),
                                    __shfl_sync(kFull, ang, leader), lane, cnt))
                    return -1.0f;
            }
        }
    }
    int last_x = -1, last_z = -1;  // the reference's last tested cell
    float cost = start_cost;
    for (int base = 0; base < np; base += 32) {
        const int i = base + lane;
        const double t = h.sample_t(i);
        double px, pz;
        h.ref_pos(t, px, pz);
        // A sample counts when it lies in the frame and so does its cell.  The
        // reference tests the cell's bounds after the position's (they differ
        // for a NaN position: with numPoints == 1, t = 0 / 0); a sample that
        // fails either is skipped and leaves the last tested cell as it was.
        int cx = 0, cz = 0;
        bool valid = false;
        if (i < np && !(px < 0 || px >= h.W) && !(pz < 0 || pz >= h.H)) {
            cx = (int)(px);
            cz = (int)(pz);
            valid = cx >= 0 && cx < h.W && cz >= 0 && cz < h.H;
        }
        const unsigned im = __ballot_sync(kFull, valid);
        const unsigned below = im & lower;
        const int src = below ? 31 - __clz(below) : lane;
        const int qx = __shfl_sync(kFull, cx, src), qz = __shfl_sync(kFull, cz, src);
        const int pcx = below ? qx : last_x, pcz = below ? qz : last_z;
        const bool tested = valid && !(cx == pcx && cz == pcz);
        float v = 0.0f;
        bool over = false, hard = false;
        float ang = 0.0f;
        unsigned long long pl = 0;  // this lane's probes (feasible footprints)
        double ddx = 0, ddz = 0, dd2x = 0, dd2z = 0;
        if (tested) {
            v = (h.intrinsic ? h.intrinsic[(long)cz * h.W + cx] : 0.0f) + 1;
            h.ref_deriv(t, ddx, ddz, dd2x, dd2z);
            over = max_curv > 0 && h.ref_over(ddx, ddz, dd2x, dd2z, h.kap_hi2, h.kap_lo2);
        }
        // a curvature failure anywhere in the chunk decides the answer (no
        // connection) whatever the footprints before it give; the chunk's
        // feasible footprints are then left uncounted
        if (__any_sync(kFull, over))
            return -1.0f;
        if (tested && !skip_foot && !quick_feasible(f, cx, cz, pl)) {
            const double s2 = ddx * ddx + ddz * ddz;
            bool box = false;
            if (f.sat && s2 > 0.0) {
                const float inv = rsqrtf((float)s2);
                box = box_feasible(f, cx, cz, fabsf((float)ddz) * inv, fabsf((float)ddx) * inv, pl);
            }
            if (!box) {
                hard = true;
                ang = atan2f(ddz, ddx) + kHalfPi;
            }
        }
        unsigned hm = __ballot_sync(kFull, hard);
        int ff = 32;  // first footprint failure
        unsigned fcnt = 0;
        while (hm) {
            const int leader = __ffs(hm) - 1;
            hm &= hm - 1;
            unsigned cnt = 0;
            const bool ok = footprint_call<kOut>(f, __shfl_sync(kFull, cx, leader), __shfl_sync(kFull, cz, leader),
                                           __shfl_sync(kFull, ang, leader), lane, cnt);
            if (!ok) {
                ff = leader;
                fcnt = cnt;
                break;
            }
            if (lane == leader)
                pl += cnt;
        }
        if (lane < ff)
            probes += pl;
        if (ff < 32) {
            if (lane == 0)
                probes += fcnt;
            return -1.0f;
        }
        unsigned tm = __ballot_sync(kFull, tested);
        while (tm) {
            const int k = __ffs(tm) - 1;
            tm &= tm - 1;
            cost += __shfl_sync(kFull, v, k);
        }
        if (im) {
            const int hi = 31 - __clz(im);
            last_x = __shfl_sync(kFull, cx, hi);
            last_z = __shfl_sync(kFull, cz, hi);
        }
    }
    if (np <= 0 || (last_x != gx && last_z != gz))
        return -1.0f;
    return cost;
}

// computeHeading (graph.cu:219-234)
__device__ inline double compute_heading(int x1, int z1, int x2, int z2)
{
    double dz = z2 - z1;
    double dx = x2 - x1;
    if (dx == 0 && dz == 0)
        return 0;
    double v1 = 0;
    if (dz != 0)
        v1 = atan2f(-dz, dx);
    else
        v1 = atan2f(0, dx);
    return kHalfPi - v1;
}

// ---------------------------------------------------------------------------
// shared-memory staging of the frame masks with the Blackwell bulk copy
// engine (cp.async.bulk, completion on an mbarrier, bounded waits)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned phase)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

constexpr long kWaitLimit = 1L << 22;  // try_wait rounds before giving up

// Loads `words` 32-bit words of the two masks into shared memory.  Called by
// the whole block; returns false (and the caller falls back to the global
// copies, after draining the copy with a second bounded wait) if the copy did
// not complete within `limit` rounds.
__device__ inline bool stage_masks(uint32_t *s_blk, uint32_t *s_clr, const uint32_t *g_blk,
                                   const uint32_t *g_clr, int words, uint64_t *bar, unsigned &phase,
                                   long limit = kWaitLimit)
{
    __syncthreads();  // every warp finished reading the previous masks
    if (threadIdx.x == 0) {
        fence_proxy_async_smem();
        const unsigned bytes = (unsigned)words * 4u;
        mbar_expect_tx(bar, 2u * bytes);
        bulk_g2s(s_blk, g_blk, bytes, bar);
        bulk_g2s(s_clr, g_clr, bytes, bar);
    }
    bool done = false;
    for (long k = 0; k < limit; k++)
        if (mbar_try_wait(bar, phase)) {
            done = true;
            break;
        }
    phase ^= 1u;
    return __syncthreads_and(done) != 0;
}

}  // namespace frrt
