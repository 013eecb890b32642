// ref_capi.cu -- TEST INFRASTRUCTURE ONLY.
//
// Linked into oracle/_ref/libfastrrt_ref.so together with the reference's
// own sources (compiled from their location in the reference tree by
// oracle/ref/Makefile).  It exposes, through a flat C ABI for the tests:
//   ref_h_* : the reference's `__device__ __host__` per-candidate functions
//             run on the host CPU;
//   ref_d_* : the same reference functions run on the GPU, one thread per
//             candidate (the bit-exact checker for the product kernels);
//   ref_frame_* : a shim SearchFrame for the reference's own FastRRT C ABI
//             (fastrrt_initialize / set_plan_data / loop ...), which the
//             reference's python_bind.cpp exports from the same library.
#include <cuda_runtime.h>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <driveless/cuda_params.h>
#include <driveless/search_frame.h>

// reference function signatures (kinematics.cu:123-125, path_feasible.cu:18,
// graph_direct_goal_connection.cu:16, graph.cu:219)
extern __device__ __host__ float4 check_kinematic_new_path(int4 *graph, float4 *graphData,
    double *physicalParams, int *searchSpaceParams, float3 *frame, float *classCosts,
    float3 *ogStart, int2 start, float steeringAngle, float pathSize, float velocity_m_s);
extern __device__ __host__ bool __computeFeasibleForAngle(float3 *frame, int *params,
    float *classCost, int minDistX, int minDistZ, int x, int z, float angle_radians);
extern __device__ __host__ float checkDirectConnectionToGoal(float4 *graphData, float3 *frame,
    float *classCosts, int *searchSpaceParams, float max_curvature, int x, int z,
    float local_heading, int goal_x, int goal_z, float goal_heading, bool isSafeZoneChecked,
    bool isDistanceToGoalProcessed);
extern __device__ __host__ double computeHeading(int x1, int z1, int x2, int z2);

namespace {

struct Inputs {
    int W, H;
    std::vector<float3> frame;
    std::vector<float> costs;
    std::vector<int4> graph;
    std::vector<float4> data;
    double pp[16];
    int sp[16];
    float3 og;
};

void fill(Inputs &in, int W, int H, const float *frame_xyz, const float *costs, int ncls,
          const float *heading, const float *cost, double max_steer_rad, double lr, int mdx,
          int mdz, int lbx, int lbz, int ubx, int ubz, float og_x, float og_z)
{
    in.W = W;
    in.H = H;
    const long n = (long)W * H;
    in.frame.resize(n);
    for (long i = 0; i < n; i++)
        in.frame[i] = make_float3(frame_xyz[3 * i], frame_xyz[3 * i + 1], frame_xyz[3 * i + 2]);
    in.costs.assign(costs, costs + ncls);
    in.graph.assign(n, make_int4(0, 0, 0, 0));
    in.data.assign(n, make_float4(0, 0, 0, 0));
    for (long i = 0; i < n; i++) {
        in.data[i].x = heading ? heading[i] : 0.0f;
        in.data[i].y = cost ? cost[i] : 0.0f;
    }
    memset(in.pp, 0, sizeof(in.pp));
    memset(in.sp, 0, sizeof(in.sp));
    in.pp[PHYSICAL_PARAMS_MAX_STEERING_RAD] = max_steer_rad;
    in.pp[PHYSICAL_PARAMS_LR] = lr;
    in.sp[FRAME_PARAM_WIDTH] = W;
    in.sp[FRAME_PARAM_HEIGHT] = H;
    in.sp[FRAME_PARAM_MIN_DIST_X] = mdx;
    in.sp[FRAME_PARAM_MIN_DIST_Z] = mdz;
    in.sp[FRAME_PARAM_LOWER_BOUND_X] = lbx;
    in.sp[FRAME_PARAM_LOWER_BOUND_Z] = lbz;
    in.sp[FRAME_PARAM_UPPER_BOUND_X] = ubx;
    in.sp[FRAME_PARAM_UPPER_BOUND_Z] = ubz;
    in.og = make_float3(og_x, og_z, 0.0f);
}

template <typename T>
T *dev_copy(const T *h, size_t n)
{
    T *d = nullptr;
    if (cudaMalloc((void **)&d, n * sizeof(T) + 16) != cudaSuccess)
        return nullptr;
    if (n)
        cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

// plain pointers passed by value to the kernels
struct DevPtrs {
    float3 *frame;
    float *costs;
    int4 *graph;
    float4 *data;
    double *pp;
    int *sp;
    float3 *og;
};

// owns the device copies of one Inputs set
struct DevInputs {
    DevPtrs p{};
    bool ok() const { return p.frame && p.costs && p.graph && p.data && p.pp && p.sp && p.og; }
    void up(const Inputs &in)
    {
        p.frame = dev_copy(in.frame.data(), in.frame.size());
        p.costs = dev_copy(in.costs.data(), in.costs.size());
        p.graph = dev_copy(in.graph.data(), in.graph.size());
        p.data = dev_copy(in.data.data(), in.data.size());
        p.pp = dev_copy(in.pp, 16);
        p.sp = dev_copy(in.sp, 16);
        p.og = dev_copy(&in.og, 1);
    }
    ~DevInputs()
    {
        cudaFree(p.frame); cudaFree(p.costs); cudaFree(p.graph); cudaFree(p.data);
        cudaFree(p.pp); cudaFree(p.sp); cudaFree(p.og);
    }
};

__global__ void k_ref_kinematic(DevPtrs d, int n, const int *sx, const int *sz, const float *st,
                                const float *len, float v, float4 *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    out[i] = check_kinematic_new_path(d.graph, d.data, d.pp, d.sp, d.frame, d.costs, d.og,
                                      make_int2(sx[i], sz[i]), st[i], len[i], v);
}

__global__ void k_ref_feasible(DevPtrs d, int n, const int *x, const int *z, const float *a,
                               int *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    out[i] = __computeFeasibleForAngle(d.frame, d.sp, d.costs, d.sp[FRAME_PARAM_MIN_DIST_X],
                                       d.sp[FRAME_PARAM_MIN_DIST_Z], x[i], z[i], a[i]);
}

__global__ void k_ref_direct(DevPtrs d, float maxc, int n, const int *x, const int *z,
                             const float *lh, const int *gx, const int *gz, const float *gh,
                             int safe, float *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    // safe: bit 0 isSafeZoneChecked, bit 1 isDistanceToGoalProcessed
    out[i] = checkDirectConnectionToGoal(d.data, d.frame, d.costs, d.sp, maxc, x[i], z[i], lh[i],
                                         gx[i], gz[i], gh[i], (safe & 1) != 0, (safe & 2) != 0);
}

__global__ void k_ref_heading(int n, const int *x, const int *z, const int *gx, const int *gz,
                              float *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    out[i] = (float)computeHeading(x[i], z[i], gx[i], gz[i]);
}

int grid_of(int n) { return (n + 127) / 128; }

} // namespace

#define REF_COMMON_ARGS                                                                  \
    int W, int H, const float *frame_xyz, const float *costs, int ncls, const float *heading, \
        const float *cost, double max_steer_rad, double lr, int mdx, int mdz, int lbx, int lbz, \
        int ubx, int ubz, float og_x, float og_z
#define REF_COMMON_PASS                                                                      \
    W, H, frame_xyz, costs, ncls, heading, cost, max_steer_rad, lr, mdx, mdz, lbx, lbz, ubx, ubz, \
        og_x, og_z

extern "C" {

int ref_h_kinematic(REF_COMMON_ARGS, int n, const int *sx, const int *sz, const float *steer,
                    const float *len, float velocity, float *out)
{
    Inputs in;
    fill(in, REF_COMMON_PASS);
    for (int i = 0; i < n; i++) {
        float4 r = check_kinematic_new_path(in.graph.data(), in.data.data(), in.pp, in.sp,
                                            in.frame.data(), in.costs.data(), &in.og,
                                            make_int2(sx[i], sz[i]), steer[i], len[i], velocity);
        out[4 * i] = r.x; out[4 * i + 1] = r.y; out[4 * i + 2] = r.z; out[4 * i + 3] = r.w;
    }
    return 0;
}

int ref_h_feasible(REF_COMMON_ARGS, int n, const int *x, const int *z, const float *a, int *out)
{
    Inputs in;
    fill(in, REF_COMMON_PASS);
    for (int i = 0; i < n; i++)
        out[i] = __computeFeasibleForAngle(in.frame.data(), in.sp, in.costs.data(), mdx, mdz, x[i],
                                           z[i], a[i]);
    return 0;
}

int ref_h_direct(REF_COMMON_ARGS, float maxc, int n, const int *x, const int *z, const float *lh,
                 const int *gx, const int *gz, const float *gh, int safe, float *out)
{
    Inputs in;
    fill(in, REF_COMMON_PASS);
    for (int i = 0; i < n; i++)
        out[i] = checkDirectConnectionToGoal(in.data.data(), in.frame.data(), in.costs.data(), in.sp,
                                             maxc, x[i], z[i], lh[i], gx[i], gz[i], gh[i],
                                             (safe & 1) != 0, (safe & 2) != 0);
    return 0;
}

float ref_h_compute_heading(int x1, int z1, int x2, int z2)
{
    return (float)computeHeading(x1, z1, x2, z2);
}

int ref_d_kinematic(REF_COMMON_ARGS, int n, const int *sx, const int *sz, const float *steer,
                    const float *len, float velocity, float *out)
{
    Inputs in;
    fill(in, REF_COMMON_PASS);
    DevInputs d;
    d.up(in);
    int *dsx = dev_copy(sx, n), *dsz = dev_copy(sz, n);
    float *dst = dev_copy(steer, n), *dln = dev_copy(len, n);
    float4 *dout = nullptr;
    cudaMalloc((void **)&dout, sizeof(float4) * (size_t)(n + 1));
    int rc = -1;
    if (d.ok() && dsx && dsz && dst && dln && dout) {
        k_ref_kinematic<<<grid_of(n), 128>>>(d.p, n, dsx, dsz, dst, dln, velocity, dout);
        if (cudaDeviceSynchronize() == cudaSuccess &&
            cudaMemcpy(out, dout, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToHost) == cudaSuccess)
            rc = 0;
    }
    cudaFree(dsx); cudaFree(dsz); cudaFree(dst); cudaFree(dln); cudaFree(dout);
    return rc;
}

int ref_d_feasible(REF_COMMON_ARGS, int n, const int *x, const int *z, const float *a, int *out)
{
    Inputs in;
    fill(in, REF_COMMON_PASS);
    DevInputs d;
    d.up(in);
    int *dx = dev_copy(x, n), *dz = dev_copy(z, n), *dout = nullptr;
    float *da = dev_copy(a, n);
    cudaMalloc((void **)&dout, sizeof(int) * (size_t)(n + 1));
    int rc = -1;
    if (d.ok() && dx && dz && da && dout) {
        k_ref_feasible<<<grid_of(n), 128>>>(d.p, n, dx, dz, da, dout);
        if (cudaDeviceSynchronize() == cudaSuccess &&
            cudaMemcpy(out, dout, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost) == cudaSuccess)
            rc = 0;
    }
    cudaFree(dx); cudaFree(dz); cudaFree(da); cudaFree(dout);
    return rc;
}

int ref_d_direct(REF_COMMON_ARGS, float maxc, int n, const int *x, const int *z, const float *lh,
                 const int *gx, const int *gz, const float *gh, int safe, float *out)
{
    Inputs in;
    fill(in, REF_COMMON_PASS);
    DevInputs d;
    d.up(in);
    int *dx = dev_copy(x, n), *dz = dev_copy(z, n), *dgx = dev_copy(gx, n), *dgz = dev_copy(gz, n);
    float *dlh = dev_copy(lh, n), *dgh = dev_copy(gh, n), *dout = nullptr;
    cudaMalloc((void **)&dout, sizeof(float) * (size_t)(n + 1));
    int rc = -1;
    if (d.ok() && dx && dz && dgx && dgz && dlh && dgh && dout) {
        k_ref_direct<<<grid_of(n), 128>>>(d.p, maxc, n, dx, dz, dlh, dgx, dgz, dgh, safe, dout);
        if (cudaDeviceSynchronize() == cudaSuccess &&
            cudaMemcpy(out, dout, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost) == cudaSuccess)
            rc = 0;
    }
    cudaFree(dx); cudaFree(dz); cudaFree(dgx); cudaFree(dgz);
    cudaFree(dlh); cudaFree(dgh); cudaFree(dout);
    return rc;
}

int ref_d_compute_heading(int n, const int *x, const int *z, const int *gx, const int *gz, float *out)
{
    int *dx = dev_copy(x, n), *dz = dev_copy(z, n), *dgx = dev_copy(gx, n), *dgz = dev_copy(gz, n);
    float *dout = nullptr;
    cudaMalloc((void **)&dout, sizeof(float) * (size_t)(n + 1));
    int rc = -1;
    if (dx && dz && dgx && dgz && dout) {
        k_ref_heading<<<grid_of(n), 128>>>(n, dx, dz, dgx, dgz, dout);
        if (cudaDeviceSynchronize() == cudaSuccess &&
            cudaMemcpy(out, dout, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost) == cudaSuccess)
            rc = 0;
    }
    cudaFree(dx); cudaFree(dz); cudaFree(dgx); cudaFree(dgz); cudaFree(dout);
    return rc;
}

// a SearchFrame for the reference's own set_plan_data(); frame_xyz holds
// (class id, distance, traversability) per pixel
void *ref_frame_new(int W, int H, const float *frame_xyz, const float *costs, int ncls, int lbx,
                    int lbz, int ubx, int ubz, int mdx, int mdz)
{
    SearchFrame *f = new SearchFrame(W, H, {lbx, lbz}, {ubx, ubz});
    f->setClassCosts(std::vector<float>(costs, costs + ncls));
    f->copyFrom(frame_xyz);
    f->setHalfMinDistance(mdx, mdz);
    return f;
}

void ref_frame_free(void *f) { delete (SearchFrame *)f; }

} // extern "C"
