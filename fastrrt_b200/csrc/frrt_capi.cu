// frrt_capi.cu -- extern "C" ABI of libfastrrt_b200.so (include/fastrrt_b200.h).
#include "fastrrt_b200.h"

#include <algorithm>
#include <chrono>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "frrt_engine.h"
#include "frrt_mlp.h"

using namespace frrt;

namespace {

constexpr double kPiD = 3.14159265358979323846;

double now_ms()
{
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

uint64_t wall_ms()
{
    return (uint64_t)std::chrono::duration_cast<std::chrono::milliseconds>(
               std::chrono::system_clock::now().time_since_epoch())
        .count();
}

float *path_array(const std::vector<float> &xyh)
{
    const int n = (int)xyh.size() / 3;
    float *r = new (std::nothrow) float[3 * n + 1];
    if (!r)
        return nullptr;
    r[0] = (float)n;
    for (int i = 0; i < 3 * n; i++)
        r[1 + i] = xyh[i];
    return r;
}

// The drop-in planner: FastRRT (fastrrt.cpp:35-297) over a one-slot engine.
struct Planner {
    std::unique_ptr<Engine> eng;
    int W, H;
    Physical phys{};
    PlanRequest req{};
    std::vector<float> default_costs;
    const Frame *frame = nullptr;
    bool has_plan = false;
    int timeout_ms = 0;
    double start_ms = 0;
    uint64_t seed;
    bool seed_set = false;

    bool timed_out() const { return timeout_ms > 0 && now_ms() - start_ms > timeout_ms; }
};

Planner *as_planner(void *p)
{
    if (!p)
        set_error("null planner handle");
    return static_cast<Planner *>(p);
}

}  // namespace

namespace {
struct Candidates {
    std::unique_ptr<Engine> eng;
    int W, H;
};

bool cells_in_frame(const Candidates *c, int n, const int32_t *x, const int32_t *z)
{
    for (int i = 0; i < n; i++)
        if (x[i] < 0 || x[i] >= c->W || z[i] < 0 || z[i] >= c->H) {
            set_error("candidates: cell outside the frame");
            return false;
        }
    return true;
}

template <typename T>
struct DevBuf {
    T *p = nullptr;
    bool alloc(size_t n) { return cudaMalloc(&p, sizeof(T) * (n ? n : 1)) == cudaSuccess; }
    ~DevBuf() { cudaFree(p); }
};
}  // namespace

namespace {
struct Batch {
    std::unique_ptr<Engine> eng;
    std::vector<int> admitted;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.0f;
    ~Batch()
    {
        if (ev0)
            cudaEventDestroy(ev0);
        if (ev1)
            cudaEventDestroy(ev1);
    }
};

bool load_request(Engine &e, int slot, const fastrrt_request &r, int timeout_ms = 0)
{
    Physical ph{};
    ph.pw_m = r.perception_w_m;
    ph.ph_m = r.perception_h_m;
    ph.max_steer_rad = (double)r.max_steering_deg * (kPiD / 180.0);
    ph.vehicle_len = r.vehicle_length_m;
    ph.max_curvature = r.max_curvature;
    ph.lbx = r.lb_x;
    ph.lbz = r.lb_z;
    ph.ubx = r.ub_x;
    ph.ubz = r.ub_z;
    e.set_physical(slot, ph);
    PlanRequest q{};
    q.start_x = r.start_x;
    q.start_z = r.start_z;
    q.start_heading = r.start_heading;
    q.goal_x = r.goal_x;
    q.goal_z = r.goal_z;
    q.goal_heading = r.goal_heading;
    q.velocity = r.velocity_m_s;
    q.min_dist_x = r.min_dist_x;
    q.min_dist_z = r.min_dist_z;
    q.max_path = r.max_path_size;
    q.dist_tol = r.dist_to_goal_tol;
    q.heading_tol = r.heading_tol_rad;
    q.seed = r.seed;
    q.smart = r.smart;
    q.max_iter = r.max_iterations;
    q.stop_on_goal = 1;
    q.timeout_ms = r.timeout_ms > 0 ? r.timeout_ms : timeout_ms;
    e.set_request(slot, q);
    return e.copy_frame(slot, r.width, r.height, r.class_ids, r.class_costs, r.n_classes,
                        r.class_ids_on_device != 0);
}
}  // namespace

extern "C" {

const char *fastrrt_last_error(void) { return last_error(); }

// ---------------------------------------------------------------------------
// frames
// ---------------------------------------------------------------------------

void *fastrrt_frame_create(int width, int height, const uint8_t *class_ids, const float *class_costs,
                           int n_classes, const int32_t *trav_bits)
{
    return frame_create(width, height, class_ids, class_costs, n_classes, trav_bits);
}

void *fastrrt_frame_create_f3(int width, int height, const float *xyz, const float *class_costs,
                              int n_classes)
{
    return frame_create_f3(width, height, xyz, class_costs, n_classes);
}

void fastrrt_frame_destroy(void *frame) { delete static_cast<Frame *>(frame); }

int fastrrt_frame_process_distance_to_goal(void *frame, int goal_x, int goal_z)
{
    return frame_process_distance_to_goal(static_cast<Frame *>(frame), goal_x, goal_z) ? 0 : -1;
}

int fastrrt_frame_process_safe_zone(void *frame, int min_dist_x, int min_dist_z)
{
    return frame_process_safe_zone(static_cast<Frame *>(frame), min_dist_x, min_dist_z) ? 0 : -1;
}

int fastrrt_frame_flags(void *frame, int *safe_zone_checked, int *distance_to_goal_processed)
{
    const Frame *f = static_cast<const Frame *>(frame);
    if (!f) {
        set_error("frame: null");
        return -1;
    }
    if (safe_zone_checked)
        *safe_zone_checked = f->safe_zone_checked;
    if (distance_to_goal_processed)
        *distance_to_goal_processed = f->distance_processed;
    return 0;
}

int fastrrt_frame_channels(void *frame, float *distance, int32_t *traversability)
{
    const Frame *f = static_cast<const Frame *>(frame);
    if (!f) {
        set_error("frame: null");
        return -1;
    }
    const size_t n = (size_t)f->W * f->H;
    bool ok = true;
    if (distance)
        ok = f->d_dist ? cudaMemcpy(distance, f->d_dist, 4 * n, cudaMemcpyDeviceToHost) == cudaSuccess
                       : (memset(distance, 0, 4 * n), true);
    if (traversability && ok)
        ok = f->d_trav ? cudaMemcpy(traversability, f->d_trav, 4 * n, cudaMemcpyDeviceToHost) == cudaSuccess
                       : (memset(traversability, 0, 4 * n), true);
    if (!ok)
        set_error("frame: channel download failed");
    return ok ? 0 : -1;
}

// ---------------------------------------------------------------------------
// planner
// ---------------------------------------------------------------------------

void *fastrrt_initialize(int width, int height, float perceptionWidthSize_m,
                         float perceptionHeightSize_m, float maxSteeringAngle_deg,
                         float vehicleLength, int lowerBound_x, int lowerBound_z,
                         int upperBound_x, int upperBound_z, float *classCosts,
                         float max_curvature)
{
    auto *p = new (std::nothrow) Planner();
    if (!p) {
        set_error("out of host memory");
        return nullptr;
    }
    p->eng.reset(new (std::nothrow) Engine(1, width, height));
    if (!p->eng || !p->eng->ok()) {
        delete p;
        return nullptr;
    }
    p->W = width;
    p->H = height;
    if (classCosts) {
        const int n = (int)classCosts[0];
        if (n > 0 && n <= 256)
            p->default_costs.assign(classCosts + 1, classCosts + 1 + n);
    }
    p->phys.pw_m = perceptionWidthSize_m;
    p->phys.ph_m = perceptionHeightSize_m;
    // angle::deg(maxSteeringAngle_deg).rad()
    p->phys.max_steer_rad = (double)maxSteeringAngle_deg * (kPiD / 180.0);
    p->phys.vehicle_len = vehicleLength;
    p->phys.max_curvature = max_curvature;
    p->phys.lbx = lowerBound_x;
    p->phys.lbz = lowerBound_z;
    p->phys.ubx = upperBound_x;
    p->phys.ubz = upperBound_z;
    p->eng->set_physical(0, p->phys);
    // heading tolerance default 10 degrees (fastrrt.cpp:39)
    p->req.heading_tol = (float)(10.0 * kPiD / 180.0);
    p->seed = wall_ms();
    return p;
}

void fastrrt_destroy(void *ptr) { delete static_cast<Planner *>(ptr); }

int fastrrt_debug_set_stage_wait_limit(int64_t rounds)
{
    if (rounds < 0) {
        set_error("stage wait limit: negative");
        return -1;
    }
    if (!set_stage_wait_limit((long)rounds)) {
        set_error("stage wait limit: symbol copy failed");
        return -1;
    }
    return 0;
}

int fastrrt_debug_stage_timeouts(uint64_t *count)
{
    unsigned long long c = 0;
    if (!take_stage_timeouts(c)) {
        set_error("stage timeouts: symbol copy failed");
        return -1;
    }
    if (count)
        *count = c;
    return 0;
}

int fastrrt_set_frame_preprocessing(void *ptr, int use)
{
    Planner *p = as_planner(ptr);
    if (!p)
        return -1;
    p->eng->set_use_frame_preprocessing(0, use != 0);
    return 0;
}

int fastrrt_set_seed(void *ptr, uint64_t seed)
{
    Planner *p = as_planner(ptr);
    if (!p)
        return -1;
    p->seed = seed;
    p->seed_set = true;
    p->req.seed = seed;
    p->eng->set_request(0, p->req);
    return 0;
}

void set_plan_data(void *ptr, void *frame, int start_x, int start_z, float start_heading_rad,
                   int goal_x, int goal_z, float goal_heading_rad, float velocity_m_s,
                   int min_dist_x, int min_dist_z, int timeout_ms, float maxPathSize,
                   float distToGoalTolerance, float headingErrorTolerance_rad)
{
    set_error("");
    Planner *p = as_planner(ptr);
    if (!p)
        return;
    const Frame *f = static_cast<const Frame *>(frame);
    if (!f) {
        set_error("set_plan_data: null frame");
        return;
    }
    if (f->W != p->W || f->H != p->H) {
        set_error("set_plan_data: frame size differs from the planner's");
        return;
    }
    p->frame = f;
    p->req.start_x = start_x;
    p->req.start_z = start_z;
    p->req.start_heading = start_heading_rad;
    p->req.goal_x = goal_x;
    p->req.goal_z = goal_z;
    p->req.goal_heading = goal_heading_rad;
    p->req.velocity = velocity_m_s;
    p->req.min_dist_x = min_dist_x;
    p->req.min_dist_z = min_dist_z;
    p->req.max_path = maxPathSize;
    p->req.dist_tol = distToGoalTolerance;
    p->req.heading_tol = headingErrorTolerance_rad;
    p->req.seed = p->seed;
    p->req.smart = 0;
    p->req.max_iter = 0;
    p->req.stop_on_goal = 0;
    p->timeout_ms = timeout_ms;
    Engine &e = *p->eng;
    e.set_request(0, p->req);
    if (!e.bind_frame(0, f) || !e.prepare({0}, 0.8f))
        return;
    p->has_plan = true;
}

void search_init(void *ptr, bool copyIntrinsicCostsFromFrame)
{
    (void)copyIntrinsicCostsFromFrame;  // accepted and ignored, as in fastrrt.cpp:85-98
    Planner *p = as_planner(ptr);
    if (!p)
        return;
    if (!p->has_plan) {
        set_error("unable to initialize planning without planning data");
        return;
    }
    p->start_ms = now_ms();
    // clear() keeps the region densities (graph.cu:416-427)
    if (!p->eng->search_init({0}, false))
        return;
    p->eng->fetch_states(true);
}

bool goal_reached(void *ptr)
{
    Planner *p = as_planner(ptr);
    if (!p || !p->has_plan)
        return false;
    Engine &e = *p->eng;
    if (!e.fetch_states(true))
        return false;
    if (e.state(0).goal_reached)
        return true;
    if (!e.goal_check(0))
        return false;
    return e.state(0).goal_reached != 0;
}

bool loop(void *ptr, bool smartExpansion)
{
    Planner *p = as_planner(ptr);
    if (!p || !p->has_plan)
        return false;
    if (p->timed_out())
        return false;
    Engine &e = *p->eng;
    if (p->req.smart != (smartExpansion ? 1 : 0)) {
        p->req.smart = smartExpansion ? 1 : 0;
        e.set_request(0, p->req);
    }
    if (!e.iterate() || !e.fetch_states(true))
        return false;
    if (e.state(0).error) {
        set_error("loop: device wait limit reached");
        return false;
    }
    return e.state(0).goal_reached == 0;
}

static std::vector<float> planned_path(Planner *p)
{
    std::vector<float> xyh;
    if (!p->has_plan || !goal_reached(p))
        return xyh;
    p->eng->extract_path(0, xyh);
    return xyh;
}

bool path_optimize(void *ptr)
{
    Planner *p = as_planner(ptr);
    if (!p || !p->has_plan || p->timed_out())
        return false;
    if (!goal_reached(p))
        return false;
    int changed = 0;
    if (!p->eng->optimize(0, changed))
        return false;
    return changed != 0;
}

float *get_planned_path(void *ptr)
{
    Planner *p = as_planner(ptr);
    if (!p)
        return nullptr;
    return path_array(planned_path(p));
}

float *interpolate_planned_path(void *ptr)
{
    Planner *p = as_planner(ptr);
    if (!p)
        return nullptr;
    return path_array(interpolate_path(planned_path(p), p->W, p->H));
}

void release_planned_path_data(float *ptr) { delete[] ptr; }

float *interpolate_planned_path_p(void *ptr, float *pts, int size)
{
    Planner *p = as_planner(ptr);
    if (!p || (!pts && size > 0))
        return nullptr;
    std::vector<float> xyh;
    for (int i = 0; i + 2 < size; i += 3) {
        // Waypoint(int, int, angle) of the given triple
        xyh.push_back((float)(int)pts[i]);
        xyh.push_back((float)(int)pts[i + 1]);
        xyh.push_back(pts[i + 2]);
    }
    return path_array(interpolate_path(xyh, p->W, p->H));
}

float *ideal_curve(void *ptr, int goal_x, int goal_z, float goal_heading_rad)
{
    Planner *p = as_planner(ptr);
    if (!p)
        return nullptr;
    // from the coordinate origin (frame centre, heading 0), fastrrt.cpp:270-281
    const Inst &I = p->eng->inst(0);
    const int ox = (int)(I.W ? I.og_x : p->W / 2), oz = (int)(I.H ? I.og_z : p->H / 2);
    return path_array(interpolate_hermite(p->W, p->H, ox, oz, 0.0f, goal_x, goal_z, goal_heading_rad));
}

int *export_graph_nodes(void *ptr)
{
    Planner *p = as_planner(ptr);
    if (!p)
        return nullptr;
    std::vector<int8_t> type;
    std::vector<int32_t> parent, child;
    std::vector<float> heading, cost, intr, direct;
    if (p->eng->inst(0).W == 0 ||
        !p->eng->grid_download(0, type, parent, child, heading, cost, intr, direct)) {
        int *r = new int[1];
        r[0] = 0;
        return r;
    }
    std::vector<int> out;
    for (int z = 0; z < p->H; z++)
        for (int x = 0; x < p->W; x++) {
            const int t = type[(size_t)z * p->W + x];
            if (t == T_NULL)
                continue;
            out.push_back(x);
            out.push_back(z);
            out.push_back(t);
        }
    int *r = new int[out.size() + 1];
    r[0] = (int)(out.size() / 3);
    for (size_t i = 0; i < out.size(); i++)
        r[1 + i] = out[i];
    return r;
}

void release_export_graph_nodes(int *ptr) { delete[] ptr; }

int fastrrt_apf_repulsion(void *ptr, void *frame, float kr, int radius)
{
    Planner *p = as_planner(ptr);
    if (!p)
        return -1;
    return p->eng->apf_repulsion(0, static_cast<const Frame *>(frame), kr, radius) ? 0 : -1;
}

int fastrrt_apf_attraction(void *ptr, void *frame, float ka, int goal_x, int goal_z)
{
    Planner *p = as_planner(ptr);
    if (!p)
        return -1;
    return p->eng->apf_attraction(0, static_cast<const Frame *>(frame), ka, goal_x, goal_z) ? 0 : -1;
}

int fastrrt_intrinsic_costs(void *ptr, float *out)
{
    Planner *p = as_planner(ptr);
    if (!p || !out) {
        set_error("intrinsic costs: bad arguments");
        return -1;
    }
    std::vector<float> v;
    if (!p->eng->intrinsic_download(0, v))
        return -1;
    std::copy(v.begin(), v.end(), out);
    return (int)v.size();
}

int fastrrt_check_graph_consistent(void *ptr)
{
    Planner *p = as_planner(ptr);
    if (!p)
        return -1;
    if (p->eng->inst(0).W == 0) {
        set_error("check_graph_consistent: set_plan_data first");
        return -1;
    }
    int ok = 0;
    return p->eng->check_graph(0, ok) ? ok : -1;
}

int fastrrt_validate_path(void *ptr, const float *xyh, int n)
{
    Planner *p = as_planner(ptr);
    if (!p || n < 0 || (n > 0 && !xyh)) {
        set_error("validate_path: bad arguments");
        return -1;
    }
    if (p->eng->inst(0).W == 0) {
        set_error("validate_path: set_plan_data first");
        return -1;
    }
    int ok = 0;
    return p->eng->check_path(0, xyh, n, ok) ? ok : -1;
}

void compute_region_debug_performance(void *ptr)
{
    // computeGraphRegionDensity (graph_expansion_search_zones.cu:111-159)
    Planner *p = as_planner(ptr);
    if (!p || p->eng->inst(0).W == 0)
        return;
    std::vector<int8_t> type;
    std::vector<int32_t> parent, child;
    std::vector<float> heading, cost, intr, direct;
    if (!p->eng->grid_download(0, type, parent, child, heading, cost, intr, direct))
        return;
    const int dw = p->W / kRegion + 1, dh = p->H / kRegion + 1;
    std::vector<unsigned> counts((size_t)dw * dh, 0u);
    for (int z = 0; z < p->H; z++)
        for (int x = 0; x < p->W; x++) {
            const int t = type[(size_t)z * p->W + x];
            if (t == T_NULL || t == T_PROCESSING)
                continue;
            counts[(z / kRegion) * dw + x / kRegion]++;
        }
    p->eng->regions_upload(0, counts);
}

void save_current_graph_state(void *ptr, const char *filename)
{
    // CudaGraph::dumpGraph (graph.cu:496-520)
    Planner *p = as_planner(ptr);
    if (!p || !filename || p->eng->inst(0).W == 0)
        return;
    std::vector<int8_t> type;
    std::vector<int32_t> parent, child;
    std::vector<float> heading, cost, intr, direct;
    if (!p->eng->grid_download(0, type, parent, child, heading, cost, intr, direct))
        return;
    FILE *fp = fopen(filename, "w");
    if (!fp) {
        set_error(std::string("cannot open ") + filename);
        return;
    }
    for (size_t i = 0; i < type.size(); i++)
        fprintf(fp, "%d %d %d %d %f %f %f %f\n", unpack_x(parent[i]), unpack_z(parent[i]), (int)type[i],
                child[i], heading[i], cost[i], intr[i], direct[i]);
    fclose(fp);
}

void load_graph_state(void *ptr, const char *filename)
{
    // CudaGraph::readfromDump (graph.cu:522-546) + FastRRT::loadGraphState
    // (fastrrt.cpp:293-297)
    Planner *p = as_planner(ptr);
    if (!p || !filename)
        return;
    Engine &e = *p->eng;
    if (e.inst(0).W == 0) {
        set_error("load_graph_state: set_plan_data first");
        return;
    }
    FILE *fp = fopen(filename, "r");
    if (!fp) {
        set_error(std::string("cannot open ") + filename);
        return;
    }
    const size_t n = (size_t)p->W * p->H;
    std::vector<int8_t> type(n);
    std::vector<int32_t> parent(n), child(n);
    std::vector<float> heading(n), cost(n), intr(n), direct(n);
    int temps = 0;
    for (size_t i = 0; i < n; i++) {
        int px = 0, pz = 0, t = 0, c = 0;
        float h = 0, co = 0, in = 0, d = 0;
        if (fscanf(fp, "%d %d %d %d %f %f %f %f\n", &px, &pz, &t, &c, &h, &co, &in, &d) != 8)
            break;
        type[i] = (int8_t)t;
        parent[i] = pack_xz(px, pz);
        child[i] = c;
        heading[i] = h;
        cost[i] = co;
        intr[i] = in;
        direct[i] = d;
        temps += t == T_TEMP;
    }
    fclose(fp);
    if (e.grid_upload(0, type, parent, child, heading, cost, intr, direct))
        e.set_state_field_last_expanded(0, temps);
}

int fastrrt_probe_count(void *ptr, uint64_t *probes)
{
    Planner *p = as_planner(ptr);
    if (!p || !probes)
        return -1;
    if (!p->eng->fetch_states(true))
        return -1;
    const State &S = p->eng->state(0);
    *probes = S.probes + S.probes_goal + S.probes_pre;
    return 0;
}

int fastrrt_loop_count(void *ptr)
{
    Planner *p = as_planner(ptr);
    if (!p || !p->eng->fetch_states(true))
        return -1;
    return p->eng->state(0).loops;
}

// ---------------------------------------------------------------------------
// per-candidate kernels
// ---------------------------------------------------------------------------


void *fastrrt_candidates_create(void *frame, int min_dist_x, int min_dist_z, int lowerBound_x,
                                int lowerBound_z, int upperBound_x, int upperBound_z,
                                double max_steering_rad, double lr_m, const float *heading_grid,
                                const float *cost_grid)
{
    const Frame *f = static_cast<const Frame *>(frame);
    if (!f) {
        set_error("candidates: null frame");
        return nullptr;
    }
    auto *c = new (std::nothrow) Candidates();
    if (!c)
        return nullptr;
    c->eng.reset(new (std::nothrow) Engine(1, f->W, f->H));
    if (!c->eng || !c->eng->ok()) {
        delete c;
        return nullptr;
    }
    c->W = f->W;
    c->H = f->H;
    Engine &e = *c->eng;
    Physical ph{};
    ph.pw_m = (float)f->W;
    ph.ph_m = (float)f->H;
    ph.max_steer_rad = max_steering_rad;
    ph.vehicle_len = (float)(2 * lr_m);
    ph.max_curvature = -1;
    ph.lbx = lowerBound_x;
    ph.lbz = lowerBound_z;
    ph.ubx = upperBound_x;
    ph.ubz = upperBound_z;
    e.set_physical(0, ph);
    e.inst(0).lr = lr_m;  // exact lr, not round-tripped through a float length
    PlanRequest r{};
    r.min_dist_x = min_dist_x;
    r.min_dist_z = min_dist_z;
    r.velocity = 1.0f;
    r.max_path = 40.0f;
    r.dist_tol = 20.0f;
    r.heading_tol = 0.1745329f;
    r.goal_x = f->W / 2;
    r.goal_z = 0;
    e.set_request(0, r);
    if (!e.bind_frame(0, f) || !e.commit()) {
        delete c;
        return nullptr;
    }
    const size_t n = (size_t)f->W * f->H;
    std::vector<float> zeros(n, 0.0f);
    const Inst &I = e.inst(0);
    bool ok = cudaMemcpy(I.heading, heading_grid ? heading_grid : zeros.data(), 4 * n,
                         cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(I.cost, cost_grid ? cost_grid : zeros.data(), 4 * n, cudaMemcpyHostToDevice) ==
                  cudaSuccess;
    // masks only (the goal precompute is not needed here); the precompute
    // runs as part of prepare() and is cheap for one frame
    if (!ok || !e.prepare({0}, 0.8f)) {
        if (!ok)
            set_error("candidates: grid upload failed");
        delete c;
        return nullptr;
    }
    return c;
}

void fastrrt_candidates_destroy(void *ctx) { delete static_cast<Candidates *>(ctx); }

int fastrrt_candidates_kinematic_device(void *ctx, int n, const int32_t *sx, const int32_t *sz,
                                        const float *steer, const float *length, float velocity_m_s,
                                        float *out4, uint64_t *probes, void *stream)
{
    auto *c = static_cast<Candidates *>(ctx);
    if (!c || n < 0) {
        set_error("candidates: bad arguments");
        return -1;
    }
    (void)stream;
    if (!c->eng->candidates(0, n, sx, sz, steer, length, velocity_m_s,
                            reinterpret_cast<float4 *>(out4),
                            reinterpret_cast<unsigned long long *>(probes)))
        return -1;
    return 0;
}

int fastrrt_candidates_kinematic(void *ctx, int n, const int32_t *sx, const int32_t *sz,
                                 const float *steer, const float *length, float velocity_m_s,
                                 float *out4, uint64_t *probes)
{
    auto *c = static_cast<Candidates *>(ctx);
    if (!c || n < 0 || (n > 0 && (!sx || !sz || !steer || !length || !out4))) {
        set_error("candidates: bad arguments");
        return -1;
    }
    if (n == 0)
        return 0;
    if (!cells_in_frame(c, n, sx, sz))
        return -1;
    cudaStream_t st = c->eng->stream();
    DevBuf<int32_t> dsx, dsz;
    DevBuf<float> dst, dln, dout;
    DevBuf<unsigned long long> dpr;
    if (!dsx.alloc(n) || !dsz.alloc(n) || !dst.alloc(n) || !dln.alloc(n) || !dout.alloc(4 * (size_t)n) ||
        !dpr.alloc(1)) {
        set_error("candidates: device allocation failed");
        return -1;
    }
    bool ok = cudaMemcpyAsync(dsx.p, sx, 4 * (size_t)n, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(dsz.p, sz, 4 * (size_t)n, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(dst.p, steer, 4 * (size_t)n, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(dln.p, length, 4 * (size_t)n, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemsetAsync(dpr.p, 0, 8, st) == cudaSuccess;
    ok = ok && c->eng->candidates(0, n, dsx.p, dsz.p, dst.p, dln.p, velocity_m_s,
                                  reinterpret_cast<float4 *>(dout.p), dpr.p);
    unsigned long long pr = 0;
    ok = ok && cudaMemcpyAsync(out4, dout.p, 16 * (size_t)n, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaMemcpyAsync(&pr, dpr.p, 8, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) {
        set_error(std::string("candidates: ") + cudaGetErrorString(cudaGetLastError()));
        return -1;
    }
    if (probes)
        *probes = pr;
    return 0;
}

int fastrrt_candidates_hermite_device(void *ctx, int n, const int32_t *x, const int32_t *z,
                                      const float *local_heading, const int32_t *goal_x,
                                      const int32_t *goal_z, const float *goal_heading,
                                      float max_curvature, int safe_zone_checked, float *out,
                                      uint64_t *probes, void *stream)
{
    auto *c = static_cast<Candidates *>(ctx);
    if (!c || n < 0) {
        set_error("candidates: bad arguments");
        return -1;
    }
    (void)stream;
    return c->eng->hermite(0, n, x, z, local_heading, goal_x, goal_z, goal_heading, max_curvature,
                           safe_zone_checked, out, reinterpret_cast<unsigned long long *>(probes))
               ? 0
               : -1;
}

int fastrrt_candidates_hermite(void *ctx, int n, const int32_t *x, const int32_t *z,
                               const float *local_heading, const int32_t *goal_x,
                               const int32_t *goal_z, const float *goal_heading,
                               float max_curvature, int safe_zone_checked, float *out,
                               uint64_t *probes)
{
    auto *c = static_cast<Candidates *>(ctx);
    if (!c || n < 0 || (n > 0 && (!x || !z || !local_heading || !goal_x || !goal_z || !goal_heading || !out))) {
        set_error("candidates: bad arguments");
        return -1;
    }
    if (n == 0)
        return 0;
    if (!cells_in_frame(c, n, x, z))
        return -1;
    cudaStream_t st = c->eng->stream();
    DevBuf<int32_t> dx, dz, dgx, dgz;
    DevBuf<float> dlh, dgh, dout;
    DevBuf<unsigned long long> dpr;
    if (!dx.alloc(n) || !dz.alloc(n) || !dgx.alloc(n) || !dgz.alloc(n) || !dlh.alloc(n) ||
        !dgh.alloc(n) || !dout.alloc(n) || !dpr.alloc(1)) {
        set_error("candidates: device allocation failed");
        return -1;
    }
    const size_t b = 4 * (size_t)n;
    bool ok = cudaMemcpyAsync(dx.p, x, b, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(dz.p, z, b, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(dgx.p, goal_x, b, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(dgz.p, goal_z, b, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(dlh.p, local_heading, b, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(dgh.p, goal_heading, b, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemsetAsync(dpr.p, 0, 8, st) == cudaSuccess;
    ok = ok && c->eng->hermite(0, n, dx.p, dz.p, dlh.p, dgx.p, dgz.p, dgh.p, max_curvature,
                               safe_zone_checked, dout.p, dpr.p);
    unsigned long long pr = 0;
    ok = ok && cudaMemcpyAsync(out, dout.p, b, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaMemcpyAsync(&pr, dpr.p, 8, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) {
        set_error(std::string("candidates: ") + cudaGetErrorString(cudaGetLastError()));
        return -1;
    }
    if (probes)
        *probes = pr;
    return 0;
}

int fastrrt_candidates_feasible(void *ctx, int n, const int32_t *x, const int32_t *z,
                                const float *angle, int32_t *out, uint64_t *probes)
{
    auto *c = static_cast<Candidates *>(ctx);
    if (!c || n < 0 || (n > 0 && (!x || !z || !angle || !out))) {
        set_error("candidates: bad arguments");
        return -1;
    }
    if (n == 0)
        return 0;
    if (!cells_in_frame(c, n, x, z))
        return -1;
    cudaStream_t st = c->eng->stream();
    DevBuf<int32_t> dx, dz, dout;
    DevBuf<float> da;
    DevBuf<unsigned long long> dpr;
    if (!dx.alloc(n) || !dz.alloc(n) || !dout.alloc(n) || !da.alloc(n) || !dpr.alloc(1)) {
        set_error("candidates: device allocation failed");
        return -1;
    }
    const size_t b = 4 * (size_t)n;
    bool ok = cudaMemcpyAsync(dx.p, x, b, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(dz.p, z, b, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(da.p, angle, b, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemsetAsync(dpr.p, 0, 8, st) == cudaSuccess;
    ok = ok && c->eng->feasible(0, n, dx.p, dz.p, da.p, dout.p, dpr.p);
    unsigned long long pr = 0;
    ok = ok && cudaMemcpyAsync(out, dout.p, b, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaMemcpyAsync(&pr, dpr.p, 8, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) {
        set_error(std::string("candidates: ") + cudaGetErrorString(cudaGetLastError()));
        return -1;
    }
    if (probes)
        *probes = pr;
    return 0;
}

// ---------------------------------------------------------------------------
// batched planner
// ---------------------------------------------------------------------------


void *fastrrt_batch_create(int n_slots, int max_width, int max_height)
{
    auto *b = new (std::nothrow) Batch();
    if (!b)
        return nullptr;
    b->eng.reset(new (std::nothrow) Engine(n_slots, max_width, max_height));
    if (!b->eng || !b->eng->ok() || cudaEventCreate(&b->ev0) != cudaSuccess ||
        cudaEventCreate(&b->ev1) != cudaSuccess) {
        delete b;
        return nullptr;
    }
    return b;
}

void *fastrrt_batch_create_budget(int max_slots, int max_width, int max_height, uint64_t budget_bytes)
{
    if (budget_bytes == 0) {
        set_error("batch create: a memory budget of 0 bytes");
        return nullptr;
    }
    auto *b = new (std::nothrow) Batch();
    if (!b)
        return nullptr;
    b->eng.reset(new (std::nothrow) Engine(max_slots, max_width, max_height, -1, (size_t)budget_bytes));
    if (!b->eng || !b->eng->ok() || cudaEventCreate(&b->ev0) != cudaSuccess ||
        cudaEventCreate(&b->ev1) != cudaSuccess) {
        delete b;
        return nullptr;
    }
    return b;
}

int fastrrt_batch_memory(void *batch, uint64_t *budget, uint64_t *used, uint64_t *peak)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b) {
        set_error("batch memory: bad arguments");
        return -1;
    }
    if (budget)
        *budget = b->eng->budget();
    if (used)
        *used = b->eng->used();
    if (peak)
        *peak = b->eng->peak_used();
    return 0;
}

uint64_t fastrrt_slot_bytes(int width, int height)
{
    return width > 0 && height > 0 ? (uint64_t)Engine::slot_bytes(width, height) : 0;
}

void fastrrt_batch_destroy(void *batch) { delete static_cast<Batch *>(batch); }

int fastrrt_batch_admit_many(void *batch, int n, const fastrrt_request *reqs, int timeout_ms)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || !reqs || n < 0 || n > b->eng->n_slots()) {
        set_error("batch admit: bad arguments");
        return -1;
    }
    Engine &e = *b->eng;
    std::vector<int> slots;
    for (int k = 0; k < n; k++) {
        if (!load_request(e, k, reqs[k], timeout_ms))
            return -1;
        slots.push_back(k);
    }
    if (!e.prepare(slots, 0.8f, true) || !e.search_init(slots, true) || !e.sync())
        return -1;
    b->admitted = slots;
    return 0;
}

int fastrrt_batch_admit(void *batch, int slot, const fastrrt_request *req, int timeout_ms)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || !req || slot < 0 || slot >= b->eng->n_slots()) {
        set_error("batch admit: bad arguments");
        return -1;
    }
    Engine &e = *b->eng;
    if (!load_request(e, slot, *req, timeout_ms) || !e.prepare({slot}, 0.8f, true) || !e.search_init({slot}, true) ||
        !e.sync())
        return -1;
    return 0;
}

int fastrrt_batch_step(void *batch)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b)
        return -1;
    return b->eng->iterate() ? 0 : -1;
}

int fastrrt_batch_run(void *batch, int max_launches, int check_every)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b)
        return -1;
    Engine &e = *b->eng;
    if (check_every <= 0)
        check_every = 1;
    int launches = 0;
    cudaEventRecord(b->ev0, e.stream());
    while (launches < max_launches) {
        for (int k = 0; k < check_every && launches < max_launches; k++, launches++)
            if (!e.iterate())
                return -1;
        if (!e.fetch_states(true))
            return -1;
        bool all_done = true;
        for (int s = 0; s < e.n_slots(); s++) {
            const State &S = e.state(s);
            if (S.active && !S.done) {
                all_done = false;
                break;
            }
        }
        if (all_done)
            break;
    }
    cudaEventRecord(b->ev1, e.stream());
    cudaEventSynchronize(b->ev1);
    cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
    return launches;
}

float fastrrt_batch_last_ms(void *batch)
{
    auto *b = static_cast<Batch *>(batch);
    return b ? b->last_ms : -1.0f;
}

int fastrrt_batch_status(void *batch, int32_t *done, int32_t *goal, int32_t *loops)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b)
        return -1;
    Engine &e = *b->eng;
    if (!e.fetch_states(true))
        return -1;
    for (int s = 0; s < e.n_slots(); s++) {
        const State &S = e.state(s);
        if (done)
            done[s] = S.active ? S.done : 1;
        if (goal)
            goal[s] = S.goal_reached;
        if (loops)
            loops[s] = S.loops;
    }
    return 0;
}

int fastrrt_batch_collect(void *batch, int n, const int32_t *slots, int32_t *valid, float *length,
                          int32_t *path_n)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || n < 0 || (n > 0 && !slots)) {
        set_error("batch collect: bad arguments");
        return -1;
    }
    Engine &e = *b->eng;
    std::vector<int> list(slots, slots + n);
    if (!e.extract_and_validate(list, 1024))
        return -1;
    int good = 0;
    for (int k = 0; k < n; k++) {
        // a path only counts when the slot reached its goal
        const int v = e.valid()[k] && e.state(list[k]).goal_reached;
        if (valid)
            valid[k] = v;
        if (length)
            length[k] = e.lengths()[k];
        if (path_n)
            path_n[k] = e.paths_n()[k];
        good += v;
    }
    return good;
}

int fastrrt_batch_path(void *batch, int k, float *xyh, int cap)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || k < 0 || k >= (int)b->eng->paths_n().size()) {
        set_error("batch path: bad index");
        return -1;
    }
    const int m = std::min(b->eng->paths_n()[k], cap);
    const size_t stride = b->eng->paths().size() / b->eng->paths_n().size();
    for (int i = 0; i < 3 * m; i++)
        xyh[i] = b->eng->paths()[(size_t)k * stride + i];
    return m;
}

int fastrrt_batch_interpolate(void *batch, int cap, float *length, float *jerk, int32_t *tan_disc)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || cap <= 0) {
        set_error("batch interpolate: bad arguments");
        return -1;
    }
    Engine &e = *b->eng;
    if (!e.interpolate_last(cap))
        return -1;
    const int n = (int)e.interp_n().size();
    for (int k = 0; k < n; k++) {
        if (length)
            length[k] = e.interp_length()[k];
        if (jerk)
            jerk[k] = e.interp_jerk()[k];
        if (tan_disc)
            tan_disc[k] = e.interp_disc()[k];
    }
    return n;
}

int fastrrt_batch_interpolated_path(void *batch, int k, float *xyh, int cap)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || k < 0 || k >= (int)b->eng->interp_n().size() || !xyh || cap < 0) {
        set_error("batch interpolated path: bad index");
        return -1;
    }
    const Engine &e = *b->eng;
    const int m = std::min(e.interp_n()[k], cap);
    const size_t stride = (size_t)3 * e.interp_cap();
    for (int i = 0; i < 3 * m; i++)
        xyh[i] = e.interp_points()[(size_t)k * stride + i];
    return m;
}

int fastrrt_batch_plan(void *batch, int n, const fastrrt_request *reqs, int max_launches,
                       int check_every, int32_t *valid, float *length, float *latency_ms,
                       float *device_ms)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || !reqs || n <= 0 || n > b->eng->n_slots()) {
        set_error("batch plan: bad arguments");
        return -1;
    }
    Engine &e = *b->eng;
    cudaEvent_t e0 = b->ev0, e_adm = nullptr;
    if (cudaEventCreate(&e_adm) != cudaSuccess) {
        set_error("batch plan: event");
        return -1;
    }
    cudaEventRecord(e0, e.stream());
    std::vector<int> slots;
    for (int k = 0; k < n; k++) {
        if (!load_request(e, k, reqs[k])) {
            cudaEventDestroy(e_adm);
            return -1;
        }
        slots.push_back(k);
    }
    for (int s = n; s < e.n_slots(); s++)
        if (e.state(s).active)
            e.deactivate(s);
    const bool adm = e.prepare(slots, 0.8f, true) && e.search_init(slots, true);
    cudaEventRecord(e_adm, e.stream());
    if (!adm) {
        cudaEventDestroy(e_adm);
        return -1;
    }
    int launches = 0;
    if (check_every <= 0)
        check_every = 1;
    bool ok = true;
    while (ok && launches < max_launches) {
        for (int k = 0; k < check_every && launches < max_launches && ok; k++, launches++)
            ok = e.iterate();
        ok = ok && e.fetch_states(true);
        if (!ok)
            break;
        bool all_done = true;
        for (int s = 0; s < n; s++)
            if (e.state(s).active && !e.state(s).done) {
                all_done = false;
                break;
            }
        if (all_done)
            break;
    }
    ok = ok && e.extract_and_validate(slots, 1024);
    cudaEventRecord(b->ev1, e.stream());
    cudaEventSynchronize(b->ev1);
    float adm_ms = 0, total_ms = 0;
    cudaEventElapsedTime(&adm_ms, e0, e_adm);
    cudaEventElapsedTime(&total_ms, e0, b->ev1);
    cudaEventDestroy(e_adm);
    if (!ok)
        return -1;
    b->last_ms = total_ms;
    if (device_ms)
        *device_ms = total_ms;
    int good = 0;
    for (int k = 0; k < n; k++) {
        const State &S = e.state(k);
        const int v = e.valid()[k] && S.goal_reached;
        good += v;
        if (valid)
            valid[k] = v;
        if (length)
            length[k] = e.lengths()[k];
        if (latency_ms) {
            const long long fin = S.finish_ns ? S.finish_ns : S.start_ns;
            latency_ms[k] = adm_ms + (float)((fin - S.start_ns) * 1e-6);
        }
    }
    return good;
}

int fastrrt_batch_serve(void *batch, int n, const fastrrt_request *reqs, const double *arrival_ms,
                        int timeout_ms, int check_every, int32_t *valid, float *length,
                        float *latency_ms, float *service_ms, int32_t *loops, double *wall_ms,
                        float *device_ms, float *result_ms)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || n < 0 || (n > 0 && !reqs)) {
        set_error("batch serve: bad arguments");
        return -1;
    }
    if (arrival_ms)
        for (int k = 0; k < n; k++)
            if (!(arrival_ms[k] >= 0.0) || (k > 0 && arrival_ms[k] < arrival_ms[k - 1])) {
                set_error("batch serve: arrival times must be finite, >= 0 and non-decreasing");
                return -1;
            }
    Engine &e = *b->eng;
    const int n_slots = e.n_slots();
    if (check_every <= 0)
        check_every = 1;
    // slots left live by an earlier call take no part
    if (!e.fetch_states(true))
        return -1;
    for (int s = 0; s < n_slots; s++) {
        if (e.state(s).active && !e.state(s).done && !e.deactivate(s))
            return -1;
        e.release_storage(s);  // budget mode: the whole arena for this call
    }
    // device clock -> host clock: one read bracketed by host reads
    long long dev0 = 0;
    const double ha = now_ms();
    if (!e.device_clock(dev0))
        return -1;
    const double host_at_dev0 = 0.5 * (ha + now_ms());
    const double t0 = now_ms();
    cudaEventRecord(b->ev0, e.stream());
    auto finish_ms = [&](long long ns) { return host_at_dev0 + (double)(ns - dev0) * 1e-6 - t0; };

    std::vector<int> free_slots, owner(n_slots, -1), list;
    for (int s = n_slots - 1; s >= 0; s--)
        free_slots.push_back(s);
    std::vector<double> admitted_at(n, 0.0);
    int next = 0, finished = 0, in_flight = 0, good = 0;
    while (finished < n) {
        // admit every request that has arrived while a slot is free
        const double now = now_ms() - t0;
        list.clear();
        while (next < n && !free_slots.empty() && (!arrival_ms || arrival_ms[next] <= now)) {
            const int s = free_slots.back();
            // admission by device memory: the request waits (in arrival
            // order) until the arena has room for its frame's storage
            if (!e.ensure_storage(s, reqs[next].width, reqs[next].height)) {
                if (!e.out_of_budget())
                    return -1;
                if (in_flight == 0 && list.empty()) {
                    set_error("batch serve: a request needs more memory than the whole budget");
                    return -1;
                }
                break;
            }
            free_slots.pop_back();
            if (!load_request(e, s, reqs[next], timeout_ms))
                return -1;
            owner[s] = next;
            admitted_at[next] = now;
            list.push_back(s);
            next++;
        }
        if (!list.empty()) {
            if (!e.prepare(list, 0.8f, true) || !e.search_init(list, true))
                return -1;
            in_flight += (int)list.size();
        }
        if (in_flight == 0) {
            if (!arrival_ms || next >= n) {
                set_error("batch serve: no free slot");
                return -1;
            }
            // nothing on the GPU: wait for the next arrival
            const double wait = arrival_ms[next] - (now_ms() - t0);
            if (wait > 0)
                std::this_thread::sleep_for(std::chrono::microseconds(
                    (long long)std::min(wait * 1000.0, 200.0)));
            continue;
        }
        for (int k = 0; k < check_every; k++)
            if (!e.iterate())
                return -1;
        if (!e.fetch_states(true))
            return -1;
        // harvest finished slots and free them
        list.clear();
        for (int s = 0; s < n_slots; s++)
            if (owner[s] >= 0 && e.state(s).done)
                list.push_back(s);
        if (list.empty())
            continue;
        if (!e.extract_and_validate(list, 1024, false))
            return -1;
        // the paths and verdicts of these requests are on the host now
        const double ready = now_ms() - t0;
        for (size_t k = 0; k < list.size(); k++) {
            const int s = list[k];
            const int r = owner[s];
            const State &S = e.state(s);
            if (result_ms)
                result_ms[r] = (float)(ready - (arrival_ms ? arrival_ms[r] : 0.0));
            const int v = e.valid()[k] && S.goal_reached;
            good += v;
            const double fin = finish_ms(S.finish_ns);
            if (valid)
                valid[r] = v;
            if (length)
                length[r] = e.lengths()[k];
            if (latency_ms)
                latency_ms[r] = (float)(fin - (arrival_ms ? arrival_ms[r] : 0.0));
            if (service_ms)
                service_ms[r] = (float)(fin - admitted_at[r]);
            if (loops)
                loops[r] = S.loops;
            owner[s] = -1;
            free_slots.push_back(s);
            e.release_storage(s);  // budget mode: back to the arena
            in_flight--;
            finished++;
        }
    }
    cudaEventRecord(b->ev1, e.stream());
    cudaEventSynchronize(b->ev1);
    if (wall_ms)
        *wall_ms = now_ms() - t0;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    b->last_ms = ms;
    if (device_ms)
        *device_ms = ms;
    return good;
}

int fastrrt_batch_set_launch(void *batch, int sweep_blocks_per_sm, int work_blocks_per_sm)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b) {
        set_error("batch set_launch: bad arguments");
        return -1;
    }
    return b->eng->set_launch(sweep_blocks_per_sm, work_blocks_per_sm) ? 0 : -1;
}

int fastrrt_batch_set_proposal(void *batch, void *mlp, float mix, int cap)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || (mlp && (cap <= 0 || !(mix >= 0.0f && mix <= 1.0f)))) {
        set_error("batch set_proposal: bad arguments");
        return -1;
    }
    if (!mlp)
        return b->eng->set_proposal(nullptr, 0.0f, 0) ? 0 : -1;
    const MlpWeights w = static_cast<Mlp *>(mlp)->weights();
    return b->eng->set_proposal(&w, mix, cap) ? 0 : -1;
}

int fastrrt_batch_log_paths(void *batch, void *X_bf16, int32_t *labels, int offset, int cap)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || !X_bf16 || !labels || offset < 0 || cap < offset) {
        set_error("batch log_paths: bad arguments");
        return -1;
    }
    return b->eng->log_paths(static_cast<__nv_bfloat16 *>(X_bf16), labels, offset, cap);
}

int fastrrt_batch_log_nodes(void *batch, void *X_bf16, int32_t *labels, int offset, int cap)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || !X_bf16 || !labels || offset < 0 || cap < offset) {
        set_error("batch log_nodes: bad arguments");
        return -1;
    }
    return b->eng->log_paths(static_cast<__nv_bfloat16 *>(X_bf16), labels, offset, cap, true);
}

int fastrrt_batch_probes(void *batch, uint64_t *expand, uint64_t *goal, uint64_t *precompute)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || !b->eng->fetch_states(true))
        return -1;
    uint64_t a = 0, g = 0, p = 0;
    for (int s = 0; s < b->eng->n_slots(); s++) {
        a += b->eng->state(s).probes;
        g += b->eng->state(s).probes_goal;
        p += b->eng->state(s).probes_pre;
    }
    if (expand)
        *expand = a;
    if (goal)
        *goal = g;
    if (precompute)
        *precompute = p;
    return 0;
}

int fastrrt_batch_direct_connections(void *batch, int slot, uint8_t *flag, float *cost,
                                     float *heading)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || slot < 0 || slot >= b->eng->n_slots() || !flag || !cost || !heading) {
        set_error("batch_direct_connections: bad arguments");
        return -1;
    }
    Engine &e = *b->eng;
    if (!e.sync())
        return -1;
    const Inst &I = e.inst(slot);
    const size_t cells = (size_t)I.W * I.H;
    cudaError_t err = cudaMemcpy(flag, I.gd_flag, cells, cudaMemcpyDeviceToHost);
    if (err == cudaSuccess)
        err = cudaMemcpy(cost, I.gd_cost, cells * sizeof(float), cudaMemcpyDeviceToHost);
    if (err == cudaSuccess)
        err = cudaMemcpy(heading, I.gd_heading, cells * sizeof(float), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) {
        set_error(std::string("batch_direct_connections: ") + cudaGetErrorString(err));
        return -1;
    }
    return 0;
}

int fastrrt_batch_profile(void *batch, int on)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b)
        return -1;
    return b->eng->set_profiling(on != 0) ? 0 : -1;
}

int fastrrt_kernel_count(void) { return kIterKernels + 1; }

const char *fastrrt_kernel_name(int k)
{
    if (k >= 0 && k < kIterKernels)
        return kIterKernelNames[k];
    if (k == kIterKernels)
        return "k_gd_reset";
    return "";
}

int fastrrt_batch_kernel_times(void *batch, double *ms, int64_t *launches)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || !ms || !launches)
        return -1;
    Engine &e = *b->eng;
    if (e.kernel_ms().size() < (size_t)kIterKernels) {
        set_error("kernel times: profiling is off");
        return -1;
    }
    for (int k = 0; k < kIterKernels; k++) {
        ms[k] = e.kernel_ms()[k];
        launches[k] = e.kernel_launches()[k];
    }
    ms[kIterKernels] = e.precompute_ms();
    launches[kIterKernels] = e.precompute_launches();
    return 0;
}

int fastrrt_batch_release(void *batch, int slot)
{
    auto *b = static_cast<Batch *>(batch);
    if (!b || slot < 0 || slot >= b->eng->n_slots())
        return -1;
    if (!b->eng->deactivate(slot))
        return -1;
    b->eng->release_storage(slot);
    return 0;
}

}  // extern "C"
