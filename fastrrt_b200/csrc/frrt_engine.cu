// frrt_engine.cu -- host runtime of the B200 FastRRT planner.
#include "frrt_engine.h"

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace frrt {

namespace {
thread_local std::string g_last_error;

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

constexpr int kMaxClasses = 256;
constexpr int kOptCap = 1024;          // path_optimize handles paths up to this many waypoints
constexpr int kSmemLimit = 200 * 1024; // dynamic shared memory for the two staged masks
constexpr size_t kStateHead = sizeof(State);
}  // namespace

void set_error(const std::string &msg) { g_last_error = msg; }
const char *last_error() { return g_last_error.c_str(); }

// ---------------------------------------------------------------------------
// frames
// ---------------------------------------------------------------------------

Frame::~Frame()
{
    cudaFree(d_cls);
    cudaFree(d_costs);
    cudaFree(d_trav);
    cudaFree(d_dist);
}

bool frame_process_distance_to_goal(Frame *f, int goal_x, int goal_z)
{
    if (!f) {
        set_error("frame: null");
        return false;
    }
    if (!f->d_dist && cudaMalloc(&f->d_dist, sizeof(float) * (size_t)f->W * f->H) != cudaSuccess) {
        set_error("frame: distance channel allocation failed");
        return false;
    }
    launch_frame_distance(f->W, f->H, goal_x, goal_z, f->d_dist, 0);
    if (cudaDeviceSynchronize() != cudaSuccess) {
        set_error(std::string("frame: distance to goal: ") + cudaGetErrorString(cudaGetLastError()));
        return false;
    }
    f->distance_processed = true;
    return true;
}

bool frame_process_safe_zone(Frame *f, int min_dist_x, int min_dist_z)
{
    if (!f || min_dist_x < 0 || min_dist_z < 0) {
        set_error("frame: bad safe-zone arguments");
        return false;
    }
    const size_t n = (size_t)f->W * f->H;
    if (!f->d_trav) {
        if (cudaMalloc(&f->d_trav, sizeof(int32_t) * n) != cudaSuccess ||
            cudaMemset(f->d_trav, 0, sizeof(int32_t) * n) != cudaSuccess) {
            set_error("frame: traversability channel allocation failed");
            return false;
        }
    }
    uint8_t *rows = nullptr;
    if (cudaMalloc(&rows, n) != cudaSuccess) {
        set_error("frame: safe-zone scratch allocation failed");
        return false;
    }
    // setSearchParams (graph.cu:306-314): half extents TO_INT((float)min / 2)
    const int mdx = (int)((float)min_dist_x / 2), mdz = (int)((float)min_dist_z / 2);
    const int rc = (int)std::floor(std::sqrt((double)mdx * mdx + (double)mdz * mdz)) + 2;
    launch_frame_safe_zone(f->W, f->H, f->d_cls, f->d_costs, f->n_classes, rc, rows, f->d_trav, 0);
    const cudaError_t e = cudaDeviceSynchronize();
    cudaFree(rows);
    if (e != cudaSuccess) {
        set_error(std::string("frame: safe zone: ") + cudaGetErrorString(e));
        return false;
    }
    f->safe_zone_checked = true;
    return true;
}

Frame *frame_create(int W, int H, const uint8_t *cls, const float *costs, int n_classes,
                    const int32_t *trav)
{
    if (W <= 0 || H <= 0 || W > 4095 || H > 4095) {
        set_error("frame size must be within 1..4095");
        return nullptr;
    }
    if (!cls || !costs || n_classes <= 0 || n_classes > kMaxClasses) {
        set_error("frame needs class ids and 1..256 class costs");
        return nullptr;
    }
    const long n = (long)W * H;
    for (long i = 0; i < n; i++)
        if (cls[i] >= n_classes) {
            set_error("frame class id outside the class-cost table");
            return nullptr;
        }
    Frame *f = new Frame();
    f->W = W;
    f->H = H;
    f->n_classes = n_classes;
    f->h_costs.assign(costs, costs + n_classes);
    const size_t padded = align_up((size_t)n, 4096);
    bool ok = cudaMalloc(&f->d_cls, padded) == cudaSuccess &&
              cudaMalloc(&f->d_costs, sizeof(float) * kMaxClasses) == cudaSuccess;
    ok = ok && cudaMemset(f->d_cls, 0, padded) == cudaSuccess &&
         cudaMemcpy(f->d_cls, cls, (size_t)n, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(f->d_costs, 0, sizeof(float) * kMaxClasses) == cudaSuccess &&
         cudaMemcpy(f->d_costs, costs, sizeof(float) * n_classes, cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok && trav)
        ok = cudaMalloc(&f->d_trav, sizeof(int32_t) * (size_t)n) == cudaSuccess &&
             cudaMemcpy(f->d_trav, trav, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) {
        set_error(std::string("frame upload failed: ") + cudaGetErrorString(cudaGetLastError()));
        delete f;
        return nullptr;
    }
    return f;
}

Frame *frame_create_f3(int W, int H, const float *xyz, const float *costs, int n_classes)
{
    if (!xyz || W <= 0 || H <= 0) {
        set_error("frame data is null or empty");
        return nullptr;
    }
    const long n = (long)W * H;
    std::vector<uint8_t> cls((size_t)n);
    std::vector<int32_t> trav((size_t)n);
    bool any_trav = false;
    for (long i = 0; i < n; i++) {
        const int c = (int)xyz[3 * i];  // TO_INT(frame.x)
        if (c < 0 || c >= kMaxClasses) {
            set_error("frame class id outside 0..255");
            return nullptr;
        }
        cls[i] = (uint8_t)c;
        trav[i] = (int32_t)xyz[3 * i + 2];  // TO_INT(frame.z)
        any_trav = any_trav || trav[i] != 0;
    }
    Frame *f = frame_create(W, H, cls.data(), costs, n_classes, any_trav ? trav.data() : nullptr);
    if (!f)
        return nullptr;
    // the distance channel (frame.y), kept for isDistanceToGoalProcessed
    std::vector<float> dist((size_t)n);
    for (long i = 0; i < n; i++)
        dist[i] = xyz[3 * i + 1];
    if (cudaMalloc(&f->d_dist, sizeof(float) * (size_t)n) != cudaSuccess ||
        cudaMemcpy(f->d_dist, dist.data(), sizeof(float) * (size_t)n, cudaMemcpyHostToDevice) != cudaSuccess) {
        set_error("frame: distance channel upload failed");
        delete f;
        return nullptr;
    }
    return f;
}

// ---------------------------------------------------------------------------
// engine
// ---------------------------------------------------------------------------

bool Engine::check(cudaError_t e, const char *what)
{
    if (e == cudaSuccess)
        return true;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

// byte sizes of the parts of one slot's storage for a W x H frame (C = cells
// rounded up to a sweep chunk), each part 256-byte aligned
namespace {
constexpr int kParts = 37;
void slot_parts(int W, int H, size_t parts[kParts])
{
    const size_t C = align_up((size_t)W * H, kSweepCells);
    const size_t mw = align_up((size_t)((W + 31) / 32) * H, 4);
    const size_t p[kParts] = {
        C,                                  // 0 type
        4 * C, 4 * C,                       // 1 parent, 2 child
        4 * C, 4 * C, 4 * C, 4 * C,         // 3 heading, 4 cost, 5 intrinsic, 6 direct
        C, 4 * C, 4 * C,                    // 7 gd flag, 8 heading, 9 cost
        4 * C,                              // 10 claim
        4 * C, 4 * C, 4 * C, 4 * C,         // 11 cand, 12 end, 13 heading, 14 cost
        4 * C, 8 * C, 4 * C, 4 * C,         // 15 nodes, 16 best key, 17 pending, 18 pruned
        C,                                  // 19 own class ids
        4 * mw,                             // 20 blocked
        4 * mw,                             // 21 clear
        4 * (size_t)kMaxRegions,            // 22 region_count
        4 * (size_t)kMaxRegions,            // 23 region_new
        4 * mw,                             // 24 clear-mask scratch
        C / 8, 4 * C,                       // 25 gd request bits, 26 gd cell list
        8 * C, 8 * C,                       // 27 memo key, 28 memo result
        2 * (size_t)(W + 1) * (H + 1),      // 29 obstacle summed-area table
        4 * C, 4 * C, 0, 4 * C, 4 * C,      // 30 cand steer, 31 cand len, 32 (unused), 33/34 prop
        4 * C, 4 * C,                       // 35 exp steer, 36 exp len
    };
    for (int k = 0; k < kParts; k++)
        parts[k] = align_up(p[k], 256);
}
}  // namespace

size_t Engine::slot_bytes(int W, int H)
{
    size_t parts[kParts], total = 0;
    slot_parts(W, H, parts);
    for (size_t b : parts)
        total += b;
    return align_up(total, 4096);
}

// points the slot's record at its storage (store_off_ in the arena) laid out
// for a W x H frame; the claim array starts free
bool Engine::layout_slot(int s, int W, int H)
{
    size_t parts[kParts];
    slot_parts(W, H, parts);
    void *ptr[kParts];
    char *base = (char *)arena_ + store_off_[s];
    for (int k = 0; k < kParts; k++) {
        ptr[k] = base;
        base += parts[k];
    }
    Inst &I = h_inst_[s];
    I.type = (int8_t *)ptr[0];
    I.parent = (int32_t *)ptr[1];
    I.child = (int32_t *)ptr[2];
    I.heading = (float *)ptr[3];
    I.cost = (float *)ptr[4];
    intrinsic_[s] = (float *)ptr[5];
    I.intrinsic = nullptr;  // zero intrinsic costs: the reference's default
    I.direct = (float *)ptr[6];
    I.gd_flag = (uint8_t *)ptr[7];
    I.gd_heading = (float *)ptr[8];
    I.gd_cost = (float *)ptr[9];
    I.claim = (int32_t *)ptr[10];
    I.cand = (int32_t *)ptr[11];
    I.cand_end = (int32_t *)ptr[12];
    I.cand_heading = (float *)ptr[13];
    I.cand_cost = (float *)ptr[14];
    I.nodes = (int32_t *)ptr[15];
    I.node_key = (unsigned long long *)ptr[16];
    I.node_pending = (int32_t *)ptr[17];
    I.node_pruned = (int32_t *)ptr[18];
    own_cls_[s] = (uint8_t *)ptr[19];
    I.cls = own_cls_[s];
    I.blocked = (const uint32_t *)ptr[20];
    I.clear = (const uint32_t *)ptr[21];
    I.region_count = (unsigned *)ptr[22];
    I.region_new = (unsigned *)ptr[23];
    I.rowdil = (uint32_t *)ptr[24];
    I.gd_req = (uint32_t *)ptr[25];
    I.gd_list = (int32_t *)ptr[26];
    I.memo_key = (unsigned long long *)ptr[27];
    I.memo_result = (unsigned long long *)ptr[28];
    I.sat = (const uint16_t *)ptr[29];
    I.cand_steer = (float *)ptr[30];
    I.cand_len = (float *)ptr[31];
    I.prop_steer = (float *)ptr[33];
    I.prop_len = (float *)ptr[34];
    I.exp_steer = (float *)ptr[35];
    I.exp_len = (float *)ptr[36];
    dirty_ = true;
    return check(cudaMemsetAsync(I.claim, 0x7F, parts[10], stream_), "claim init");
}

bool Engine::ensure_storage(int slot, int W, int H)
{
    out_of_budget_ = false;
    if (!budget_)
        return W <= max_w_ && H <= max_h_;
    if (store_bytes_[slot] && store_w_[slot] == W && store_h_[slot] == H)
        return true;
    release_storage(slot);
    const size_t need = slot_bytes(W, H);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
        if (it->second < need)
            continue;
        const size_t off = it->first, len = it->second;
        free_.erase(it);
        if (len > need)
            free_[off + need] = len - need;
        store_off_[slot] = off;
        store_bytes_[slot] = need;
        store_w_[slot] = W;
        store_h_[slot] = H;
        used_ += need;
        peak_used_ = std::max(peak_used_, used_);
        return layout_slot(slot, W, H);
    }
    out_of_budget_ = true;
    set_error("admission: device memory budget exhausted (" + std::to_string(need) + " bytes needed, " +
              std::to_string(budget_ - used_) + " of " + std::to_string(budget_) + " free)");
    return false;
}

void Engine::release_storage(int slot)
{
    if (!budget_ || !store_bytes_[slot])
        return;
    size_t off = store_off_[slot], len = store_bytes_[slot];
    used_ -= len;
    // merge with the free neighbours
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + len == next->first) {
        len += next->second;
        next = free_.erase(next);
    }
    if (next != free_.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == off) {
            off = prev->first;
            len += prev->second;
            free_.erase(prev);
        }
    }
    free_[off] = len;
    store_bytes_[slot] = 0;
    store_w_[slot] = store_h_[slot] = 0;
    // no frame: no sweep chunks, no pointers
    Inst &I = h_inst_[slot];
    const Physical ph = h_phys_[slot];
    const double ms = I.max_steer, lr = I.lr;
    const float mc = I.max_curvature;
    const float *costs = I.class_costs;
    memset(&I, 0, sizeof(Inst));
    I.class_costs = costs;
    I.max_steer = ms;
    I.lr = lr;
    I.max_curvature = mc;
    I.lbx = ph.lbx;
    I.lbz = ph.lbz;
    I.ubx = ph.ubx;
    I.ubz = ph.ubz;
    I.stop_on_goal = 1;
    own_cls_[slot] = nullptr;
    intrinsic_[slot] = nullptr;
    dirty_ = true;
}

Engine::Engine(int n_slots, int max_w, int max_h, int device, size_t budget_bytes)
{
    if (n_slots <= 0 || max_w <= 0 || max_h <= 0 || max_w > 4095 || max_h > 4095) {
        set_error("engine: bad slot count or frame size (frames up to 4095 x 4095)");
        return;
    }
    n_slots_ = n_slots;
    max_w_ = max_w;
    max_h_ = max_h;
    max_cells_ = max_w * max_h;
    if (device >= 0 && !check(cudaSetDevice(device), "cudaSetDevice"))
        return;
    if (!check(cudaGetDevice(&device_), "cudaGetDevice"))
        return;
    int sms = 0;
    if (!check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_), "device query"))
        return;
    if (!check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate"))
        return;

    const int rw = (max_w + 31) / 32;
    mask_words_ = (int)align_up((size_t)rw * max_h, 4);
    h_inst_.assign(n_slots, Inst{});
    h_phys_.assign(n_slots, Physical{});
    own_cls_.assign(n_slots, nullptr);
    intrinsic_.assign(n_slots, nullptr);
    ncls_.assign(n_slots, 0);
    use_preproc_.assign(n_slots, 0);
    store_off_.assign(n_slots, 0);
    store_bytes_.assign(n_slots, 0);
    store_w_.assign(n_slots, 0);
    store_h_.assign(n_slots, 0);
    for (int s = 0; s < n_slots; s++) {
        Inst &I = h_inst_[s];
        memset(&I, 0, sizeof(Inst));
        I.lbx = I.lbz = I.ubx = I.ubz = -1;
        I.stop_on_goal = 1;
    }
    if (budget_bytes > 0) {
        // slots get their storage on admission, sized by the frame
        budget_ = align_up(budget_bytes, 4096);
        arena_bytes_ = budget_;
        if (!check(cudaMalloc(&arena_, arena_bytes_), "arena cudaMalloc"))
            return;
        free_[0] = budget_;
    } else {
        // every slot holds the largest frame, for good
        const size_t per_slot = slot_bytes(max_w, max_h);
        arena_bytes_ = per_slot * n_slots;
        if (!check(cudaMalloc(&arena_, arena_bytes_), "arena cudaMalloc"))
            return;
        if (!check(cudaMemsetAsync(arena_, 0, arena_bytes_, stream_), "arena memset"))
            return;
        for (int s = 0; s < n_slots; s++) {
            store_off_[s] = per_slot * s;
            store_bytes_[s] = per_slot;
            store_w_[s] = max_w;
            store_h_[s] = max_h;
            if (!layout_slot(s, max_w, max_h))
                return;
        }
    }
    bool ok = check(cudaMalloc(&d_inst_, sizeof(Inst) * n_slots), "inst table") &&
              check(cudaMalloc(&d_state_, sizeof(State) * n_slots), "state table") &&
              check(cudaMemsetAsync(d_state_, 0, sizeof(State) * n_slots, stream_), "state init") &&
              check(cudaMallocHost(&h_state_, sizeof(State) * n_slots), "pinned state") &&
              check(cudaMalloc(&d_sched_, sizeof(Sched)), "sched") &&
              check(cudaMalloc(&d_sched_arrays_, sizeof(int) * 6 * (n_slots + 1)), "sched arrays") &&
              check(cudaMalloc(&d_grab_, sizeof(unsigned) * 4), "grab counters") &&
              check(cudaMalloc(&d_slots_, sizeof(int) * n_slots), "slot list") &&
              check(cudaMalloc(&d_class_costs_, sizeof(float) * kMaxClasses * n_slots), "class costs") &&
              check(cudaMalloc(&d_bad_, sizeof(int)), "flag") &&
              check(cudaMalloc(&d_clock_, sizeof(long long)), "clock") &&
              check(cudaMallocHost(&h_small_, sizeof(int) * 64), "pinned scratch") &&
              check(cudaMallocHost(&h_costs_pin_, sizeof(float) * kMaxClasses * n_slots), "pinned costs") &&
              check(cudaEventCreateWithFlags(&stage_ev_, cudaEventDisableTiming), "staging event") &&
              check(cudaMalloc(&d_newcost_, sizeof(float) * kOptCap * kOptCap), "optimize scratch") &&
              check(cudaMalloc(&d_changed_, sizeof(int)), "optimize flag") &&
              check(cudaMemsetAsync(d_sched_arrays_, 0, sizeof(int) * 6 * (n_slots + 1), stream_), "sched init") &&
              check(cudaMemsetAsync(d_grab_, 0, sizeof(unsigned) * 4, stream_), "grab init") &&
              check(cudaMemsetAsync(d_class_costs_, 0, sizeof(float) * kMaxClasses * n_slots, stream_), "costs init");
    if (!ok)
        return;
    memset(h_state_, 0, sizeof(State) * n_slots);
    for (int s = 0; s < n_slots; s++)
        h_inst_[s].class_costs = d_class_costs_ + (size_t)s * kMaxClasses;
    // stage both bit-packed masks of a slot in shared memory when they fit
    const int smem_bytes = 2 * 4 * mask_words_;
    L_.sms = sms;
    L_.smem_words = smem_bytes <= kSmemLimit ? mask_words_ : 0;
    if (L_.smem_words) {
        configure_kernels(smem_bytes);
        if (!check(cudaGetLastError(), "kernel attributes"))
            return;
    }
    L_.work_blocks = sms * work_per_sm_;
    L_.sweep_blocks = sms * sweep_per_sm_;
    // FRRT_NO_PDL=1: every iteration kernel waits for the end of the one
    // before it (no programmatic dependent launch), for measurement
    const char *no_pdl = getenv("FRRT_NO_PDL");
    L_.pdl = (no_pdl && atoi(no_pdl)) ? 0 : 1;
    ok_ = true;
    ok_ = commit();
}

Engine::~Engine()
{
    if (stream_)
        cudaStreamSynchronize(stream_);
    if (graph_exec_)
        cudaGraphExecDestroy(graph_exec_);
    if (graph_)
        cudaGraphDestroy(graph_);
    cudaFree(arena_);
    cudaFree(d_inst_);
    cudaFree(d_state_);
    if (h_state_)
        cudaFreeHost(h_state_);
    cudaFree(d_sched_);
    cudaFree(d_sched_arrays_);
    cudaFree(d_grab_);
    cudaFree(d_slots_);
    cudaFree(d_class_costs_);
    cudaFree(d_bad_);
    cudaFree(d_clock_);
    cudaFree(pb_.X);
    cudaFree(pb_.logits);
    cudaFree(d_log_cells_);
    cudaFree(d_log_slots_);
    cudaFree(d_log_count_);
    if (h_small_)
        cudaFreeHost(h_small_);
    if (h_costs_pin_)
        cudaFreeHost(h_costs_pin_);
    if (h_stage_)
        cudaFreeHost(h_stage_);
    if (stage_ev_)
        cudaEventDestroy(stage_ev_);
    cudaFree(d_paths_);
    cudaFree(d_path_n_);
    cudaFree(d_interp_);
    cudaFree(d_interp_n_);
    cudaFree(d_qscratch_);
    cudaFree(d_qlen_);
    cudaFree(d_qjerk_);
    cudaFree(d_qdisc_);
    cudaFree(d_keys_);
    cudaFree(d_counts_);
    cudaFree(d_valid_);
    cudaFree(d_length_);
    cudaFree(d_newcost_);
    cudaFree(d_changed_);
    if (stream_)
        cudaStreamDestroy(stream_);
}

void Engine::set_physical(int slot, const Physical &p)
{
    Inst &I = h_inst_[slot];
    h_phys_[slot] = p;
    I.max_steer = p.max_steer_rad;
    I.lr = p.vehicle_len / 2;
    // setPhysicalParams (graph.cu:286-304): 2 t / (0.5 L sqrtf(4 + t))
    const float t = tanf((float)p.max_steer_rad);
    const double mc = p.max_curvature < 0 ? 2 * t / (0.5 * p.vehicle_len * sqrtf(4 + t))
                                          : (double)p.max_curvature;
    I.max_curvature = (float)mc;
    I.lbx = p.lbx;
    I.lbz = p.lbz;
    I.ubx = p.ubx;
    I.ubz = p.ubz;
    dirty_ = true;
}

static void set_geometry(Inst &I, int W, int H)
{
    I.W = W;
    I.H = H;
    I.mask_rw = (W + 31) / 32;
    I.mask_words = (int)align_up((size_t)I.mask_rw * H, 4);
    // default coordinate origin: the frame centre (graph.cu:279)
    I.og_x = (float)(W / 2);
    I.og_z = (float)(H / 2);
}

bool Engine::bind_frame(int slot, const Frame *f)
{
    if (!f || f->W > max_w_ || f->H > max_h_) {
        set_error("frame larger than the engine's slots");
        return false;
    }
    if (!ensure_storage(slot, f->W, f->H))
        return false;
    Inst &I = h_inst_[slot];
    set_geometry(I, f->W, f->H);
    I.cls = f->d_cls;  // read in place
    I.trav = f->d_trav;
    const bool pre = use_preproc_[slot] != 0;
    I.frame_dist = f->d_dist;
    I.gd_dist = pre && f->distance_processed ? f->d_dist : nullptr;
    I.gd_safe = pre && f->safe_zone_checked ? 1 : 0;
    ncls_[slot] = f->n_classes;
    I.n_classes = f->n_classes;
    dirty_ = true;
    return check(cudaMemcpyAsync(d_class_costs_ + (size_t)slot * kMaxClasses, f->d_costs,
                                 sizeof(float) * kMaxClasses, cudaMemcpyDeviceToDevice, stream_),
                 "class costs");
}

bool Engine::copy_frame(int slot, int W, int H, const uint8_t *cls, const float *costs_host,
                        int n_classes, bool cls_on_device)
{
    if (W <= 0 || H <= 0 || W > max_w_ || H > max_h_ || n_classes <= 0 || n_classes > kMaxClasses) {
        set_error("frame larger than the engine's slots or bad class table");
        return false;
    }
    if (!ensure_storage(slot, W, H))
        return false;
    Inst &I = h_inst_[slot];
    set_geometry(I, W, H);
    I.cls = own_cls_[slot];
    I.trav = nullptr;
    I.frame_dist = nullptr;
    I.gd_dist = nullptr;
    I.gd_safe = 0;
    ncls_[slot] = n_classes;
    I.n_classes = n_classes;
    dirty_ = true;
    return check(cudaMemcpyAsync(own_cls_[slot], cls, (size_t)W * H,
                                 cls_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                 stream_),
                 "frame upload") &&
           (memcpy(h_costs_pin_ + (size_t)slot * kMaxClasses, costs_host, sizeof(float) * n_classes),
            check(cudaMemcpyAsync(d_class_costs_ + (size_t)slot * kMaxClasses,
                                  h_costs_pin_ + (size_t)slot * kMaxClasses, sizeof(float) * n_classes,
                                  cudaMemcpyHostToDevice, stream_),
                  "class costs"));
}

void Engine::set_request(int slot, const PlanRequest &r)
{
    Inst &I = h_inst_[slot];
    I.start_x = r.start_x;
    I.start_z = r.start_z;
    I.start_heading = r.start_heading;
    I.goal_x = r.goal_x;
    I.goal_z = r.goal_z;
    I.goal_heading = r.goal_heading;
    I.velocity = r.velocity;
    // setSearchParams (graph.cu:306-314): TO_INT((float)min / 2)
    I.mdx = (int)((float)r.min_dist_x / 2);
    I.mdz = (int)((float)r.min_dist_z / 2);
    // every probe lies within floor(sqrt(mdx^2 + mdz^2)) + 2 of the cell
    I.rc = (int)std::floor(std::sqrt((double)I.mdx * I.mdx + (double)I.mdz * I.mdz)) + 2;
    I.max_path = r.max_path;
    I.dist_tol = r.dist_tol;
    I.heading_tol = r.heading_tol;
    I.seed = r.seed;
    I.smart = r.smart;
    I.max_iter = r.max_iter;
    I.stop_on_goal = r.stop_on_goal;
    I.timeout_ns = r.timeout_ms > 0 ? (long long)r.timeout_ms * 1000000LL : 0;
    // a window spans at most (int)(2 r) + 2 cells per axis
    const long wmax = (long)(2.0f * r.dist_tol) + 2;
    I.win_chunks = (int)std::max(1L, (wmax * wmax + 31) / 32);
    dirty_ = true;
}

bool Engine::set_intrinsic(int slot, const float *host_costs)
{
    Inst &I = h_inst_[slot];
    dirty_ = true;
    if (!host_costs) {
        I.intrinsic = nullptr;
        return true;
    }
    I.intrinsic = intrinsic_[slot];
    return check(cudaMemcpyAsync(intrinsic_[slot], host_costs, sizeof(float) * (size_t)I.W * I.H,
                                 cudaMemcpyHostToDevice, stream_),
                 "intrinsic costs");
}

bool Engine::commit()
{
    if (!ok_)
        return false;
    std::vector<int> arrays(n_slots_ + 1, 0);
    int run = 0;
    for (int s = 0; s < n_slots_; s++) {
        arrays[s] = run;
        const long cells = (long)h_inst_[s].W * h_inst_[s].H;
        run += (int)((cells + kSweepCells - 1) / kSweepCells);
    }
    arrays[n_slots_] = run;
    h_sched_.n_slots = n_slots_;
    h_sched_.sweep_total = run;
    h_sched_.sweep_start = d_sched_arrays_;
    h_sched_.cand_start = d_sched_arrays_ + (n_slots_ + 1);
    h_sched_.node_start = d_sched_arrays_ + 2 * (n_slots_ + 1);
    h_sched_.goal_start = d_sched_arrays_ + 4 * (n_slots_ + 1);
    h_sched_.cand_exact = d_sched_arrays_ + 5 * (n_slots_ + 1);
    h_sched_.grab = d_grab_;
    const int sweep_blocks = std::max(1, std::min(L_.sms * sweep_per_sm_, run));
    if (sweep_blocks != L_.sweep_blocks) {
        L_.sweep_blocks = sweep_blocks;
        if (graph_exec_) {
            cudaGraphExecDestroy(graph_exec_);
            graph_exec_ = nullptr;
        }
        if (graph_) {
            cudaGraphDestroy(graph_);
            graph_ = nullptr;
        }
    }
    // stage the three tables in pinned memory (the previous upload from it
    // has to be done first) and upload them without waiting for the stream
    const size_t inst_b = sizeof(Inst) * n_slots_, arr_b = sizeof(int) * (n_slots_ + 1);
    const size_t need = inst_b + arr_b + sizeof(Sched);
    if (need > stage_bytes_) {
        if (h_stage_ && !check(cudaEventSynchronize(stage_ev_), "staging wait"))
            return false;
        if (h_stage_)
            cudaFreeHost(h_stage_);
        h_stage_ = nullptr;
        if (!check(cudaMallocHost(&h_stage_, need), "pinned staging"))
            return false;
        stage_bytes_ = need;
    } else if (!check(cudaEventSynchronize(stage_ev_), "staging wait")) {
        return false;
    }
    memcpy(h_stage_, h_inst_.data(), inst_b);
    memcpy(h_stage_ + inst_b, arrays.data(), arr_b);
    memcpy(h_stage_ + inst_b + arr_b, &h_sched_, sizeof(Sched));
    const bool ok =
        check(cudaMemcpyAsync(d_inst_, h_stage_, inst_b, cudaMemcpyHostToDevice, stream_), "inst upload") &&
        check(cudaMemcpyAsync(d_sched_arrays_, h_stage_ + inst_b, arr_b, cudaMemcpyHostToDevice, stream_),
              "sched upload") &&
        check(cudaMemcpyAsync(d_sched_, h_stage_ + inst_b + arr_b, sizeof(Sched), cudaMemcpyHostToDevice,
                              stream_),
              "sched upload") &&
        check(cudaEventRecord(stage_ev_, stream_), "staging event");
    dirty_ = !ok;
    return ok;
}

bool Engine::upload_slots_list(const std::vector<int> &slots)
{
    return check(cudaMemcpyAsync(d_slots_, slots.data(), sizeof(int) * slots.size(),
                                 cudaMemcpyHostToDevice, stream_),
                 "slot list upload");
}

bool Engine::prepare(const std::vector<int> &slots, float direct_max_curvature, bool fresh)
{
    for (int sl : slots) {
        if (h_inst_[sl].gd_max_curvature != direct_max_curvature) {
            h_inst_[sl].gd_max_curvature = direct_max_curvature;
            dirty_ = true;
        }
    }
    if (dirty_ && !commit())
        return false;
    if (slots.empty())
        return true;
    if (!check(cudaMemsetAsync(d_bad_, 0, sizeof(int), stream_), "flag reset"))
        return false;
    int max_cells = 0, max_words = 0, max_w = 0, max_h = 0;
    for (int s : slots) {
        const Inst &I = h_inst_[s];
        if (I.W <= 0) {
            set_error("slot has no frame");
            return false;
        }
        max_cells = std::max(max_cells, I.W * I.H);
        max_words = std::max(max_words, I.mask_rw * I.H);
        max_w = std::max(max_w, I.W);
        max_h = std::max(max_h, I.H);
    }
    if (!upload_slots_list(slots))
        return false;
    launch_frame_masks(d_inst_, d_state_, d_slots_, (int)slots.size(), max_words, kMaxClasses, d_bad_,
                       stream_, max_w, max_h);
    if (profiling_)
        cudaEventRecord(prof_ev_[kIterKernels + 1], stream_);
    launch_direct_goal_reset(d_inst_, d_slots_, (int)slots.size(), max_cells, fresh ? 1 : 0, stream_);
    if (profiling_) {
        cudaEventRecord(prof_ev_[kIterKernels + 2], stream_);
        float ms = 0;
        if (check(cudaEventSynchronize(prof_ev_[kIterKernels + 2]), "profiling sync") &&
            check(cudaEventElapsedTime(&ms, prof_ev_[kIterKernels + 1], prof_ev_[kIterKernels + 2]),
                  "profiling time")) {
            prof_pre_ms_ += ms;
            prof_pre_n_ += 1;
        }
    }
    if (!check(cudaGetLastError(), "precompute launch") ||
        !check(cudaMemcpyAsync(h_small_, d_bad_, sizeof(int), cudaMemcpyDeviceToHost, stream_), "flag") ||
        !check(cudaStreamSynchronize(stream_), "precompute"))
        return false;
    if (h_small_[0]) {
        set_error("frame class id outside the class-cost table");
        return false;
    }
    return true;
}

bool Engine::search_init(const std::vector<int> &slots, bool fresh)
{
    if (dirty_ && !commit())
        return false;
    if (slots.empty())
        return true;
    int max_cells = 0;
    for (int s : slots)
        max_cells = std::max(max_cells, h_inst_[s].W * h_inst_[s].H);
    if (!upload_slots_list(slots))
        return false;
    launch_search_init(d_inst_, d_state_, d_slots_, (int)slots.size(), max_cells, fresh ? 1 : 0,
                       stream_);
    return check(cudaGetLastError(), "search_init launch");
}

bool Engine::ensure_graph()
{
    if (graph_exec_)
        return true;
    if (!check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "graph capture"))
        return false;
    launch_iteration(d_inst_, d_state_, d_sched_, n_slots_, L_, stream_, nullptr,
                     use_proposal_ ? &pb_ : nullptr);
    const cudaError_t launch_err = cudaGetLastError();
    const cudaError_t end_err = cudaStreamEndCapture(stream_, &graph_);
    if (!check(launch_err, "iteration capture") || !check(end_err, "graph capture end"))
        return false;
    return check(cudaGraphInstantiate(&graph_exec_, graph_, 0), "graph instantiate");
}

bool Engine::set_profiling(bool on)
{
    profiling_ = on;
    if (on && prof_ev_.empty()) {
        prof_ev_.resize(kIterKernels + 3);
        for (auto &e : prof_ev_)
            if (!check(cudaEventCreate(&e), "profiling events"))
                return false;
    }
    prof_ms_.assign(kIterKernels, 0.0);
    prof_n_.assign(kIterKernels, 0);
    prof_pre_ms_ = 0;
    prof_pre_n_ = 0;
    return true;
}

bool Engine::iterate()
{
    if (dirty_ && !commit())
        return false;
    if (profiling_) {
        launch_iteration(d_inst_, d_state_, d_sched_, n_slots_, L_, stream_, prof_ev_.data(),
                         use_proposal_ ? &pb_ : nullptr);
        if (!check(cudaGetLastError(), "iteration launch") || !sync())
            return false;
        for (int k = 0; k < kIterKernels; k++) {
            float ms = 0;
            cudaEventElapsedTime(&ms, prof_ev_[k], prof_ev_[k + 1]);
            prof_ms_[k] += ms;
            prof_n_[k] += 1;
        }
        return true;
    }
    if (!ensure_graph())
        return false;
    return check(cudaGraphLaunch(graph_exec_, stream_), "graph launch");
}

bool Engine::sync() { return check(cudaStreamSynchronize(stream_), "stream sync"); }

bool Engine::fetch_states(bool synchronous)
{
    if (!check(cudaMemcpyAsync(h_state_, d_state_, sizeof(State) * n_slots_, cudaMemcpyDeviceToHost,
                               stream_),
               "state download"))
        return false;
    if (!synchronous)
        return true;
    if (!sync())
        return false;
    // the proposal network's GEMMs of the iterations since the last check
    if (use_proposal_)
        if (const char *e = gemm_take_error()) {
            set_error(std::string("proposal: ") + e);
            return false;
        }
    return true;
}

bool Engine::deactivate(int slot)
{
    const int zero = 0;
    h_state_[slot].active = 0;
    return check(cudaMemcpyAsync(&d_state_[slot].active, &zero, sizeof(int), cudaMemcpyHostToDevice,
                                 stream_),
                 "deactivate") &&
           sync();
}

bool Engine::goal_check(int slot)
{
    if (!upload_slots_list({slot}))
        return false;
    launch_goal_check(d_inst_, d_state_, d_slots_, 1, h_inst_[slot].W * h_inst_[slot].H, stream_);
    return check(cudaGetLastError(), "goal check") && fetch_states(true);
}

int Engine::count(int slot, int type)
{
    if (!d_counts_ && !check(cudaMalloc(&d_counts_, sizeof(unsigned) * n_slots_), "count scratch"))
        return -1;
    if (!upload_slots_list({slot}))
        return -1;
    launch_count(d_inst_, d_slots_, 1, h_inst_[slot].W * h_inst_[slot].H, type, d_counts_, stream_);
    if (!check(cudaMemcpyAsync(h_small_, d_counts_, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_),
               "count") ||
        !sync())
        return -1;
    return h_small_[0];
}

bool Engine::extract_and_validate(const std::vector<int> &slots, int cap, bool copy_paths)
{
    const int n = (int)slots.size();
    if (cap > cap_ || !d_paths_) {
        cudaFree(d_paths_);
        cudaFree(d_path_n_);
        cudaFree(d_keys_);
        cudaFree(d_valid_);
        cudaFree(d_length_);
        if (!d_counts_ && !check(cudaMalloc(&d_counts_, sizeof(unsigned) * n_slots_), "count scratch"))
            return false;
        cap_ = std::max(cap, 64);
        if (!check(cudaMalloc(&d_paths_, sizeof(float) * 3 * (size_t)cap_ * n_slots_), "path buffers") ||
            !check(cudaMalloc(&d_path_n_, sizeof(int) * n_slots_), "path counts") ||
            !check(cudaMalloc(&d_keys_, sizeof(long long) * n_slots_), "best keys") ||
            !check(cudaMalloc(&d_valid_, sizeof(int) * n_slots_), "valid flags") ||
            !check(cudaMalloc(&d_length_, sizeof(float) * n_slots_), "lengths"))
            return false;
    }
    if (n == 0)
        return true;
    last_list_ = slots;
    int max_cells = 0;
    for (int s : slots)
        max_cells = std::max(max_cells, h_inst_[s].W * h_inst_[s].H);
    if (!upload_slots_list(slots))
        return false;
    launch_extract_paths(d_inst_, d_state_, d_slots_, n, max_cells, d_paths_, d_path_n_, d_keys_, cap_,
                         stream_);
    launch_validate(d_inst_, d_state_, d_slots_, n, max_cells, d_paths_, d_path_n_, cap_, d_counts_,
                    d_valid_, d_length_, stream_);
    h_path_n_.resize(n);
    h_valid_.resize(n);
    h_length_.resize(n);
    if (copy_paths)
        h_paths_.resize((size_t)3 * cap_ * n);
    return check(cudaGetLastError(), "extract launch") &&
           check(cudaMemcpyAsync(h_path_n_.data(), d_path_n_, sizeof(int) * n, cudaMemcpyDeviceToHost,
                                 stream_), "path counts") &&
           check(cudaMemcpyAsync(h_valid_.data(), d_valid_, sizeof(int) * n, cudaMemcpyDeviceToHost,
                                 stream_), "valid flags") &&
           check(cudaMemcpyAsync(h_length_.data(), d_length_, sizeof(float) * n, cudaMemcpyDeviceToHost,
                                 stream_), "lengths") &&
           (!copy_paths ||
            check(cudaMemcpyAsync(h_paths_.data(), d_paths_, sizeof(float) * 3 * (size_t)cap_ * n,
                                  cudaMemcpyDeviceToHost, stream_), "paths")) &&
           sync();
}

// the slot's intrinsic-cost array made current (zeroed when the costs were
// all zero) after the deferred goal connections that read the old costs
bool Engine::intrinsic_for_update(int slot, const Frame *f)
{
    Inst &I = h_inst_[slot];
    if (!f || I.W == 0 || f->W != I.W || f->H != I.H) {
        set_error("apf: the frame must have the planner's size (set_plan_data first)");
        return false;
    }
    if (!gd_complete(slot) ||
        !check(cudaMemsetAsync(I.memo_key, 0xFF, 8 * (size_t)I.W * I.H, stream_), "memo reset"))
        return false;
    if (!I.intrinsic) {
        if (!check(cudaMemsetAsync(intrinsic_[slot], 0, 4 * (size_t)I.W * I.H, stream_), "intrinsic init"))
            return false;
        I.intrinsic = intrinsic_[slot];
        dirty_ = true;
    }
    return true;
}

bool Engine::apf_repulsion(int slot, const Frame *f, float kr, int radius)
{
    if (radius < 1) {
        set_error("apf: radius must be at least 1");
        return false;
    }
    if (!intrinsic_for_update(slot, f))
        return false;
    const Inst &I = h_inst_[slot];
    uint8_t *scratch = nullptr;
    if (!check(cudaMallocAsync((void **)&scratch, (size_t)I.W * I.H, stream_), "apf scratch"))
        return false;
    launch_apf_repulsion(I.W, I.H, f->d_cls, f->d_costs, f->n_classes, I.lbx, I.lbz, I.ubx, I.ubz, kr, radius,
                         scratch, intrinsic_[slot], stream_);
    const bool ok = check(cudaGetLastError(), "apf launch");
    cudaFreeAsync(scratch, stream_);
    return ok && commit() && sync();
}

bool Engine::apf_attraction(int slot, const Frame *f, float ka, int goal_x, int goal_z)
{
    if (!intrinsic_for_update(slot, f))
        return false;
    const Inst &I = h_inst_[slot];
    launch_apf_attraction(I.W, I.H, f->d_cls, f->d_costs, f->n_classes, ka, goal_x, goal_z, intrinsic_[slot],
                          stream_);
    return check(cudaGetLastError(), "apf launch") && commit() && sync();
}

bool Engine::intrinsic_download(int slot, std::vector<float> &out)
{
    const Inst &I = h_inst_[slot];
    out.assign((size_t)I.W * I.H, 0.0f);
    if (!I.intrinsic || out.empty())
        return true;
    return check(cudaMemcpyAsync(out.data(), I.intrinsic, 4 * out.size(), cudaMemcpyDeviceToHost, stream_),
                 "intrinsic download") &&
           sync();
}

bool Engine::interpolate_last(int out_cap)
{
    const int n = (int)last_list_.size();
    if (n == 0 || !d_paths_) {
        set_error("interpolate: no extracted paths");
        return false;
    }
    if (out_cap <= 0) {
        set_error("interpolate: bad capacity");
        return false;
    }
    if (out_cap > interp_cap_) {
        cudaFree(d_interp_);
        cudaFree(d_interp_n_);
        cudaFree(d_qscratch_);
        cudaFree(d_qlen_);
        cudaFree(d_qjerk_);
        cudaFree(d_qdisc_);
        d_interp_ = d_qlen_ = d_qjerk_ = nullptr;
        d_interp_n_ = d_qdisc_ = nullptr;
        d_qscratch_ = nullptr;
        interp_cap_ = 0;
        const size_t ns = (size_t)n_slots_;
        if (!check(cudaMalloc(&d_interp_, sizeof(float) * 3 * (size_t)out_cap * ns), "interpolation buffers") ||
            !check(cudaMalloc(&d_interp_n_, sizeof(int) * ns), "interpolation counts") ||
            !check(cudaMalloc(&d_qscratch_, sizeof(double) * 2 * (size_t)out_cap * ns), "quality scratch") ||
            !check(cudaMalloc(&d_qlen_, sizeof(float) * ns), "quality") ||
            !check(cudaMalloc(&d_qjerk_, sizeof(float) * ns), "quality") ||
            !check(cudaMalloc(&d_qdisc_, sizeof(int) * ns), "quality"))
            return false;
        interp_cap_ = out_cap;
    }
    if (!upload_slots_list(last_list_))
        return false;
    launch_interpolate(d_inst_, d_slots_, n, d_paths_, d_path_n_, cap_, d_interp_, d_interp_n_, interp_cap_,
                       d_qscratch_, d_qlen_, d_qjerk_, d_qdisc_, stream_);
    h_interp_.resize((size_t)3 * interp_cap_ * n);
    h_interp_n_.resize(n);
    h_qlen_.resize(n);
    h_qjerk_.resize(n);
    h_qdisc_.resize(n);
    return check(cudaGetLastError(), "interpolate launch") &&
           check(cudaMemcpyAsync(h_interp_.data(), d_interp_, sizeof(float) * h_interp_.size(),
                                 cudaMemcpyDeviceToHost, stream_), "interpolated points") &&
           check(cudaMemcpyAsync(h_interp_n_.data(), d_interp_n_, sizeof(int) * n, cudaMemcpyDeviceToHost,
                                 stream_), "interpolated counts") &&
           check(cudaMemcpyAsync(h_qlen_.data(), d_qlen_, sizeof(float) * n, cudaMemcpyDeviceToHost, stream_),
                 "quality") &&
           check(cudaMemcpyAsync(h_qjerk_.data(), d_qjerk_, sizeof(float) * n, cudaMemcpyDeviceToHost, stream_),
                 "quality") &&
           check(cudaMemcpyAsync(h_qdisc_.data(), d_qdisc_, sizeof(int) * n, cudaMemcpyDeviceToHost, stream_),
                 "quality") &&
           sync();
}

bool Engine::check_graph(int slot, int &ok)
{
    ok = 0;
    // the path buffers hold the validity flags and node counts
    if (!extract_and_validate({}, 64) || !upload_slots_list({slot}))
        return false;
    launch_check_graphs(d_inst_, d_slots_, 1, h_inst_[slot].W * h_inst_[slot].H, d_counts_, d_valid_,
                        stream_);
    return check(cudaGetLastError(), "graph check launch") &&
           check(cudaMemcpyAsync(h_small_, d_valid_, sizeof(int), cudaMemcpyDeviceToHost, stream_),
                 "graph check") &&
           sync() && ((ok = h_small_[0]), true);
}

bool Engine::check_path(int slot, const float *xyh, int m, int &ok)
{
    ok = 0;
    if (m < 0 || (m > 0 && !xyh)) {
        set_error("path check: bad path");
        return false;
    }
    if (!extract_and_validate({}, std::max(m, 64)) || !upload_slots_list({slot}))
        return false;
    h_small_[0] = m;
    if (!check(cudaMemcpyAsync(d_path_n_, h_small_, sizeof(int), cudaMemcpyHostToDevice, stream_),
               "path upload") ||
        (m > 0 && !check(cudaMemcpyAsync(d_paths_, xyh, sizeof(float) * 3 * (size_t)m,
                                         cudaMemcpyHostToDevice, stream_),
                         "path upload")))
        return false;
    launch_check_paths(d_inst_, d_slots_, 1, d_paths_, d_path_n_, cap_, d_valid_, d_length_, stream_);
    return check(cudaGetLastError(), "path check launch") &&
           check(cudaMemcpyAsync(h_small_ + 1, d_valid_, sizeof(int), cudaMemcpyDeviceToHost, stream_),
                 "path check") &&
           sync() && ((ok = h_small_[1]), true);
}

int Engine::extract_path(int slot, std::vector<float> &xyh)
{
    xyh.clear();
    if (!extract_and_validate({slot}, 4096))
        return -1;
    const int m = h_path_n_[0];
    xyh.assign(h_paths_.begin(), h_paths_.begin() + 3 * m);
    return m;
}

bool Engine::optimize(int slot, int &changed)
{
    changed = 0;
    std::vector<float> path;
    const int m = extract_path(slot, path);
    if (m < 0)
        return false;
    if (m < 3 || m > kOptCap)
        return true;  // nothing to shortcut (or path beyond the optimiser's size)
    // the extracted path sits at index 0 of the path buffers
    launch_optimize(d_inst_, slot, h_inst_[slot].W * h_inst_[slot].H, d_paths_, d_path_n_, d_newcost_,
                    d_changed_, kOptCap, L_, stream_);
    if (!check(cudaGetLastError(), "optimize launch") ||
        !check(cudaMemcpyAsync(h_small_, d_changed_, sizeof(int), cudaMemcpyDeviceToHost, stream_),
               "optimize flag") ||
        !sync())
        return false;
    changed = h_small_[0];
    if (changed) {
        // clear() also resets the goal flag (graph.cu:425)
        return clear_goal_flag(slot);
    }
    return true;
}

bool Engine::clear_goal_flag(int slot)
{
    const int zero = 0;
    h_state_[slot].goal_reached = 0;
    return check(cudaMemcpyAsync(&d_state_[slot].goal_reached, &zero, sizeof(int),
                                 cudaMemcpyHostToDevice, stream_),
                 "goal flag") &&
           sync();
}

bool Engine::set_state_field_last_expanded(int slot, int v)
{
    h_state_[slot].last_expanded = v;
    return check(cudaMemcpyAsync(&d_state_[slot].last_expanded, &v, sizeof(int),
                                 cudaMemcpyHostToDevice, stream_),
                 "state field") &&
           sync();
}

bool Engine::grid_download(int slot, std::vector<int8_t> &type, std::vector<int32_t> &parent,
                           std::vector<int32_t> &child, std::vector<float> &heading,
                           std::vector<float> &cost, std::vector<float> &intrinsic,
                           std::vector<float> &direct)
{
    const Inst &I = h_inst_[slot];
    const size_t n = (size_t)I.W * I.H;
    type.resize(n);
    parent.resize(n);
    child.resize(n);
    heading.resize(n);
    cost.resize(n);
    intrinsic.assign(n, 0.0f);
    direct.resize(n);
    bool ok = check(cudaMemcpyAsync(type.data(), I.type, n, cudaMemcpyDeviceToHost, stream_), "type") &&
              check(cudaMemcpyAsync(parent.data(), I.parent, 4 * n, cudaMemcpyDeviceToHost, stream_), "parent") &&
              check(cudaMemcpyAsync(child.data(), I.child, 4 * n, cudaMemcpyDeviceToHost, stream_), "child") &&
              check(cudaMemcpyAsync(heading.data(), I.heading, 4 * n, cudaMemcpyDeviceToHost, stream_), "heading") &&
              check(cudaMemcpyAsync(cost.data(), I.cost, 4 * n, cudaMemcpyDeviceToHost, stream_), "cost") &&
              check(cudaMemcpyAsync(direct.data(), I.direct, 4 * n, cudaMemcpyDeviceToHost, stream_), "direct");
    if (ok && I.intrinsic)
        ok = check(cudaMemcpyAsync(intrinsic.data(), I.intrinsic, 4 * n, cudaMemcpyDeviceToHost, stream_),
                   "intrinsic");
    return ok && sync();
}

bool Engine::grid_upload(int slot, const std::vector<int8_t> &type, const std::vector<int32_t> &parent,
                         const std::vector<int32_t> &child, const std::vector<float> &heading,
                         const std::vector<float> &cost, const std::vector<float> &intrinsic,
                         const std::vector<float> &direct)
{
    Inst &I = h_inst_[slot];
    const size_t n = (size_t)I.W * I.H;
    bool any_intr = false;
    for (float v : intrinsic)
        any_intr = any_intr || v != 0.0f;
    bool ok = check(cudaMemcpyAsync(I.type, type.data(), n, cudaMemcpyHostToDevice, stream_), "type") &&
              check(cudaMemcpyAsync(I.parent, parent.data(), 4 * n, cudaMemcpyHostToDevice, stream_), "parent") &&
              check(cudaMemcpyAsync(I.child, child.data(), 4 * n, cudaMemcpyHostToDevice, stream_), "child") &&
              check(cudaMemcpyAsync(I.heading, heading.data(), 4 * n, cudaMemcpyHostToDevice, stream_), "heading") &&
              check(cudaMemcpyAsync(I.cost, cost.data(), 4 * n, cudaMemcpyHostToDevice, stream_), "cost") &&
              check(cudaMemcpyAsync(I.direct, direct.data(), 4 * n, cudaMemcpyHostToDevice, stream_), "direct");
    // the deferred goal direct connections read the intrinsic costs of
    // set_plan_data time: evaluate the rest before they are replaced; kept
    // goal-search results depend on them too
    ok = ok && gd_complete(slot) &&
         check(cudaMemsetAsync(I.memo_key, 0xFF, 8 * n, stream_), "memo reset");
    if (ok)
        ok = set_intrinsic(slot, any_intr ? intrinsic.data() : nullptr);
    return ok && commit();
}

bool Engine::set_launch(int sweep_per_sm, int work_per_sm)
{
    if (sweep_per_sm < 1 || sweep_per_sm > 64 || work_per_sm < 1 || work_per_sm > 8) {
        set_error("launch shape out of range (sweep 1..64, work 1..8 blocks per SM)");
        return false;
    }
    sweep_per_sm_ = sweep_per_sm;
    work_per_sm_ = work_per_sm;
    L_.work_blocks = L_.sms * work_per_sm;
    L_.sweep_blocks = -1;  // recomputed (and the graph recaptured) by commit()
    if (graph_exec_) {
        cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
    }
    if (graph_) {
        cudaGraphDestroy(graph_);
        graph_ = nullptr;
    }
    dirty_ = true;
    return commit();
}

bool Engine::set_proposal(const MlpWeights *w, float mix, int cap)
{
    if (w && !umma_init()) {
        const char *e = gemm_take_error();
        set_error(std::string("proposal: ") + (e ? e : "tensor-core GEMM unavailable"));
        return false;
    }
    if (w && cap > 0 && cap != pb_.cap) {
        cudaFree(pb_.X);
        cudaFree(pb_.logits);
        pb_ = ProposalBufs{};
        const size_t c = (size_t)cap;
        if (!check(cudaMalloc(&pb_.X, 2 * c * kMlpInPad), "proposal buffers") ||
            !check(cudaMalloc(&pb_.logits, 4 * c * kMlpOut), "proposal buffers"))
            return false;
        pb_.cap = cap;
    }
    use_proposal_ = w != nullptr && pb_.cap > 0;
    if (use_proposal_) {
        pb_.w = *w;
        pb_.mix = mix;
        pb_.count = h_sched_.cand_exact + n_slots_;  // the iteration's candidate count
    }
    h_sched_.prop_cap = use_proposal_ ? pb_.cap : 0;
    for (auto &I : h_inst_)
        I.proposal = use_proposal_ ? 1 : 0;
    dirty_ = true;
    // the iteration graph changes
    if (graph_exec_) {
        cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
    }
    if (graph_) {
        cudaGraphDestroy(graph_);
        graph_ = nullptr;
    }
    return commit();
}

int Engine::log_paths(__nv_bfloat16 *X, int32_t *labels, int offset, int cap, bool all_nodes)
{
    const int n = (int)h_path_n_.size();
    if (n == 0 || cap <= offset)
        return 0;
    const int rows_max = cap - offset;
    if (rows_max > log_cap_) {
        cudaFree(d_log_cells_);
        cudaFree(d_log_slots_);
        if (!d_log_count_ && !check(cudaMalloc(&d_log_count_, sizeof(int)), "log counter"))
            return -1;
        if (!check(cudaMalloc(&d_log_cells_, 4 * (size_t)rows_max), "log rows") ||
            !check(cudaMalloc(&d_log_slots_, 4 * (size_t)rows_max), "log rows"))
            return -1;
        log_cap_ = rows_max;
    }
    if (!check(cudaMemsetAsync(d_log_count_, 0, sizeof(int), stream_), "log counter"))
        return -1;
    if (all_nodes)
        launch_log_nodes(d_inst_, d_state_, d_slots_, n, d_valid_, d_log_cells_, d_log_slots_, labels + offset,
                         d_log_count_, rows_max, stream_);
    else
        launch_log_paths(d_inst_, d_state_, d_slots_, n, d_paths_, d_path_n_, d_valid_, cap_, d_log_cells_,
                         d_log_slots_, labels + offset, d_log_count_, rows_max, stream_);
    int rows = 0;
    if (!check(cudaMemcpyAsync(&h_small_[4], d_log_count_, sizeof(int), cudaMemcpyDeviceToHost, stream_),
               "log counter") ||
        !sync())
        return -1;
    rows = std::min(h_small_[4], rows_max);
    launch_features(d_inst_, d_log_cells_, d_log_slots_, rows, X + (size_t)offset * kMlpInPad, stream_);
    if (!check(cudaGetLastError(), "log features") || !sync())
        return -1;
    return rows;
}

bool Engine::device_clock(long long &ns)
{
    launch_clock(d_clock_, stream_);
    return check(cudaGetLastError(), "clock launch") &&
           check(cudaMemcpyAsync(&h_small_[2], d_clock_, sizeof(long long), cudaMemcpyDeviceToHost,
                                 stream_),
                 "clock read") &&
           sync() && (memcpy(&ns, &h_small_[2], sizeof(long long)), true);
}

bool Engine::gd_complete(int slot)
{
    const Inst &I = h_inst_[slot];
    if (I.W <= 0)
        return true;
    const std::vector<int> one{slot};
    if (!upload_slots_list(one))
        return false;
    launch_direct_goal_complete(d_inst_, d_state_, d_slots_, 1, I.W * I.H, stream_);
    return check(cudaGetLastError(), "goal direct-connection completion") && sync();
}

bool Engine::gd_download(int slot, std::vector<uint8_t> &flag, std::vector<float> &heading,
                         std::vector<float> &cost)
{
    if (!gd_complete(slot))
        return false;
    const Inst &I = h_inst_[slot];
    const size_t n = (size_t)I.W * I.H;
    flag.resize(n);
    heading.resize(n);
    cost.resize(n);
    return check(cudaMemcpyAsync(flag.data(), I.gd_flag, n, cudaMemcpyDeviceToHost, stream_), "gd") &&
           check(cudaMemcpyAsync(heading.data(), I.gd_heading, 4 * n, cudaMemcpyDeviceToHost, stream_), "gd") &&
           check(cudaMemcpyAsync(cost.data(), I.gd_cost, 4 * n, cudaMemcpyDeviceToHost, stream_), "gd") &&
           sync();
}

bool Engine::regions_upload(int slot, const std::vector<unsigned> &counts)
{
    const Inst &I = h_inst_[slot];
    std::vector<unsigned> full(kMaxRegions, 0u);
    std::copy(counts.begin(), counts.begin() + std::min<size_t>(counts.size(), kMaxRegions), full.begin());
    return check(cudaMemcpyAsync(I.region_count, full.data(), sizeof(unsigned) * kMaxRegions,
                                 cudaMemcpyHostToDevice, stream_),
                 "regions") &&
           sync();
}

bool Engine::candidates(int slot, int n, const int32_t *sx, const int32_t *sz, const float *steer,
                        const float *len, float velocity, float4 *out, unsigned long long *probes)
{
    if (dirty_ && !commit())
        return false;
    launch_candidates(d_inst_, slot, n, sx, sz, steer, len, velocity, out, probes, L_, stream_);
    return check(cudaGetLastError(), "candidates launch");
}

bool Engine::hermite(int slot, int n, const int32_t *x, const int32_t *z, const float *lh,
                     const int32_t *gx, const int32_t *gz, const float *gh, float max_curvature,
                     int safe, float *out, unsigned long long *probes)
{
    if (dirty_ && !commit())
        return false;
    launch_hermite_pairs(d_inst_, slot, n, x, z, lh, gx, gz, gh, max_curvature, safe, out, probes, L_,
                         stream_);
    return check(cudaGetLastError(), "hermite launch");
}

bool Engine::feasible(int slot, int n, const int32_t *x, const int32_t *z, const float *a,
                      int32_t *out, unsigned long long *probes)
{
    if (dirty_ && !commit())
        return false;
    launch_feasible(d_inst_, slot, n, x, z, a, out, probes, stream_);
    return check(cudaGetLastError(), "feasible launch");
}

// ---------------------------------------------------------------------------
// host Hermite interpolation of the output path (interpolation.cpp:36-135):
// float arithmetic on the host, round() to cells
// ---------------------------------------------------------------------------

std::vector<float> interpolate_hermite(int W, int H, int p1x, int p1z, float p1h, int p2x, int p2z,
                                       float p2h)
{
    std::vector<float> curve;
    const double ddx = p2x - p1x, ddz = p2z - p1z;
    const int numPoints = (int)std::sqrt(ddx * ddx + ddz * ddz);
    const float dx = (float)(p2x - p1x), dz = (float)(p2z - p1z);
    const float d = sqrtf(dx * dx + dz * dz);
    const double kPiD = 3.14159265358979323846;
    const float a1 = (float)(p1h - kPiD / 2), a2 = (float)(p2h - kPiD / 2);
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
        const float heading = (float)(atan2f(ddz2, ddx2) + kPiD / 2);
        curve.push_back((float)cx);
        curve.push_back((float)cz);
        curve.push_back(heading);
        lx = cx;
        lz = cz;
    }
    return curve;
}

std::vector<float> interpolate_path(const std::vector<float> &xyh, int W, int H)
{
    std::vector<float> out;
    const int n = (int)xyh.size() / 3;
    if (n < 2)
        return out;
    for (int s = 1; s < n; s++) {
        std::vector<float> c = interpolate_hermite(W, H, (int)xyh[3 * (s - 1)], (int)xyh[3 * (s - 1) + 1],
                                                   xyh[3 * (s - 1) + 2], (int)xyh[3 * s],
                                                   (int)xyh[3 * s + 1], xyh[3 * s + 2]);
        out.insert(out.end(), c.begin(), c.end());
    }
    return out;
}

}  // namespace frrt
