// frrt_engine.h -- host runtime of the B200 FastRRT planner.
//
// An Engine owns a device arena of `n_slots` planning slots, each with the
// node grid, frame masks and scratch of one instance of up to max_w x max_h
// cells, plus the scheduling tables and a captured CUDA graph of one
// planning iteration over all slots.  The drop-in FastRRT planner is an
// Engine with one slot; the batched and served planners use many.
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "frrt_common.cuh"
#include "frrt_kernels.cuh"
#include "frrt_mlp.cuh"

namespace frrt {

void set_error(const std::string &msg);
const char *last_error();

// A BEV frame in device memory: class ids, class costs, optional
// traversability bits (the reference SearchFrame's three channels, minus the
// unused distance channel).
struct Frame {
    int W = 0, H = 0;
    uint8_t *d_cls = nullptr;
    float *d_costs = nullptr;
    int n_classes = 0;
    int32_t *d_trav = nullptr;
    float *d_dist = nullptr;         // distance-to-goal channel or nullptr
    bool safe_zone_checked = false;  // the SearchFrame's isSafeZoneChecked()
    bool distance_processed = false; // the SearchFrame's isDistanceToGoalProcessed()
    std::vector<float> h_costs;
    ~Frame();
};

// SearchFrame preprocessing on the device (the driveless SearchFrame's
// processDistanceToGoal / processSafeDistanceZone, whose sources are not in
// the reference tree; semantics from their uses in the reference):
// the distance channel gets the Euclidean distance of every cell to the goal
// as checkDirectConnectionToGoal computes it, sqrtf(dx * dx + dz * dz); the
// safe zone sets traversability bit 0x100 on every cell whose footprint of
// half extents (min_dist_x / 2, min_dist_z / 2) holds no obstacle at any
// heading (no obstacle within the Chebyshev radius that bounds every probe).
bool frame_process_distance_to_goal(Frame *f, int goal_x, int goal_z);
bool frame_process_safe_zone(Frame *f, int min_dist_x, int min_dist_z);

Frame *frame_create(int W, int H, const uint8_t *cls, const float *costs, int n_classes,
                    const int32_t *trav);
// from the reference SearchFrame's float3 layout (class, distance, bits)
Frame *frame_create_f3(int W, int H, const float *xyz, const float *costs, int n_classes);

struct PlanRequest {
    int start_x, start_z;
    float start_heading;
    int goal_x, goal_z;
    float goal_heading;
    float velocity;
    int min_dist_x, min_dist_z;
    float max_path;
    float dist_tol;
    float heading_tol;
    unsigned long long seed;
    int smart;
    int max_iter;
    int stop_on_goal;
    int timeout_ms;   // > 0: the slot stops this long after search_init (device clock)
};

struct Physical {
    float pw_m, ph_m;
    double max_steer_rad;
    float vehicle_len;
    float max_curvature;  // < 0: derived from steering and length
    int lbx, lbz, ubx, ubz;
};

class Engine {
public:
    // budget_bytes == 0: every slot holds storage for the largest frame for
    // the engine's life.  budget_bytes > 0: slots hold no storage until a
    // frame is bound to them; each then gets storage sized by its frame from
    // one arena of budget_bytes, and gives it back when released.
    Engine(int n_slots, int max_w, int max_h, int device = -1, size_t budget_bytes = 0);
    ~Engine();
    bool ok() const { return ok_; }

    int n_slots() const { return n_slots_; }
    int max_cells() const { return max_cells_; }
    cudaStream_t stream() const { return stream_; }
    const Launch &launch() const { return L_; }

    // device memory of one slot's storage (node grid, frame copy, masks,
    // scratch) for a W x H frame
    static size_t slot_bytes(int W, int H);
    // budget mode: storage for a W x H frame in `slot` (kept when it already
    // holds that layout); false with out_of_budget() when the arena has no
    // room.  Without a budget: whether the frame fits the preallocated slots.
    bool ensure_storage(int slot, int W, int H);
    bool out_of_budget() const { return out_of_budget_; }
    // budget mode: gives the slot's storage back to the arena
    void release_storage(int slot);
    size_t budget() const { return budget_; }
    size_t used() const { return budget_ ? used_ : arena_bytes_; }
    size_t peak_used() const { return budget_ ? peak_used_ : arena_bytes_; }

    // the goal direct connections of the slot follow its frame's
    // preprocessing flags (the reference's processDirectGoalConnection passes
    // false for both, fastrrt.cpp:79 -> graph_direct_goal_connection.cu:222)
    void set_use_frame_preprocessing(int slot, bool on) { use_preproc_[slot] = on; }

    // slot configuration (host side; uploaded by commit())
    void set_physical(int slot, const Physical &p);
    // frame owned by the caller (must outlive its use) or copied into the slot
    bool bind_frame(int slot, const Frame *f);
    // copies class ids (host or device memory) into the slot's own buffer
    bool copy_frame(int slot, int W, int H, const uint8_t *cls, const float *costs_host,
                    int n_classes, bool cls_on_device = false);
    void set_request(int slot, const PlanRequest &r);
    // intrinsic costs: nullptr keeps them zero (the planner's default)
    bool set_intrinsic(int slot, const float *host_costs);
    bool commit();  // upload Inst table + scheduling tables

    // set_plan_data for listed slots: masks + goal direct-connection precompute
    // frame masks and the reset of the goal direct connections; `fresh` (a
    // new request in a slot) takes the curves' start costs from a newly
    // constructed planner (zero) instead of the slot's current grid
    bool prepare(const std::vector<int> &slots, float direct_max_curvature = 0.8f,
                 bool fresh = false);
    // search_init for listed slots
    // fresh = a new request: the slot starts like a newly constructed planner
    bool search_init(const std::vector<int> &slots, bool fresh);
    // one loop() over every live slot (graph launch); no host sync
    bool iterate();
    // kernel timing mode: iterate() launches the kernels one by one between
    // CUDA events and accumulates each kernel's device time
    bool set_profiling(bool on);
    const std::vector<double> &kernel_ms() const { return prof_ms_; }
    const std::vector<long> &kernel_launches() const { return prof_n_; }
    // device time spent in the direct-goal precompute by prepare() (profiling mode)
    double precompute_ms() const { return prof_pre_ms_; }
    long precompute_launches() const { return prof_pre_n_; }
    bool sync();
    // copy the small head of the state of every slot to host memory
    bool fetch_states(bool synchronous = true);
    const State &state(int slot) const { return h_state_[slot]; }
    bool deactivate(int slot);

    // per-slot operations (drop-in API)
    bool goal_check(int slot);
    int extract_path(int slot, std::vector<float> &xyh);
    bool optimize(int slot, int &changed);
    int count(int slot, int type);
    bool grid_download(int slot, std::vector<int8_t> &type, std::vector<int32_t> &parent,
                       std::vector<int32_t> &child, std::vector<float> &heading,
                       std::vector<float> &cost, std::vector<float> &intrinsic,
                       std::vector<float> &direct);
    bool grid_upload(int slot, const std::vector<int8_t> &type, const std::vector<int32_t> &parent,
                     const std::vector<int32_t> &child, const std::vector<float> &heading,
                     const std::vector<float> &cost, const std::vector<float> &intrinsic,
                     const std::vector<float> &direct);
    // device clock (ns) read now; the stream is synchronised
    bool device_clock(long long &ns);
    // evaluates every goal direct connection of the slot still unknown
    bool gd_complete(int slot);
    bool gd_download(int slot, std::vector<uint8_t> &flag, std::vector<float> &heading,
                     std::vector<float> &cost);
    bool regions_upload(int slot, const std::vector<unsigned> &counts);
    // artificial potential fields (apf.cu:23-154) of frame f added to the
    // slot's intrinsic costs (the deferred goal direct connections of the
    // current plan are evaluated first, with the costs they were set up with)
    bool apf_repulsion(int slot, const Frame *f, float kr, int radius);
    bool apf_attraction(int slot, const Frame *f, float ka, int goal_x, int goal_z);
    bool intrinsic_download(int slot, std::vector<float> &out);
    bool set_state_field_last_expanded(int slot, int v);
    bool clear_goal_flag(int slot);

    // batched extraction + validation of listed slots
    // copy_paths = false leaves the paths on the device (counts, validity and
    // lengths still come to the host)
    bool extract_and_validate(const std::vector<int> &slots, int cap, bool copy_paths = true);
    // learned expansion proposal: network weights (device), the probability
    // of sampling from it, rows per iteration; w == nullptr detaches it
    bool set_proposal(const MlpWeights *w, float mix, int cap);
    // launch shape: blocks per SM of the sweep kernels and of the persistent
    // expansion kernel (the autotuner's knobs)
    bool set_launch(int sweep_per_sm, int work_per_sm);
    // training rows of the last extracted list: for each valid path, one row
    // per expansion on it (features of the parent, the bin of the draw that
    // made the child) appended at X[offset..], labels[offset..] (device, at
    // most cap rows in all); returns the rows added or -1.  all_nodes: one
    // row per node of each solved graph but the start instead
    int log_paths(__nv_bfloat16 *X, int32_t *labels, int offset, int cap, bool all_nodes = false);
    // the validator's halves on one slot: checkGraphIsConsistent of its
    // graph (graph_check_dag_consistency.cpp:33-76), and the per-path checks
    // of a host path [x, z, heading] * m against its frame, grid and goal;
    // `ok` gets 1 (passes) or 0
    bool check_graph(int slot, int &ok);
    bool check_path(int slot, const float *xyh, int m, int &ok);
    // interpolation of the paths of the last extract_and_validate list and
    // their curve-quality metrics, on the device; up to out_cap points per
    // path; results in interp_* (host copies)
    bool interpolate_last(int out_cap);
    const std::vector<float> &interp_points() const { return h_interp_; }
    const std::vector<int> &interp_n() const { return h_interp_n_; }
    const std::vector<float> &interp_length() const { return h_qlen_; }
    const std::vector<float> &interp_jerk() const { return h_qjerk_; }
    const std::vector<int> &interp_disc() const { return h_qdisc_; }
    int interp_cap() const { return interp_cap_; }
    const std::vector<int> &paths_n() const { return h_path_n_; }
    const std::vector<int> &valid() const { return h_valid_; }
    const std::vector<float> &lengths() const { return h_length_; }
    const std::vector<float> &paths() const { return h_paths_; }

    // per-candidate microbenchmarks on one slot's frame
    bool candidates(int slot, int n, const int32_t *sx, const int32_t *sz, const float *steer,
                    const float *len, float velocity, float4 *out, unsigned long long *probes);
    bool hermite(int slot, int n, const int32_t *x, const int32_t *z, const float *lh,
                 const int32_t *gx, const int32_t *gz, const float *gh, float max_curvature,
                 int safe, float *out, unsigned long long *probes);
    bool feasible(int slot, int n, const int32_t *x, const int32_t *z, const float *a, int32_t *out,
                  unsigned long long *probes);

    Inst &inst(int slot) { return h_inst_[slot]; }
    const Inst *d_inst() const { return d_inst_; }
    State *d_state() const { return d_state_; }

private:
    ProposalBufs pb_{};
    int sweep_per_sm_ = 8, work_per_sm_ = 2;
    bool use_proposal_ = false;
    int32_t *d_log_cells_ = nullptr, *d_log_slots_ = nullptr;
    int *d_log_count_ = nullptr;
    int log_cap_ = 0;
    bool check(cudaError_t e, const char *what);
    bool layout_slot(int slot, int W, int H);
    bool intrinsic_for_update(int slot, const Frame *f);
    bool ensure_graph();
    bool upload_slots_list(const std::vector<int> &slots);

    bool ok_ = false;
    int device_ = 0;
    int n_slots_ = 0, max_w_ = 0, max_h_ = 0, max_cells_ = 0, mask_words_ = 0;
    cudaStream_t stream_ = nullptr;
    Launch L_{};
    void *arena_ = nullptr;
    size_t arena_bytes_ = 0;
    // slot storage: offset and bytes in the arena, the frame size it is laid
    // out for; budget mode keeps the arena's free ranges (offset -> bytes)
    size_t budget_ = 0, used_ = 0, peak_used_ = 0;
    bool out_of_budget_ = false;
    std::map<size_t, size_t> free_;
    std::vector<size_t> store_off_, store_bytes_;
    std::vector<int> store_w_, store_h_;
    std::vector<Inst> h_inst_;
    std::vector<Physical> h_phys_;
    Inst *d_inst_ = nullptr;
    State *d_state_ = nullptr;
    State *h_state_ = nullptr;  // pinned
    Sched h_sched_{};
    // pinned staging of the tables commit() uploads and of class costs, so
    // the uploads do not wait for the stream (pageable copies would)
    unsigned char *h_stage_ = nullptr;
    size_t stage_bytes_ = 0;
    cudaEvent_t stage_ev_ = nullptr;
    float *h_costs_pin_ = nullptr;
    Sched *d_sched_ = nullptr;
    int *d_sched_arrays_ = nullptr;
    unsigned *d_grab_ = nullptr;
    int *d_slots_ = nullptr;
    float *d_class_costs_ = nullptr;  // per slot, 256 entries
    int *d_bad_ = nullptr;
    std::vector<uint8_t *> own_cls_;  // per slot frame copies
    std::vector<float *> intrinsic_;  // per slot intrinsic-cost arrays
    std::vector<int> ncls_;           // class count of each slot's frame
    std::vector<char> use_preproc_;   // set_use_frame_preprocessing
    // path extraction / validation scratch
    int cap_ = 0;
    float *d_paths_ = nullptr;
    int *d_path_n_ = nullptr;
    long long *d_keys_ = nullptr;
    unsigned *d_counts_ = nullptr;
    int *d_valid_ = nullptr;
    float *d_length_ = nullptr;
    float *d_newcost_ = nullptr;
    int *d_changed_ = nullptr;
    int *h_small_ = nullptr;          // pinned scratch
    long long *d_clock_ = nullptr;    // device clock read-out
    std::vector<int> h_path_n_, h_valid_;
    std::vector<float> h_length_, h_paths_;
    std::vector<int> last_list_;      // slots of the last extraction
    int interp_cap_ = 0;
    float *d_interp_ = nullptr, *d_qlen_ = nullptr, *d_qjerk_ = nullptr;
    int *d_interp_n_ = nullptr, *d_qdisc_ = nullptr;
    double *d_qscratch_ = nullptr;
    std::vector<float> h_interp_, h_qlen_, h_qjerk_;
    std::vector<int> h_interp_n_, h_qdisc_;
    bool profiling_ = false;
    std::vector<cudaEvent_t> prof_ev_;
    std::vector<double> prof_ms_;
    std::vector<long> prof_n_;
    double prof_pre_ms_ = 0;
    long prof_pre_n_ = 0;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    bool dirty_ = true;
};

// host Hermite interpolation (interpolation.cpp:36-135)
std::vector<float> interpolate_hermite(int W, int H, int p1x, int p1z, float p1h, int p2x, int p2z,
                                       float p2h);
std::vector<float> interpolate_path(const std::vector<float> &xyh, int W, int H);

}  // namespace frrt
