// frrt_kernels.cuh -- kernel launch interface of the planner engine.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "frrt_common.cuh"

namespace frrt {

constexpr int kSweepCells = 4096;   // cells per sweep chunk (256 threads x 16)
constexpr int kCandChunk = 256;     // candidates per expansion chunk (one per thread)
constexpr int kNodeChunk = 8;       // listed nodes per goal-search chunk (one per warp)
// resident blocks per SM of the warp-grab kernels (their register budgets);
// build-time knobs for measurement
#ifndef FRRT_EVAL_BLOCKS
#define FRRT_EVAL_BLOCKS 2
#endif
#ifndef FRRT_GOAL_BLOCKS
#define FRRT_GOAL_BLOCKS 2
#endif
constexpr int kEvalBlocks = FRRT_EVAL_BLOCKS;
constexpr int kGoalBlocks = FRRT_GOAL_BLOCKS;
constexpr int32_t kClaimFree = 0x7F7F7F7F;

// Scheduling tables shared by the iteration kernels (device memory).
struct Sched {
    int n_slots;
    int sweep_total;          // total sweep chunks
    int *sweep_start;         // [n_slots + 1] prefix of sweep chunks per slot
    int *cand_start;          // [n_slots + 1] prefix of candidate chunks per slot
    int *node_start;          // [n_slots + 1] prefix of node chunks per slot
    int *goal_start;          // [n_slots + 1] prefix of (node, window chunk) units per slot
    int *cand_exact;          // [n_slots + 1] prefix of candidates per slot
    unsigned *grab;           // [4] dynamic work counters
    int prop_cap;             // proposal rows per iteration (0: no network attached); the
                              // candidate idx of slot s is row cand_exact[s] + idx
};

// the slot whose prefix range [prefix[s], prefix[s + 1]) holds `chunk`
// (the last of equal entries: slots with nothing are skipped)
__device__ __forceinline__ int find_slot(const int *prefix, int n, int chunk)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= chunk)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

struct Launch {
    int sms;                  // multiprocessors
    int sweep_blocks;         // grid of the sweep kernels
    int work_blocks;          // grid of the persistent expansion / goal kernels
    int smem_words;           // words per mask staged in shared memory (0 = global masks)
    int pdl = 1;              // iteration kernels launched as programmatic dependents
};

// a kernel launch, as a programmatic dependent of the previous kernel on the
// stream when `pdl` (the kernel starts with griddep_wait())
template <typename... KArgs, typename... Args>
inline cudaError_t launch_dep(bool pdl, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

// writes the device clock of the state timestamps (ns) to *d_out
void launch_clock(long long *d_out, cudaStream_t st);

// allows `smem_bytes` of dynamic shared memory on the mask-staging kernels
void configure_kernels(int smem_bytes);

// frame preparation for listed slots: obstacle and clear masks, and the
// obstacle summed-area table of slots that have one (max_w / max_h bound the
// listed frames; 0 skips the table)
void launch_frame_masks(const Inst *d_inst, State *d_state, const int *d_slots, int n, int max_words,
                        int ncls_max, int *d_bad_class, cudaStream_t st, int max_w = 0,
                        int max_h = 0);
// processDirectGoalConnection for the n listed slots, deferred: marks every
// cell's goal direct connection as not evaluated; the iterations evaluate
// the cells that goal-search windows reach
void launch_direct_goal_reset(const Inst *d_inst, const int *d_slots, int n, int max_cells,
                              int fresh, cudaStream_t st);
// evaluates every cell of the listed slots whose goal direct connection is
// still unknown
void launch_direct_goal_complete(const Inst *d_inst, State *d_state, const int *d_slots, int n,
                                 int max_cells, cudaStream_t st);
// search_init for listed slots: reset node types, add the start, reset state;
// `fresh` (a new request) also zeroes the rest of the node grid and the
// density-region counts
void launch_search_init(const Inst *d_inst, State *d_state, const int *d_slots, int n,
                        int max_cells, int fresh, cudaStream_t st);
// one planning iteration (loop()) over all active slots; with `ev` (an array
// of kIterKernels + 1 events) an event is recorded before each kernel and
// after the last one
constexpr int kIterKernels = 14;
extern const char *const kIterKernelNames[kIterKernels];
struct ProposalBufs;
// with `pb`, candidates of slots that use the learned proposal get their
// (steering, length) from the network before the expansion
void launch_iteration(const Inst *d_inst, State *d_state, Sched *d_sched, int n_slots,
                      const Launch &L, cudaStream_t st, cudaEvent_t *ev = nullptr,
                      const ProposalBufs *pb = nullptr);
// standalone goal check (checkGoalReached) for listed slots
void launch_goal_check(const Inst *d_inst, State *d_state, const int *d_slots, int n,
                       int max_cells, cudaStream_t st);
// best node (findBestNode) + parent walk into per-slot path buffers of
// `cap` (x, z, heading) triples; d_path_n[k] gets the count
void launch_extract_paths(const Inst *d_inst, State *d_state, const int *d_slots, int n,
                          int max_cells, float *d_paths, int *d_path_n, long long *d_keys, int cap,
                          cudaStream_t st);
// one path_optimize() pass on the path of one slot; d_changed gets 0/1
void launch_optimize(const Inst *d_inst, int slot, int cells, float *d_path, int *d_path_n,
                     float *d_newcost, int *d_changed, int cap, const Launch &L, cudaStream_t st);
// validator over listed slots: DAG + waypoint footprint + curvature + goal
void launch_validate(const Inst *d_inst, State *d_state, const int *d_slots, int n, int max_cells,
                     const float *d_paths, const int *d_path_n, int cap, unsigned *d_counts,
                     int *d_valid, float *d_length, cudaStream_t st);
// interpolation of extracted paths (interpolation.cpp:36-135) and the
// curve-quality metrics of the interpolated curves (the reference's
// tests/python_dataset/curve_quality.py): out_cap points of (x, z, heading)
// per path, their count, length, jerk (NaN where undefined) and tangential
// discontinuity (1, 0, or -1 where undefined); scratch holds 2 * out_cap
// doubles per path
void launch_interpolate(const Inst *d_inst, const int *d_slots, int n, const float *d_paths,
                        const int *d_path_n, int cap, float *d_out, int *d_out_n, int out_cap,
                        double *d_scratch, float *d_length, float *d_jerk, int *d_disc, cudaStream_t st);
// training rows (parent cell, slot, label) of the valid paths of the last
// extraction, appended through *count (at most cap_rows)
void launch_log_paths(const Inst *d_inst, const State *d_state, const int *d_slots, int n,
                      const float *d_paths, const int *d_path_n, const int *d_valid, int cap,
                      int32_t *cells, int32_t *slot_of, int32_t *labels, int *count, int cap_rows,
                      cudaStream_t st);
// the same for every accepted expansion (NODE cell but the start) of the
// solved slots of the list
void launch_log_nodes(const Inst *d_inst, const State *d_state, const int *d_slots, int n, const int *d_valid,
                      int32_t *cells, int32_t *slot_of, int32_t *labels, int *count, int cap_rows,
                      cudaStream_t st);
// count cells of `type` (type < 0: all non-NULL) for listed slots into d_out[k]
void launch_count(const Inst *d_inst, const int *d_slots, int n, int max_cells, int type,
                  unsigned *d_out, cudaStream_t st);
// the two halves of launch_validate on their own: the DAG consistency of the
// listed slots' graphs, and the per-path checks of given paths
void launch_check_graphs(const Inst *d_inst, const int *d_slots, int n, int max_cells, unsigned *d_counts,
                         int *d_valid, cudaStream_t st);
void launch_check_paths(const Inst *d_inst, const int *d_slots, int n, const float *d_paths,
                        const int *d_path_n, int cap, int *d_valid, float *d_length, cudaStream_t st);

// SearchFrame preprocessing: the distance-to-goal channel and the safe-zone
// bit (0x100) of the traversability channel
void launch_frame_distance(int W, int H, int gx, int gz, float *dist, cudaStream_t st);
void launch_frame_safe_zone(int W, int H, const uint8_t *cls, const float *costs, int ncls, int rc,
                            uint8_t *rows, int32_t *trav, cudaStream_t st);

// the bounded wait of the per-candidate kernels for their staged masks: its
// limit in rounds (a test hook; the default is kWaitLimit) and the number of
// blocks that gave up since the last call (reset by the read)
bool set_stage_wait_limit(long rounds);
bool take_stage_timeouts(unsigned long long &count);

// artificial potential field intrinsic costs (apf.cu:23-154): the repulsive
// field of the frame's obstacles within `radius` cells (scratch: W*H bytes)
// and the attractive field of the goal, added to intr (W*H floats)
void launch_apf_repulsion(int W, int H, const uint8_t *cls, const float *costs, int ncls, int lbx, int lbz, int ubx,
                          int ubz, float kr, int radius, uint8_t *scratch, float *intr, cudaStream_t st);
void launch_apf_attraction(int W, int H, const uint8_t *cls, const float *costs, int ncls, float ka, int gx, int gz,
                           float *intr, cudaStream_t st);

// per-candidate microbenchmarks over one frame slot
void launch_candidates(const Inst *d_inst, int slot, int n, const int32_t *sx, const int32_t *sz,
                       const float *steer, const float *len, float velocity, float4 *out,
                       unsigned long long *probes, const Launch &L, cudaStream_t st,
                       int *bad_cell = nullptr);
void launch_hermite_pairs(const Inst *d_inst, int slot, int n, const int32_t *x, const int32_t *z,
                          const float *lh, const int32_t *gx, const int32_t *gz, const float *gh,
                          float max_curvature, int safe, float *out, unsigned long long *probes,
                          const Launch &L, cudaStream_t st);
void launch_feasible(const Inst *d_inst, int slot, int n, const int32_t *x, const int32_t *z,
                     const float *a, int32_t *out, unsigned long long *probes, cudaStream_t st);

}  // namespace frrt
