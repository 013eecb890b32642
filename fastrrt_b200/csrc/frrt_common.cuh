// frrt_common.cuh -- shared types of the B200 FastRRT planner.
//
// Node grid of one planning instance (structure of arrays, W*H cells each):
//   type    int8   node type (NULL/NODE/TEMP/PROCESSING/COLLISION/CONNECT)
//   parent  int32  parent cell packed as (x & 0xffff) | (z << 16); (-1,-1) = root
//   child   int32  child count
//   heading f32, cost f32, intrinsic f32, direct f32
//   gd_*    goal direct-connection data (flag u8, heading f32, cost f32),
//           evaluated lazily: flag kGdUnknown until a goal-search window
//           first covers the cell
//   memo_*  goal-search result of a node, keyed by its heading and cost bits
// Frame of one instance: class ids (u8), a bit-packed obstacle mask
// (class cost < 0), a bit-packed "clear" mask (no obstacle within the
// footprint's circumscribed square), a summed-area table of the obstacle mask
// (u16) for footprint bounding-box tests, optional traversability bits (int32).
// Masks are row-padded: row z starts at word z * mask_rw, pixel x is bit
// (x & 31) of word (x >> 5).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace frrt {

enum : int8_t {
    T_NULL = 0,
    T_NODE = 1,
    T_TEMP = 2,
    T_PROCESSING = 3,
    T_COLLISION = 4,
    T_CONNECT_TO_GOAL = 5
};

constexpr int kRegion = 128;          // density region edge (graph_expansion_search_zones.cu:32)
constexpr int kMaxRegions = 1024;     // supports frames up to 4095 x 4095
constexpr int kFrontierThreshold = 100;  // fastrrt.cpp:116
constexpr long long kBigCost = 99999999999LL;
constexpr uint8_t kGdUnknown = 0xFF;  // gd_flag of a cell not evaluated yet
constexpr unsigned long long kMemoNone = ~0ull;  // memo_key of a cell without a result
constexpr unsigned long long kNoConnection = ~0ull;  // node_key without a connection
constexpr unsigned kFull = 0xffffffffu;

__host__ __device__ inline int32_t pack_xz(int x, int z)
{
    return (int32_t)(((uint32_t)x & 0xffffu) | ((uint32_t)z << 16));
}
__host__ __device__ inline int unpack_x(int32_t p) { return (int)(int16_t)(p & 0xffff); }
__host__ __device__ inline int unpack_z(int32_t p) { return (int)(int16_t)((uint32_t)p >> 16); }

// Static description of one planning instance (read-only inside an iteration).
struct Inst {
    int W, H;
    // frame
    const uint8_t *cls;
    const uint32_t *blocked;   // bit i: class cost of pixel i < 0
    const uint32_t *clear;     // bit i: no blocked pixel within Chebyshev radius rc
    const int32_t *trav;       // traversability bits or nullptr
    const uint16_t *sat;       // (W+1) x (H+1) summed-area table of the obstacle
                               // mask, counts mod 2^16, or nullptr
    int mask_rw;               // words per mask row = ceil(W / 32)
    int mask_words;            // words per mask, padded to a multiple of 4
    // node grid
    int8_t *type;
    int32_t *parent;
    int32_t *child;
    float *heading;
    float *cost;
    float *intrinsic;          // nullptr when all zero
    float *direct;
    uint8_t *gd_flag;          // 0 / 1, or kGdUnknown
    float *gd_heading;
    float *gd_cost;
    uint32_t *gd_req;          // bit per cell: evaluation requested
    int32_t *gd_list;          // cells to evaluate this iteration
    // goal search of a node is a pure function of (cell, heading, cost) for a
    // fixed frame, goal and intrinsic costs: results of complete (unpruned)
    // searches are kept per cell and reused while the node keeps that key
    unsigned long long *memo_key;     // (heading bits << 32) | cost bits, or kMemoNone
    unsigned long long *memo_result;  // the search's result key (see node_key)
    // per-iteration scratch
    int32_t *claim;
    int32_t *cand;
    int32_t *cand_end;
    float *cand_heading;
    float *cand_cost;
    float *cand_steer, *cand_len;  // per candidate: the draw it was integrated with
    float *prop_steer, *prop_len;  // per candidate: the proposal (prop_len < 0: uniform)
    float *exp_steer, *exp_len;    // per cell: the draw of the expansion that made the node
    int32_t *nodes;
    // per listed node: best connection as (floor(100 * total) << 32) |
    // (0xffffffff - cell), so the minimum is the cheapest, ties to the highest
    // cell; kNoConnection when none
    unsigned long long *node_key;
    int32_t *node_pending;     // window chunks of the node not searched yet
    int32_t *node_pruned;      // a chunk skipped cells by the bound
    unsigned *region_count;    // [kMaxRegions] density used by the gate
    unsigned *region_new;      // [kMaxRegions] density counted after this expansion
    uint32_t *rowdil;          // mask scratch of the clear-mask dilation
    const float *class_costs;  // class-cost table of the frame
    int n_classes;
    // parameters
    float og_x, og_z;          // coordinate origin (frame centre)
    int mdx, mdz;              // half footprint
    int lbx, lbz, ubx, ubz;    // ego box
    int rc;                    // clear-mask radius
    double max_steer;          // rad
    double lr;                 // vehicle length / 2 (m)
    float max_curvature;       // PHYSICAL_MAX_CURVATURE as float
    float gd_max_curvature;    // curvature limit of the goal direct connections
    // SearchFrame preprocessing used by the goal direct connections: the
    // frame's distance-to-goal channel (nullptr: computed) and the safe-zone
    // skip of the traversability bit 0x100 (isDistanceToGoalProcessed,
    // isSafeZoneChecked; graph_direct_goal_connection.cu:16-36, 124-135)
    const float *gd_dist;
    int gd_safe;
    const float *frame_dist;   // the frame's distance-to-goal channel or nullptr
    int win_chunks;            // 32-cell chunks covering a node's goal-search window
    float velocity, max_path, dist_tol, heading_tol;
    int start_x, start_z;
    float start_heading;
    int goal_x, goal_z;
    float goal_heading;
    unsigned long long seed;
    int smart;
    int max_iter;              // 0 = unlimited
    int stop_on_goal;          // batched planning stops a slot at its goal
    int proposal;              // expansions may come from the learned proposal
    long long timeout_ns;      // > 0: deadline after search_init (device clock)
};

// Mutable per-instance state.
struct State {
    int active;                // instance is being planned
    int done;                  // planning finished (goal or budget)
    int goal_reached;
    int collision;
    unsigned iter;             // expansion passes run (RNG counter)
    int last_expanded;         // TEMP count of the last pass
    int n_cand;
    int node_count;            // NODE count after expansion (erase bound)
    int temp_count;
    int all_count;
    int n_nodes;               // listed NODE cells for the goal search (nodes[0, n_nodes))
    int n_memo;                // listed nodes with a kept search result, at the list's end
                               // (nodes[W H - n_memo, W H)), resolved when listed
    int n_gd;                  // cells listed for goal direct-connection evaluation
    int skip;                  // graph was empty: start re-added, rest skipped
    int found;                 // goal connection found this iteration
    unsigned long long winner; // (cell << 32) | listed index of the best connection
    long long best;            // best floor(100 * total) this iteration
    int loops;                 // loop() calls run
    int error;                 // bounded-wait / consistency error code
    long long deadline_ns;     // device-clock deadline (0 = none)
    long long start_ns;        // device clock at search_init
    long long finish_ns;       // device clock when the slot finished
    unsigned long long probes;        // footprint probes of the reference algorithm: expansion
    unsigned long long probes_goal;   // ... goal-connection search
    unsigned long long probes_pre;    // ... goal direct-connection precompute
};

}  // namespace frrt
