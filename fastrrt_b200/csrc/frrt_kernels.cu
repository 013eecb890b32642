// frrt_kernels.cu -- planner kernels for sm_100a.
//
// One planning iteration (FastRRT::loop, fastrrt.cpp:108-181) over every
// active slot is a fixed sequence of kernels, captured once into a CUDA
// graph by the engine:
//
//   k_scan        gate + candidate list             (graph_expansion.cu:148-183,
//                                                    graph_expansion_search_zones.cu:161-194)
//   k_plan        per-slot candidate prefixes (1 block)
//   [proposal]    features, network, sampling (learned proposal only)
//   k_expand      integrate + footprint + claim     (expand_node, graph_expansion.cu:103-145)
//   k_apply       claim winners change the grid
//   k_post        NODE count + region density       (graph_expansion_search_zones.cu:42-66)
//   k_erase       colliding subtree erase           (graph_collision.cu:32-83)
//   k_accept      COLLISION -> NODE (graph_collision.cu:84-104), TEMP count, all
//                 count, TEMP->NODE, node list      (graph_list.cu:7-60, graph_expansion.cu:36-65)
//   k_plan        node and goal-window work prefixes
//   k_gd_demand   window cells whose goal direct connection is unknown
//   k_gd_eval     their direct connections (graph_direct_goal_connection.cu:16-167)
//   k_goal        goal check + best node->cell goal connection
//                                                   (graph_best_node.cu:181-222,
//                                                    graph_check_goal_reached.cu:17-139)
//   k_select      tie-break of the best connection
//   k_finish      connection / start adds, loop bookkeeping (fastrrt.cpp:130-180)
//
// Sweep kernels read the int8 type grid 16 cells at a time (one 16-byte
// load per thread).  The expansion and goal kernels are persistent: warps
// pull work from global counters across all slots and read the slots'
// bit-packed frame masks through L1 (a slot's masks are 16 KB at 256 x 256).
// Concurrent claims on one target cell are resolved by atomicMin on the
// expanding cell index, which makes every iteration deterministic for a
// given seed.
#include <algorithm>
#include <climits>
#include <cstdio>

#include "frrt_device.cuh"
#include "frrt_kernels.cuh"
#include "frrt_mlp.cuh"

namespace frrt {

namespace {



__device__ __forceinline__ bool live(const State &S) { return S.active && !S.done; }

// rounds the per-candidate kernels wait for their staged masks before they
// give up and read the global copies (a test hook lowers it), and how many
// blocks gave up
__device__ long g_stage_wait_limit = kWaitLimit;
__device__ unsigned long long g_stage_timeouts = 0;

// Items a warp of the warp-per-item kernels takes from its work counter at
// once: one while the items are few next to the grid's warps (every item on
// a warp of its own, the shortest launch), more when there are many (fewer
// atomics on the one counter).
__device__ __forceinline__ int grab_batch(int total)
{
    const int warps = (int)(gridDim.x * (blockDim.x >> 5));
    return total >= 16 * warps ? 4 : total >= 4 * warps ? 2 : 1;
}

// warp-aggregated append: returns this lane's first output index
__device__ __forceinline__ int warp_append(int *counter, int n)
{
    const int lane = threadIdx.x & 31;
    int incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(kFull, incl, o);
        if (lane >= o)
            incl += v;
    }
    const int total = __shfl_sync(kFull, incl, 31);
    int base = 0;
    if (lane == 31 && total)
        base = atomicAdd(counter, total);
    base = __shfl_sync(kFull, base, 31);
    return base + incl - n;
}

__device__ __forceinline__ int warp_sum(int v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1)
        v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1)
        v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ void load16(const int8_t *p, int8_t out[16])
{
    const int4 v = *reinterpret_cast<const int4 *>(p);
    const int8_t *b = reinterpret_cast<const int8_t *>(&v);
#pragma unroll
    for (int k = 0; k < 16; k++)
        out[k] = b[k];
}

// CudaGraph::add (graph.cu:364-374): bounds, parent child count, overriding set
__device__ void grid_add(const Inst &I, int x, int z, float heading, int ppx, int ppz, float cost)
{
    if (x < 0 || x >= I.W || z < 0 || z >= I.H)
        return;
    if (ppx != -1 && ppz != -1 && ppx >= 0 && ppx < I.W && ppz >= 0 && ppz < I.H)
        I.child[(long)ppz * I.W + ppx]++;
    const long pos = (long)z * I.W + x;
    I.type[pos] = T_NODE;
    I.parent[pos] = pack_xz(ppx, ppz);
    I.heading[pos] = heading;
    I.cost[pos] = cost;
}

__device__ __forceinline__ long long global_ns()
{
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

}  // namespace

// ---------------------------------------------------------------------------
// frame preparation
// ---------------------------------------------------------------------------

// one thread per mask word of every listed slot: bit set when class cost < 0
__global__ void k_blocked(const Inst *insts, State *states, const int *slots, int *bad_class)
{
    const Inst &I = insts[slots[blockIdx.y]];
    if (blockIdx.x == 0 && threadIdx.x == 0)
        states[slots[blockIdx.y]].probes_pre = 0;
    const long words = (long)I.mask_rw * I.H;
    for (long w = blockIdx.x * (long)blockDim.x + threadIdx.x; w < words;
         w += (long)gridDim.x * blockDim.x) {
        const int z = (int)(w / I.mask_rw);
        const int x0 = (int)(w - (long)z * I.mask_rw) * 32;
        uint32_t bits = 0;
        for (int b = 0; b < 32; b++) {
            const int x = x0 + b;
            if (x >= I.W)
                break;
            const int c = I.cls[(long)z * I.W + x];
            if (c >= I.n_classes) {
                atomicExch(bad_class, 1);
                continue;
            }
            if (I.class_costs[c] < 0)
                bits |= 1u << b;
        }
        const_cast<uint32_t *>(I.blocked)[w] = bits;
    }
}

// 32 row bits starting at bit `start` (may be negative / beyond the row)
__device__ __forceinline__ uint32_t row_bits(const uint32_t *row, int rw, int start)
{
    const int q = start >= 0 ? start >> 5 : -((-start + 31) >> 5);
    const int r = start - q * 32;
    const uint32_t lo = (q >= 0 && q < rw) ? row[q] : 0u;
    const uint32_t hi = (q + 1 >= 0 && q + 1 < rw) ? row[q + 1] : 0u;
    return r ? (lo >> r) | (hi << (32 - r)) : lo;
}

// horizontal dilation of the obstacle mask by rc
__global__ void k_rowdil(const Inst *insts, const int *slots)
{
    const Inst &I = insts[slots[blockIdx.y]];
    const long words = (long)I.mask_rw * I.H;
    for (long w = blockIdx.x * (long)blockDim.x + threadIdx.x; w < words;
         w += (long)gridDim.x * blockDim.x) {
        const int z = (int)(w / I.mask_rw);
        const int q = (int)(w - (long)z * I.mask_rw);
        const uint32_t *row = I.blocked + (long)z * I.mask_rw;
        uint32_t acc = 0;
        for (int d = -I.rc; d <= I.rc; d++)
            acc |= row_bits(row, I.mask_rw, q * 32 + d);
        I.rowdil[w] = acc;
    }
}

// vertical dilation + complement: clear = no obstacle within Chebyshev rc
__global__ void k_clear(const Inst *insts, const int *slots)
{
    const Inst &I = insts[slots[blockIdx.y]];
    const long words = (long)I.mask_rw * I.H;
    for (long w = blockIdx.x * (long)blockDim.x + threadIdx.x; w < words;
         w += (long)gridDim.x * blockDim.x) {
        const int z = (int)(w / I.mask_rw);
        const int q = (int)(w - (long)z * I.mask_rw);
        uint32_t acc = 0;
        const int z0 = max(0, z - I.rc), z1 = min(I.H - 1, z + I.rc);
        for (int zz = z0; zz <= z1; zz++)
            acc |= I.rowdil[(long)zz * I.mask_rw + q];
        uint32_t valid = 0xffffffffu;
        const int left = I.W - q * 32;
        if (left < 32)
            valid = left <= 0 ? 0u : ((1u << left) - 1u);
        const_cast<uint32_t *>(I.clear)[w] = ~acc & valid;
    }
}

// Summed-area table of the obstacle mask, one block per slot: each warp scans
// rows (lanes over 32-pixel words, popcount prefix across the warp), then each
// thread runs down columns.  Row 0 and column 0 are zero; counts wrap mod 2^16.
__global__ void __launch_bounds__(256) k_sat(const Inst *insts, const int *slots)
{
    const Inst &I = insts[slots[blockIdx.x]];
    if (!I.sat)
        return;
    uint16_t *S = const_cast<uint16_t *>(I.sat);
    const int w = I.W + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int z = warp; z <= I.H; z += nwarps) {
        uint16_t *row = S + (long)z * w;
        if (z == 0) {
            for (int x = lane; x < w; x += 32)
                row[x] = 0;
            continue;
        }
        if (lane == 0)
            row[0] = 0;
        const uint32_t *m = I.blocked + (long)(z - 1) * I.mask_rw;
        unsigned carry = 0;
        for (int q0 = 0; q0 < I.mask_rw; q0 += 32) {
            const int q = q0 + lane;
            const uint32_t bits = q < I.mask_rw ? m[q] : 0u;
            const int c = __popc(bits);
            int incl = c;
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(kFull, incl, o);
                if (lane >= o)
                    incl += v;
            }
            if (q < I.mask_rw) {
                unsigned run = carry + (unsigned)(incl - c);
                const int nb = min(32, I.W - q * 32);
                for (int b = 0; b < nb; b++) {
                    run += (bits >> b) & 1u;
                    row[q * 32 + b + 1] = (uint16_t)run;
                }
            }
            carry += (unsigned)__shfl_sync(kFull, incl, 31);
        }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < w; x += blockDim.x) {
        uint16_t run = 0;
        int z = 1;
        for (; z + 7 <= I.H; z += 8) {
            uint16_t v[8];
#pragma unroll
            for (int k = 0; k < 8; k++)
                v[k] = S[(long)(z + k) * w + x];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                run = (uint16_t)(run + v[k]);
                S[(long)(z + k) * w + x] = run;
            }
        }
        for (; z <= I.H; z++) {
            run = (uint16_t)(run + S[(long)z * w + x]);
            S[(long)z * w + x] = run;
        }
    }
}

void launch_frame_masks(const Inst *d_inst, State *d_state, const int *d_slots, int n, int max_words,
                        int ncls_max, int *d_bad_class, cudaStream_t st, int max_w, int max_h)
{
    if (n <= 0)
        return;
    const dim3 grid((max_words + 255) / 256, n);
    (void)ncls_max;
    k_blocked<<<grid, 256, 0, st>>>(d_inst, d_state, d_slots, d_bad_class);
    k_rowdil<<<grid, 256, 0, st>>>(d_inst, d_slots);
    k_clear<<<grid, 256, 0, st>>>(d_inst, d_slots);
    if (max_w > 0 && max_h > 0)
        k_sat<<<n, 256, 0, st>>>(d_inst, d_slots);
}

// ---------------------------------------------------------------------------
// goal direct-connection precompute (graph_direct_goal_connection.cu:169-227)
// ---------------------------------------------------------------------------

// Deferred precompute.  Only the goal search reads a cell's direct connection
// (graph_check_goal_reached.cu:53-63), and only for cells inside the window
// of a node it searches, so each cell is evaluated the first time such a
// window covers it, with the same function and arguments as the eager pass
// (graph_direct_goal_connection.cu:169-227).
__global__ void k_gd_reset(const Inst *insts, const int *slots, int fresh)
{
    const Inst &I = insts[slots[blockIdx.y]];
    const long cells = (long)I.W * I.H;
    const long words = (cells + 31) / 32;
    const int4 ones = make_int4(-1, -1, -1, -1);
    for (long base = ((long)blockIdx.x * blockDim.x + threadIdx.x) * 16; base < cells;
         base += (long)gridDim.x * blockDim.x * 16) {
        *reinterpret_cast<int4 *>(I.gd_flag + base) = ones;
#pragma unroll
        for (int q = 0; q < 16; q += 2)
            *reinterpret_cast<int4 *>(I.memo_key + base + q) = ones;
        // the eager pass starts each curve from the cell's graph cost at
        // set_plan_data time (zero in a newly constructed planner): keep it
        // until the cell is evaluated
#pragma unroll
        for (int q = 0; q < 16; q += 4)
            *reinterpret_cast<int4 *>(I.gd_cost + base + q) =
                fresh ? make_int4(0, 0, 0, 0) : *reinterpret_cast<const int4 *>(I.cost + base + q);
    }
    for (long w = (long)blockIdx.x * blockDim.x + threadIdx.x; w < words;
         w += (long)gridDim.x * blockDim.x)
        I.gd_req[w] = 0u;
}

void launch_direct_goal_reset(const Inst *d_inst, const int *d_slots, int n, int max_cells,
                              int fresh, cudaStream_t st)
{
    if (n <= 0)
        return;
    const int bx = (max_cells / 16 + 255) / 256;
    k_gd_reset<<<dim3(bx, n), 256, 0, st>>>(d_inst, d_slots, fresh);
}

// Evaluates the goal direct connection of one cell with the whole warp and
// stores it as __CUDA_direct_connection does (graph_direct_goal_connection.cu:
// 169-193).  Every lane passes the same cell.
__device__ void gd_eval_cell(const Inst &I, const Foot &f, int pos, int lane, unsigned long long &probes)
{
    const int z = pos / I.W;
    const int x = pos - z * I.W;
    const float lh = compute_heading(x, z, I.goal_x, I.goal_z);
    const float c = curve_warp(I, f, I.gd_max_curvature, x, z, lh, I.goal_x, I.goal_z, I.goal_heading,
                               I.gd_safe, I.gd_cost[pos], kCoarseStride, lane, probes, I.gd_dist);
    if (lane == 0) {
        if (c >= 0) {
            I.gd_heading[pos] = lh;
            I.gd_cost[pos] = c;
        }
        I.gd_flag[pos] = c >= 0 ? 1 : 0;
    }
}

// every still unknown cell of the listed slots (before the intrinsic costs
// that the deferred evaluation reads are replaced); a warp takes 32 cells at
// a time and evaluates their unknown ones one after another
__global__ void __launch_bounds__(256) k_gd_complete(const Inst *insts, State *states,
                                                     const int *slots)
{
    const int slot = slots[blockIdx.y];
    const Inst &I = insts[slot];
    const int cells = I.W * I.H;
    if ((long)blockIdx.x * blockDim.x >= cells)
        return;
    const Foot f = foot_of(I, I.blocked, I.clear);
    const int lane = threadIdx.x & 31;
    unsigned long long probes = 0;
    for (long base = (long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < cells;
         base += (long)gridDim.x * blockDim.x) {
        const long pos = base + lane;
        unsigned m = __ballot_sync(kFull, pos < cells && I.gd_flag[pos] == kGdUnknown);
        while (m) {
            const int k = __ffs(m) - 1;
            m &= m - 1;
            gd_eval_cell(I, f, (int)(base + k), lane, probes);
        }
    }
    probes = warp_sum64(probes);
    if (lane == 0 && probes)
        atomicAdd(&states[slot].probes_pre, probes);
}

void launch_direct_goal_complete(const Inst *d_inst, State *d_state, const int *d_slots, int n,
                                 int max_cells, cudaStream_t st)
{
    if (n <= 0)
        return;
    k_gd_complete<<<dim3((max_cells + 255) / 256, n), 256, 0, st>>>(d_inst, d_state, d_slots);
}

// ---------------------------------------------------------------------------
// search_init (fastrrt.cpp:85-98): clear() only resets the type
// (graph.cu:400-427), then the start node is added
// ---------------------------------------------------------------------------

// CudaGraph::clear (graph.cu:400-427) sets only the node types to NULL, so a
// planner that is reused keeps the derive counts, parents, headings and costs
// of earlier plans in its NULL cells (the derive count steers frontier
// expansion, graph_expansion.cu:160).  `fresh` zeroes those too, which is the
// state of a newly constructed planner: a batch slot that takes a new request
// then plans exactly like a new FastRRT.
__global__ void k_clear_types(const Inst *insts, const int *slots, int fresh)
{
    const Inst &I = insts[slots[blockIdx.y]];
    const long cells = (long)I.W * I.H;
    const int4 zero = make_int4(0, 0, 0, 0);
    if (blockIdx.x == 0)
        for (int r = threadIdx.x; r < kMaxRegions; r += blockDim.x) {
            if (fresh)
                I.region_count[r] = 0;
            I.region_new[r] = 0;
        }
    for (long base = ((long)blockIdx.x * blockDim.x + threadIdx.x) * 16; base < cells;
         base += (long)gridDim.x * blockDim.x * 16) {
        *reinterpret_cast<int4 *>(I.type + base) = zero;
        // the intrinsic costs that goal searches read may change here
#pragma unroll
        for (int q = 0; q < 16; q += 2)
            *reinterpret_cast<int4 *>(I.memo_key + base + q) = make_int4(-1, -1, -1, -1);
        if (fresh) {
#pragma unroll
            for (int q = 0; q < 16; q += 4) {
                *reinterpret_cast<int4 *>(I.child + base + q) = zero;
                *reinterpret_cast<int4 *>(I.parent + base + q) = zero;
                *reinterpret_cast<int4 *>(I.heading + base + q) = zero;
                *reinterpret_cast<int4 *>(I.cost + base + q) = zero;
            }
        }
    }
}

__global__ void k_init_state(const Inst *insts, State *states, const int *slots, int n,
                             int reset_regions)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const int slot = slots[k];
    const Inst &I = insts[slot];
    State &S = states[slot];
    grid_add(I, I.start_x, I.start_z, I.start_heading, -1, -1, 0.0f);
    S.active = 1;
    S.done = 0;
    S.goal_reached = 0;
    S.collision = 0;
    S.iter = 0;
    S.last_expanded = 0;
    S.n_cand = 0;
    S.node_count = 0;
    S.temp_count = 0;
    S.all_count = 0;
    S.n_nodes = 0;
    S.n_memo = 0;
    S.n_gd = 0;
    S.skip = 0;
    S.found = 0;
    S.winner = 0;
    S.best = kBigCost;
    S.loops = 0;
    S.error = 0;
    S.probes = 0;
    S.probes_goal = 0;
    S.start_ns = global_ns();
    S.finish_ns = 0;
    S.deadline_ns = I.timeout_ns > 0 ? S.start_ns + I.timeout_ns : 0;
    (void)reset_regions;  // region counters are reset by k_clear_types
}

void launch_search_init(const Inst *d_inst, State *d_state, const int *d_slots, int n,
                        int max_cells, int fresh, cudaStream_t st)
{
    if (n <= 0)
        return;
    const int bx = (max_cells / 16 + 255) / 256;
    k_clear_types<<<dim3(bx, n), 256, 0, st>>>(d_inst, d_slots, fresh);
    k_init_state<<<(n + 127) / 128, 128, 0, st>>>(d_inst, d_state, d_slots, n, fresh);
}

// ---------------------------------------------------------------------------
// iteration kernels
// ---------------------------------------------------------------------------

// candidate gate + list (graph_expansion.cu:157-164,
// graph_expansion_search_zones.cu:358-368, 461-473)
__global__ void __launch_bounds__(256) k_scan(const Inst *insts, State *states, const Sched *sc)
{
    griddep_wait();  // the previous kernel of the iteration has finished
    const int n = sc->n_slots;
    const int total = sc->sweep_total;
    for (int c = blockIdx.x; c < total; c += gridDim.x) {
        const int slot = find_slot(sc->sweep_start, n, c);
        State &S = states[slot];
        if (!live(S))
            continue;
        const Inst &I = insts[slot];
        const int cells = I.W * I.H;
        const int base = (c - sc->sweep_start[slot]) * kSweepCells + threadIdx.x * 16;
        const int last = S.last_expanded;
        const bool frontier = last >= kFrontierThreshold;
        const bool force = last == 0;
        const int dw = I.W / kRegion + 1;
        int32_t mine[16];
        int cnt = 0;
        if (base < cells) {
            int8_t t[16];
            load16(I.type + base, t);
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const int pos = base + k;
                if (t[k] != T_NODE || pos >= cells)
                    continue;
                bool take;
                if (I.smart) {
                    if (force)
                        take = true;
                    else if (frontier)
                        take = I.child[pos] == 0;
                    else {
                        const int z = pos / I.W, x = pos - z * I.W;
                        take = I.region_count[(z / kRegion) * dw + x / kRegion] <= 0.5 * kRegion;
                    }
                } else {
                    take = !(frontier && I.child[pos] > 0);
                }
                if (take)
                    mine[cnt++] = pos;
            }
        }
        const int at = warp_append(&S.n_cand, cnt);
        for (int k = 0; k < cnt; k++)
            I.cand[at + k] = mine[k];
    }
}

// 32-cell window chunks per goal-search unit, and the units of one node.
// One: with four, the units of a first iteration (one start window per
// request) were too few to balance, and the launch ended with 8 % of its
// warps active (2.1 ms against 0.7 ms, 512 fresh 256 x 256 requests).
constexpr int kGoalGroup = 1;
__device__ __forceinline__ int goal_groups(const Inst &I)
{
    return (I.win_chunks + kGoalGroup - 1) / kGoalGroup;
}

// work units of one slot: 0 candidate chunks, 1 listed-node chunks (both
// ends of the list), 2 listed cells, 3 (node to search, window chunk group),
// 4 candidates
__device__ __forceinline__ long long chunks_of(const Inst &I, const State &S, int which)
{
    switch (which) {
    case 0: return (S.n_cand + kCandChunk - 1) / kCandChunk;
    case 1: return (S.n_nodes + S.n_memo + kNodeChunk - 1) / kNodeChunk;
    case 2: return S.n_gd;
    case 3: return (long long)S.n_nodes * goal_groups(I);
    default: return S.n_cand;
    }
}

// exclusive prefix over the slots of their work units (one block)
__device__ void plan_prefix(const Inst *insts, State *states, int n, int which, int *out)
{
    __shared__ long long warp_tot[32];
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int s0 = threadIdx.x * per;
    long long local = 0;
    for (int s = s0; s < s0 + per && s < n; s++) {
        const State &S = states[s];
        if (!live(S))
            continue;
        local += chunks_of(insts[s], S, which);
    }
    // block exclusive scan of `local`
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    long long incl = local;
    for (int o = 1; o < 32; o <<= 1) {
        const long long v = __shfl_up_sync(kFull, incl, o);
        if (lane >= o)
            incl += v;
    }
    __syncthreads();  // warp_tot is free (an earlier call is done with it)
    if (lane == 31)
        warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        long long v = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const long long u = __shfl_up_sync(kFull, v, o);
            if (lane >= o)
                v += u;
        }
        warp_tot[lane] = v;
    }
    __syncthreads();
    // the work counters are 32-bit: a pass beyond 2^31 units is refused
    // (state error 2 on every live slot) instead of wrapping
    const bool fits = warp_tot[(blockDim.x >> 5) - 1] <= 0x7fffffffLL;
    long long run = incl - local + (wid ? warp_tot[wid - 1] : 0);
    for (int s = s0; s < s0 + per && s < n; s++) {
        out[s] = fits ? (int)run : 0;
        State &S = states[s];
        if (live(S)) {
            run += chunks_of(insts[s], S, which);
            if (!fits)
                S.error = 2;
        }
    }
    if (threadIdx.x == blockDim.x - 1)
        out[n] = fits ? (int)run : 0;
}

// prefix of per-slot work (one block) for kernels of the iteration, and the
// reset of their work counters; which = 0 (candidates) writes the chunk
// prefix and the exact candidate prefix, which = 1 (node chunks) also the
// prefix of the goal search's (node, window chunk) units, which counts the
// same listed nodes (k_gd_eval scans its own listed cells)
__global__ void __launch_bounds__(1024) k_plan(const Inst *insts, State *states, Sched *sc,
                                              int which)
{
    griddep_wait();  // the previous kernel of the iteration has finished
    const int n = sc->n_slots;
    int *out = which == 0 ? sc->cand_start : sc->node_start;
    plan_prefix(insts, states, n, which, out);
    if (which == 0)
        plan_prefix(insts, states, n, 4, sc->cand_exact);
    if (which == 1)
        plan_prefix(insts, states, n, 3, sc->goal_start);
    if (threadIdx.x == 0) {
        sc->grab[which] = 0;
        if (which == 1) {  // the direct-connection evaluation and the goal search follow
            sc->grab[2] = 0;
            sc->grab[3] = 0;
        }
    }
}


// the winner of each claimed cell applies expand_node's transitions
__global__ void __launch_bounds__(256) k_apply(const Inst *insts, State *states, const Sched *sc)
{
    griddep_wait();  // the previous kernel of the iteration has finished
    const int n = sc->n_slots;
    const int total = sc->cand_start[n];
    for (int c = blockIdx.x; c < total; c += gridDim.x) {
        const int slot = find_slot(sc->cand_start, n, c);
        const Inst &I = insts[slot];
        State &S = states[slot];
        const int idx = (c - sc->cand_start[slot]) * kCandChunk + threadIdx.x;
        if (idx >= S.n_cand)
            continue;
        const int end = I.cand_end[idx];
        if (end < 0)
            continue;
        const int pos = I.cand[idx];
        if (I.claim[end] != pos)
            continue;
        I.claim[end] = kClaimFree;
        const int z = pos / I.W, x = pos - z * I.W;
        const int8_t t = I.type[end];
        if (t == T_NULL) {
            I.child[pos] += 1;
            I.type[end] = T_TEMP;
        } else if (t == T_NODE) {
            I.type[end] = T_COLLISION;
            S.collision = 1;
            I.child[pos] -= 1;
        } else {
            continue;
        }
        I.parent[end] = pack_xz(x, z);
        I.heading[end] = I.cand_heading[idx];
        I.cost[end] = I.cand_cost[idx];
        I.exp_steer[end] = I.cand_steer[idx];
        I.exp_len[end] = I.cand_len[idx];
    }
}

// NODE count (erase bound) and region density after the expansion
__global__ void __launch_bounds__(256) k_post(const Inst *insts, State *states, const Sched *sc)
{
    griddep_wait();  // the previous kernel of the iteration has finished
    const int n = sc->n_slots;
    const int total = sc->sweep_total;
    for (int c = blockIdx.x; c < total; c += gridDim.x) {
        const int slot = find_slot(sc->sweep_start, n, c);
        State &S = states[slot];
        if (!live(S))
            continue;
        const Inst &I = insts[slot];
        const int cells = I.W * I.H;
        const int base = (c - sc->sweep_start[slot]) * kSweepCells + threadIdx.x * 16;
        int nodes = 0;
        // the last two (region, count) runs of the thread's 16 cells (a run
        // before those, possible when the cells span a row end, is added
        // directly)
        int reg[2] = {-1, -1};
        unsigned cnt[2] = {0u, 0u};
        if (base < cells) {
            int8_t t[16];
            load16(I.type + base, t);
            const int dw = I.W / kRegion + 1;
            int run = -1;
            for (int k = 0; k < 16; k++) {
                const int pos = base + k;
                if (pos >= cells)
                    break;
                nodes += t[k] == T_NODE;
                if (I.smart && t[k] != T_NULL && t[k] != T_PROCESSING) {
                    const int z = pos / I.W, x = pos - z * I.W;
                    const int r = (z / kRegion) * dw + x / kRegion;
                    if (run < 0 || r != reg[run]) {
                        if (run == 1) {
                            atomicAdd(&I.region_new[reg[0]], cnt[0]);
                            reg[0] = reg[1];
                            cnt[0] = cnt[1];
                            cnt[1] = 0u;
                            run = 0;
                        }
                        reg[++run] = r;
                    }
                    cnt[run]++;
                }
            }
        }
        // density of the new nodes by region (graph_expansion_search_zones.cu:
        // 42-66): the warp's 512 consecutive cells fall in a few regions; the
        // lanes of each region sum their counts and one adds them
        if (I.smart) {
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const bool has = cnt[q] > 0;
                const unsigned act = __ballot_sync(kFull, has);
                if (has) {
                    const unsigned m = __match_any_sync(act, reg[q]);
                    const unsigned sum = __reduce_add_sync(m, cnt[q]);
                    if ((threadIdx.x & 31) == __ffs(m) - 1)
                        atomicAdd(&I.region_new[reg[q]], sum);
                }
            }
        }
        nodes = warp_sum(nodes);
        if ((threadIdx.x & 31) == 0 && nodes)
            atomicAdd(&S.node_count, nodes);
    }
}

// erase every node whose ancestor chain meets a COLLISION or NULL node within
// numNodes + 4 hops (graph_collision.cu:32-83; an exhausted walk keeps the node)
__global__ void __launch_bounds__(256) k_erase(const Inst *insts, State *states, const Sched *sc)
{
    griddep_wait();  // the previous kernel of the iteration has finished
    // the chunk's non-NULL cells (offsets in the chunk), walked one per thread
    __shared__ uint16_t list[kSweepCells];
    __shared__ int count;
    const int n = sc->n_slots;
    const int total = sc->sweep_total;
    for (int c = blockIdx.x; c < total; c += gridDim.x) {
        const int slot = find_slot(sc->sweep_start, n, c);
        const State &S = states[slot];
        if (!live(S) || !S.collision || S.node_count <= 2)
            continue;  // uniform across the block
        const Inst &I = insts[slot];
        volatile int8_t *type = I.type;
        const int cells = I.W * I.H;
        const int base0 = (c - sc->sweep_start[slot]) * kSweepCells;
        if (threadIdx.x == 0)
            count = 0;
        __syncthreads();
        const int base = base0 + threadIdx.x * 16;
        int8_t t[16];
        int mine = 0;
        if (base < cells) {
            load16(I.type + base, t);
            for (int k = 0; k < 16; k++)
                mine += (base + k < cells && t[k] != T_NULL) ? 1 : 0;
        }
        // warp-aggregated append into the block's list
        const int lane = threadIdx.x & 31;
        int incl = mine;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(kFull, incl, o);
            if (lane >= o)
                incl += v;
        }
        const int wsum = __shfl_sync(kFull, incl, 31);
        int at = 0;
        if (lane == 31 && wsum)
            at = atomicAdd(&count, wsum);
        at = __shfl_sync(kFull, at, 31) + incl - mine;
        if (mine) {
            for (int k = 0; k < 16; k++)
                if (base + k < cells && t[k] != T_NULL)
                    list[at++] = (uint16_t)(threadIdx.x * 16 + k);
        }
        __syncthreads();
        const int m = count;
        for (int e = threadIdx.x; e < m; e += blockDim.x) {
            const int pos = base0 + list[e];
            int curr = pos;
            int i = S.node_count + 4;
            while (i-- > 0) {
                const int32_t p = I.parent[curr];
                const int px = unpack_x(p), pz = unpack_z(p);
                if (px == -1 && pz == -1)
                    break;
                if (px < 0 || px >= I.W || pz < 0 || pz >= I.H)
                    break;
                const int next = pz * I.W + px;
                const int8_t tn = type[next];
                if (tn == T_COLLISION || tn == T_NULL) {
                    type[pos] = T_NULL;
                    break;
                }
                curr = next;
            }
        }
        __syncthreads();  // the list is rebuilt for the next chunk
    }
}

// COLLISION -> NODE, child count reset, parent child count + 1
// (graph_collision.cu:84-104)
// COLLISION -> NODE of a thread's 16 cells with the child-count updates
// (graph_collision.cu:90-110), run by k_accept before it reads them; the
// collision pass needs k_erase's walks over the whole grid done, which the
// kernel boundary before k_accept provides
__device__ __forceinline__ void set_collision_nodes(const Inst &I, int base, int cells)
{
    int8_t t[16];
    load16(I.type + base, t);
    for (int k = 0; k < 16; k++) {
        const int pos = base + k;
        if (pos >= cells || t[k] != T_COLLISION)
            continue;
        I.type[pos] = T_NODE;
        I.child[pos] = 0;
        const int32_t p = I.parent[pos];
        const int px = unpack_x(p), pz = unpack_z(p);
        if (px >= 0 && px < I.W && pz >= 0 && pz < I.H)
            atomicAdd(&I.child[pz * I.W + px], 1);
    }
}

// TEMP count, non-NULL count, TEMP -> NODE, and the NODE list
__device__ __forceinline__ unsigned long long memo_key_of(const Inst &I, int pos)
{
    return ((unsigned long long)__float_as_uint(I.heading[pos]) << 32) |
           (unsigned long long)__float_as_uint(I.cost[pos]);
}

// checkGoalReached for one node (graph_best_node.cu:181-222)
__device__ __forceinline__ void goal_check_node(const Inst &I, State &S, int pos)
{
    const int z = pos / I.W, x = pos - z * I.W;
    const double dx = I.goal_x - x, dz = I.goal_z - z;
    if (!(sqrt(dx * dx + dz * dz) > I.dist_tol) && fabsf(I.heading[pos] - I.goal_heading) <= I.heading_tol)
        S.goal_reached = 1;
}

__global__ void __launch_bounds__(256) k_accept(const Inst *insts, State *states, const Sched *sc)
{
    griddep_wait();  // the previous kernel of the iteration has finished
    const int n = sc->n_slots;
    const int total = sc->sweep_total;
    for (int c = blockIdx.x; c < total; c += gridDim.x) {
        const int slot = find_slot(sc->sweep_start, n, c);
        State &S = states[slot];
        if (!live(S))
            continue;
        const Inst &I = insts[slot];
        const int cells = I.W * I.H;
        const int base = (c - sc->sweep_start[slot]) * kSweepCells + threadIdx.x * 16;
        int temps = 0, all = 0, cnt = 0, kept = 0;
        int32_t mine[16];
        int32_t mine_kept[16];
        if (base < cells && S.collision && S.node_count > 2)
            set_collision_nodes(I, base, cells);  // this thread's own 16 cells, before it reads them
        if (base < cells) {
            int4 v = *reinterpret_cast<const int4 *>(I.type + base);
            int8_t *t = reinterpret_cast<int8_t *>(&v);
            bool changed = false;
#pragma unroll
            for (int k = 0; k < 16; k++) {
                if (base + k >= cells)
                    continue;
                temps += t[k] == T_TEMP;
                all += t[k] != T_NULL;
                if (t[k] == T_TEMP) {
                    t[k] = T_NODE;
                    changed = true;
                }
                if (t[k] != T_NODE)
                    continue;
                const int pos = base + k;
                if (I.memo_key[pos] == memo_key_of(I, pos)) {
                    // searched before with this heading and cost: the goal
                    // check runs here, and a kept connection is listed as
                    // the node's result without a search
                    goal_check_node(I, S, pos);
                    const unsigned long long r = I.memo_result[pos];
                    if (r != kNoConnection) {
                        mine_kept[kept++] = pos;
                        atomicMin(&S.best, (long long)(r >> 32));
                    }
                    continue;
                }
                mine[cnt++] = pos;
            }
            if (changed)
                *reinterpret_cast<int4 *>(I.type + base) = v;
        }
        const int at = warp_append(&S.n_nodes, cnt);
        for (int k = 0; k < cnt; k++) {
            I.nodes[at + k] = mine[k];
            I.node_key[at + k] = kNoConnection;
            I.node_pending[at + k] = goal_groups(I);
            I.node_pruned[at + k] = 0;
        }
        // kept results from the end of the list: the two ends never meet, as
        // both hold distinct NODE cells of the frame
        const int kat = warp_append(&S.n_memo, kept);
        for (int k = 0; k < kept; k++) {
            const int idx = cells - 1 - (kat + k);
            I.nodes[idx] = mine_kept[k];
            I.node_key[idx] = I.memo_result[mine_kept[k]];
        }
        temps = warp_sum(temps);
        all = warp_sum(all);
        if ((threadIdx.x & 31) == 0) {
            if (temps)
                atomicAdd(&S.temp_count, temps);
            if (all)
                atomicAdd(&S.all_count, all);
        }
    }
}

__device__ __forceinline__ int window_count(int c, float r, int &lo)
{
    lo = (int)(c - r);
    const float hi = c + r;
    const int k0 = (int)ceilf(hi);
    return k0 > lo ? k0 - lo : 0;
}

// Lists, once per cell, the cells inside the windows of the nodes that the
// goal search will search this iteration whose direct connection is unknown.
// One warp per unit of the goal search (node to search, group of window
// chunks), one window cell per lane and chunk: a node's window is spread
// over many warps, so the pass costs a few memory round trips at any load.
__global__ void __launch_bounds__(256) k_gd_demand(const Inst *insts, State *states, const Sched *sc)
{
    griddep_wait();  // the previous kernel of the iteration has finished
    const int n = sc->n_slots;
    const int total = sc->goal_start[n];
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int u = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); u < total; u += warps) {
        const int slot = find_slot(sc->goal_start, n, u);
        const Inst &I = insts[slot];
        State &S = states[slot];
        const int local = u - sc->goal_start[slot];
        const int groups = goal_groups(I);
        const int idx = local / groups;
        const int wg = local - idx * groups;
        const int pos = I.nodes[idx];  // a node to search: no kept result
        const int z = pos / I.W, x = pos - z * I.W;
        int zlo, xlo;
        const int nz = window_count(z, I.dist_tol, zlo);
        const int nx = window_count(x, I.dist_tol, xlo);
        const int wtotal = nx > 0 ? nz * nx : 0;
        for (int q = 0; q < kGoalGroup; q++) {
            const int w = (wg * kGoalGroup + q) * 32 + lane;
            int cell = -1;
            if (w < wtotal) {
                const int zp = zlo + w / nx, xp = xlo + w % nx;
                if (zp >= 0 && zp < I.H && xp >= 0 && xp < I.W) {
                    const int cc = zp * I.W + xp;
                    if (I.gd_flag[cc] == kGdUnknown) {
                        const uint32_t bit = 1u << (cc & 31);
                        if (!(atomicOr(&I.gd_req[cc >> 5], bit) & bit))
                            cell = cc;
                    }
                }
            }
            const unsigned m = __ballot_sync(kFull, cell >= 0);
            if (!m)
                continue;
            int at = 0;
            if (lane == 0)
                at = atomicAdd(&S.n_gd, __popc(m));
            at = __shfl_sync(kFull, at, 0);
            if (cell >= 0)
                I.gd_list[at + __popc(m & ((1u << lane) - 1u))] = cell;
        }
    }
}

// A full footprint probe for lane `leader`, answered by the whole warp; the
// leader's footprint may belong to another slot than the other lanes' tasks.
__device__ inline bool coop_probe(const Foot &mine, int leader, int lane, int x, int z, float angle,
                                  unsigned &cnt)
{
    Foot f;
    f.W = __shfl_sync(kFull, mine.W, leader);
    f.H = __shfl_sync(kFull, mine.H, leader);
    f.mdx = __shfl_sync(kFull, mine.mdx, leader);
    f.mdz = __shfl_sync(kFull, mine.mdz, leader);
    f.lbx = __shfl_sync(kFull, mine.lbx, leader);
    f.lbz = __shfl_sync(kFull, mine.lbz, leader);
    f.ubx = __shfl_sync(kFull, mine.ubx, leader);
    f.ubz = __shfl_sync(kFull, mine.ubz, leader);
    f.rw = __shfl_sync(kFull, mine.rw, leader);
    f.blocked = reinterpret_cast<const uint32_t *>(
        __shfl_sync(kFull, reinterpret_cast<unsigned long long>(mine.blocked), leader));
    f.clear = nullptr;
    f.trav = nullptr;
    f.sat = nullptr;
    const int bx = __shfl_sync(kFull, x, leader);
    const int bz = __shfl_sync(kFull, z, leader);
    const float ba = __shfl_sync(kFull, angle, leader);
    if (rows_clear_warp(f, bx, bz, cosf(ba), sinf(ba), lane)) {
        cnt = full_probes(f);  // feasible: the reference runs all its probes
        return true;
    }
    return probe_warp(f, bx, bz, ba, lane, cnt);
}

// One listed cell per warp at a time, grabbed from a counter over all slots:
// the warp evaluates the cell's curve to the goal sample-parallel
// (curve_warp), so a launch with few cells still spreads each curve over 32
// lanes, and lanes never wait for a longer curve of another lane.  Masks are
// read through L1.
__global__ void __launch_bounds__(256, kEvalBlocks) k_gd_eval(const Inst *insts, State *states, Sched *sc)
{
    griddep_wait();  // the previous kernel of the iteration has finished
    const int n = sc->n_slots;
    // every block scans the slots' listed-cell counts into its own prefix
    // (n + 1 ints of dynamic shared memory) instead of a separate launch
    extern __shared__ int gd_start[];
    plan_prefix(insts, states, n, 2, gd_start);
    __syncthreads();
    const int total = gd_start[n];
    const int lane = threadIdx.x & 31;
    const int batch = grab_batch(total);
    for (int e0 = 0, e1 = 0, e = 0, slot = 0;; e++) {
        if (e >= e1) {
            if (lane == 0)
                e0 = (int)atomicAdd(&sc->grab[2], (unsigned)batch);
            e0 = __shfl_sync(kFull, e0, 0);
            if (e0 >= total)
                break;
            e = e0;
            e1 = min(e0 + batch, total);
            slot = find_slot(gd_start, n, e);
        }
        while (e >= gd_start[slot + 1])
            slot++;
        const Inst &I = insts[slot];
        const int pos = I.gd_list[e - gd_start[slot]];
        const Foot f = foot_of(I, I.blocked, I.clear);
        const int z = pos / I.W;
        const int x = pos - z * I.W;
        const float lh = compute_heading(x, z, I.goal_x, I.goal_z);
        unsigned long long probes = 0;
        // the full footprint test out of line (8 % less time per launch,
        // same answers)
        const float c = curve_warp<true>(I, f, I.gd_max_curvature, x, z, lh, I.goal_x, I.goal_z,
                                         I.goal_heading, I.gd_safe, I.gd_cost[pos], kCoarseStride, lane,
                                         probes, I.gd_dist);
        probes = warp_sum64(probes);
        if (lane == 0) {
            // __CUDA_direct_connection (graph_direct_goal_connection.cu:169-193)
            if (c >= 0) {
                I.gd_heading[pos] = lh;
                I.gd_cost[pos] = c;
            }
            I.gd_flag[pos] = c >= 0 ? 1 : 0;
            if (probes)
                atomicAdd(&states[slot].probes_pre, probes);
        }
    }
}

// Expansion: one candidate per warp at a time, grabbed over all slots: the
// warp integrates the candidate
// step-parallel (kin_warp), so a launch with few candidates still spreads
// each over 32 lanes.  Masks are read through L1.
__global__ void __launch_bounds__(256) k_expand(const Inst *insts, State *states, Sched *sc)
{
    griddep_wait();  // the previous kernel of the iteration has finished
    const int n = sc->n_slots;
    const int total = sc->cand_exact[n];
    const int lane = threadIdx.x & 31;
    const int batch = grab_batch(total);
    for (int e0 = 0, e1 = 0, e = 0, slot = 0;; e++) {
        if (e >= e1) {
            if (lane == 0)
                e0 = (int)atomicAdd(&sc->grab[0], (unsigned)batch);
            e0 = __shfl_sync(kFull, e0, 0);
            if (e0 >= total)
                break;
            e = e0;
            e1 = min(e0 + batch, total);
            slot = find_slot(sc->cand_exact, n, e);
        }
        while (e >= sc->cand_exact[slot + 1])
            slot++;
        const int idx = e - sc->cand_exact[slot];
        const Inst &I = insts[slot];
        const Foot f = foot_of(I, I.blocked, I.clear);
        const int pos = I.cand[idx];
        const int z = pos / I.W, x = pos - z * I.W;
        float steer, len;
        if (I.proposal && e < sc->prop_cap && I.prop_len[idx] >= 0.0f) {
            steer = I.prop_steer[idx];
            len = I.prop_len[idx];
        } else {
            draw_expansion(I.seed, (uint32_t)pos, states[slot].iter, (float)I.max_steer, I.max_path, steer,
                           len);
        }
        unsigned long long probes = 0;
        const KinResult r = kin_warp(I, f, x, z, steer, len, I.velocity, I.heading[pos], I.cost[pos], lane,
                                     probes);
        probes = warp_sum64(probes);
        if (lane == 0) {
            // expand_node (graph_expansion.cu:103-145): no end cell at the
            // coordinate origin or on the expanding cell itself
            int end = -1;
            if (r.ok && !(r.last_x == I.og_x && r.last_z == I.og_z)) {
                const int ep = r.last_z * I.W + r.last_x;
                if (ep != pos)
                    end = ep;
            }
            I.cand_steer[idx] = steer;
            I.cand_len[idx] = len;
            I.cand_end[idx] = end;
            I.cand_heading[idx] = r.heading;
            I.cand_cost[idx] = r.cost;
            if (end >= 0)
                atomicMin(&I.claim[end], pos);
            if (probes)
                atomicAdd(&states[slot].probes, probes);
        }
    }
}

__device__ __forceinline__ unsigned long long connection_key(long long lc, int cell)
{
    return ((unsigned long long)lc << 32) | (unsigned long long)(0xffffffffu - (unsigned)cell);
}

// Goal search (findBestGoalDirectConnection, graph_check_goal_reached.cu:
// 17-70, plus checkGoalReached for the node, graph_best_node.cu:181-222),
// one warp per (listed node, group of kGoalGroup 32-cell chunks of its
// window) unit, each warp grabbing units on its own: a node's window is
// spread over many warps, so a few nodes with busy windows do not hold a
// launch back.  The warp lists the unit's cells that have a direct goal
// connection (a few percent of a window) and evaluates the node's curve to
// each of them in window order, sample-parallel (curve_warp).  The best
// connection keeps the lowest fixed-point cost, ties to the later (higher)
// cell.  Consecutive units a warp takes of one node are merged before they
// are published; the node's last unit to finish keeps the node's result when
// no unit skipped a cell by the bound.  Masks are read through L1.
__global__ void __launch_bounds__(256, kGoalBlocks) k_goal(const Inst *insts, State *states, Sched *sc)
{
    griddep_wait();  // the previous kernel of the iteration has finished
    const int n = sc->n_slots;
    const int total = sc->goal_start[n];
    const int lane = threadIdx.x & 31;
    const int batch = grab_batch(total);
    // the node whose units this warp is merging
    int cur_slot = -1, cur_idx = -1, cur_units = 0;
    long long best = kBigCost;
    int best_cell = -1;
    bool pruned = false;
    unsigned long long probes = 0, key = 0;
    int cur_pos = 0;
    auto publish = [&]() {
        if (cur_idx < 0)
            return;
        const Inst &I = insts[cur_slot];
        State &S = states[cur_slot];
        probes = warp_sum64(probes);
        if (lane == 0) {
            if (probes)
                atomicAdd(&S.probes_goal, probes);
            if (best < kBigCost) {
                const unsigned long long k = connection_key(best, best_cell);
                atomicMin(&I.node_key[cur_idx], k);
                atomicMin(&S.best, (long long)(k >> 32));
            }
            if (pruned)
                atomicOr(&I.node_pruned[cur_idx], 1);
            __threadfence();
            if (atomicSub(&I.node_pending[cur_idx], cur_units) == cur_units) {
                // every unit of the node is done
                __threadfence();
                const unsigned long long r = atomicAdd(&I.node_key[cur_idx], 0ull);
                if (!atomicAdd(&I.node_pruned[cur_idx], 0)) {
                    I.memo_result[cur_pos] = r;
                    I.memo_key[cur_pos] = key;
                }
            }
        }
        probes = 0;
        best = kBigCost;
        best_cell = -1;
        pruned = false;
        cur_idx = -1;
        cur_units = 0;
    };
    for (int e0 = 0, e1 = 0, e = 0, slot = 0;; e++) {
        if (e >= e1) {
            if (lane == 0)
                e0 = (int)atomicAdd(&sc->grab[3], (unsigned)batch);
            e0 = __shfl_sync(kFull, e0, 0);
            if (e0 >= total)
                break;
            e = e0;
            e1 = min(e0 + batch, total);
            slot = find_slot(sc->goal_start, n, e);
        }
        while (e >= sc->goal_start[slot + 1])
            slot++;
        const Inst &I = insts[slot];
        State &S = states[slot];
        const int local = e - sc->goal_start[slot];
        const int groups = goal_groups(I);
        const int idx = local / groups;
        const int wg = local - idx * groups;
        // a node to search (nodes with a kept result were resolved when
        // listed); the key of this heading and cost marks a complete result
        const int pos = I.nodes[idx];
        if (slot != cur_slot || idx != cur_idx) {
            publish();
            cur_slot = slot;
            cur_idx = idx;
            cur_pos = pos;
            key = memo_key_of(I, pos);
        }
        cur_units++;
        if (wg == 0 && lane == 0)
            goal_check_node(I, S, pos);
        const Foot f = foot_of(I, I.blocked, I.clear);
        const int z = pos / I.W, x = pos - z * I.W;
        const float heading = I.heading[pos];
        const float cost = I.cost[pos];
        int zlo, xlo;
        const int nz = window_count(z, I.dist_tol, zlo);
        const int nx = window_count(x, I.dist_tol, xlo);
        const int wtotal = nx > 0 ? nz * nx : 0;
        const bool prune = I.intrinsic == nullptr;
        const volatile long long *global_best = &S.best;
        for (int q = 0; q < kGoalGroup; q++) {
            const int w = (wg * kGoalGroup + q) * 32 + lane;
            int cell = -1;
            if (w < wtotal) {
                const int zp = zlo + w / nx, xp = xlo + w % nx;
                if (zp >= 0 && zp < I.H && xp >= 0 && xp < I.W) {
                    const int cc = zp * I.W + xp;
                    if (I.gd_flag[cc] == 1)
                        cell = cc;
                }
            }
            unsigned m = __ballot_sync(kFull, cell >= 0);
            while (m) {
                const int k = __ffs(m) - 1;
                m &= m - 1;
                const int cc = __shfl_sync(kFull, cell, k);
                const float gdc = I.gd_cost[cc];
                if (prune) {
                    // the connection costs at least cost + 1 (the first sample)
                    const float lb_total = (cost + 1.0f) + gdc;
                    const long long lb = __float2ll_rd(100 * lb_total);
                    // one read for the whole warp, so its lanes agree
                    long long gb = 0;
                    if (lane == 0)
                        gb = *global_best;
                    gb = __shfl_sync(kFull, gb, 0);
                    if (lb > gb) {
                        pruned = true;
                        continue;
                    }
                }
                const int zp = cc / I.W, xp = cc - zp * I.W;
                const float seg = curve_warp(I, f, I.max_curvature, x, z, heading, xp, zp, I.gd_heading[cc],
                                             1, cost, 0, lane, probes);
                if (seg < 0)
                    continue;
                const float total_cost = seg + gdc;
                const long long lc = __float2ll_rd(100 * total_cost);
                if (lc <= best) {
                    best = lc;
                    best_cell = cc;
                }
            }
        }
    }
    publish();
}

// among listed nodes with the minimum, the highest node cell index wins
__global__ void __launch_bounds__(256) k_select(const Inst *insts, State *states, const Sched *sc)
{
    griddep_wait();  // the previous kernel of the iteration has finished
    const int n = sc->n_slots;
    const long entries = (long)sc->node_start[n] * kNodeChunk;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < entries;
         e += (long)gridDim.x * blockDim.x) {
        const int chunk = (int)(e / kNodeChunk);
        const int slot = find_slot(sc->node_start, n, chunk);
        const Inst &I = insts[slot];
        State &S = states[slot];
        int idx = (chunk - sc->node_start[slot]) * kNodeChunk + (int)(e % kNodeChunk);
        if (idx >= S.n_nodes + S.n_memo || S.best >= kBigCost)
            continue;
        if (idx >= S.n_nodes)
            idx = I.W * I.H - 1 - (idx - S.n_nodes);  // a kept result
        const unsigned long long nk = I.node_key[idx];
        if (nk != kNoConnection && (long long)(nk >> 32) == S.best) {
            const unsigned long long key =
                ((unsigned long long)(unsigned)I.nodes[idx] << 32) | (unsigned)idx;
            atomicMax(&S.winner, key);
        }
    }
}

// The cost of the curve from node ppos to the goal-connected cell, as the goal
// search computed it (graph_direct_goal_connection.cu:16-167 from the node),
// by the calling warp.  Every lane of the warp calls it.
__device__ float connection_segment_cost(const Inst &I, int ppos, int cell, int lane)
{
    const Foot f = foot_of(I, I.blocked, I.clear);
    const int pz = ppos / I.W, px = ppos - pz * I.W;
    const int cz = cell / I.W, cx = cell - cz * I.W;
    unsigned long long unused = 0;
    return curve_warp(I, f, I.max_curvature, px, pz, I.heading[ppos], cx, cz, I.gd_heading[cell], 1,
                      I.cost[ppos], 0, lane, unused);
}

// the host-side tail of FastRRT::loop, one warp per slot (the warp helps
// lane 0 re-run the winning connection's curve)
__global__ void k_finish(const Inst *insts, State *states, int n)
{
    griddep_wait();  // the previous kernel of the iteration has finished
    const int slot = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (slot >= n)
        return;  // uniform across the warp
    State &S = states[slot];
    if (!live(S))
        return;  // uniform across the warp
    const Inst &I = insts[slot];
    const bool connect = !(S.temp_count == 0 && S.all_count == 0) && S.best < kBigCost;
    float seg = 0.0f;
    if (connect) {
        const int widx = (int)(S.winner & 0xffffffffu);
        const int wcell = (int)(0xffffffffu - (unsigned)(I.node_key[widx] & 0xffffffffu));
        seg = connection_segment_cost(I, I.nodes[widx], wcell, lane);
    }
    if (lane != 0)
        return;
    S.last_expanded = S.temp_count;
    if (S.temp_count == 0 && S.all_count == 0) {
        // empty graph: the start is added again (fastrrt.cpp:132-139)
        grid_add(I, I.start_x, I.start_z, I.start_heading, -1, -1, 0.0f);
    } else if (S.best < kBigCost) {
        // fastrrt.cpp:145-167
        const int idx = (int)(S.winner & 0xffffffffu);
        const int ppos = I.nodes[idx];
        const int pz = ppos / I.W, px = ppos - pz * I.W;
        const int cell = (int)(0xffffffffu - (unsigned)(I.node_key[idx] & 0xffffffffu));
        const int cz = cell / I.W, cx = cell - cz * I.W;
        const float base = I.cost[ppos];
        const float child_heading = I.gd_heading[cell];
        grid_add(I, cx, cz, child_heading, px, pz, seg + base);
        const float child_cost = child_heading + base;
        grid_add(I, I.goal_x, I.goal_z, I.goal_heading, cx, cz, child_cost);
        if (I.goal_x >= 0 && I.goal_x < I.W && I.goal_z >= 0 && I.goal_z < I.H &&
            !(0.0 > I.dist_tol) && fabsf(I.goal_heading - I.goal_heading) <= I.heading_tol)
            S.goal_reached = 1;
        S.found = 1;
    }
    S.loops++;
    S.iter++;
    const long long now = global_ns();
    if (S.goal_reached && I.stop_on_goal)
        S.done = 1;
    else if (I.max_iter > 0 && S.loops >= I.max_iter)
        S.done = 1;
    else if (S.deadline_ns > 0 && now > S.deadline_ns)
        S.done = 1;
    if (S.done)
        S.finish_ns = now;
    // per-iteration resets
    S.n_cand = 0;
    S.node_count = 0;
    S.temp_count = 0;
    S.all_count = 0;
    S.n_nodes = 0;
    S.n_memo = 0;
    S.n_gd = 0;
    S.collision = 0;
    S.best = kBigCost;
    S.winner = 0;
    if (I.smart) {
        const int regions = (I.W / kRegion + 1) * (I.H / kRegion + 1);
        for (int r = 0; r < regions; r++) {
            I.region_count[r] = I.region_new[r];
            I.region_new[r] = 0;
        }
    }
}

const char *const kIterKernelNames[kIterKernels] = {
    "k_scan", "k_plan(cand)", "k_propose(mlp)", "k_expand", "k_apply", "k_post", "k_erase",
    "k_accept", "k_plan(nodes, windows)", "k_gd_demand", "k_gd_eval", "k_goal", "k_select",
    "k_finish"};

// ---------------------------------------------------------------------------
// learned expansion proposal inside an iteration
// ---------------------------------------------------------------------------

// One warp per listed candidate: with probability mix (the third Philox word
// of the candidate's draw) the (steering, length) bin is sampled from the
// softmax of the network's logits (fourth word, inverse CDF) and the value
// uniformly inside the bin (first two words); otherwise prop_len = -1 and
// the expansion draws uniformly as without the network.
__device__ void prop_sample_row(const Inst *insts, const State *states, const Sched *sc, const ProposalBufs &pb,
                                int r, int lane)
{
    const int slot = find_slot(sc->cand_exact, sc->n_slots, r);
    const int idx = r - sc->cand_exact[slot];
    const Inst &I = insts[slot];
    const int pos = I.cand[idx];
    const State &S = states[slot];
    uint32_t w[4];
    philox4x32((uint32_t)pos, S.iter, kRngTag, 0u, (uint32_t)I.seed, (uint32_t)(I.seed >> 32), w);
    if (!(u01(w[2]) < pb.mix)) {
        if (lane == 0)
            I.prop_len[idx] = -1.0f;
        return;
    }
    const float *l = pb.logits + (long)r * kMlpOut;
    float v[kMlpOut / 32];
    float mx = -1e30f;
#pragma unroll
    for (int q = 0; q < kMlpOut / 32; q++) {
        v[q] = l[lane * (kMlpOut / 32) + q];  // lane owns bins lane*4 .. lane*4+3
        mx = fmaxf(mx, v[q]);
    }
    for (int o = 16; o; o >>= 1)
        mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, o));
    float mine = 0.0f;
#pragma unroll
    for (int q = 0; q < kMlpOut / 32; q++) {
        v[q] = __expf(v[q] - mx);
        mine += v[q];
    }
    float incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const float t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o)
            incl += t;
    }
    const float total = __shfl_sync(kFull, incl, 31);
    const float target = u01(w[3]) * total;
    // the first bin whose cumulative mass reaches the target
    const float before = incl - mine;
    int bin = -1;
    if (target < incl && target >= before) {
        float run = before;
        bin = lane * (kMlpOut / 32) + kMlpOut / 32 - 1;
#pragma unroll
        for (int q = 0; q < kMlpOut / 32; q++) {
            run += v[q];
            if (target < run) {
                bin = lane * (kMlpOut / 32) + q;
                break;
            }
        }
    }
    const unsigned found = __ballot_sync(kFull, bin >= 0);
    const int owner = found ? __ffs(found) - 1 : 31;
    bin = __shfl_sync(kFull, bin, owner);
    if (bin < 0)
        bin = kMlpOut - 1;
    if (lane != 0)
        return;
    const float ms = (float)I.max_steer;
    const int sb = bin / kLenBins, lb = bin - sb * kLenBins;
    const float sw = 2.0f * ms / kSteerBins;
    const float lo = 5.0f, hi = fmaxf(I.max_path, 5.0f);
    const float lw = (hi - lo) / kLenBins;
    I.prop_steer[idx] = -ms + (sb + u01(w[0])) * sw;
    I.prop_len[idx] = fmaxf(5.0f, lo + (lb + u01(w[1])) * lw);
}

// rows grid-strided over a machine-sized grid (the row count is on the device)
__global__ void __launch_bounds__(256) k_prop_sample(const Inst *insts, const State *states, const Sched *sc,
                                                     ProposalBufs pb)
{
    griddep_wait();  // the previous kernel of the iteration has finished
    const int lane = threadIdx.x & 31;
    const int rows = min(sc->cand_exact[sc->n_slots], pb.cap);
    const int warps = (int)((gridDim.x * (long)blockDim.x) >> 5);
    for (int r = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5); r < rows; r += warps)
        prop_sample_row(insts, states, sc, pb, r, lane);
}

// the proposal step: every candidate of the iteration has its row (the exact
// candidate prefix of its slot + its index), so features, the network and
// the sampling read their rows' candidates directly; *count is the number
// of candidates (the last entry of the exact prefix, on the device)
void launch_proposal(const Inst *d_inst, State *d_state, const Sched *d_sched, const ProposalBufs &pb,
                     const Launch &L, cudaStream_t st, bool dep)
{
    (void)L;
    launch_features_sched(d_inst, d_sched, pb.cap, pb.X, st, pb.count, dep);
    launch_mlp_forward(pb.w, pb.X, pb.cap, pb.count, nullptr, nullptr, pb.logits, st, dep);
    launch_dep(dep, k_prop_sample, std::min((pb.cap * 32 + 255) / 256, kMlpGridBlocks), 256, 0, st, d_inst,
               d_state, d_sched, pb);
}

void launch_iteration(const Inst *d_inst, State *d_state, Sched *d_sched, int n_slots,
                      const Launch &L, cudaStream_t st, cudaEvent_t *ev, const ProposalBufs *pb)
{
    // programmatic dependent launches, except in the kernel-timing mode
    // (events between the kernels)
    const bool dep = L.pdl && !ev;
    int k = 0;
    auto mark = [&]() {
        if (ev)
            cudaEventRecord(ev[k], st);
        k++;
    };
    mark();
    launch_dep(dep, k_scan, L.sweep_blocks, 256, 0, st, d_inst, d_state, d_sched);
    mark();
    launch_dep(dep, k_plan, 1, 1024, 0, st, d_inst, d_state, d_sched, 0);
    mark();
    if (pb)
        launch_proposal(d_inst, d_state, d_sched, *pb, L, st, dep);
    mark();
    launch_dep(dep, k_expand, L.work_blocks, 256, 0, st, d_inst, d_state, d_sched);
    mark();
    launch_dep(dep, k_apply, L.sweep_blocks, 256, 0, st, d_inst, d_state, d_sched);
    mark();
    launch_dep(dep, k_post, L.sweep_blocks, 256, 0, st, d_inst, d_state, d_sched);
    mark();
    launch_dep(dep, k_erase, L.sweep_blocks, 256, 0, st, d_inst, d_state, d_sched);
    mark();
    launch_dep(dep, k_accept, L.sweep_blocks, 256, 0, st, d_inst, d_state, d_sched);
    mark();
    launch_dep(dep, k_plan, 1, 1024, 0, st, d_inst, d_state, d_sched, 1);
    mark();
    // one warp per (node, window chunk): its grid follows the machine, not
    // the frame's sweep chunks (16 for one 256 x 256 slot)
    launch_dep(dep, k_gd_demand, L.sms * 8, 256, 0, st, d_inst, d_state, d_sched);
    mark();
    launch_dep(dep, k_gd_eval, L.sms * kEvalBlocks, 256, sizeof(int) * (n_slots + 1), st, d_inst, d_state,
               d_sched);
    mark();
    launch_dep(dep, k_goal, L.sms * kGoalBlocks, 256, 0, st, d_inst, d_state, d_sched);
    mark();
    launch_dep(dep, k_select, L.sweep_blocks, 256, 0, st, d_inst, d_state, d_sched);
    mark();
    launch_dep(dep, k_finish, (n_slots * 32 + 127) / 128, 128, 0, st, d_inst, d_state, n_slots);
    mark();
}

// ---------------------------------------------------------------------------
// standalone goal check, path extraction, optimisation, validation
// ---------------------------------------------------------------------------

// checkGoalReached (graph_best_node.cu:181-250); sticky flag
__global__ void k_goal_check(const Inst *insts, State *states, const int *slots)
{
    const int slot = slots[blockIdx.y];
    const Inst &I = insts[slot];
    State &S = states[slot];
    if (S.goal_reached)
        return;
    const long cells = (long)I.W * I.H;
    for (long pos = blockIdx.x * (long)blockDim.x + threadIdx.x; pos < cells;
         pos += (long)gridDim.x * blockDim.x) {
        if (I.type[pos] != T_NODE)
            continue;
        const int z = (int)(pos / I.W), x = (int)(pos - (long)z * I.W);
        const double dx = I.goal_x - x, dz = I.goal_z - z;
        if (sqrt(dx * dx + dz * dz) > I.dist_tol)
            continue;
        if (fabsf(I.heading[pos] - I.goal_heading) <= I.heading_tol)
            S.goal_reached = 1;
    }
}

void launch_goal_check(const Inst *d_inst, State *d_state, const int *d_slots, int n,
                       int max_cells, cudaStream_t st)
{
    if (n <= 0)
        return;
    k_goal_check<<<dim3((max_cells + 255) / 256, n), 256, 0, st>>>(d_inst, d_state, d_slots);
}

// findBestNode pass 1 (graph_best_node.cu:15-75): key = cost * 2^32 +
// (2^32 - 1 - cell), so the minimum is the lowest cost and, among equal
// costs, the highest cell index (the last writer of the sequential pass 2)
// Only the NODE cells within dist_tol of the goal qualify, so one block per
// slot scans the goal's window (the cells within dist_tol on each axis); the
// minimum key does not depend on the order of the scan.
__global__ void k_best_node(const Inst *insts, const int *slots, long long *keys)
{
    const int k = blockIdx.y;
    const Inst &I = insts[slots[k]];
    const Foot f = foot_of(I, I.blocked, I.clear);
    int zlo, xlo;
    const int nz = window_count(I.goal_z, I.dist_tol, zlo);
    const int nx = window_count(I.goal_x, I.dist_tol, xlo);
    const int wtotal = nx > 0 ? nz * nx : 0;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < wtotal; w += gridDim.x * blockDim.x) {
        const int z = zlo + w / nx, x = xlo + w % nx;
        if (z < 0 || z >= I.H || x < 0 || x >= I.W)
            continue;
        const long pos = (long)z * I.W + x;
        if (I.type[pos] != T_NODE)
            continue;
        const int dx = I.goal_x - x, dz = I.goal_z - z;
        const float dist = sqrtf(dx * dx + dz * dz);
        if (dist > I.dist_tol)
            continue;
        const float heading = I.heading[pos];
        if (fabsf(heading - I.goal_heading) > I.heading_tol)
            continue;
        unsigned long long pr = 0;
        if (!feasible_scalar(f, x, z, heading, pr))
            continue;
        // __compute_cost_findBestNode (graph_best_node.cu:16-18)
        const long long cost = __float2ll_rd(1 * dist + 3 * kToDeg * heading + 1 * I.cost[pos]);
        const long long key = cost * 4294967296LL + (long long)(0xffffffffu - (unsigned)pos);
        atomicMin(&keys[k], key);
    }
}

// parent walk from the best node (fastrrt.cpp:214-231), one thread per slot
__global__ void k_walk(const Inst *insts, const int *slots, int n, const long long *keys,
                       float *paths, int *path_n, int cap)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const Inst &I = insts[slots[k]];
    float *out = paths + (long)k * cap * 3;
    path_n[k] = 0;
    const long long key = keys[k];
    if (key == LLONG_MAX)
        return;
    const unsigned inv = (unsigned)(key & 0xffffffffLL);
    int pos = (int)(0xffffffffu - inv);
    int bx = pos % I.W, bz = pos / I.W;
    int m = 0;
    long i = 0;
    while (bx != -1 && bz != -1) {
        if (m < cap) {
            out[3 * m] = (float)bx;
            out[3 * m + 1] = (float)bz;
            out[3 * m + 2] = I.heading[(long)bz * I.W + bx];
        }
        m++;
        // CudaGraph::getParent (graph.cu:446-453)
        int nx = -1, nz = -1;
        if (bx >= 0 && bx < I.W && bz >= 0 && bz < I.H && I.type[(long)bz * I.W + bx] != T_NULL) {
            const int32_t p = I.parent[(long)bz * I.W + bx];
            nx = unpack_x(p);
            nz = unpack_z(p);
        }
        bx = nx;
        bz = nz;
        if (i++ >= 1000000) {
            m = 0;
            break;
        }
    }
    if (m > cap)
        m = cap;
    for (int a = 0, b = m - 1; a < b; a++, b--)
        for (int q = 0; q < 3; q++) {
            const float t = out[3 * a + q];
            out[3 * a + q] = out[3 * b + q];
            out[3 * b + q] = t;
        }
    path_n[k] = m;
}

__global__ void k_fill_keys(long long *keys, int n)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n)
        keys[k] = LLONG_MAX;
}

void launch_extract_paths(const Inst *d_inst, State *d_state, const int *d_slots, int n,
                          int max_cells, float *d_paths, int *d_path_n, long long *d_keys, int cap,
                          cudaStream_t st)
{
    (void)d_state;
    if (n <= 0)
        return;
    k_fill_keys<<<(n + 255) / 256, 256, 0, st>>>(d_keys, n);
    (void)max_cells;
    k_best_node<<<dim3(1, n), 256, 0, st>>>(d_inst, d_slots, d_keys);
    k_walk<<<(n + 63) / 64, 64, 0, st>>>(d_inst, d_slots, n, d_keys, d_paths, d_path_n, cap);
}

// optimizePathLoop (graph_optimization.cu:25-56, 92-195): every pair (i, j),
// j >= i + 2, of path waypoints is tested with checkDirectConnectionToGoal,
// one pair per warp at a time (curve_warp)
__global__ void k_opt_pairs(const Inst *insts, int slot, const float *path, const int *path_n,
                            float *newcost)
{
    const Inst &I = insts[slot];
    const int n = *path_n;
    const long pairs = (long)n * n;
    const Foot f = foot_of(I, I.blocked, I.clear);
    const int lane = threadIdx.x & 31;
    const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long warps = ((long)gridDim.x * blockDim.x) >> 5;
    unsigned long long probes = 0;
    for (long p = warp; p < pairs; p += warps) {
        const int i = (int)(p / n), j = (int)(p - (long)i * n);
        float r = -1.0f;
        if (j >= i + 2 && i < n - 2) {
            const int x = (int)path[3 * i], z = (int)path[3 * i + 1];
            r = curve_warp(I, f, I.max_curvature, x, z, path[3 * i + 2], (int)path[3 * j],
                           (int)path[3 * j + 1], path[3 * j + 2], 1, I.cost[(long)z * I.W + x], 0, lane,
                           probes);
        }
        if (lane == 0)
            newcost[p] = r;
    }
}

__global__ void k_opt_select(const Inst *insts, int slot, float *path, int *path_n,
                             float *newcost, int *changed, int cap)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    const Inst &I = insts[slot];
    int n = *path_n;
    *changed = 0;
    // path[].w = getCost of each waypoint (convertPlannedPath, graph_optimization.cu:76-90)
    float maxGain = -1;
    int mg = -1, mg_j = -1;
    float mg_cost = 0;
    for (int i = 0; i < n - 2; i++) {
        int sel = -1;
        float sel_cost = 0, sel_gain = 0;
        for (int j = i + 2; j < n; j++) {
            const int xj = (int)path[3 * j], zj = (int)path[3 * j + 1];
            const float cur = (xj >= 0 && xj < I.W && zj >= 0 && zj < I.H) ? I.cost[(long)zj * I.W + xj] : -1.0f;
            const float nc = newcost[(long)i * n + j];
            if (nc > 0 && nc < cur) {
                sel = j;
                sel_cost = nc;
                sel_gain = cur - nc;
            }
        }
        if (sel >= 0 && maxGain < sel_gain) {
            maxGain = sel_gain;
            mg = i;
            mg_j = sel;
            mg_cost = sel_cost;
        }
    }
    if (mg < 0)
        return;
    const int next_pos = mg_j;
    // the waypoint costs (path[].w) travel in newcost[0, n) from here on,
    // because the grid is cleared before the path is added back
    for (int j = 0; j < n; j++) {
        const int xj = (int)path[3 * j], zj = (int)path[3 * j + 1];
        newcost[j] = (xj >= 0 && xj < I.W && zj >= 0 && zj < I.H) ? I.cost[(long)zj * I.W + xj] : -1.0f;
    }
    if (next_pos > mg + 1) {
        newcost[next_pos] = mg_cost;
        const int rm = next_pos - mg - 1;
        for (int i = mg + 1; i + rm < n; ++i) {
            path[3 * i] = path[3 * (i + rm)];
            path[3 * i + 1] = path[3 * (i + rm) + 1];
            path[3 * i + 2] = path[3 * (i + rm) + 2];
            newcost[i] = newcost[i + rm];
        }
        n -= rm;
    }
    *path_n = n;
    *changed = 1;
    (void)cap;
}

__global__ void k_opt_rebuild(const Inst *insts, int slot, const float *path, const int *path_n,
                              const float *costs, const int *changed)
{
    if (threadIdx.x != 0 || blockIdx.x != 0 || !*changed)
        return;
    const Inst &I = insts[slot];
    const int n = *path_n;
    int ppx = (int)path[0], ppz = (int)path[1];
    grid_add(I, ppx, ppz, path[2], -1, -1, costs[0]);
    for (int i = 1; i < n; i++) {
        const int x = (int)path[3 * i], z = (int)path[3 * i + 1];
        grid_add(I, x, z, path[3 * i + 2], ppx, ppz, costs[i]);
        ppx = x;
        ppz = z;
    }
}

__global__ void k_clear_types_if(const Inst *insts, int slot, const int *changed)
{
    if (!*changed)
        return;
    const Inst &I = insts[slot];
    const long cells = (long)I.W * I.H;
    for (long base = ((long)blockIdx.x * blockDim.x + threadIdx.x) * 16; base < cells;
         base += (long)gridDim.x * blockDim.x * 16)
        *reinterpret_cast<int4 *>(I.type + base) = make_int4(0, 0, 0, 0);
}

void launch_optimize(const Inst *d_inst, int slot, int cells, float *d_path, int *d_path_n,
                     float *d_newcost, int *d_changed, int cap, const Launch &L, cudaStream_t st)
{
    const long pairs = (long)cap * cap;
    int grid = (int)((pairs + 7) / 8);  // one pair per warp
    if (grid > L.sms * 8)
        grid = L.sms * 8;
    k_opt_pairs<<<grid, 256, 0, st>>>(d_inst, slot, d_path, d_path_n, d_newcost);
    k_opt_select<<<1, 32, 0, st>>>(d_inst, slot, d_path, d_path_n, d_newcost, d_changed, cap);
    k_clear_types_if<<<(cells / 16 + 255) / 256, 256, 0, st>>>(d_inst, slot, d_changed);
    k_opt_rebuild<<<1, 32, 0, st>>>(d_inst, slot, d_path, d_path_n, d_newcost, d_changed);
}

// count of one node type (type < 0: all non-NULL) per listed slot
__global__ void k_count(const Inst *insts, const int *slots, int type, unsigned *out)
{
    const Inst &I = insts[slots[blockIdx.y]];
    const long cells = (long)I.W * I.H;
    int c = 0;
    for (long pos = blockIdx.x * (long)blockDim.x + threadIdx.x; pos < cells;
         pos += (long)gridDim.x * blockDim.x) {
        const int8_t t = I.type[pos];
        c += type < 0 ? t != T_NULL : t == type;
    }
    c = warp_sum(c);
    if ((threadIdx.x & 31) == 0 && c)
        atomicAdd(&out[blockIdx.y], (unsigned)c);
}

void launch_count(const Inst *d_inst, const int *d_slots, int n, int max_cells, int type,
                  unsigned *d_out, cudaStream_t st)
{
    if (n <= 0)
        return;
    cudaMemsetAsync(d_out, 0, sizeof(unsigned) * n, st);
    k_count<<<dim3((max_cells + 255) / 256, n), 256, 0, st>>>(d_inst, d_slots, type, d_out);
}

// checkGraphIsConsistent (graph_check_dag_consistency.cpp:33-76) in parallel:
// every non-NULL cell walks at most count(NODE) + 4 parents
__global__ void k_dag(const Inst *insts, const int *slots, const unsigned *node_counts, int *valid)
{
    const int k = blockIdx.y;
    const Inst &I = insts[slots[k]];
    const long cells = (long)I.W * I.H;
    const int maxLoop = (int)node_counts[k] + 4;
    for (long pos = blockIdx.x * (long)blockDim.x + threadIdx.x; pos < cells;
         pos += (long)gridDim.x * blockDim.x) {
        if (I.type[pos] == T_NULL)
            continue;
        int cx = (int)(pos % I.W), cz = (int)(pos / I.W);
        int i = maxLoop;
        bool bad = false;
        while (i-- > 0) {
            int px = -1, pz = -1;
            if (I.type[(long)cz * I.W + cx] != T_NULL) {
                const int32_t p = I.parent[(long)cz * I.W + cx];
                px = unpack_x(p);
                pz = unpack_z(p);
            }
            if (px == cx && pz == cz) {
                bad = true;
                break;
            }
            if (px == -1)
                break;
            const bool in = px >= 0 && px < I.W && pz >= 0 && pz < I.H;
            const int pt = in ? I.type[(long)pz * I.W + px] : -1;
            if (pt != T_NODE && pt != T_COLLISION && pt != T_CONNECT_TO_GOAL) {
                bad = true;
                break;
            }
            cx = px;
            cz = pz;
        }
        // the reference reports an inconsistency whenever the counter ends <= 0
        if (bad || i <= 0)
            valid[k] = 0;
    }
}

__device__ __forceinline__ float wrap_pi(float a)
{
    const float tp = (float)(2 * kPi);
    while (a > (float)kPi)
        a -= tp;
    while (a < -(float)kPi)
        a += tp;
    return a;
}

// The validator on one path per warp: lane k checks waypoints k, k + 32, ...
// (cell in the frame, parent link, no repeated cell, heading change within
// the curvature bound, footprint feasible outside the ego box); footprints
// the quick tests cannot clear are probed by the whole warp.
__global__ void __launch_bounds__(128) k_path_check(const Inst *insts, const int *slots, int n,
                                                    const float *paths, const int *path_n, int cap,
                                                    int *valid, float *length)
{
    const int k = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (k >= n)
        return;  // uniform across the warp
    const Inst &I = insts[slots[k]];
    const float *p = paths + (long)k * cap * 3;
    const int m = path_n[k];
    if (m < 2 || (int)p[0] != I.start_x || (int)p[1] != I.start_z) {
        if (lane == 0) {
            valid[k] = 0;
            length[k] = 0.0f;
        }
        return;
    }
    const Foot f = foot_of(I, I.blocked, I.clear);
    const double steer = tan(I.max_steer), beta = atan(steer / 2);
    double kappa = cos(beta) * steer / (2 * I.lr);
    if (I.max_curvature > kappa)
        kappa = I.max_curvature;
    if (0.8 > kappa)
        kappa = 0.8;
    float len = 0.0f;
    bool bad = false;
    for (int i0 = 0; i0 < m; i0 += 32) {
        const int i = i0 + lane;
        bool need = false;
        int x = 0, z = 0;
        float h = 0.0f;
        if (i < m) {
            x = (int)p[3 * i];
            z = (int)p[3 * i + 1];
            h = p[3 * i + 2];
            if (x < 0 || x >= I.W || z < 0 || z >= I.H) {
                bad = true;
            } else {
                const bool in_ego = x >= I.lbx && x <= I.ubx && z >= I.ubz && z <= I.lbz;
                unsigned long long pr = 0;
                if (!in_ego && !quick_feasible(f, x, z, pr)) {
                    float sn, cs;
                    sincosf(h, &sn, &cs);
                    need = !box_feasible(f, x, z, fabsf(cs), fabsf(sn), pr);
                }
                if (i > 0) {
                    const int px = (int)p[3 * (i - 1)], pz = (int)p[3 * (i - 1) + 1];
                    const int32_t par = I.parent[(long)z * I.W + x];
                    const double chord =
                        sqrt((double)(x - px) * (x - px) + (double)(z - pz) * (z - pz));
                    const float dh = wrap_pi(h - p[3 * (i - 1) + 2]);
                    if ((px == x && pz == z) || I.type[(long)z * I.W + x] == T_NULL ||
                        unpack_x(par) != px || unpack_z(par) != pz ||
                        fabs(dh) > (kPi / 2) * kappa * chord + 1e-3)
                        bad = true;
                    len += sqrtf((float)((x - px) * (x - px) + (z - pz) * (z - pz)));
                }
            }
        }
        unsigned mm = __ballot_sync(kFull, need);
        while (mm) {
            const int leader = __ffs(mm) - 1;
            mm &= mm - 1;
            unsigned cnt = 0;
            const bool ok = coop_probe(f, leader, lane, x, z, h, cnt);
            if (lane == leader && !ok)
                bad = true;
        }
    }
    bad = __any_sync(kFull, bad);
    for (int o = 16; o; o >>= 1)
        len += __shfl_xor_sync(kFull, len, o);
    if (lane != 0)
        return;
    if (!bad) {
        const int lx = (int)p[3 * (m - 1)], lz = (int)p[3 * (m - 1) + 1];
        const double gdx = lx - I.goal_x, gdz = lz - I.goal_z;
        if (sqrt(gdx * gdx + gdz * gdz) > I.dist_tol)
            bad = true;
        if (fabsf(p[3 * (m - 1) + 2] - I.goal_heading) > I.heading_tol)
            bad = true;
    }
    if (bad)
        valid[k] = 0;
    length[k] = len;
}

// ---------------------------------------------------------------------------
// interpolation of extracted paths and curve quality, one warp per path
// ---------------------------------------------------------------------------

// interpolate (interpolation.cpp:112-135) of the listed paths: for every pair
// of consecutive waypoints, interpolateHermiteCurve (interpolation.cpp:36-110)
// with the reference's float arithmetic, each product and sum rounded on its
// own (the reference is host code: no fused multiply-adds), samples across
// the lanes; a sample keeps its rounded cell when it lies in the frame and
// the cell differs from the last kept one (a ballot over the chunk, the last
// kept cell carried).  Then the curve-quality metrics of the interpolated
// curve (tests/python_dataset/curve_quality.py:92-99, 179-294, in double as
// the reference's Python): length, jerk of the windowed direction, and the
// tangential discontinuity against the path's start heading.
__global__ void __launch_bounds__(128) k_interp(const Inst *insts, const int *slots, int n,
                                                const float *paths, const int *path_n, int cap,
                                                float *out, int *out_n, int out_cap, double *scratch,
                                                float *length, float *jerk, int *tan_disc)
{
    const int k = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (k >= n)
        return;  // uniform across the warp
    const Inst &I = insts[slots[k]];
    const float *p = paths + (long)k * cap * 3;
    const int m = path_n[k];
    float *o = out + (long)k * out_cap * 3;
    const unsigned lower = (1u << lane) - 1u;
    int cnt = 0, last_x = -1, last_z = -1;
    bool full = false;
    for (int s = 1; s < m && !full; s++) {
        // each segment's samples are deduplicated on their own: the end cell
        // of one segment and the start cell of the next are both kept
        last_x = last_z = -1;
        const int p1x = (int)p[3 * (s - 1)], p1z = (int)p[3 * (s - 1) + 1];
        const int p2x = (int)p[3 * s], p2z = (int)p[3 * s + 1];
        const float p1h = p[3 * (s - 1) + 2], p2h = p[3 * s + 2];
        const double dxd = p2x - p1x, dzd = p2z - p1z;
        const int numPoints = (int)sqrt(dxd * dxd + dzd * dzd);
        const float dx = (float)(p2x - p1x), dz = (float)(p2z - p1z);
        const float d = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dz, dz)));
        const float a1 = (float)(p1h - kPi / 2), a2 = (float)(p2h - kPi / 2);
        // the host's float trigonometry, rounded from double (the correctly
        // rounded float value but in rare halfway cases)
        const float t1x = __fmul_rn(d, (float)cos((double)a1)), t1y = __fmul_rn(d, (float)sin((double)a1));
        const float t2x = __fmul_rn(d, (float)cos((double)a2)), t2y = __fmul_rn(d, (float)sin((double)a2));
        const float fx1 = (float)p1x, fz1 = (float)p1z, fx2 = (float)p2x, fz2 = (float)p2z;
        // x = h00 p1 + h10 tan1 + h01 p2 + h11 tan2, summed left to right
        auto mix = [](float a, float b, float c, float d4, float u, float v, float w, float q) {
            return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(a, u), __fmul_rn(b, v)), __fmul_rn(c, w)),
                             __fmul_rn(d4, q));
        };
        for (int base = 0; base < numPoints && !full; base += 32) {
            const int i = base + lane;
            const float t = __fdiv_rn((float)i, (float)(numPoints - 1));
            const float t2 = __fmul_rn(t, t), t3 = __fmul_rn(t2, t);
            const float h00 = __fadd_rn(__fsub_rn(__fmul_rn(2.0f, t3), __fmul_rn(3.0f, t2)), 1.0f);
            const float h10 = __fadd_rn(__fsub_rn(t3, __fmul_rn(2.0f, t2)), t);
            const float h01 = __fadd_rn(__fmul_rn(-2.0f, t3), __fmul_rn(3.0f, t2));
            const float h11 = __fsub_rn(t3, t2);
            const float x = mix(h00, h10, h01, h11, fx1, t1x, fx2, t2x);
            const float z = mix(h00, h10, h01, h11, fz1, t1y, fz2, t2y);
            int cx = 0, cz = 0;
            bool valid = false;
            if (i < numPoints && !(x < 0 || x >= I.W) && !(z < 0 || z >= I.H)) {
                cx = (int)roundf(x);
                cz = (int)roundf(z);
                valid = cx >= 0 && cx < I.W && cz >= 0 && cz < I.H;
            }
            const unsigned vm = __ballot_sync(kFull, valid);
            const unsigned below = vm & lower;
            const int src = below ? 31 - __clz(below) : lane;
            const int qx = __shfl_sync(kFull, cx, src), qz = __shfl_sync(kFull, cz, src);
            const bool keep = valid && !(cx == (below ? qx : last_x) && cz == (below ? qz : last_z));
            const unsigned km = __ballot_sync(kFull, keep);
            if (keep) {
                const float t00 = __fsub_rn(__fmul_rn(6.0f, t2), __fmul_rn(6.0f, t));
                const float t10 = __fadd_rn(__fsub_rn(__fmul_rn(3.0f, t2), __fmul_rn(4.0f, t)), 1.0f);
                const float t01 = __fadd_rn(__fmul_rn(-6.0f, t2), __fmul_rn(6.0f, t));
                const float t11 = __fsub_rn(__fmul_rn(3.0f, t2), __fmul_rn(2.0f, t));
                const float ddx = mix(t00, t10, t01, t11, fx1, t1x, fx2, t2x);
                const float ddz = mix(t00, t10, t01, t11, fz1, t1y, fz2, t2y);
                const float heading = (float)((double)(float)atan2((double)ddz, (double)ddx) + kPi / 2);
                const int at = cnt + __popc(km & lower);
                if (at < out_cap) {
                    o[3 * at] = (float)cx;
                    o[3 * at + 1] = (float)cz;
                    o[3 * at + 2] = heading;
                }
            }
            if (vm) {
                const int hi = 31 - __clz(vm);
                last_x = __shfl_sync(kFull, cx, hi);
                last_z = __shfl_sync(kFull, cz, hi);
            }
            cnt += __popc(km);
            full = cnt >= out_cap;
        }
    }
    cnt = min(cnt, out_cap);
    __syncwarp();
    // curve quality of the cnt interpolated cells
    double len = 0.0;
    for (int i = 1 + lane; i < cnt; i += 32) {
        const double ex = o[3 * i] - o[3 * (i - 1)], ez = o[3 * i + 1] - o[3 * (i - 1) + 1];
        len += sqrt(ex * ex + ez * ez);
    }
    for (int q = 16; q; q >>= 1)
        len += __shfl_xor_sync(kFull, len, q);
    // the window of point `pos` (curve_quality.py:191-201), positions below
    // zero wrap to the curve's end as Python's do; below -cnt they fail
    auto window = [cnt](int pos, int &i0, int &j0) {
        int i = pos - 4, j = pos + 4;
        if (i < 0) {
            j -= i;
            i = 0;
        }
        if (j >= cnt) {
            i = i - (j - cnt) - 1;
            j = cnt - 1;
        }
        i0 = i;
        j0 = j;
    };
    double *v = scratch + (long)k * out_cap * 2, *g = v + out_cap;
    bool ok = cnt >= 3, disc = false;
    const double thr = 15.0 * kPi / 180.0;
    const float sh = m > 0 ? p[2] : 0.0f;
    for (int i = lane; i < cnt && ok; i += 32) {
        int i0, j0;
        window(i, i0, j0);
        if (i0 < -cnt) {
            ok = false;
            break;
        }
        const double px = o[3 * i], pz = o[3 * i + 1];
        double dv = 0.0, mh = 0.0;
        int c = 0;
        for (int q = i0; q <= j0; q++) {
            if (q == i)
                continue;
            const int r = q < 0 ? q + cnt : q;
            const double rx = o[3 * r], rz = o[3 * r + 1];
            // direction (curve_quality.py:243-246), from the earlier point
            const double ax = q < i ? px - rx : rx - px, az = q < i ? pz - rz : rz - pz;
            dv += atan2(az, ax);
            // heading (curve_quality.py:179-189): 0 for a repeated point
            double hd = 0.0;
            if (!(ax == 0.0 && az == 0.0)) {
                hd = kPi / 2 - atan2(-az, ax);
                if (hd > kPi)
                    hd -= 2 * kPi;
            }
            mh += hd;
            c++;
        }
        v[i] = c ? dv / c : 0.0;
        g[i] = c ? mh / c : 0.0;
    }
    ok = __all_sync(kFull, ok);
    __syncwarp();
    // tangential discontinuity (curve_quality.py:227-241): any step of the
    // windowed heading above 15 degrees, from the start heading on
    for (int i = 1 + lane; i < cnt && ok; i += 32) {
        const double before = i == 1 ? (double)sh : g[i - 1];
        if (fabs(g[i] - before) > thr)
            disc = true;
    }
    disc = __any_sync(kFull, disc);
    __syncwarp();
    // jerk (curve_quality.py:290-294): np.gradient twice (one-sided at the
    // ends), then the sum of magnitudes
    auto grad = [cnt](const double *f, int i) {
        if (i == 0)
            return f[1] - f[0];
        if (i == cnt - 1)
            return f[cnt - 1] - f[cnt - 2];
        return (f[i + 1] - f[i - 1]) / 2.0;
    };
    for (int i = lane; i < cnt && ok; i += 32)
        g[i] = grad(v, i);
    __syncwarp();
    double js = 0.0;
    for (int i = lane; i < cnt && ok; i += 32)
        js += fabs(grad(g, i));
    for (int q = 16; q; q >>= 1)
        js += __shfl_xor_sync(kFull, js, q);
    if (lane == 0) {
        out_n[k] = cnt;
        length[k] = (float)len;
        jerk[k] = ok ? (float)fabs(js) : __int_as_float(0x7fc00000);
        tan_disc[k] = ok ? (disc ? 1 : 0) : -1;
    }
}

void launch_interpolate(const Inst *d_inst, const int *d_slots, int n, const float *d_paths,
                        const int *d_path_n, int cap, float *d_out, int *d_out_n, int out_cap,
                        double *d_scratch, float *d_length, float *d_jerk, int *d_disc, cudaStream_t st)
{
    if (n <= 0)
        return;
    k_interp<<<(n * 32 + 127) / 128, 128, 0, st>>>(d_inst, d_slots, n, d_paths, d_path_n, cap, d_out,
                                                   d_out_n, out_cap, d_scratch, d_length, d_jerk, d_disc);
}

// Training rows of valid paths: one per expansion on the path (waypoints 1 ..
// m - 3; the last two are the goal connection and the goal): the parent cell,
// its slot, and the bin of the draw that made the child.  One warp per path.
__global__ void __launch_bounds__(128) k_log_list(const Inst *insts, const State *states,
                                                  const int *slots, int n, const float *paths,
                                                  const int *path_n, const int *valid, int cap,
                                                  int32_t *cells, int32_t *slot_of, int32_t *labels,
                                                  int *count, int cap_rows)
{
    const int k = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (k >= n)
        return;
    const int slot = slots[k];
    const Inst &I = insts[slot];
    if (!valid[k] || !states[slot].goal_reached)
        return;
    const float *p = paths + (long)k * cap * 3;
    const int m = path_n[k];
    for (int i = 1 + lane; i <= m - 3; i += 32) {
        const int cx = (int)p[3 * i], cz = (int)p[3 * i + 1];
        const int px = (int)p[3 * (i - 1)], pz = (int)p[3 * (i - 1) + 1];
        const int child = cz * I.W + cx;
        const int row = atomicAdd(count, 1);
        if (row >= cap_rows)
            continue;
        cells[row] = pz * I.W + px;
        slot_of[row] = slot;
        labels[row] = proposal_bin(I.exp_steer[child], I.exp_len[child], (float)I.max_steer, I.max_path);
    }
}

// Training rows of every accepted expansion of the solved slots: each NODE
// cell but the start, with its parent cell, its slot, and the bin of the draw
// that made it.  blockIdx.y = list entry; the blocks of an entry stride over
// its cells; rows appended warp by warp (their order is not deterministic).
__global__ void __launch_bounds__(256) k_log_nodes(const Inst *insts, const State *states, const int *slots,
                                                   const int *valid, int32_t *cells, int32_t *slot_of,
                                                   int32_t *labels, int *count, int cap_rows)
{
    const int k = blockIdx.y;
    const int slot = slots[k];
    if (!valid[k] || !states[slot].goal_reached)
        return;  // uniform across the block
    const Inst &I = insts[slot];
    const int lane = threadIdx.x & 31;
    const int n_cells = I.W * I.H, start = I.start_z * I.W + I.start_x;
    for (int base = blockIdx.x * blockDim.x; base < n_cells; base += gridDim.x * blockDim.x) {
        const int c = base + threadIdx.x;
        const bool is = c < n_cells && c != start && I.type[c] == T_NODE;
        const unsigned m = __ballot_sync(kFull, is);
        if (!m)
            continue;
        int b0 = 0;
        if (lane == 0)
            b0 = atomicAdd(count, __popc(m));
        b0 = __shfl_sync(kFull, b0, 0);
        if (!is)
            continue;
        const int row = b0 + __popc(m & ((1u << lane) - 1u));
        if (row >= cap_rows)
            continue;
        const int32_t par = I.parent[c];
        cells[row] = unpack_z(par) * I.W + unpack_x(par);
        slot_of[row] = slot;
        labels[row] = proposal_bin(I.exp_steer[c], I.exp_len[c], (float)I.max_steer, I.max_path);
    }
}

void launch_log_nodes(const Inst *d_inst, const State *d_state, const int *d_slots, int n, const int *d_valid,
                      int32_t *cells, int32_t *slot_of, int32_t *labels, int *count, int cap_rows,
                      cudaStream_t st)
{
    if (n <= 0)
        return;
    k_log_nodes<<<dim3(16, n), 256, 0, st>>>(d_inst, d_state, d_slots, d_valid, cells, slot_of, labels, count,
                                             cap_rows);
}

void launch_log_paths(const Inst *d_inst, const State *d_state, const int *d_slots, int n,
                      const float *d_paths, const int *d_path_n, const int *d_valid, int cap,
                      int32_t *cells, int32_t *slot_of, int32_t *labels, int *count, int cap_rows,
                      cudaStream_t st)
{
    if (n <= 0)
        return;
    k_log_list<<<(n * 32 + 127) / 128, 128, 0, st>>>(d_inst, d_state, d_slots, n, d_paths, d_path_n,
                                                      d_valid, cap, cells, slot_of, labels, count,
                                                      cap_rows);
}

__global__ void k_fill_int(int *v, int n, int value)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n)
        v[k] = value;
}

void launch_validate(const Inst *d_inst, State *d_state, const int *d_slots, int n, int max_cells,
                     const float *d_paths, const int *d_path_n, int cap, unsigned *d_counts,
                     int *d_valid, float *d_length, cudaStream_t st)
{
    (void)d_state;
    if (n <= 0)
        return;
    k_fill_int<<<(n + 255) / 256, 256, 0, st>>>(d_valid, n, 1);
    launch_count(d_inst, d_slots, n, max_cells, T_NODE, d_counts, st);
    k_dag<<<dim3((max_cells + 255) / 256, n), 256, 0, st>>>(d_inst, d_slots, d_counts, d_valid);
    k_path_check<<<(n * 32 + 127) / 128, 128, 0, st>>>(d_inst, d_slots, n, d_paths, d_path_n, cap,
                                                       d_valid, d_length);
}

void launch_check_graphs(const Inst *d_inst, const int *d_slots, int n, int max_cells, unsigned *d_counts,
                         int *d_valid, cudaStream_t st)
{
    if (n <= 0)
        return;
    k_fill_int<<<(n + 255) / 256, 256, 0, st>>>(d_valid, n, 1);
    launch_count(d_inst, d_slots, n, max_cells, T_NODE, d_counts, st);
    k_dag<<<dim3((max_cells + 255) / 256, n), 256, 0, st>>>(d_inst, d_slots, d_counts, d_valid);
}

void launch_check_paths(const Inst *d_inst, const int *d_slots, int n, const float *d_paths,
                        const int *d_path_n, int cap, int *d_valid, float *d_length, cudaStream_t st)
{
    if (n <= 0)
        return;
    k_fill_int<<<(n + 255) / 256, 256, 0, st>>>(d_valid, n, 1);
    k_path_check<<<(n * 32 + 127) / 128, 128, 0, st>>>(d_inst, d_slots, n, d_paths, d_path_n, cap,
                                                       d_valid, d_length);
}

// ---------------------------------------------------------------------------
// per-candidate microbenchmarks (one frame slot)
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_candidates(const Inst *insts, int slot, int n,
                                                    const int32_t *sx, const int32_t *sz,
                                                    const float *steer, const float *len,
                                                    float velocity, float4 *out,
                                                    unsigned long long *probes_out, int smem_words,
                                                    int *bad_cell)
{
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ __align__(8) uint64_t bar;
    const Inst &I = insts[slot];
    const uint32_t *blk = I.blocked, *clr = I.clear;
    unsigned phase = 0;
    if (smem_words > 0 && I.mask_words <= smem_words) {
        if (threadIdx.x == 0)
            mbar_init(&bar, 1);
        __syncthreads();
        if (stage_masks(smem, smem + smem_words, I.blocked, I.clear, I.mask_words, &bar, phase,
                        g_stage_wait_limit)) {
            blk = smem;
            clr = smem + smem_words;
        } else {
            // the copy did not land in time: count it, let it finish (its
            // shared memory must outlive it) and read the global masks
            if (threadIdx.x == 0)
                atomicAdd(&g_stage_timeouts, 1ull);
            for (long k = 0; k < kWaitLimit; k++)
                if (mbar_try_wait(&bar, phase ^ 1u))
                    break;
            __syncthreads();
        }
    }
    const Foot f = foot_of(I, blk, clr);
    const int lane = threadIdx.x & 31;
    const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long warps = ((long)gridDim.x * blockDim.x) >> 5;
    unsigned long long probes = 0;
    // one candidate per warp at a time (kin_warp)
    for (long i = warp; i < n; i += warps) {
        // a start cell outside the frame is rejected (and reported) without
        // reading the grids at it
        const int cx = sx[i], cz = sz[i];
        if (!(cx >= 0 && cx < I.W && cz >= 0 && cz < I.H)) {
            if (lane == 0) {
                out[i] = make_float4(-1.0f, -1.0f, 0.0f, 0.0f);
                if (bad_cell)
                    atomicOr(bad_cell, 1);
            }
            continue;
        }
        const long pos = (long)cz * I.W + cx;
        const KinResult r = kin_warp(I, f, cx, cz, steer[i], len[i], velocity, I.heading[pos], I.cost[pos],
                                     lane, probes);
        if (lane == 0)
            out[i] = r.ok ? make_float4((float)r.last_x, (float)r.last_z, r.cost, r.heading)
                          : make_float4(-1.0f, -1.0f, 0.0f, 0.0f);
    }
    probes = warp_sum64(probes);
    if (lane == 0 && probes && probes_out)
        atomicAdd(probes_out, probes);
}

void launch_candidates(const Inst *d_inst, int slot, int n, const int32_t *sx, const int32_t *sz,
                       const float *steer, const float *len, float velocity, float4 *out,
                       unsigned long long *probes, const Launch &L, cudaStream_t st, int *bad_cell)
{
    if (n <= 0)
        return;
    // one candidate per warp: 8 per block
    int grid = (n + 7) / 8;
    if (grid > L.sms * 8)
        grid = L.sms * 8;
    const size_t smem = (size_t)L.smem_words * 2 * 4;
    k_candidates<<<grid, 256, smem, st>>>(d_inst, slot, n, sx, sz, steer, len, velocity, out, probes,
                                          L.smem_words, bad_cell);
}

// One pose pair per warp at a time (curve_warp, samples across the lanes, no
// coarse pass: the probe count is the reference's exact count).
__global__ void __launch_bounds__(256) k_hermite(const Inst *insts, int slot, int n, const int32_t *x,
                                                 const int32_t *z, const float *lh, const int32_t *gx,
                                                 const int32_t *gz, const float *gh, float maxc,
                                                 int safe, float *out, unsigned long long *probes_out,
                                                 int smem_words)
{
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ __align__(8) uint64_t bar;
    const Inst &I = insts[slot];
    const uint32_t *blk = I.blocked, *clr = I.clear;
    unsigned phase = 0;
    if (smem_words > 0 && I.mask_words <= smem_words) {
        if (threadIdx.x == 0)
            mbar_init(&bar, 1);
        __syncthreads();
        if (stage_masks(smem, smem + smem_words, I.blocked, I.clear, I.mask_words, &bar, phase,
                        g_stage_wait_limit)) {
            blk = smem;
            clr = smem + smem_words;
        } else {
            // the copy did not land in time: count it, let it finish (its
            // shared memory must outlive it) and read the global masks
            if (threadIdx.x == 0)
                atomicAdd(&g_stage_timeouts, 1ull);
            for (long k = 0; k < kWaitLimit; k++)
                if (mbar_try_wait(&bar, phase ^ 1u))
                    break;
            __syncthreads();
        }
    }
    const Foot f = foot_of(I, blk, clr);
    const int lane = threadIdx.x & 31;
    const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long warps = ((long)gridDim.x * blockDim.x) >> 5;
    unsigned long long probes = 0;
    for (long i = warp; i < n; i += warps) {
        // a start cell outside the frame is not connected (its cost and
        // traversability are not read)
        const int cx = x[i], cz = z[i];
        float r = -1.0f;
        if (cx >= 0 && cx < I.W && cz >= 0 && cz < I.H)
            r = curve_warp(I, f, maxc, cx, cz, lh[i], gx[i], gz[i], gh[i], safe & 1,
                           I.cost[(long)cz * I.W + cx], 0, lane, probes,
                           (safe & 2) ? I.frame_dist : nullptr);
        if (lane == 0)
            out[i] = r;
    }
    probes = warp_sum64(probes);
    if (lane == 0 && probes && probes_out)
        atomicAdd(probes_out, probes);
}

void launch_hermite_pairs(const Inst *d_inst, int slot, int n, const int32_t *x, const int32_t *z,
                          const float *lh, const int32_t *gx, const int32_t *gz, const float *gh,
                          float max_curvature, int safe, float *out, unsigned long long *probes,
                          const Launch &L, cudaStream_t st)
{
    if (n <= 0)
        return;
    // one pair per warp: 8 per block
    int grid = (n + 7) / 8;
    if (grid > L.sms * 8)
        grid = L.sms * 8;
    const size_t smem = (size_t)L.smem_words * 2 * 4;
    k_hermite<<<grid, 256, smem, st>>>(d_inst, slot, n, x, z, lh, gx, gz, gh, max_curvature, safe, out,
                                       probes, L.smem_words);
}

__global__ void k_feasible(const Inst *insts, int slot, int n, const int32_t *x, const int32_t *z,
                           const float *a, int32_t *out, unsigned long long *probes_out)
{
    const Inst &I = insts[slot];
    const Foot f = foot_of(I, I.blocked, I.clear);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long pr = 0;
    // a cell outside the frame is reported infeasible without reading it
    if (i < n)
        out[i] = (x[i] >= 0 && x[i] < I.W && z[i] >= 0 && z[i] < I.H && feasible_scalar(f, x[i], z[i], a[i], pr))
                     ? 1
                     : 0;
    pr = warp_sum64(pr);
    if ((threadIdx.x & 31) == 0 && pr && probes_out)
        atomicAdd(probes_out, pr);
}

// ---------------------------------------------------------------------------
// SearchFrame preprocessing
// ---------------------------------------------------------------------------

// distance channel: the distance of every cell to the goal as
// checkDirectConnectionToGoal computes it (graph_direct_goal_connection.cu:33-35)
__global__ void k_frame_distance(int W, int H, int gx, int gz, float *dist)
{
    const long n = (long)W * H;
    for (long pos = blockIdx.x * (long)blockDim.x + threadIdx.x; pos < n; pos += (long)gridDim.x * blockDim.x) {
        const int z = (int)(pos / W), x = (int)(pos - (long)z * W);
        const int dx = gx - x, dz = gz - z;
        dist[pos] = sqrtf(dx * dx + dz * dz);
    }
}

void launch_frame_distance(int W, int H, int gx, int gz, float *dist, cudaStream_t st)
{
    const long n = (long)W * H;
    k_frame_distance<<<(int)std::min<long>((n + 255) / 256, 148 * 16), 256, 0, st>>>(W, H, gx, gz, dist);
}

// safe zone, pass 1: per cell, an obstacle (class cost < 0) within rc cells
// of it in its row
__global__ void k_frame_rows(int W, int H, const uint8_t *cls, const float *costs, int ncls, int rc,
                             uint8_t *rows)
{
    const long n = (long)W * H;
    for (long pos = blockIdx.x * (long)blockDim.x + threadIdx.x; pos < n; pos += (long)gridDim.x * blockDim.x) {
        const int z = (int)(pos / W), x = (int)(pos - (long)z * W);
        uint8_t hit = 0;
        for (int xx = max(0, x - rc); xx <= min(W - 1, x + rc) && !hit; xx++) {
            const int c = cls[(long)z * W + xx];
            hit = (c < ncls && costs[c] < 0) ? 1 : 0;
        }
        rows[pos] = hit;
    }
}

// pass 2: no row hit within rc rows -> no obstacle within Chebyshev radius
// rc -> every footprint probe at every heading misses: bit 0x100
__global__ void k_frame_safe(int W, int H, int rc, const uint8_t *rows, int32_t *trav)
{
    const long n = (long)W * H;
    for (long pos = blockIdx.x * (long)blockDim.x + threadIdx.x; pos < n; pos += (long)gridDim.x * blockDim.x) {
        const int z = (int)(pos / W), x = (int)(pos - (long)z * W);
        bool hit = false;
        for (int zz = max(0, z - rc); zz <= min(H - 1, z + rc) && !hit; zz++)
            hit = rows[(long)zz * W + x] != 0;
        trav[pos] = hit ? (trav[pos] & ~0x100) : (trav[pos] | 0x100);
    }
}

void launch_frame_safe_zone(int W, int H, const uint8_t *cls, const float *costs, int ncls, int rc,
                            uint8_t *rows, int32_t *trav, cudaStream_t st)
{
    const long n = (long)W * H;
    const int grid = (int)std::min<long>((n + 255) / 256, 148 * 16);
    k_frame_rows<<<grid, 256, 0, st>>>(W, H, cls, costs, ncls, rc, rows);
    k_frame_safe<<<grid, 256, 0, st>>>(W, H, rc, rows, trav);
}

// ---------------------------------------------------------------------------
// artificial potential field intrinsic costs (apf.cu:23-154)
// ---------------------------------------------------------------------------

__device__ __forceinline__ bool apf_obstacle(const uint8_t *cls, const float *costs, int ncls, int W, int H,
                                             int x, int z)
{
    if (x < 0 || x >= W || z < 0 || z >= H)
        return true;  // check_is_obstacle (apf.cu:17-21): outside is an obstacle
    const int c = cls[(long)z * W + x];
    return c < ncls && costs[c] < 0;
}

__device__ __forceinline__ bool apf_ego(int x, int z, int lbx, int lbz, int ubx, int ubz)
{
    return x >= lbx && x <= ubx && z >= ubz && z <= lbz;
}

// sources of the repulsive field: obstacle cells outside the ego box with a
// free 4-neighbour (apf.cu:37-57)
__global__ void k_apf_sources(int W, int H, const uint8_t *cls, const float *costs, int ncls, int lbx, int lbz,
                              int ubx, int ubz, uint8_t *src)
{
    const long n = (long)W * H;
    for (long pos = blockIdx.x * (long)blockDim.x + threadIdx.x; pos < n; pos += (long)gridDim.x * blockDim.x) {
        const int z = (int)(pos / W), x = (int)(pos - (long)z * W);
        bool s = false;
        if (!apf_ego(x, z, lbx, lbz, ubx, ubz) && apf_obstacle(cls, costs, ncls, W, H, x, z))
            s = !(apf_obstacle(cls, costs, ncls, W, H, x - 1, z) && apf_obstacle(cls, costs, ncls, W, H, x + 1, z) &&
                  apf_obstacle(cls, costs, ncls, W, H, x, z - 1) && apf_obstacle(cls, costs, ncls, W, H, x, z + 1));
        src[pos] = s ? 1 : 0;
    }
}

// __CUDA_KERNEL_repulsive_force (apf.cu:23-91) as a gather, one cell per
// thread: an obstacle cell outside the ego box is set to 100 Kr/2 (apf.cu:49),
// then every cell outside the ego box adds Kr/2 (1/p - 1/r)^2 for each source
// within distance r (p = the distance, not the cell itself; apf.cu:59-89), one
// source after another in the sources' row-major order, each product and sum
// rounded on its own.  The reference scatters these adds with float atomics
// and its obstacle sets race with them; this order is one it can produce.
__global__ void k_apf_repulse(int W, int H, const uint8_t *cls, const float *costs, int ncls, int lbx, int lbz,
                              int ubx, int ubz, const uint8_t *src, float kr_half, int radius, float *intr)
{
    const long n = (long)W * H;
    const float p0 = (float)radius;
    for (long pos = blockIdx.x * (long)blockDim.x + threadIdx.x; pos < n; pos += (long)gridDim.x * blockDim.x) {
        const int z = (int)(pos / W), x = (int)(pos - (long)z * W);
        if (apf_ego(x, z, lbx, lbz, ubx, ubz))
            continue;
        float v = apf_obstacle(cls, costs, ncls, W, H, x, z) ? __fmul_rn(100.0f, kr_half) : intr[pos];
        for (int sz = z - radius; sz <= z + radius; sz++) {
            if (sz < 0 || sz >= H)
                continue;
            for (int sx = x - radius; sx <= x + radius; sx++) {
                if (sx < 0 || sx >= W || (sx == x && sz == z) || !src[(long)sz * W + sx])
                    continue;
                const float p = __fsqrt_rn((float)((x - sx) * (x - sx) + (z - sz) * (z - sz)));
                if (p > p0)
                    continue;
                const float f = __fsub_rn(__fdiv_rn(1.0f, p), __fdiv_rn(1.0f, p0));
                v = __fadd_rn(v, __fmul_rn(__fmul_rn(kr_half, f), f));
            }
        }
        intr[pos] = v;
    }
}

// __CUDA_KERNEL_attractive_force (apf.cu:93-121): every free cell loses
// Ka/2 times its squared distance to the goal
__global__ void k_apf_attract(int W, int H, const uint8_t *cls, const float *costs, int ncls, float ka_half,
                              int gx, int gz, float *intr)
{
    const long n = (long)W * H;
    for (long pos = blockIdx.x * (long)blockDim.x + threadIdx.x; pos < n; pos += (long)gridDim.x * blockDim.x) {
        const int z = (int)(pos / W), x = (int)(pos - (long)z * W);
        const int c = cls[pos];
        if (c < ncls && costs[c] < 0)
            continue;  // obstacle
        const int dx = gx - x, dz = gz - z;
        const float dcost = (float)(dx * dx + dz * dz) * ka_half;
        const float current_cost = intr[pos];
        intr[pos] = current_cost - dcost;
    }
}

void launch_apf_repulsion(int W, int H, const uint8_t *cls, const float *costs, int ncls, int lbx, int lbz, int ubx,
                          int ubz, float kr, int radius, uint8_t *scratch, float *intr, cudaStream_t st)
{
    const long n = (long)W * H;
    const int grid = (int)std::min<long>((n + 255) / 256, 148 * 16);
    k_apf_sources<<<grid, 256, 0, st>>>(W, H, cls, costs, ncls, lbx, lbz, ubx, ubz, scratch);
    k_apf_repulse<<<grid, 256, 0, st>>>(W, H, cls, costs, ncls, lbx, lbz, ubx, ubz, scratch, kr * 0.5f, radius, intr);
}

void launch_apf_attraction(int W, int H, const uint8_t *cls, const float *costs, int ncls, float ka, int gx, int gz,
                           float *intr, cudaStream_t st)
{
    const long n = (long)W * H;
    k_apf_attract<<<(int)std::min<long>((n + 255) / 256, 148 * 16), 256, 0, st>>>(W, H, cls, costs, ncls, ka * 0.5f,
                                                                                gx, gz, intr);
}

// the device clock that the state timestamps use (%globaltimer, ns)
__global__ void k_clock(long long *out) { *out = global_ns(); }

void launch_clock(long long *d_out, cudaStream_t st) { k_clock<<<1, 1, 0, st>>>(d_out); }

bool set_stage_wait_limit(long rounds)
{
    return cudaMemcpyToSymbol(g_stage_wait_limit, &rounds, sizeof(long)) == cudaSuccess;
}

bool take_stage_timeouts(unsigned long long &count)
{
    const unsigned long long zero = 0;
    return cudaMemcpyFromSymbol(&count, g_stage_timeouts, sizeof(count)) == cudaSuccess &&
           cudaMemcpyToSymbol(g_stage_timeouts, &zero, sizeof(zero)) == cudaSuccess;
}

void configure_kernels(int smem_bytes)
{
    cudaFuncSetAttribute(k_candidates, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
    cudaFuncSetAttribute(k_hermite, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
}

void launch_feasible(const Inst *d_inst, int slot, int n, const int32_t *x, const int32_t *z,
                     const float *a, int32_t *out, unsigned long long *probes, cudaStream_t st)
{
    if (n <= 0)
        return;
    k_feasible<<<(n + 255) / 256, 256, 0, st>>>(d_inst, slot, n, x, z, a, out, probes);
}

}  // namespace frrt
