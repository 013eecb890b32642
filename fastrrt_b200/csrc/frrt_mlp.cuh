// frrt_mlp.cuh -- the learned expansion proposal: a BF16 MLP (1030 -> 256 ->
// 256 -> 128, ReLU, FP32 accumulation) with a hand-written tcgen05 GEMM, its
// training kernels, and the planner-side feature extraction and proposal
// sampling.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "frrt_common.cuh"

namespace frrt {

constexpr int kMlpPatch = 32;                     // patch side (samples)
constexpr int kMlpPatchStride = 2;                // pixels between patch samples
constexpr int kMlpScalars = 6;                    // goal (u, v), distance, sin h, cos h, steer limit
constexpr int kMlpIn = kMlpPatch * kMlpPatch + kMlpScalars;  // 1030
constexpr int kMlpInPad = 1040;                   // K of layer 1, a multiple of 16
constexpr int kMlpHidden = 256;
constexpr int kSteerBins = 16;
constexpr int kLenBins = 8;
constexpr int kMlpOut = kSteerBins * kLenBins;    // 128
// blocks of the planner-side network kernels, whose row count is a device
// value below the row capacity (a build-time knob for measurement)
#ifndef FRRT_MLP_GRID_BLOCKS
#define FRRT_MLP_GRID_BLOCKS 1184
#endif
constexpr int kMlpGridBlocks = FRRT_MLP_GRID_BLOCKS;

// Weights of the three layers: W[l] is out x in (row-major, bf16), b[l] f32.
struct MlpWeights {
    const __nv_bfloat16 *w1, *w2, *w3;
    const float *b1, *b2, *b3;
};

// C(M x N) = epilogue(sum_k A(m, k) B(k, n)).  A(m, k) = A[m * lda + k], or
// A[k * lda + m] with transA; B(k, n) = B[n * ldb + k] (a weight matrix, out
// x in), or B[k * ldb + n] with transB.  Epilogue: + bias[n] when bias,
// ReLU when relu, times (mask[m * ldm + n] > 0) when mask (ReLU backward);
// the result is written as f32 (cf) or bf16 (cb), row-major with ldc.
struct GemmArgs {
    int M, N, K;
    const int *dM;             // device row count capping M, or nullptr
    const __nv_bfloat16 *A;
    int lda, transA;
    const __nv_bfloat16 *B;
    int ldb, transB;
    const float *bias;
    int relu;
    const __nv_bfloat16 *mask;
    int ldm;
    float *cf;
    __nv_bfloat16 *cb;
    int ldc;
    // optional f32 workspace (split_floats floats) for a split over K: a raw
    // f32 GEMM (no bias, ReLU or mask) of few output tiles and a long K is
    // computed as partial sums of K ranges by more CTAs, then reduced in a
    // fixed order (deterministic)
    float *split_ws;
    size_t split_floats;
};
// on the 5th-generation tensor cores (frrt_umma.cu); a launch that cannot be
// made, or a block whose pipeline wait ran out, leaves an error for
// gemm_take_error().  dep: launched as a programmatic dependent of the
// previous kernel on the stream
void launch_gemm(const GemmArgs &g, cudaStream_t st, bool dep = false);
// the GEMM's runtime (driver tensor-map entry point, kernel attributes,
// error flag); false when it cannot run here
bool umma_init();
// the first GEMM error since the last call (launch or device), or nullptr;
// read after the stream of the launches was synchronised
const char *gemm_take_error();

// softmax cross-entropy over rows of logits (M x 128, f32): per-row loss
// (f32, summed into *loss), d logits = (softmax - onehot) * scale as bf16
void launch_softmax_xent(const float *logits, const int32_t *labels, int M, float scale,
                         __nv_bfloat16 *dlogits, float *loss, cudaStream_t st);
// db[n] = sum_m dY[m * ld + n] (bf16 in, f32 out)
void launch_bias_grad(const __nv_bfloat16 *dY, int M, int N, int ld, float *db, cudaStream_t st);
// Adam on f32 master weights; refreshes the bf16 copy.  The step number
// (for the bias corrections) is `step`, or *d_step when d_step is given (a
// captured training step reads it on the device)
void launch_adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *w16, int n, float lr,
                 float b1, float b2, float eps, int step, cudaStream_t st, const int *d_step = nullptr);
void launch_f32_to_bf16(const float *src, __nv_bfloat16 *dst, int n, cudaStream_t st);
// X rows and labels of a minibatch gathered by index: idx[*d_base + r] when
// d_base is given (a captured training step reads its batch offset on the
// device), else idx[r]
void launch_gather_rows(const __nv_bfloat16 *X, const int32_t *labels, const int32_t *idx, int n,
                        __nv_bfloat16 *Xb, int32_t *lb, cudaStream_t st, const int *d_base = nullptr);
// the end of a captured training step: *d_base += batch, *d_step += 1
void launch_train_advance(int *d_base, int *d_step, int batch, cudaStream_t st);

// the network's forward pass: logits (n x 128, f32) of X (n x kMlpInPad);
// d_count, when given, caps n on the device; the hidden activations go to h1
// / h2 when they are not null (training's backward pass reads them).  One
// kernel (frrt_umma.cu): the activations stay in shared memory between the
// layers.
void launch_mlp_forward(const MlpWeights &w, const __nv_bfloat16 *X, int n, const int *d_count,
                        __nv_bfloat16 *h1, __nv_bfloat16 *h2, float *logits, cudaStream_t st, bool dep = false);
void launch_mlp_fused(const MlpWeights &w, const __nv_bfloat16 *X, int n, const int *d_count,
                      __nv_bfloat16 *h1, __nv_bfloat16 *h2, float *logits, cudaStream_t st, bool dep);

// Buffers of the proposal step inside a planning iteration (cap rows).
struct ProposalBufs {
    int cap;                   // candidates the network proposes for per iteration
    float mix;                 // probability of sampling from the network (else uniform)
    const int *count;          // candidates this iteration (device: the exact prefix's last entry)
    __nv_bfloat16 *X;
    float *logits;
    MlpWeights w;
};

// Features of expansion candidates: for candidate k of the listed ones, the
// 32 x 32 obstacle patch around its parent cell in the parent's heading frame
// (stride 2 px, forward = heading), the goal in that frame, the distance to
// the goal, sin / cos of the heading and the steering limit; bf16, rows of
// kMlpInPad (zero padded).  cells[k] / slots[k] name the parent.
void launch_features(const Inst *d_inst, const int32_t *cells, const int32_t *slot_of, int n,
                     __nv_bfloat16 *X, cudaStream_t st, const int *d_count = nullptr, bool dep = false);
struct Sched;
// the same for the planner's proposal rows: row r is candidate
// r - cand_exact[s] of the slot s whose exact candidate prefix holds r
void launch_features_sched(const Inst *d_inst, const Sched *d_sched, int n, __nv_bfloat16 *X, cudaStream_t st,
                           const int *d_count, bool dep);

// The (steering, length) bin of a draw, the training label
__host__ __device__ inline int proposal_bin(float steer, float len, float max_steer, float max_path)
{
    int sb = (int)floorf((steer + max_steer) / (2.0f * max_steer) * kSteerBins);
    sb = sb < 0 ? 0 : (sb >= kSteerBins ? kSteerBins - 1 : sb);
    const float lo = 5.0f, hi = max_path > 5.0f ? max_path : 5.0f + 1e-3f;
    int lb = (int)floorf((len - lo) / (hi - lo) * kLenBins);
    lb = lb < 0 ? 0 : (lb >= kLenBins ? kLenBins - 1 : lb);
    return sb * kLenBins + lb;
}

}  // namespace frrt
