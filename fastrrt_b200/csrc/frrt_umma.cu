// frrt_umma.cu -- the proposal network's BF16 GEMM on the 5th-generation
// tensor cores: operand tiles loaded by TMA (cp.async.bulk.tensor, 128-byte
// swizzle) into a 4-stage shared-memory ring, tcgen05.mma (kind::f16, BF16 in,
// FP32 accumulate) issued by one thread into a double-buffered TMEM
// accumulator, and an epilogue of four warps that reads TMEM with tcgen05.ld
// and applies bias / ReLU / ReLU-mask before the f32 or bf16 store.
//
// C(M x N) = epilogue(sum_k A(m, k) B(k, n)) with the operand conventions of
// GemmArgs: A(m, k) = A[m * lda + k] (K-major) or A[k * lda + m] (transA,
// MN-major); B(k, n) = B[n * ldb + k] (K-major: a weight matrix, out x in) or
// B[k * ldb + n] (transB, MN-major).  The instruction descriptor's major bits
// select the layout, so no operand is transposed in memory.
//
// Block: 6 warps.  Warp 4 lane 0 issues the TMA loads, warp 5 lane 0 the
// MMAs and their commits, warps 0-3 (TMEM lanes 0-127, one output row per
// thread) the epilogue.  Persistent over 128 x 128 output tiles (N tile
// fastest, so the tiles that share an A row block run side by side and the
// second read of A comes from L2); one block per SM (128 KB of operand ring).
// Every wait on an mbarrier is bounded: when one runs out the block sets the
// error flag, stops issuing, waits (bounded) for its own copies and MMAs in
// flight, frees its TMEM and returns.
#include <cuda.h>

#include <algorithm>
#include <mutex>

#include "frrt_device.cuh"
#include "frrt_kernels.cuh"
#include "frrt_mlp.cuh"

namespace frrt {

namespace {

// stages of the operand ring (32 KB each; a build-time knob for measurement)
#ifndef FRRT_UMMA_STAGES
#define FRRT_UMMA_STAGES 4
#endif
constexpr int kUM = 128, kUN = 128, kUK = 64, kUStages = FRRT_UMMA_STAGES;
constexpr int kUOpBytes = kUM * kUK * 2;  // one operand tile of one stage: 16 KB
constexpr int kUThreads = 192;
constexpr int kUTmemCols = 2 * kUN;       // two accumulators of 128 f32 columns
constexpr long kUWaitLimit = 1L << 22;    // try_wait rounds before a wait gives up

struct UmmaParams {
    int M, N, K;
    const int *dM;
    int a_mn, b_mn;
    const float *bias;
    int relu;
    const __nv_bfloat16 *mask;
    int ldm;
    float *cf;
    __nv_bfloat16 *cb;
    int ldc;
    int vec;  // rows of C and of the mask start on 16-byte boundaries
    int splits, kb_per;  // K split: partial sums of kb_per k-blocks each, into cf + split * M * ldc
    int *err;
};

struct UmmaSmem {
    __nv_bfloat16 a[kUStages][kUM * kUK];
    __nv_bfloat16 b[kUStages][kUN * kUK];
    uint64_t full[kUStages], empty[kUStages], tfull[2], tempty[2], drain;
    uint32_t tmem_base;
    int abort;
};
constexpr size_t kUSmemBytes = sizeof(UmmaSmem) + 1024;  // + alignment of the ring to 1024 B

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// bounded wait; gives up early once another role of the block has given up
__device__ __forceinline__ bool wait_bounded(uint64_t *bar, unsigned parity, volatile int *abort)
{
    for (long k = 0; k < kUWaitLimit; k++) {
        if (mbar_try_wait(bar, parity))
            return true;
        if ((k & 255) == 255 && *abort)
            return false;
    }
    *abort = 1;
    return false;
}

__device__ __forceinline__ void wait_drain(uint64_t *bar, unsigned parity)
{
    for (long k = 0; k < kUWaitLimit; k++)
        if (mbar_try_wait(bar, parity))
            return;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// arrives on `bar` once every MMA this thread issued before it has completed
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
          "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
          "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory matrix descriptor of a 128-byte-swizzled operand tile:
// start address, leading and stride byte offsets (16-byte units), the
// descriptor version of this architecture (bit 46) and the 128-byte swizzle
// mode (2 in bits 61-63).
//   K-major tile: rows of 64 bf16 (128 B), 8-row swizzle atoms 1024 B apart
//     (stride offset); the leading offset is unused (1).  The k-th 16-element
//     slice starts 32 B further.
//   MN-major tile: 64-element (128 B) MN runs per k, 8 k-rows to a 1024-B
//     atom (stride offset 1024 B); the second 64-element MN block of the tile
//     lies 8 KB further (leading offset).  The k-th slice of 16 starts
//     16 rows (2048 B) further.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46) | (2ull << 61);
}

// Instruction descriptor of kind::f16: f32 accumulator (bits 4-5 = 1), bf16
// A and B (bits 7-9, 10-12 = 1), the major of A (bit 15) and B (bit 16),
// N / 8 (bits 17-22), M / 16 (bits 24-28).
__host__ __device__ constexpr uint32_t instr_desc(int a_mn, int b_mn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(kUN >> 3) << 17) | ((uint32_t)(kUM >> 4) << 24);
}

__device__ __forceinline__ void store_chunk(const UmmaParams &p, int row, int n, const uint32_t (&r)[32])
{
    float v[32];
#pragma unroll
    for (int j = 0; j < 32; j++)
        v[j] = __uint_as_float(r[j]);
    const int nv = min(32, p.N - n);
    const bool full = p.vec && nv == 32;
    if (p.bias) {
#pragma unroll
        for (int j = 0; j < 32; j++)
            if (j < nv)
                v[j] += p.bias[n + j];
    }
    if (p.relu) {
#pragma unroll
        for (int j = 0; j < 32; j++)
            v[j] = fmaxf(v[j], 0.0f);
    }
    if (p.mask) {
        const __nv_bfloat16 *mk = p.mask + (long)row * p.ldm + n;
        if (full) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint4 w = reinterpret_cast<const uint4 *>(mk)[q];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const uint32_t word = e < 2 ? w.x : e < 4 ? w.y : e < 6 ? w.z : w.w;
                    const unsigned short h = (unsigned short)(word >> ((e & 1) * 16));
                    if (!(__bfloat162float(__ushort_as_bfloat16(h)) > 0.0f))
                        v[q * 8 + e] = 0.0f;
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < 32; j++)
                if (j < nv && !(__bfloat162float(mk[j]) > 0.0f))
                    v[j] = 0.0f;
        }
    }
    if (p.cf) {
        float *o = p.cf + (long)row * p.ldc + n;
        if (full) {
#pragma unroll
            for (int q = 0; q < 8; q++)
                reinterpret_cast<float4 *>(o)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        } else {
#pragma unroll
            for (int j = 0; j < 32; j++)
                if (j < nv)
                    o[j] = v[j];
        }
    } else {
        __nv_bfloat16 *o = p.cb + (long)row * p.ldc + n;
        if (full) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                uint32_t w[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const __nv_bfloat16 lo = __float2bfloat16(v[q * 8 + 2 * e]);
                    const __nv_bfloat16 hi = __float2bfloat16(v[q * 8 + 2 * e + 1]);
                    w[e] = (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
                }
                reinterpret_cast<uint4 *>(o)[q] = make_uint4(w[0], w[1], w[2], w[3]);
            }
        } else {
#pragma unroll
            for (int j = 0; j < 32; j++)
                if (j < nv)
                    o[j] = __float2bfloat16(v[j]);
        }
    }
}

__global__ void __launch_bounds__(kUThreads, 1)
    k_umma(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, UmmaParams p)
{
    griddep_wait();  // the producer of A (and of the row count) has finished
    extern __shared__ uint8_t smem_raw[];
    const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
    UmmaSmem &S = *reinterpret_cast<UmmaSmem *>(smem_raw + pad);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int M = p.M;
    if (p.dM) {
        const int c = *p.dM;
        M = c < M ? c : M;
    }
    const int ntn = (p.N + kUN - 1) / kUN, ntm = (M + kUM - 1) / kUM;
    const int nk = (p.K + kUK - 1) / kUK;
    const int ntiles_mn = ntm * ntn, ntiles = ntiles_mn * p.splits;
    // work unit t: K split t / ntiles_mn, output tile t % ntiles_mn (N fastest)
    auto k_range = [&](int t, int &kb0, int &kb1) {
        kb0 = (t / ntiles_mn) * p.kb_per;
        kb1 = min(nk, kb0 + p.kb_per);
    };
    if (threadIdx.x == 0) {
        for (int s = 0; s < kUStages; s++) {
            mbar_init(&S.full[s], 1);
            mbar_init(&S.empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&S.tfull[b], 1);
            mbar_init(&S.tempty[b], 4 * 32);
        }
        mbar_init(&S.drain, 1);
        S.abort = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&S.tmem_base)),
                     "r"(kUTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = S.tmem_base;
    volatile int *abort = &S.abort;
    bool ok = true;

    if (warp == 4 && lane == 0) {
        // TMA producer
        long it = 0;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
            const int tm = t % ntiles_mn;
            const int m0 = (tm / ntn) * kUM, n0 = (tm % ntn) * kUN;
            int kb0, kb1;
            k_range(t, kb0, kb1);
            for (int kb = kb0; kb < kb1; kb++) {
                const int s = (int)(it % kUStages);
                const long round = it / kUStages;
                if (round > 0 && !wait_bounded(&S.empty[s], (unsigned)((round - 1) & 1), abort)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(&S.full[s], 2u * kUOpBytes);
                const int k0 = kb * kUK;
                if (p.a_mn) {
                    tma_load_2d(S.a[s], &ta, m0, k0, &S.full[s]);
                    tma_load_2d(S.a[s] + 64 * kUK, &ta, m0 + 64, k0, &S.full[s]);
                } else {
                    tma_load_2d(S.a[s], &ta, k0, m0, &S.full[s]);
                }
                if (p.b_mn) {
                    tma_load_2d(S.b[s], &tb, n0, k0, &S.full[s]);
                    tma_load_2d(S.b[s] + 64 * kUK, &tb, n0 + 64, k0, &S.full[s]);
                } else {
                    tma_load_2d(S.b[s], &tb, k0, n0, &S.full[s]);
                }
                it++;
            }
        }
        // the copies issued land before the block exits (each stage's last
        // phase is the one of its last copy)
        for (long j = it > kUStages ? it - kUStages : 0; j < it; j++)
            wait_drain(&S.full[j % kUStages], (unsigned)((j / kUStages) & 1));
    } else if (warp == 5 && lane == 0) {
        // MMA issuer
        const uint32_t idesc = instr_desc(p.a_mn, p.b_mn);
        long it = 0;
        int tl = 0;
        bool issued = false;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, tl++) {
            const int b = tl & 1, u = tl >> 1;
            if (u > 0 && !wait_bounded(&S.tempty[b], (unsigned)((u - 1) & 1), abort)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t d = tbase + (uint32_t)(b * kUN);
            int kb0, kb1;
            k_range(t, kb0, kb1);
            for (int kb = kb0; kb < kb1; kb++, it++) {
                const int s = (int)(it % kUStages);
                if (!wait_bounded(&S.full[s], (unsigned)((it / kUStages) & 1), abort)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t sa = smem_u32(S.a[s]), sb = smem_u32(S.b[s]);
#pragma unroll
                for (int kk = 0; kk < kUK / 16; kk++) {
                    const uint64_t ad = p.a_mn ? smem_desc(sa + kk * 2048, 8192, 1024) : smem_desc(sa + kk * 32, 16, 1024);
                    const uint64_t bd = p.b_mn ? smem_desc(sb + kk * 2048, 8192, 1024) : smem_desc(sb + kk * 32, 16, 1024);
                    umma_bf16(d, ad, bd, idesc, (uint32_t)((kb - kb0) | kk));
                }
                issued = true;
                umma_commit(&S.empty[s]);
            }
            if (!ok)
                break;
            umma_commit(&S.tfull[b]);
        }
        if (issued) {  // no MMA in flight when the TMEM is freed
            umma_commit(&S.drain);
            wait_drain(&S.drain, 0);
        }
    } else if (warp < 4) {
        // epilogue: TMEM lanes 32 * warp + lane = output row
        int tl = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, tl++) {
            const int b = tl & 1, u = tl >> 1;
            if (!__all_sync(kFull, wait_bounded(&S.tfull[b], (unsigned)(u & 1), abort))) {
                ok = false;
                break;
            }
            tc_fence_after();
            const int tm = t % ntiles_mn;
            const int m0 = (tm / ntn) * kUM, n0 = (tm % ntn) * kUN;
            const int row = m0 + warp * 32 + lane;
            const uint32_t taddr = tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)(b * kUN);
            UmmaParams q = p;
            if (p.splits > 1)  // this split's partial sums
                q.cf = p.cf + (long)(t / ntiles_mn) * p.M * p.ldc;
            for (int c0 = 0; c0 < kUN && n0 + c0 < p.N; c0 += 32) {
                uint32_t r[32];
                tmem_ld32(taddr + (uint32_t)c0, r);
                if (row < M)
                    store_chunk(q, row, n0 + c0, r);
            }
            tc_fence_before();
            mbar_arrive(&S.tempty[b]);
        }
    }
    if (!ok) {
        *abort = 1;
        *reinterpret_cast<volatile int *>(p.err) = 1;
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kUTmemCols)
                     : "memory");
    }
}

// C[m][n] = sum over splits s (in order) of ws[s][m][n] (rows of N floats)
__global__ void __launch_bounds__(256) k_split_reduce(const float *ws, int splits, int M, int N, float *C,
                                                      int ldc)
{
    const long total = (long)M * N;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int k = 0; k < splits; k++)
            s += ws[(long)k * total + i];
        const long m = i / N;
        C[m * ldc + (i - m * N)] = s;
    }
}

// ---------------------------------------------------------------------------
// The network's forward pass in one kernel (the planner's proposal step):
// per 128-row tile, layer 1 streams X and W1 through a 3-stage TMA ring into
// one N = 256 accumulator; the epilogue writes bias + ReLU as bf16 into a
// shared-memory activation tile in the 128-byte-swizzled K-major layout the
// tensor core reads (the layout TMA writes), layer 2 takes its A operand from
// there and W2 from the ring, layer 3 likewise with W3, and the epilogue
// writes the logits.  The hidden activations go to global memory only when
// asked (training needs them).  Same instruction sequence per output element
// as three launches of k_umma, so the same results.
// ---------------------------------------------------------------------------

constexpr int kFStages = 3;
constexpr int kFK1 = (kMlpInPad + kUK - 1) / kUK;  // 17 k-blocks of layer 1
constexpr int kFK2 = kMlpHidden / kUK;             // 4 of layers 2 and 3
constexpr int kFUnits = kFK1 + 2 * kFK2;           // ring stages per tile
constexpr int kFTmemCols = kMlpHidden;             // one 128 x 256 f32 accumulator

struct FusedParams {
    int M;
    const int *dM;
    const float *b1, *b2, *b3;
    __nv_bfloat16 *h1, *h2;  // optional copies of the activations
    float *logits;
    int *err;
};

struct FusedSmem {
    __nv_bfloat16 a[kFStages][kUM * kUK];          // X tiles (layer 1)
    __nv_bfloat16 b[kFStages][kMlpHidden * kUK];   // weight tiles
    __nv_bfloat16 act[kMlpHidden / kUK][kUM * kUK]; // h1, then h2: 4 swizzled K-blocks
    uint64_t full[kFStages], empty[kFStages], acc_full, acc_free, act_ready, drain;
    uint32_t tmem_base;
    int abort;
};
constexpr size_t kFSmemBytes = sizeof(FusedSmem) + 1024;

__host__ __device__ constexpr uint32_t instr_desc_n(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kUM >> 4) << 24);
}

// bytes a ring stage of unit j (0 .. kFUnits - 1) receives
__device__ __forceinline__ unsigned fused_unit_bytes(int j)
{
    if (j < kFK1)
        return (unsigned)(kUM * kUK * 2 + kMlpHidden * kUK * 2);
    if (j < kFK1 + kFK2)
        return (unsigned)(kMlpHidden * kUK * 2);
    return (unsigned)(kMlpOut * kUK * 2);
}

// the epilogue's 32 columns c0 .. c0 + 31 of its row as bias + ReLU bf16:
// into the activation tile (128-byte swizzle: 16-byte chunk q of row r at
// chunk q ^ (r & 7)) and, when asked, to global memory
__device__ __forceinline__ void fused_store_act(FusedSmem &S, int r, int c0, const uint32_t (&v)[32],
                                                const float *bias, __nv_bfloat16 *gout, int row, int M)
{
    uint32_t w[16];
#pragma unroll
    for (int e = 0; e < 16; e++) {
        const float lo = fmaxf(__uint_as_float(v[2 * e]) + bias[c0 + 2 * e], 0.0f);
        const float hi = fmaxf(__uint_as_float(v[2 * e + 1]) + bias[c0 + 2 * e + 1], 0.0f);
        w[e] = (uint32_t)__bfloat16_as_ushort(__float2bfloat16(lo)) |
               ((uint32_t)__bfloat16_as_ushort(__float2bfloat16(hi)) << 16);
    }
    const int kb = c0 / kUK, q0 = (c0 % kUK) / 8;
    uint8_t *rowp = reinterpret_cast<uint8_t *>(S.act[kb]) + r * 128;
#pragma unroll
    for (int q = 0; q < 4; q++)
        *reinterpret_cast<uint4 *>(rowp + (((q0 + q) ^ (r & 7)) * 16)) =
            make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
    if (gout && row < M) {
        uint4 *g = reinterpret_cast<uint4 *>(gout + (long)row * kMlpHidden + c0);
#pragma unroll
        for (int q = 0; q < 4; q++)
            g[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
    }
}

__global__ void __launch_bounds__(kUThreads, 1)
    k_mlp_fused(const __grid_constant__ CUtensorMap tx, const __grid_constant__ CUtensorMap tw1,
                const __grid_constant__ CUtensorMap tw2, const __grid_constant__ CUtensorMap tw3, FusedParams p)
{
    griddep_wait();  // the features (and the row count) are written
    extern __shared__ uint8_t smem_raw[];
    const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
    FusedSmem &S = *reinterpret_cast<FusedSmem *>(smem_raw + pad);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int M = p.M;
    if (p.dM) {
        const int c = *p.dM;
        M = c < M ? c : M;
    }
    const int ntiles = (M + kUM - 1) / kUM;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kFStages; s++) {
            mbar_init(&S.full[s], 1);
            mbar_init(&S.empty[s], 1);
        }
        mbar_init(&S.acc_full, 1);
        mbar_init(&S.acc_free, 4 * 32);
        mbar_init(&S.act_ready, 4 * 32);
        mbar_init(&S.drain, 1);
        S.abort = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&S.tmem_base)),
                     "r"(kFTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = S.tmem_base;
    volatile int *abort = &S.abort;
    bool ok = true;

    if (warp == 4 && lane == 0) {
        // TMA producer: per tile 17 units of (X, W1), 4 of W2, 4 of W3
        long it = 0;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
            const int m0 = t * kUM;
            for (int j = 0; j < kFUnits; j++) {
                const int s = (int)(it % kFStages);
                const long round = it / kFStages;
                if (round > 0 && !wait_bounded(&S.empty[s], (unsigned)((round - 1) & 1), abort)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(&S.full[s], fused_unit_bytes(j));
                if (j < kFK1) {
                    tma_load_2d(S.a[s], &tx, j * kUK, m0, &S.full[s]);
                    tma_load_2d(S.b[s], &tw1, j * kUK, 0, &S.full[s]);
                } else if (j < kFK1 + kFK2) {
                    tma_load_2d(S.b[s], &tw2, (j - kFK1) * kUK, 0, &S.full[s]);
                } else {
                    tma_load_2d(S.b[s], &tw3, (j - kFK1 - kFK2) * kUK, 0, &S.full[s]);
                }
                it++;
            }
        }
        for (long j = it > kFStages ? it - kFStages : 0; j < it; j++)
            wait_drain(&S.full[j % kFStages], (unsigned)((j / kFStages) & 1));
    } else if (warp == 5 && lane == 0) {
        // MMA issuer
        long it = 0;
        int tl = 0;
        bool issued = false;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, tl++) {
            if (tl > 0 && !wait_bounded(&S.acc_free, (unsigned)((tl - 1) & 1), abort)) {
                ok = false;
                break;
            }
            tc_fence_after();
            for (int layer = 0; layer < 3 && ok; layer++) {
                const int nkb = layer == 0 ? kFK1 : kFK2;
                const uint32_t idesc = instr_desc_n(layer == 2 ? kMlpOut : kMlpHidden);
                if (layer > 0) {  // the activation tile of the layer before is written
                    if (!wait_bounded(&S.act_ready, (unsigned)(layer - 1), abort)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                }
                for (int kb = 0; kb < nkb; kb++, it++) {
                    const int s = (int)(it % kFStages);
                    if (!wait_bounded(&S.full[s], (unsigned)((it / kFStages) & 1), abort)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = layer == 0 ? smem_u32(S.a[s]) : smem_u32(S.act[kb]);
                    const uint32_t sb = smem_u32(S.b[s]);
#pragma unroll
                    for (int kk = 0; kk < kUK / 16; kk++)
                        umma_bf16(tbase, smem_desc(sa + kk * 32, 16, 1024), smem_desc(sb + kk * 32, 16, 1024),
                                  idesc, (uint32_t)(kb | kk));
                    issued = true;
                    umma_commit(&S.empty[s]);
                }
                if (ok)
                    umma_commit(&S.acc_full);
            }
        }
        if (issued) {
            umma_commit(&S.drain);
            wait_drain(&S.drain, 0);
        }
    } else if (warp < 4) {
        // epilogue: TMEM lane = tile row
        int tl = 0;
        const int r = warp * 32 + lane;
        const uint32_t taddr = tbase + ((uint32_t)(warp * 32) << 16);
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, tl++) {
            const int row = t * kUM + r;
            for (int layer = 0; layer < 3; layer++) {
                const unsigned parity = (unsigned)((3 * tl + layer) & 1);
                if (!__all_sync(kFull, wait_bounded(&S.acc_full, parity, abort))) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                if (layer < 2) {
                    const float *bias = layer == 0 ? p.b1 : p.b2;
                    __nv_bfloat16 *gout = layer == 0 ? p.h1 : p.h2;
                    for (int c0 = 0; c0 < kMlpHidden; c0 += 32) {
                        uint32_t v[32];
                        tmem_ld32(taddr + (uint32_t)c0, v);
                        fused_store_act(S, r, c0, v, bias, gout, row, M);
                    }
                    // the generic-proxy writes become visible to the tensor core
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    tc_fence_before();
                    mbar_arrive(&S.act_ready);
                } else {
                    for (int c0 = 0; c0 < kMlpOut; c0 += 32) {
                        uint32_t v[32];
                        tmem_ld32(taddr + (uint32_t)c0, v);
                        if (row < M) {
                            float4 *o = reinterpret_cast<float4 *>(p.logits + (long)row * kMlpOut + c0);
#pragma unroll
                            for (int q = 0; q < 8; q++)
                                o[q] = make_float4(__uint_as_float(v[4 * q]) + p.b3[c0 + 4 * q],
                                                   __uint_as_float(v[4 * q + 1]) + p.b3[c0 + 4 * q + 1],
                                                   __uint_as_float(v[4 * q + 2]) + p.b3[c0 + 4 * q + 2],
                                                   __uint_as_float(v[4 * q + 3]) + p.b3[c0 + 4 * q + 3]);
                        }
                    }
                    tc_fence_before();
                    mbar_arrive(&S.acc_free);
                }
            }
        }
    }
    if (!ok) {
        *abort = 1;
        *reinterpret_cast<volatile int *>(p.err) = 1;
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kFTmemCols)
                     : "memory");
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                  CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

struct UmmaRuntime {
    bool ok = false;
    EncodeTiledFn encode = nullptr;
    int sms = 0;
    int *h_err = nullptr;  // mapped pinned flag: set by a block whose wait ran out
    int *d_err = nullptr;
    std::mutex mu;
    const char *host_err = nullptr;  // the first launch error since the last check
};

// set up once per process, for the device current at the first call (one
// device per process, as the library's planners are used)
UmmaRuntime &runtime()
{
    static UmmaRuntime rt;
    static std::once_flag once;
    std::call_once(once, [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return;
        rt.encode = reinterpret_cast<EncodeTiledFn>(fn);
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&rt.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return;
        if (cudaFuncSetAttribute(k_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUSmemBytes) !=
                cudaSuccess ||
            cudaFuncSetAttribute(k_mlp_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFSmemBytes) !=
                cudaSuccess)
            return;
        if (cudaHostAlloc(reinterpret_cast<void **>(&rt.h_err), sizeof(int), cudaHostAllocMapped) != cudaSuccess)
            return;
        *rt.h_err = 0;
        if (cudaHostGetDevicePointer(reinterpret_cast<void **>(&rt.d_err), rt.h_err, 0) != cudaSuccess)
            return;
        rt.ok = true;
    });
    return rt;
}

// a 2-D bf16 tensor map of `outer` rows of `inner` elements, rows `ld`
// elements apart, a box of box_inner x box_outer, 128-byte swizzle, zero fill
bool make_map(CUtensorMap *m, const void *base, long inner, long outer, long ld, int box_inner, int box_outer)
{
    const cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)box_inner, (cuuint32_t)box_outer};
    const cuuint32_t es[2] = {1, 1};
    return runtime().encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box,
                            es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

}  // namespace

bool umma_init() { return runtime().ok; }

const char *gemm_take_error()
{
    UmmaRuntime &rt = runtime();
    if (!rt.ok)
        return "tensor-core GEMM: the driver's tensor-map entry point or the kernel attributes are unavailable";
    std::lock_guard<std::mutex> lk(rt.mu);
    const char *e = rt.host_err;
    rt.host_err = nullptr;
    if (!e && *reinterpret_cast<volatile int *>(rt.h_err)) {
        *reinterpret_cast<volatile int *>(rt.h_err) = 0;
        e = "tensor-core GEMM: a pipeline wait ran out (the launch stopped early)";
    }
    return e;
}

namespace {
void fail(const char *msg)
{
    UmmaRuntime &rt = runtime();
    std::lock_guard<std::mutex> lk(rt.mu);
    if (!rt.host_err)
        rt.host_err = msg;
}
}  // namespace

void launch_gemm(const GemmArgs &g, cudaStream_t st, bool dep)
{
    if (g.M <= 0 || g.N <= 0)
        return;
    UmmaRuntime &rt = runtime();
    if (!rt.ok)
        return fail("tensor-core GEMM: the driver's tensor-map entry point or the kernel attributes are unavailable");
    if (g.K <= 0 || (!g.cf) == (!g.cb))
        return fail("tensor-core GEMM: bad arguments");
    // TMA: 16-byte aligned bases and row strides
    if (!aligned16(g.A) || !aligned16(g.B) || g.lda % 8 || g.ldb % 8)
        return fail("tensor-core GEMM: operands must start on 16 bytes with row strides a multiple of 8 elements");
    CUtensorMap ta, tb;
    const bool okA = g.transA ? make_map(&ta, g.A, g.M, g.K, g.lda, 64, kUK)
                              : make_map(&ta, g.A, g.K, g.M, g.lda, kUK, kUM);
    const bool okB = g.transB ? make_map(&tb, g.B, g.N, g.K, g.ldb, 64, kUK)
                              : make_map(&tb, g.B, g.K, g.N, g.ldb, kUK, kUN);
    if (!okA || !okB)
        return fail("tensor-core GEMM: tensor map encoding failed");
    UmmaParams p{};
    p.M = g.M;
    p.N = g.N;
    p.K = g.K;
    p.dM = g.dM;
    p.a_mn = g.transA ? 1 : 0;
    p.b_mn = g.transB ? 1 : 0;
    p.bias = g.bias;
    p.relu = g.relu;
    p.mask = g.mask;
    p.ldm = g.ldm;
    p.cf = g.cf;
    p.cb = g.cb;
    p.ldc = g.ldc;
    p.vec = aligned16(g.cf ? (const void *)g.cf : (const void *)g.cb) && g.ldc % 8 == 0 &&
            (!g.mask || (aligned16(g.mask) && g.ldm % 8 == 0));
    p.err = rt.d_err;
    p.splits = 1;
    const long tiles = (long)((g.M + kUM - 1) / kUM) * ((g.N + kUN - 1) / kUN);
    const int nk = (g.K + kUK - 1) / kUK;
    p.kb_per = nk;
    // split over K: a raw f32 result with fewer tiles than half the SMs and
    // at least 8 k-blocks, into the caller's workspace
    if (g.split_ws && g.cf && !g.bias && !g.relu && !g.mask && !g.dM && 2 * tiles < rt.sms && nk >= 8) {
        int s = (int)std::min<long>(std::min<long>(nk / 4, rt.sms / tiles), 16);
        const int per = (nk + s - 1) / s;
        s = (nk + per - 1) / per;  // no empty split
        if (s > 1 && (size_t)s * g.M * g.N <= g.split_floats) {
            p.splits = s;
            p.kb_per = per;
            p.cf = g.split_ws;
            p.ldc = g.N;
            p.vec = g.N % 8 == 0 && aligned16(g.split_ws);
        }
    }
    const int grid = (int)std::min<long>(tiles * p.splits, rt.sms);
    launch_dep(dep, k_umma, grid, kUThreads, kUSmemBytes, st, ta, tb, p);
    if (p.splits > 1) {
        const long total = (long)g.M * g.N;
        k_split_reduce<<<(int)std::min<long>((total + 255) / 256, (long)rt.sms * 8), 256, 0, st>>>(
            g.split_ws, p.splits, g.M, g.N, g.cf, g.ldc);
    }
}

void launch_mlp_fused(const MlpWeights &w, const __nv_bfloat16 *X, int n, const int *d_count,
                      __nv_bfloat16 *h1, __nv_bfloat16 *h2, float *logits, cudaStream_t st, bool dep)
{
    if (n <= 0)
        return;
    UmmaRuntime &rt = runtime();
    if (!rt.ok)
        return fail("tensor-core GEMM: the driver's tensor-map entry point or the kernel attributes are unavailable");
    if (!aligned16(X) || !aligned16(w.w1) || !aligned16(w.w2) || !aligned16(w.w3) || !aligned16(logits) ||
        (h1 && !aligned16(h1)) || (h2 && !aligned16(h2)))
        return fail("fused forward: buffers must start on 16 bytes");
    CUtensorMap tx, t1, t2, t3;
    if (!make_map(&tx, X, kMlpInPad, n, kMlpInPad, kUK, kUM) ||
        !make_map(&t1, w.w1, kMlpInPad, kMlpHidden, kMlpInPad, kUK, kMlpHidden) ||
        !make_map(&t2, w.w2, kMlpHidden, kMlpHidden, kMlpHidden, kUK, kMlpHidden) ||
        !make_map(&t3, w.w3, kMlpHidden, kMlpOut, kMlpHidden, kUK, kMlpOut))
        return fail("fused forward: tensor map encoding failed");
    FusedParams p{};
    p.M = n;
    p.dM = d_count;
    p.b1 = w.b1;
    p.b2 = w.b2;
    p.b3 = w.b3;
    p.h1 = h1;
    p.h2 = h2;
    p.logits = logits;
    p.err = rt.d_err;
    const int grid = (int)std::min<long>((n + kUM - 1) / kUM, rt.sms);
    launch_dep(dep, k_mlp_fused, grid, kUThreads, kFSmemBytes, st, tx, t1, t2, t3, p);
}

}  // namespace frrt
