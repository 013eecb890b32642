// frrt_mlp.cu -- BF16 tensor-core GEMM, training kernels and planner-side
// feature extraction of the learned expansion proposal.
#include "frrt_mlp.cuh"
#include "frrt_device.cuh"

#include <algorithm>
#include <cmath>

namespace frrt {

namespace {

constexpr int kBM = 64, kBN = 64, kBK = 32, kPad = 8;

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi)
{
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// 64 x 64 output tile per block of 4 warps (2 x 2, 32 x 32 each), K in steps
// of 32 through shared memory (both operands K-contiguous there), fragments
// of mma.sync m16n8k16 (A row-major, B column-major).
__global__ void __launch_bounds__(128) k_gemm(GemmArgs g)
{
    __shared__ __nv_bfloat16 As[kBM][kBK + kPad];
    __shared__ __nv_bfloat16 Bs[kBN][kBK + kPad];
    if (g.dM) {
        const int cnt = *g.dM;
        g.M = cnt < g.M ? cnt : g.M;
    }
    const int n0 = blockIdx.x * kBN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int gq = lane >> 2, tq = lane & 3;
    // row tiles grid-strided: the grid is sized for the machine, the rows (a
    // device-side count in the planner) may be few (uniform across the block)
    for (int m0 = blockIdx.y * kBM; m0 < g.M; m0 += gridDim.y * kBM) {
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 4; e++)
                acc[i][j][e] = 0.0f;
    const __nv_bfloat16 zero = __float2bfloat16(0.0f);
    for (int k0 = 0; k0 < g.K; k0 += kBK) {
        for (int e = tid; e < kBM * kBK; e += blockDim.x) {
            int r, c;
            if (g.transA) {  // consecutive threads along m (contiguous in memory)
                r = e % kBM;
                c = e / kBM;
            } else {
                r = e / kBK;
                c = e % kBK;
            }
            const int m = m0 + r, k = k0 + c;
            __nv_bfloat16 v = zero;
            if (m < g.M && k < g.K)
                v = g.transA ? g.A[(long)k * g.lda + m] : g.A[(long)m * g.lda + k];
            As[r][c] = v;
        }
        for (int e = tid; e < kBN * kBK; e += blockDim.x) {
            int r, c;
            if (g.transB) {  // contiguous along n
                r = e % kBN;
                c = e / kBN;
            } else {
                r = e / kBK;
                c = e % kBK;
            }
            const int n = n0 + r, k = k0 + c;
            __nv_bfloat16 v = zero;
            if (n < g.N && k < g.K)
                v = g.transB ? g.B[(long)k * g.ldb + n] : g.B[(long)n * g.ldb + k];
            Bs[r][c] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kBK; kk += 16) {
            uint32_t a[2][4], b[4][2];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const int r = wm + i * 16 + gq, c = kk + 2 * tq;
                a[i][0] = pack_bf16(As[r][c], As[r][c + 1]);
                a[i][1] = pack_bf16(As[r + 8][c], As[r + 8][c + 1]);
                a[i][2] = pack_bf16(As[r][c + 8], As[r][c + 9]);
                a[i][3] = pack_bf16(As[r + 8][c + 8], As[r + 8][c + 9]);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int n = wn + j * 8 + gq, c = kk + 2 * tq;
                b[j][0] = pack_bf16(Bs[n][c], Bs[n][c + 1]);
                b[j][1] = pack_bf16(Bs[n][c + 8], Bs[n][c + 9]);
            }
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
                    mma_bf16(acc[i][j], a[i], b[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int m = m0 + wm + i * 16 + gq + (e >= 2 ? 8 : 0);
                const int n = n0 + wn + j * 8 + 2 * tq + (e & 1);
                if (m >= g.M || n >= g.N)
                    continue;
                float v = acc[i][j][e];
                if (g.bias)
                    v += g.bias[n];
                if (g.relu)
                    v = fmaxf(v, 0.0f);
                if (g.mask && !(__bfloat162float(g.mask[(long)m * g.ldm + n]) > 0.0f))
                    v = 0.0f;
                if (g.cf)
                    g.cf[(long)m * g.ldc + n] = v;
                else
                    g.cb[(long)m * g.ldc + n] = __float2bfloat16(v);
            }
    }
}

// one warp per row of 128 logits
__global__ void k_softmax_xent(const float *logits, const int32_t *labels, int M, float scale,
                               __nv_bfloat16 *dlogits, float *loss)
{
    const int row = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= M)
        return;
    const float *l = logits + (long)row * kMlpOut;
    float v[kMlpOut / 32];
    float mx = -1e30f;
#pragma unroll
    for (int q = 0; q < kMlpOut / 32; q++) {
        v[q] = l[q * 32 + lane];
        mx = fmaxf(mx, v[q]);
    }
    for (int o = 16; o; o >>= 1)
        mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, o));
    float sum = 0.0f;
#pragma unroll
    for (int q = 0; q < kMlpOut / 32; q++) {
        v[q] = __expf(v[q] - mx);
        sum += v[q];
    }
    for (int o = 16; o; o >>= 1)
        sum += __shfl_xor_sync(kFull, sum, o);
    const int y = labels[row];
#pragma unroll
    for (int q = 0; q < kMlpOut / 32; q++) {
        const int c = q * 32 + lane;
        const float p = v[q] / sum;
        dlogits[(long)row * kMlpOut + c] = __float2bfloat16((p - (c == y ? 1.0f : 0.0f)) * scale);
        if (c == y && loss)
            atomicAdd(loss, -__logf(fmaxf(p, 1e-30f)));
    }
}

__global__ void k_bias_grad(const __nv_bfloat16 *dY, int M, int N, int ld, float *db)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N)
        return;
    float s = 0.0f;
    for (int m = 0; m < M; m++)
        s += __bfloat162float(dY[(long)m * ld + n]);
    db[n] = s;
}

__global__ void k_adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *w16, int n,
                       float lr, float b1, float b2, float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (w16)
        w16[i] = __float2bfloat16(wi);
}

__global__ void k_f32_to_bf16(const float *src, __nv_bfloat16 *dst, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        dst[i] = __float2bfloat16(src[i]);
}

__global__ void k_gather_rows(const __nv_bfloat16 *X, const int32_t *labels, const int32_t *idx,
                              int n, __nv_bfloat16 *Xb, int32_t *lb)
{
    const int r = blockIdx.x;
    if (r >= n)
        return;
    const long src = (long)idx[r] * kMlpInPad, dst = (long)r * kMlpInPad;
    for (int c = threadIdx.x; c < kMlpInPad; c += blockDim.x)
        Xb[dst + c] = X[src + c];
    if (threadIdx.x == 0)
        lb[r] = labels[idx[r]];
}

// one warp per candidate; lanes over the 1024 patch samples
__global__ void k_features(const Inst *insts, const int32_t *cells, const int32_t *slot_of, int n,
                           __nv_bfloat16 *X, const int *d_count)
{
    const int lane = threadIdx.x & 31;
    if (d_count && *d_count < n)
        n = *d_count;
    // rows grid-strided over a machine-sized grid (the count is on the device)
    const int warps = (int)((gridDim.x * (long)blockDim.x) >> 5);
    for (int k = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5); k < n; k += warps) {
        const Inst &I = insts[slot_of[k]];
        const int pos = cells[k];
        const int z = pos / I.W, x = pos - z * I.W;
        const float h = I.heading[pos];
        float sh, ch;
        sincosf(h, &sh, &ch);
        // pixel offsets: forward (sin h, -cos h), right (cos h, sin h)
        __nv_bfloat16 *row = X + (long)k * kMlpInPad;
        const int half = kMlpPatch / 2;
        for (int s = lane; s < kMlpPatch * kMlpPatch; s += 32) {
            const int iu = s / kMlpPatch, iv = s % kMlpPatch;
            const float u = (float)((half - 1 - iu) * kMlpPatchStride);  // forward, row 0 ahead
            const float v = (float)((iv - half) * kMlpPatchStride);      // right
            const int px = (int)floorf(x + u * sh + v * ch + 0.5f);
            const int pz = (int)floorf(z - u * ch + v * sh + 0.5f);
            float val = 0.5f;  // outside the frame
            if (px >= 0 && px < I.W && pz >= 0 && pz < I.H)
                val = bit_xz(I.blocked, I.mask_rw, px, pz) ? 1.0f : 0.0f;
            row[s] = __float2bfloat16(val);
        }
        if (lane < kMlpInPad - kMlpPatch * kMlpPatch) {
            const float dx = (float)(I.goal_x - x), dz = (float)(I.goal_z - z);
            const float scale = 1.0f / (float)max(I.W, I.H);
            float val = 0.0f;
            switch (lane) {
            case 0: val = (dx * sh - dz * ch) * scale; break;  // goal ahead
            case 1: val = (dx * ch + dz * sh) * scale; break;  // goal to the right
            case 2: val = sqrtf(dx * dx + dz * dz) * scale; break;
            case 3: val = sh; break;
            case 4: val = ch; break;
            case 5: val = (float)I.max_steer; break;
            default: val = 0.0f;
            }
            row[kMlpPatch * kMlpPatch + lane] = __float2bfloat16(val);
        }
    }
}

}  // namespace

void launch_gemm(const GemmArgs &g, cudaStream_t st)
{
    if (g.M <= 0 || g.N <= 0)
        return;
    // at most kMlpGridBlocks blocks (the row tiles loop beyond that)
    const int nx = (g.N + kBN - 1) / kBN;
    const int ny = std::min((g.M + kBM - 1) / kBM, std::max(1, kMlpGridBlocks / nx));
    k_gemm<<<dim3(nx, ny), 128, 0, st>>>(g);
}

void launch_softmax_xent(const float *logits, const int32_t *labels, int M, float scale,
                         __nv_bfloat16 *dlogits, float *loss, cudaStream_t st)
{
    if (M <= 0)
        return;
    k_softmax_xent<<<(M * 32 + 255) / 256, 256, 0, st>>>(logits, labels, M, scale, dlogits, loss);
}

void launch_bias_grad(const __nv_bfloat16 *dY, int M, int N, int ld, float *db, cudaStream_t st)
{
    k_bias_grad<<<(N + 127) / 128, 128, 0, st>>>(dY, M, N, ld, db);
}

void launch_adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *w16, int n, float lr,
                 float b1, float b2, float eps, int step, cudaStream_t st)
{
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<(n + 255) / 256, 256, 0, st>>>(w, m, v, g, w16, n, lr, b1, b2, eps, c1, c2);
}

void launch_f32_to_bf16(const float *src, __nv_bfloat16 *dst, int n, cudaStream_t st)
{
    k_f32_to_bf16<<<(n + 255) / 256, 256, 0, st>>>(src, dst, n);
}

void launch_gather_rows(const __nv_bfloat16 *X, const int32_t *labels, const int32_t *idx, int n,
                        __nv_bfloat16 *Xb, int32_t *lb, cudaStream_t st)
{
    if (n > 0)
        k_gather_rows<<<n, 128, 0, st>>>(X, labels, idx, n, Xb, lb);
}

void launch_features(const Inst *d_inst, const int32_t *cells, const int32_t *slot_of, int n,
                     __nv_bfloat16 *X, cudaStream_t st, const int *d_count)
{
    if (n <= 0)
        return;
    k_features<<<std::min((n * 32 + 255) / 256, kMlpGridBlocks), 256, 0, st>>>(d_inst, cells, slot_of, n, X,
                                                                                 d_count);
}

void launch_mlp_forward(const MlpWeights &w, const __nv_bfloat16 *X, int n, const int *d_count,
                        __nv_bfloat16 *h1, __nv_bfloat16 *h2, float *logits, cudaStream_t st)
{
    GemmArgs g{};
    g.M = n;
    g.dM = d_count;
    g.N = kMlpHidden;
    g.K = kMlpInPad;
    g.A = X;
    g.lda = kMlpInPad;
    g.B = w.w1;
    g.ldb = kMlpInPad;
    g.bias = w.b1;
    g.relu = 1;
    g.cb = h1;
    g.ldc = kMlpHidden;
    launch_gemm(g, st);
    g.K = kMlpHidden;
    g.A = h1;
    g.lda = kMlpHidden;
    g.B = w.w2;
    g.ldb = kMlpHidden;
    g.bias = w.b2;
    g.cb = h2;
    launch_gemm(g, st);
    g.N = kMlpOut;
    g.A = h2;
    g.B = w.w3;
    g.bias = w.b3;
    g.relu = 0;
    g.cb = nullptr;
    g.cf = logits;
    g.ldc = kMlpOut;
    launch_gemm(g, st);
}

}  // namespace frrt
