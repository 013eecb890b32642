// frrt_mlp.cu -- training kernels, forward pass and planner-side feature
// extraction of the learned expansion proposal (the GEMM is frrt_umma.cu).
#include "frrt_mlp.cuh"
#include "frrt_device.cuh"
#include "frrt_kernels.cuh"

#include <algorithm>
#include <cmath>

namespace frrt {

namespace {

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

// db[n] = sum_m dY[m * ld + n]: one block per 32 columns; warp w sums rows
// w, w + 8, ... (lane = column, coalesced), the warps' partial sums are
// added in warp order (deterministic)
__global__ void __launch_bounds__(256) k_bias_grad(const __nv_bfloat16 *dY, int M, int N, int ld, float *db)
{
    __shared__ float part[8][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = blockIdx.x * 32 + lane;
    float s = 0.0f;
    if (n < N)
        for (int m = warp; m < M; m += 8)
            s += __bfloat162float(dY[(long)m * ld + n]);
    part[warp][lane] = s;
    __syncthreads();
    if (warp == 0 && n < N) {
        float t = 0.0f;
        for (int w = 0; w < 8; w++)
            t += part[w][lane];
        db[n] = t;
    }
}

__global__ void k_adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *w16, int n,
                       float lr, float b1, float b2, float eps, float c1, float c2, const int *d_step)
{
    if (d_step) {  // bias corrections of the device's step number
        const float t = (float)*d_step;
        c1 = 1.0f - powf(b1, t);
        c2 = 1.0f - powf(b2, t);
    }
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

__global__ void k_train_advance(int *d_base, int *d_step, int batch)
{
    *d_base += batch;
    *d_step += 1;
}

__global__ void k_f32_to_bf16(const float *src, __nv_bfloat16 *dst, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        dst[i] = __float2bfloat16(src[i]);
}

// rows of X (kMlpInPad bf16 = 130 x 16 B) and their labels gathered by index
__global__ void k_gather_rows(const __nv_bfloat16 *X, const int32_t *labels, const int32_t *idx,
                              int n, __nv_bfloat16 *Xb, int32_t *lb, const int *d_base)
{
    const int r = blockIdx.x;
    if (r >= n)
        return;
    if (d_base)
        idx += *d_base;
    static_assert(kMlpInPad * 2 % 16 == 0, "feature rows are whole 16-byte vectors");
    constexpr int kVec = kMlpInPad * 2 / 16;
    const uint4 *src = reinterpret_cast<const uint4 *>(X + (long)idx[r] * kMlpInPad);
    uint4 *dst = reinterpret_cast<uint4 *>(Xb + (long)r * kMlpInPad);
    for (int c = threadIdx.x; c < kVec; c += blockDim.x)
        dst[c] = src[c];
    if (threadIdx.x == 0)
        lb[r] = labels[idx[r]];
}

// one warp per candidate; lanes over the 1024 patch samples
// rows come from cells[k] / slot_of[k], or, with sc, from the planner's
// exact candidate prefix (row = cand_exact[slot] + candidate index)
__global__ void k_features(const Inst *insts, const int32_t *cells, const int32_t *slot_of, const Sched *sc,
                           int n, __nv_bfloat16 *X, const int *d_count)
{
    griddep_wait();  // the candidates are listed
    const int lane = threadIdx.x & 31;
    if (d_count && *d_count < n)
        n = *d_count;
    // rows grid-strided over a machine-sized grid (the count is on the device)
    const int warps = (int)((gridDim.x * (long)blockDim.x) >> 5);
    for (int k = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5); k < n; k += warps) {
        int slot, pos;
        if (sc) {
            slot = find_slot(sc->cand_exact, sc->n_slots, k);
            pos = insts[slot].cand[k - sc->cand_exact[slot]];
        } else {
            slot = slot_of[k];
            pos = cells[k];
        }
        const Inst &I = insts[slot];
        const int z = pos / I.W, x = pos - z * I.W;
        const float h = I.heading[pos];
        float sh, ch;
        sincosf(h, &sh, &ch);
        // pixel offsets: forward (sin h, -cos h), right (cos h, sin h)
        __nv_bfloat16 *row = X + (long)k * kMlpInPad;
        const int half = kMlpPatch / 2;
        // lane = patch column; the 32 rows' mask words are loaded before any
        // is used, so their latencies overlap instead of adding up
        const float v = (float)((lane - half) * kMlpPatchStride);  // right
        uint32_t word[kMlpPatch];
        int bit[kMlpPatch];
#pragma unroll
        for (int iu = 0; iu < kMlpPatch; iu++) {
            const float u = (float)((half - 1 - iu) * kMlpPatchStride);  // forward, row 0 ahead
            const int px = (int)floorf(x + u * sh + v * ch + 0.5f);
            const int pz = (int)floorf(z - u * ch + v * sh + 0.5f);
            const bool in = px >= 0 && px < I.W && pz >= 0 && pz < I.H;
            word[iu] = in ? I.blocked[(long)pz * I.mask_rw + (px >> 5)] : 0u;
            bit[iu] = in ? (px & 31) : -1;  // -1: outside the frame
        }
#pragma unroll
        for (int iu = 0; iu < kMlpPatch; iu++) {
            const float val = bit[iu] < 0 ? 0.5f : (((word[iu] >> bit[iu]) & 1u) ? 1.0f : 0.0f);
            row[iu * kMlpPatch + lane] = __float2bfloat16(val);
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

void launch_softmax_xent(const float *logits, const int32_t *labels, int M, float scale,
                         __nv_bfloat16 *dlogits, float *loss, cudaStream_t st)
{
    if (M <= 0)
        return;
    k_softmax_xent<<<(M * 32 + 255) / 256, 256, 0, st>>>(logits, labels, M, scale, dlogits, loss);
}

void launch_bias_grad(const __nv_bfloat16 *dY, int M, int N, int ld, float *db, cudaStream_t st)
{
    k_bias_grad<<<(N + 31) / 32, 256, 0, st>>>(dY, M, N, ld, db);
}

void launch_adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *w16, int n, float lr,
                 float b1, float b2, float eps, int step, cudaStream_t st, const int *d_step)
{
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<(n + 255) / 256, 256, 0, st>>>(w, m, v, g, w16, n, lr, b1, b2, eps, c1, c2, d_step);
}

void launch_train_advance(int *d_base, int *d_step, int batch, cudaStream_t st)
{
    k_train_advance<<<1, 1, 0, st>>>(d_base, d_step, batch);
}

void launch_f32_to_bf16(const float *src, __nv_bfloat16 *dst, int n, cudaStream_t st)
{
    k_f32_to_bf16<<<(n + 255) / 256, 256, 0, st>>>(src, dst, n);
}

void launch_gather_rows(const __nv_bfloat16 *X, const int32_t *labels, const int32_t *idx, int n,
                        __nv_bfloat16 *Xb, int32_t *lb, cudaStream_t st, const int *d_base)
{
    if (n > 0)
        k_gather_rows<<<n, 128, 0, st>>>(X, labels, idx, n, Xb, lb, d_base);
}

void launch_features(const Inst *d_inst, const int32_t *cells, const int32_t *slot_of, int n,
                     __nv_bfloat16 *X, cudaStream_t st, const int *d_count, bool dep)
{
    if (n <= 0)
        return;
    launch_dep(dep, k_features, std::min((n * 32 + 255) / 256, kMlpGridBlocks), 256, 0, st, d_inst, cells,
               slot_of, (const Sched *)nullptr, n, X, d_count);
}

void launch_features_sched(const Inst *d_inst, const Sched *d_sched, int n, __nv_bfloat16 *X, cudaStream_t st,
                           const int *d_count, bool dep)
{
    if (n <= 0)
        return;
    launch_dep(dep, k_features, std::min((n * 32 + 255) / 256, kMlpGridBlocks), 256, 0, st, d_inst,
               (const int32_t *)nullptr, (const int32_t *)nullptr, d_sched, n, X, d_count);
}

void launch_mlp_forward(const MlpWeights &w, const __nv_bfloat16 *X, int n, const int *d_count,
                        __nv_bfloat16 *h1, __nv_bfloat16 *h2, float *logits, cudaStream_t st, bool dep)
{
    launch_mlp_fused(w, X, n, d_count, h1, h2, logits, st, dep);
}

}  // namespace frrt
