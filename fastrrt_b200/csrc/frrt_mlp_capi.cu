// frrt_mlp_capi.cu -- the learned expansion proposal's network behind the C
// ABI: creation, weights in and out, forward pass, gradients, and training
// on a device-resident dataset.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "fastrrt_b200.h"
#include "frrt_engine.h"
#include "frrt_mlp.h"

namespace frrt {

namespace {

template <class T>
bool dalloc(T *&p, size_t n)
{
    return cudaMalloc(&p, sizeof(T) * (n ? n : 1)) == cudaSuccess;
}

bool cuda_ok(cudaError_t e, const char *what)
{
    if (e == cudaSuccess)
        return true;
    set_error(std::string("mlp: ") + what + ": " + cudaGetErrorString(e));
    return false;
}

// the GEMMs launched since the last check ran (after a stream sync)
bool gemm_ok()
{
    if (const char *e = gemm_take_error()) {
        set_error(std::string("mlp: ") + e);
        return false;
    }
    return true;
}

}  // namespace

// workspace of the weight gradients' split over K: at most 16 splits of the
// largest gradient (256 x 1040)
constexpr size_t kSplitFloats = 16 * (size_t)kMlpHidden * kMlpInPad;

const size_t Mlp::kSizes[6] = {(size_t)kMlpHidden * kMlpInPad, kMlpHidden,
                               (size_t)kMlpHidden * kMlpHidden, kMlpHidden,
                               (size_t)kMlpOut * kMlpHidden,    kMlpOut};

Mlp::Mlp(uint64_t seed, int max_batch) : max_batch_(max_batch)
{
    if (!umma_init()) {
        gemm_ok();
        return;
    }
    if (cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("mlp: stream");
        return;
    }
    bool ok = true;
    for (int t = 0; t < 6; t++) {
        ok = ok && dalloc(w_[t], kSizes[t]) && dalloc(m_[t], kSizes[t]) && dalloc(v_[t], kSizes[t]) &&
             dalloc(g_[t], kSizes[t]);
        ok = ok && cudaMemset(m_[t], 0, sizeof(float) * kSizes[t]) == cudaSuccess &&
             cudaMemset(v_[t], 0, sizeof(float) * kSizes[t]) == cudaSuccess;
    }
    for (int l = 0; l < 3; l++)
        ok = ok && dalloc(w16_[l], kSizes[2 * l]);
    const size_t B = (size_t)max_batch;
    ok = ok && dalloc(x_, B * kMlpInPad) && dalloc(h1_, B * kMlpHidden) && dalloc(h2_, B * kMlpHidden) &&
         dalloc(logits_, B * kMlpOut) && dalloc(dl_, B * kMlpOut) && dalloc(dh2_, B * kMlpHidden) &&
         dalloc(dh1_, B * kMlpHidden) && dalloc(labels_, B) && dalloc(loss_, 1) &&
         dalloc(xf_, B * kMlpInPad) && dalloc(split_ws_, kSplitFloats);
    if (!ok) {
        set_error("mlp: device allocation failed");
        return;
    }
    // He-uniform initialisation; the padding columns of layer 1 stay zero
    std::mt19937_64 rng(seed);
    std::vector<float> host;
    for (int l = 0; l < 3; l++) {
        const int fan_in = l == 0 ? kMlpIn : kMlpHidden;
        const int cols = l == 0 ? kMlpInPad : kMlpHidden;
        const size_t n = kSizes[2 * l];
        host.assign(n, 0.0f);
        std::uniform_real_distribution<float> u(-std::sqrt(6.0f / fan_in), std::sqrt(6.0f / fan_in));
        for (size_t i = 0; i < n; i++)
            if ((int)(i % cols) < fan_in)
                host[i] = u(rng);
        ok = ok && cudaMemcpy(w_[2 * l], host.data(), sizeof(float) * n, cudaMemcpyHostToDevice) ==
                       cudaSuccess;
        host.assign(kSizes[2 * l + 1], 0.0f);
        ok = ok && cudaMemcpy(w_[2 * l + 1], host.data(), sizeof(float) * kSizes[2 * l + 1],
                              cudaMemcpyHostToDevice) == cudaSuccess;
    }
    ok_ = ok && refresh();
}

Mlp::~Mlp()
{
    for (int t = 0; t < 6; t++) {
        cudaFree(w_[t]);
        cudaFree(m_[t]);
        cudaFree(v_[t]);
        cudaFree(g_[t]);
    }
    for (int l = 0; l < 3; l++)
        cudaFree(w16_[l]);
    cudaFree(x_);
    cudaFree(h1_);
    cudaFree(h2_);
    cudaFree(logits_);
    cudaFree(dl_);
    cudaFree(dh2_);
    cudaFree(dh1_);
    cudaFree(labels_);
    cudaFree(loss_);
    cudaFree(xf_);
    cudaFree(split_ws_);
    cudaFree(perm_);
    cudaFree(ctl_);
    if (stream_)
        cudaStreamDestroy(stream_);
}

bool Mlp::refresh()
{
    for (int l = 0; l < 3; l++)
        launch_f32_to_bf16(w_[2 * l], w16_[l], (int)kSizes[2 * l], stream_);
    return cuda_ok(cudaStreamSynchronize(stream_), "weight refresh");
}

MlpWeights Mlp::weights() const
{
    return MlpWeights{w16_[0], w16_[1], w16_[2], w_[1], w_[3], w_[5]};
}

void Mlp::forward(const __nv_bfloat16 *X, int n, cudaStream_t st, float *logits,
                  __nv_bfloat16 *h1, __nv_bfloat16 *h2, const int *d_count) const
{
    launch_mlp_forward(weights(), X, n, d_count, h1, h2, logits, st);
}

// forward + backward of a batch in x_ / labels_; gradients into g_
void Mlp::backward(int n)
{
    forward(x_, n, stream_, logits_, h1_, h2_, nullptr);
    cudaMemsetAsync(loss_, 0, sizeof(float), stream_);
    launch_softmax_xent(logits_, labels_, n, 1.0f / n, dl_, loss_, stream_);
    GemmArgs g{};
    // dW3 = dL^T H2 ; db3
    g.M = kMlpOut; g.N = kMlpHidden; g.K = n;
    g.A = dl_; g.lda = kMlpOut; g.transA = 1;
    g.B = h2_; g.ldb = kMlpHidden; g.transB = 1;
    g.cf = g_[4]; g.ldc = kMlpHidden;
    g.split_ws = split_ws_; g.split_floats = kSplitFloats;
    launch_gemm(g, stream_);
    launch_bias_grad(dl_, n, kMlpOut, kMlpOut, g_[5], stream_);
    // dH2 = dL W3 * (H2 > 0)
    g = GemmArgs{};
    g.M = n; g.N = kMlpHidden; g.K = kMlpOut;
    g.A = dl_; g.lda = kMlpOut;
    g.B = w16_[2]; g.ldb = kMlpHidden; g.transB = 1;
    g.mask = h2_; g.ldm = kMlpHidden;
    g.cb = dh2_; g.ldc = kMlpHidden;
    launch_gemm(g, stream_);
    // dW2 = dH2^T H1 ; db2
    g = GemmArgs{};
    g.M = kMlpHidden; g.N = kMlpHidden; g.K = n;
    g.A = dh2_; g.lda = kMlpHidden; g.transA = 1;
    g.B = h1_; g.ldb = kMlpHidden; g.transB = 1;
    g.cf = g_[2]; g.ldc = kMlpHidden;
    g.split_ws = split_ws_; g.split_floats = kSplitFloats;
    launch_gemm(g, stream_);
    launch_bias_grad(dh2_, n, kMlpHidden, kMlpHidden, g_[3], stream_);
    // dH1 = dH2 W2 * (H1 > 0)
    g = GemmArgs{};
    g.M = n; g.N = kMlpHidden; g.K = kMlpHidden;
    g.A = dh2_; g.lda = kMlpHidden;
    g.B = w16_[1]; g.ldb = kMlpHidden; g.transB = 1;
    g.mask = h1_; g.ldm = kMlpHidden;
    g.cb = dh1_; g.ldc = kMlpHidden;
    launch_gemm(g, stream_);
    // dW1 = dH1^T X ; db1
    g = GemmArgs{};
    g.M = kMlpHidden; g.N = kMlpInPad; g.K = n;
    g.A = dh1_; g.lda = kMlpHidden; g.transA = 1;
    g.B = x_; g.ldb = kMlpInPad; g.transB = 1;
    g.cf = g_[0]; g.ldc = kMlpInPad;
    g.split_ws = split_ws_; g.split_floats = kSplitFloats;
    launch_gemm(g, stream_);
    launch_bias_grad(dh1_, n, kMlpHidden, kMlpHidden, g_[1], stream_);
}

bool Mlp::step(int n, float lr)
{
    backward(n);
    step_++;
    for (int t = 0; t < 6; t++)
        launch_adam(w_[t], m_[t], v_[t], g_[t], (t % 2 == 0) ? w16_[t / 2] : nullptr, (int)kSizes[t], lr,
                    0.9f, 0.999f, 1e-8f, step_, stream_);
    return cuda_ok(cudaGetLastError(), "train step");
}

bool Mlp::load_batch_host(int n, const float *X, const int32_t *labels)
{
    if (n <= 0 || n > max_batch_) {
        set_error("mlp: batch size out of range");
        return false;
    }
    // rows of kMlpIn floats -> padded bf16 rows
    std::vector<float> pad((size_t)n * kMlpInPad, 0.0f);
    for (int r = 0; r < n; r++)
        memcpy(&pad[(size_t)r * kMlpInPad], X + (size_t)r * kMlpIn, sizeof(float) * kMlpIn);
    bool ok = cuda_ok(cudaMemcpyAsync(xf_, pad.data(), sizeof(float) * pad.size(), cudaMemcpyHostToDevice,
                                      stream_), "batch upload");
    launch_f32_to_bf16(xf_, x_, (int)pad.size(), stream_);
    if (labels)
        ok = ok && cuda_ok(cudaMemcpyAsync(labels_, labels, sizeof(int32_t) * n, cudaMemcpyHostToDevice,
                                           stream_), "label upload");
    return ok;
}

bool Mlp::train(const __nv_bfloat16 *X, const int32_t *labels, int n_total, int epochs, int batch,
                float lr, uint64_t seed, float *last_loss)
{
    if (batch <= 0 || batch > max_batch_ || n_total < batch) {
        set_error("mlp: bad training sizes");
        return false;
    }
    std::mt19937_64 rng(seed);
    std::vector<int32_t> perm(n_total);
    if (n_total > perm_cap_) {
        cudaFree(perm_);
        perm_ = nullptr;
        perm_cap_ = 0;
        if (!cuda_ok(cudaMalloc(&perm_, sizeof(int32_t) * (size_t)n_total), "permutation"))
            return false;
        perm_cap_ = n_total;
    }
    if (!ctl_ && !cuda_ok(cudaMalloc(&ctl_, 2 * sizeof(int)), "training control"))
        return false;
    // One training step as a CUDA graph: the gather of the batch (its offset
    // in the epoch's order, ctl_[0], read on the device), forward, backward,
    // Adam (the step number ctl_[1] read on the device) and the advance of
    // both; one graph launch per batch.
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (!cuda_ok(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "step capture"))
        return false;
    launch_gather_rows(X, labels, perm_, batch, x_, labels_, stream_, ctl_);
    backward(batch);
    for (int t = 0; t < 6; t++)
        launch_adam(w_[t], m_[t], v_[t], g_[t], (t % 2 == 0) ? w16_[t / 2] : nullptr, (int)kSizes[t], lr,
                    0.9f, 0.999f, 1e-8f, 1, stream_, ctl_ + 1);
    launch_train_advance(ctl_, ctl_ + 1, batch, stream_);
    const cudaError_t cap = cudaStreamEndCapture(stream_, &graph);
    if (!cuda_ok(cap, "step capture") || !cuda_ok(cudaGraphInstantiate(&exec, graph, 0), "step graph")) {
        if (graph)
            cudaGraphDestroy(graph);
        return false;
    }
    cudaGraphDestroy(graph);
    float loss = 0.0f;
    bool ok = true;
    for (int e = 0; e < epochs && ok; e++) {
        for (int i = 0; i < n_total; i++)
            perm[i] = i;
        std::shuffle(perm.begin(), perm.end(), rng);
        // the epoch's order goes to the device once; each batch gathers its rows
        const int ctl[2] = {0, step_ + 1};
        ok = cuda_ok(cudaMemcpyAsync(perm_, perm.data(), sizeof(int32_t) * (size_t)n_total,
                                     cudaMemcpyHostToDevice, stream_), "permutation upload") &&
             cuda_ok(cudaMemcpyAsync(ctl_, ctl, sizeof(ctl), cudaMemcpyHostToDevice, stream_), "step control");
        for (int b0 = 0; ok && b0 + batch <= n_total; b0 += batch) {
            ok = cuda_ok(cudaGraphLaunch(exec, stream_), "train step");
            step_++;
        }
        ok = ok && cuda_ok(cudaMemcpyAsync(&loss, loss_, sizeof(float), cudaMemcpyDeviceToHost, stream_), "loss") &&
             cuda_ok(cudaStreamSynchronize(stream_), "epoch") && gemm_ok();
    }
    cudaGraphExecDestroy(exec);
    if (ok && last_loss)
        *last_loss = loss / batch;
    return ok;
}

}  // namespace frrt

using namespace frrt;

extern "C" {

void *fastrrt_mlp_create(uint64_t seed, int max_batch)
{
    if (max_batch <= 0) {
        set_error("mlp: max_batch must be positive");
        return nullptr;
    }
    auto *m = new (std::nothrow) Mlp(seed, max_batch);
    if (!m || !m->ok()) {
        delete m;
        return nullptr;
    }
    return m;
}

void fastrrt_mlp_destroy(void *mlp) { delete static_cast<Mlp *>(mlp); }

int fastrrt_mlp_get_weights(void *mlp, float *w1, float *b1, float *w2, float *b2, float *w3, float *b3)
{
    auto *m = static_cast<Mlp *>(mlp);
    if (!m)
        return -1;
    float *out[6] = {w1, b1, w2, b2, w3, b3};
    for (int t = 0; t < 6; t++)
        if (out[t] && !cuda_ok(cudaMemcpy(out[t], m->master(t), sizeof(float) * Mlp::kSizes[t],
                                          cudaMemcpyDeviceToHost), "weights download"))
            return -1;
    return 0;
}

int fastrrt_mlp_set_weights(void *mlp, const float *w1, const float *b1, const float *w2,
                            const float *b2, const float *w3, const float *b3)
{
    auto *m = static_cast<Mlp *>(mlp);
    if (!m)
        return -1;
    const float *in[6] = {w1, b1, w2, b2, w3, b3};
    for (int t = 0; t < 6; t++)
        if (in[t] && !cuda_ok(cudaMemcpy(m->master(t), in[t], sizeof(float) * Mlp::kSizes[t],
                                         cudaMemcpyHostToDevice), "weights upload"))
            return -1;
    return m->refresh() ? 0 : -1;
}

int fastrrt_mlp_forward(void *mlp, int n, const float *X, float *logits)
{
    auto *m = static_cast<Mlp *>(mlp);
    if (!m || !X || !logits || !m->load_batch_host(n, X, nullptr))
        return -1;
    m->forward(m->x(), n, m->stream(), m->logits(), m->h1(), m->h2(), nullptr);
    return cuda_ok(cudaMemcpyAsync(logits, m->logits(), sizeof(float) * n * kMlpOut,
                                   cudaMemcpyDeviceToHost, m->stream()), "logits") &&
                   cuda_ok(cudaStreamSynchronize(m->stream()), "forward") && gemm_ok()
               ? 0
               : -1;
}

int fastrrt_mlp_gradients(void *mlp, int n, const float *X, const int32_t *labels, float *gw1,
                          float *gb1, float *gw2, float *gb2, float *gw3, float *gb3, float *loss)
{
    auto *m = static_cast<Mlp *>(mlp);
    if (!m || !X || !labels || !m->load_batch_host(n, X, labels))
        return -1;
    m->backward(n);
    float *out[6] = {gw1, gb1, gw2, gb2, gw3, gb3};
    for (int t = 0; t < 6; t++)
        if (out[t] && !cuda_ok(cudaMemcpyAsync(out[t], m->grad(t), sizeof(float) * Mlp::kSizes[t],
                                               cudaMemcpyDeviceToHost, m->stream()), "gradients"))
            return -1;
    float l = 0.0f;
    if (!cuda_ok(cudaMemcpyAsync(&l, m->loss(), sizeof(float), cudaMemcpyDeviceToHost, m->stream()),
                 "loss") ||
        !cuda_ok(cudaStreamSynchronize(m->stream()), "gradients") || !gemm_ok())
        return -1;
    if (loss)
        *loss = l / n;
    return 0;
}

int fastrrt_gemm_bf16(int M, int N, int K, const void *A, int lda, int transA, const void *B, int ldb,
                      int transB, const float *bias, int relu, const void *mask, int ldm, float *Cf, void *Cb,
                      int ldc, const int *dM, float *split_ws, uint64_t split_floats, void *stream)
{
    if (M < 0 || N < 0 || K <= 0 || !A || !B || (!Cf) == (!Cb) || ldc < N ||
        lda < (transA ? M : K) || ldb < (transB ? N : K) || (mask && ldm < N)) {
        set_error("gemm: bad arguments");
        return -1;
    }
    if (!umma_init())
        return gemm_ok() ? 0 : -1;
    GemmArgs g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.dM = dM;
    g.A = static_cast<const __nv_bfloat16 *>(A);
    g.lda = lda;
    g.transA = transA;
    g.B = static_cast<const __nv_bfloat16 *>(B);
    g.ldb = ldb;
    g.transB = transB;
    g.bias = bias;
    g.relu = relu;
    g.mask = static_cast<const __nv_bfloat16 *>(mask);
    g.ldm = ldm;
    g.cf = Cf;
    g.cb = static_cast<__nv_bfloat16 *>(Cb);
    g.ldc = ldc;
    g.split_ws = split_ws;
    g.split_floats = split_ws ? (size_t)split_floats : 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    launch_gemm(g, st);
    return cuda_ok(cudaGetLastError(), "gemm launch") && cuda_ok(cudaStreamSynchronize(st), "gemm") &&
                   gemm_ok()
               ? 0
               : -1;
}

int fastrrt_mlp_train(void *mlp, const void *X_bf16, const int32_t *labels, int n, int epochs,
                      int batch, float lr, uint64_t seed, float *last_loss)
{
    auto *m = static_cast<Mlp *>(mlp);
    if (!m || !X_bf16 || !labels)
        return -1;
    return m->train(static_cast<const __nv_bfloat16 *>(X_bf16), labels, n, epochs, batch, lr, seed,
                    last_loss)
               ? 0
               : -1;
}

}  // extern "C"
