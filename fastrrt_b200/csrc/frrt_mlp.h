// frrt_mlp.h -- host object of the learned expansion proposal's network.
#pragma once
#include <cstdint>

#include "frrt_mlp.cuh"

namespace frrt {

// The network with FP32 master weights, Adam moments, BF16 compute copies
// and the scratch of one batch (max_batch rows).
class Mlp {
public:
    static const size_t kSizes[6];  // w1, b1, w2, b2, w3, b3

    Mlp(uint64_t seed, int max_batch);
    ~Mlp();
    bool ok() const { return ok_; }
    // BF16 copies of the master weights
    bool refresh();
    MlpWeights weights() const;
    // logits (n x 128, f32) of X (n x kMlpInPad bf16); d_count: a device row
    // count that caps n (graph launches size for n, run for *d_count)
    void forward(const __nv_bfloat16 *X, int n, cudaStream_t st, float *logits, __nv_bfloat16 *h1,
                 __nv_bfloat16 *h2, const int *d_count) const;
    // forward + backward of the batch in x() / labels: gradients in grad(t)
    void backward(int n);
    bool step(int n, float lr);
    bool load_batch_host(int n, const float *X, const int32_t *labels);
    bool train(const __nv_bfloat16 *X, const int32_t *labels, int n_total, int epochs, int batch,
               float lr, uint64_t seed, float *last_loss);

    float *master(int t) { return w_[t]; }
    float *grad(int t) { return g_[t]; }
    __nv_bfloat16 *x() { return x_; }
    float *logits() { return logits_; }
    __nv_bfloat16 *h1() { return h1_; }
    __nv_bfloat16 *h2() { return h2_; }
    float *loss() { return loss_; }
    cudaStream_t stream() const { return stream_; }
    int max_batch() const { return max_batch_; }

private:
    bool ok_ = false;
    int max_batch_ = 0;
    int step_ = 0;
    cudaStream_t stream_ = nullptr;
    float *w_[6] = {}, *m_[6] = {}, *v_[6] = {}, *g_[6] = {};
    __nv_bfloat16 *w16_[3] = {};
    __nv_bfloat16 *x_ = nullptr, *h1_ = nullptr, *h2_ = nullptr, *dl_ = nullptr, *dh2_ = nullptr,
                  *dh1_ = nullptr;
    float *logits_ = nullptr, *loss_ = nullptr, *xf_ = nullptr;
    int32_t *labels_ = nullptr;
    float *split_ws_ = nullptr;  // the weight gradients' split-over-K partial sums
    int32_t *perm_ = nullptr;    // an epoch's row order on the device
    int perm_cap_ = 0;
    int *ctl_ = nullptr;         // captured training step: batch offset, step number
};

}  // namespace frrt
