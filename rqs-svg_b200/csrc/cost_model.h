// Learned cost model of fused passes (cost_model.cu).
#pragma once

#include "qcs_internal.h"

#include <vector>

namespace qcsb
{

class CostModel
{
  public:
    static constexpr int kInputs = 6;
    static constexpr int kHidden = 64;
    static constexpr int kParams = kHidden * kInputs + kHidden + kHidden * kHidden + kHidden + kHidden + 1;
    static constexpr int kScaling = 2 * kInputs + 2;

    explicit CostModel(uint32_t seed);
    ~CostModel();
    CostModel(const CostModel &) = delete;
    CostModel &operator=(const CostModel &) = delete;

    // Adam on mini-batches (one CUDA graph per step); returns the final
    // mean squared error on the standardised training set.
    float train(const float *features, const float *targets, int n, int epochs, int batch, float lr, uint32_t seed);
    // features in physical units -> targets in physical units
    void predict(const float *features, int n, float *out);
    // Gradient of the mean squared error w.r.t. all parameters for
    // already-standardised inputs and targets; returns the loss.
    float gradients(const float *x_std, const float *t_std, int n, float *grads_out);

    void get_params(float *out) const;
    void set_params(const float *in);
    // in_mean[4], in_std[4], out_mean, out_std
    void get_scaling(float *out) const;
    void set_scaling(const float *in);
    bool trained() const { return trained_; }

  private:
    void ensure_batch(int B);
    void release_batch();
    void forward(const float *X, int B, float *Y);
    void backward(int B);
    void fit_scaling(const float *features, const float *targets, int n);
    void standardise(const float *features, const float *targets, int n, std::vector<float> &x,
                     std::vector<float> &t) const;
    void predict_standardised(const float *x_std, int n, float *out);
    float evaluate_loss(const float *x_std, const float *t_std, int n);

    cudaStream_t stream_ = nullptr;
    float *params_ = nullptr;
    float *data_x_ = nullptr, *data_t_ = nullptr;
    int batch_cap_ = 0;
    float *xb_ = nullptr, *tb_ = nullptr, *z1_ = nullptr, *h1_ = nullptr, *z2_ = nullptr, *h2_ = nullptr;
    float *y_ = nullptr, *dy_ = nullptr, *dh2_ = nullptr, *dh1_ = nullptr, *sq_ = nullptr;
    float *grads_ = nullptr, *m_ = nullptr, *v_ = nullptr, *scale_ = nullptr;
    int *index_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    float in_mean_[kInputs], in_std_[kInputs];
    float out_mean_ = 0.0f, out_std_ = 1.0f;
    bool trained_ = false;
};

} // namespace qcsb
