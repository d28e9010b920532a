// Learned cost model of fused passes: a 6 -> 64 -> 64 -> 1 FP32 MLP with
// ReLU activations, trained on the GPU by the kernels below (forward,
// backward, Adam) on pass timings the simulator records itself.
//
// Inputs (per pass, PassFeatures): block width (1: gates one by one on the
// register path; 3, 4: 8 x 8 or 16 x 16 tensor stages), blocks (stages),
// arithmetic gates, light ops (diagonal phases and permutations), the
// target-qubit stride (log2 of the largest local qubit's stride) and log2 of
// the chunk count (capped). Target: log(device time per amplitude in ns).
// Inputs and target are standardised with the training set's mean and
// deviation.
//
// Parameter layout (one float buffer): W1[64x6], b1[64], W2[64x64], b2[64],
// W3[64], b3[1].
//
// One training step (gather a mini-batch, three layers forward, loss
// gradient, three layers backward, Adam) is captured once in a CUDA graph and
// replayed per mini-batch; the mini-batch indices are written to a device
// buffer the graph reads.

#include "cost_model.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>

namespace qcsb
{
namespace
{

constexpr int kIn = CostModel::kInputs;
constexpr int kHid = CostModel::kHidden;
constexpr int kW1 = 0, kB1 = kW1 + kHid * kIn, kW2 = kB1 + kHid, kB2 = kW2 + kHid * kHid, kW3 = kB2 + kHid,
              kB3 = kW3 + kHid, kParams = kB3 + 1;
static_assert(kParams == CostModel::kParams, "parameter layout");

constexpr int kThreads = 256;

// Z[b, o] = sum_i X[b, i] W[o, i] + bias[o]; H = relu(Z) when relu.
__global__ void linear_fwd_kernel(const float *X, int B, int K, const float *W, const float *bias, int N,
                                  float *Z, float *H)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * N)
        return;
    const int b = idx / N, o = idx % N;
    float acc = bias[o];
    for (int i = 0; i < K; ++i)
        acc = fmaf(X[b * K + i], W[o * K + i], acc);
    Z[idx] = acc;
    if (H)
        H[idx] = acc > 0.0f ? acc : 0.0f;
}

// dX[b, i] = sum_o dZ[b, o] W[o, i], then masked by relu'(Zprev) when given.
__global__ void linear_bwd_input_kernel(const float *dZ, int B, int N, const float *W, int K, const float *Zprev,
                                        float *dX)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * K)
        return;
    const int b = idx / K, i = idx % K;
    float acc = 0.0f;
    for (int o = 0; o < N; ++o)
        acc = fmaf(dZ[b * N + o], W[o * K + i], acc);
    if (Zprev && Zprev[idx] <= 0.0f)
        acc = 0.0f;
    dX[idx] = acc;
}

// dW[o, i] = sum_b dZ[b, o] X[b, i]; db[o] = sum_b dZ[b, o] (fixed order).
__global__ void linear_bwd_weight_kernel(const float *dZ, const float *X, int B, int N, int K, float *dW, float *db)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < N * K)
    {
        const int o = idx / K, i = idx % K;
        float acc = 0.0f;
        for (int b = 0; b < B; ++b)
            acc = fmaf(dZ[b * N + o], X[b * K + i], acc);
        dW[idx] = acc;
    }
    else if (idx < N * K + N)
    {
        const int o = idx - N * K;
        float acc = 0.0f;
        for (int b = 0; b < B; ++b)
            acc += dZ[b * N + o];
        db[o] = acc;
    }
}

// dY = 2 (Y - T) / B; loss partial per sample.
__global__ void mse_grad_kernel(const float *Y, const float *T, int B, float *dY, float *sqerr)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B)
        return;
    const float d = Y[b] - T[b];
    dY[b] = 2.0f * d / B;
    sqerr[b] = d * d;
}

__global__ void gather_kernel(const float *X, const float *T, const int *index, int B, float *Xb, float *Tb)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B)
        return;
    const int s = index[b];
    for (int i = 0; i < kIn; ++i)
        Xb[b * kIn + i] = X[s * kIn + i];
    Tb[b] = T[s];
}

__global__ void adam_kernel(float *p, const float *g, float *m, float *v, int count, float lr, float b1, float b2,
                            const float *step_scale, float eps)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    // step_scale = {1 / (1 - b1^t), 1 / (1 - b2^t)} written by the host
    const float mh = mi * step_scale[0];
    const float vh = vi * step_scale[1];
    p[i] -= lr * mh / (sqrtf(vh) + eps);
}

unsigned blocks_for(int n) { return static_cast<unsigned>((n + kThreads - 1) / kThreads); }

} // namespace

CostModel::CostModel(uint32_t seed)
{
    // He-style initialisation on the host, copied once
    std::mt19937 rng(seed);
    std::vector<float> p(kParams, 0.0f);
    std::normal_distribution<float> n1(0.0f, std::sqrt(2.0f / kIn)), n2(0.0f, std::sqrt(2.0f / kHid));
    for (int i = 0; i < kHid * kIn; ++i)
        p[kW1 + i] = n1(rng);
    for (int i = 0; i < kHid * kHid; ++i)
        p[kW2 + i] = n2(rng);
    for (int i = 0; i < kHid; ++i)
        p[kW3 + i] = n2(rng);
    QCSB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    QCSB_CUDA(cudaMalloc(&params_, sizeof(float) * kParams));
    QCSB_CUDA(cudaMemcpy(params_, p.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice));
    for (int i = 0; i < kIn; ++i)
    {
        in_mean_[i] = 0.0f;
        in_std_[i] = 1.0f;
    }
}

CostModel::~CostModel()
{
    release_batch();
    if (graph_exec_)
        cudaGraphExecDestroy(graph_exec_);
    cudaFree(params_);
    cudaFree(data_x_);
    cudaFree(data_t_);
    if (stream_)
        cudaStreamDestroy(stream_);
}

void CostModel::release_batch()
{
    for (float *p : {xb_, tb_, z1_, h1_, z2_, h2_, y_, dy_, dh2_, dh1_, sq_, grads_, m_, v_, scale_})
        cudaFree(p);
    cudaFree(index_);
    xb_ = tb_ = z1_ = h1_ = z2_ = h2_ = y_ = dy_ = dh2_ = dh1_ = sq_ = grads_ = m_ = v_ = scale_ = nullptr;
    index_ = nullptr;
    batch_cap_ = 0;
}

void CostModel::ensure_batch(int B)
{
    if (B <= batch_cap_)
        return;
    release_batch();
    if (graph_exec_)
    {
        cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
    }
    auto alloc = [](float **p, size_t n) { QCSB_CUDA(cudaMalloc(p, sizeof(float) * n)); };
    alloc(&xb_, (size_t)B * kIn);
    alloc(&tb_, B);
    alloc(&z1_, (size_t)B * kHid);
    alloc(&h1_, (size_t)B * kHid);
    alloc(&z2_, (size_t)B * kHid);
    alloc(&h2_, (size_t)B * kHid);
    alloc(&y_, B);
    alloc(&dy_, B);
    alloc(&dh2_, (size_t)B * kHid);
    alloc(&dh1_, (size_t)B * kHid);
    alloc(&sq_, B);
    alloc(&grads_, kParams);
    alloc(&m_, kParams);
    alloc(&v_, kParams);
    alloc(&scale_, 2);
    QCSB_CUDA(cudaMalloc(&index_, sizeof(int) * B));
    QCSB_CUDA(cudaMemset(m_, 0, sizeof(float) * kParams));
    QCSB_CUDA(cudaMemset(v_, 0, sizeof(float) * kParams));
    batch_cap_ = B;
}

// Forward on B standardised rows in xb_ (writes z1, h1, z2, h2, y).
void CostModel::forward(const float *X, int B, float *Y)
{
    const float *P = params_;
    linear_fwd_kernel<<<blocks_for(B * kHid), kThreads, 0, stream_>>>(X, B, kIn, P + kW1, P + kB1, kHid, z1_, h1_);
    linear_fwd_kernel<<<blocks_for(B * kHid), kThreads, 0, stream_>>>(h1_, B, kHid, P + kW2, P + kB2, kHid, z2_, h2_);
    linear_fwd_kernel<<<blocks_for(B), kThreads, 0, stream_>>>(h2_, B, kHid, P + kW3, P + kB3, 1, Y, nullptr);
}

// Gradients of the mean squared error for the batch in xb_/tb_ into grads_.
void CostModel::backward(int B)
{
    float *G = grads_;
    const float *P = params_;
    mse_grad_kernel<<<blocks_for(B), kThreads, 0, stream_>>>(y_, tb_, B, dy_, sq_);
    linear_bwd_weight_kernel<<<blocks_for(kHid + 1), kThreads, 0, stream_>>>(dy_, h2_, B, 1, kHid, G + kW3, G + kB3);
    linear_bwd_input_kernel<<<blocks_for(B * kHid), kThreads, 0, stream_>>>(dy_, B, 1, P + kW3, kHid, z2_, dh2_);
    linear_bwd_weight_kernel<<<blocks_for(kHid * kHid + kHid), kThreads, 0, stream_>>>(dh2_, h1_, B, kHid, kHid, G + kW2, G + kB2);
    linear_bwd_input_kernel<<<blocks_for(B * kHid), kThreads, 0, stream_>>>(dh2_, B, kHid, P + kW2, kHid, z1_, dh1_);
    linear_bwd_weight_kernel<<<blocks_for(kHid * kIn + kHid), kThreads, 0, stream_>>>(dh1_, xb_, B, kHid, kIn, G + kW1, G + kB1);
}

void CostModel::standardise(const float *features, const float *targets, int n, std::vector<float> &x,
                            std::vector<float> &t) const
{
    x.resize((size_t)n * kIn);
    for (int s = 0; s < n; ++s)
        for (int i = 0; i < kIn; ++i)
            x[(size_t)s * kIn + i] = (features[(size_t)s * kIn + i] - in_mean_[i]) / in_std_[i];
    if (targets)
    {
        t.resize(n);
        for (int s = 0; s < n; ++s)
            t[s] = (targets[s] - out_mean_) / out_std_;
    }
}

void CostModel::fit_scaling(const float *features, const float *targets, int n)
{
    for (int i = 0; i < kIn; ++i)
    {
        double m = 0.0, v = 0.0;
        for (int s = 0; s < n; ++s)
            m += features[(size_t)s * kIn + i];
        m /= n;
        for (int s = 0; s < n; ++s)
        {
            const double d = features[(size_t)s * kIn + i] - m;
            v += d * d;
        }
        in_mean_[i] = static_cast<float>(m);
        const double sd = std::sqrt(v / n);
        in_std_[i] = static_cast<float>(sd > 1e-6 ? sd : 1.0);
    }
    double m = 0.0, v = 0.0;
    for (int s = 0; s < n; ++s)
        m += targets[s];
    m /= n;
    for (int s = 0; s < n; ++s)
        v += (targets[s] - m) * (targets[s] - m);
    out_mean_ = static_cast<float>(m);
    const double sd = std::sqrt(v / n);
    out_std_ = static_cast<float>(sd > 1e-6 ? sd : 1.0);
}

float CostModel::train(const float *features, const float *targets, int n, int epochs, int batch, float lr,
                       uint32_t seed)
{
    if (n <= 0 || batch <= 0 || epochs <= 0)
        throw std::runtime_error("cost model train: sample count, batch and epochs must be positive");
    batch = std::min(batch, n);
    fit_scaling(features, targets, n);
    std::vector<float> x, t;
    standardise(features, targets, n, x, t);
    cudaFree(data_x_);
    cudaFree(data_t_);
    QCSB_CUDA(cudaMalloc(&data_x_, sizeof(float) * x.size()));
    QCSB_CUDA(cudaMalloc(&data_t_, sizeof(float) * t.size()));
    QCSB_CUDA(cudaMemcpy(data_x_, x.data(), sizeof(float) * x.size(), cudaMemcpyHostToDevice));
    QCSB_CUDA(cudaMemcpy(data_t_, t.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice));
    ensure_batch(batch);
    QCSB_CUDA(cudaMemset(m_, 0, sizeof(float) * kParams));
    QCSB_CUDA(cudaMemset(v_, 0, sizeof(float) * kParams));

    // capture one training step for this batch size
    if (graph_exec_)
    {
        cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
    }
    constexpr float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    cudaGraph_t graph;
    QCSB_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    gather_kernel<<<blocks_for(batch), kThreads, 0, stream_>>>(data_x_, data_t_, index_, batch, xb_, tb_);
    forward(xb_, batch, y_);
    backward(batch);
    adam_kernel<<<blocks_for(kParams), kThreads, 0, stream_>>>(params_, grads_, m_, v_, kParams, lr, b1, b2, scale_, eps);
    QCSB_CUDA(cudaStreamEndCapture(stream_, &graph));
    QCSB_CUDA(cudaGraphInstantiate(&graph_exec_, graph, 0));
    QCSB_CUDA(cudaGraphDestroy(graph));

    std::mt19937 rng(seed);
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    int *idx_host = nullptr;
    float *scale_host = nullptr;
    QCSB_CUDA(cudaMallocHost(&idx_host, sizeof(int) * batch));
    QCSB_CUDA(cudaMallocHost(&scale_host, sizeof(float) * 2));
    long step = 0;
    const int steps_per_epoch = n / batch;
    for (int e = 0; e < epochs; ++e)
    {
        std::shuffle(order.begin(), order.end(), rng);
        for (int s = 0; s < steps_per_epoch; ++s)
        {
            ++step;
            QCSB_CUDA(cudaStreamSynchronize(stream_));   // pinned inputs are reused
            std::copy(order.begin() + (size_t)s * batch, order.begin() + (size_t)(s + 1) * batch, idx_host);
            scale_host[0] = static_cast<float>(1.0 / (1.0 - std::pow(double(b1), double(step))));
            scale_host[1] = static_cast<float>(1.0 / (1.0 - std::pow(double(b2), double(step))));
            QCSB_CUDA(cudaMemcpyAsync(index_, idx_host, sizeof(int) * batch, cudaMemcpyHostToDevice, stream_));
            QCSB_CUDA(cudaMemcpyAsync(scale_, scale_host, sizeof(float) * 2, cudaMemcpyHostToDevice, stream_));
            QCSB_CUDA(cudaGraphLaunch(graph_exec_, stream_));
        }
    }
    QCSB_CUDA(cudaStreamSynchronize(stream_));
    cudaFreeHost(idx_host);
    cudaFreeHost(scale_host);
    trained_ = true;
    // loss on the whole (standardised) training set
    return evaluate_loss(x.data(), t.data(), n);
}

float CostModel::evaluate_loss(const float *x_std, const float *t_std, int n)
{
    std::vector<float> pred(n);
    predict_standardised(x_std, n, pred.data());
    double s = 0.0;
    for (int i = 0; i < n; ++i)
        s += double(pred[i] - t_std[i]) * double(pred[i] - t_std[i]);
    return static_cast<float>(s / n);
}

void CostModel::predict_standardised(const float *x_std, int n, float *out)
{
    ensure_batch(std::min(std::max(n, 1), 1 << 16));
    const int cap = batch_cap_;
    for (int off = 0; off < n; off += cap)
    {
        const int B = std::min(cap, n - off);
        QCSB_CUDA(cudaMemcpyAsync(xb_, x_std + (size_t)off * kIn, sizeof(float) * B * kIn, cudaMemcpyHostToDevice, stream_));
        forward(xb_, B, y_);
        QCSB_CUDA(cudaMemcpyAsync(out + off, y_, sizeof(float) * B, cudaMemcpyDeviceToHost, stream_));
        QCSB_CUDA(cudaStreamSynchronize(stream_));
    }
}

void CostModel::predict(const float *features, int n, float *out)
{
    std::vector<float> x, t;
    standardise(features, nullptr, n, x, t);
    predict_standardised(x.data(), n, out);
    for (int i = 0; i < n; ++i)
        out[i] = out[i] * out_std_ + out_mean_;
}

float CostModel::gradients(const float *x_std, const float *t_std, int n, float *grads_out)
{
    ensure_batch(n);
    QCSB_CUDA(cudaMemcpyAsync(xb_, x_std, sizeof(float) * n * kIn, cudaMemcpyHostToDevice, stream_));
    QCSB_CUDA(cudaMemcpyAsync(tb_, t_std, sizeof(float) * n, cudaMemcpyHostToDevice, stream_));
    forward(xb_, n, y_);
    backward(n);
    std::vector<float> sq(n);
    QCSB_CUDA(cudaMemcpyAsync(grads_out, grads_, sizeof(float) * kParams, cudaMemcpyDeviceToHost, stream_));
    QCSB_CUDA(cudaMemcpyAsync(sq.data(), sq_, sizeof(float) * n, cudaMemcpyDeviceToHost, stream_));
    QCSB_CUDA(cudaStreamSynchronize(stream_));
    double s = 0.0;
    for (float v : sq)
        s += v;
    return static_cast<float>(s / n);
}

void CostModel::get_params(float *out) const
{
    QCSB_CUDA(cudaMemcpy(out, params_, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
}

void CostModel::set_params(const float *in)
{
    QCSB_CUDA(cudaMemcpy(params_, in, sizeof(float) * kParams, cudaMemcpyHostToDevice));
}

void CostModel::get_scaling(float *out) const
{
    for (int i = 0; i < kIn; ++i)
    {
        out[i] = in_mean_[i];
        out[kIn + i] = in_std_[i];
    }
    out[2 * kIn] = out_mean_;
    out[2 * kIn + 1] = out_std_;
}

void CostModel::set_scaling(const float *in)
{
    for (int i = 0; i < kIn; ++i)
    {
        in_mean_[i] = in[i];
        in_std_[i] = in[kIn + i];
    }
    out_mean_ = in[2 * kIn];
    out_std_ = in[2 * kIn + 1];
    trained_ = true;
}

} // namespace qcsb
