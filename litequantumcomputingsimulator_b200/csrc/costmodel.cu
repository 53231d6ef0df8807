// costmodel.cu — a small FP32 MLP that predicts the device time of one device operation,
// trained on the GPU by hand-written forward / backward / Adam kernels.
//
// Network: x (kCostFeatures) -> 64 ReLU -> 64 ReLU -> 1, predicting log(time in ms per
// 2^24 amplitudes).  Parameters are one flat FP32 array: W1 [64][F], b1 [64], W2 [64][64],
// b2 [64], W3 [64], b3 [1].  Every reduction over samples runs in a fixed order (one thread
// per parameter looping over the samples), so training is deterministic.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "costmodel.hpp"
#include "engine.hpp"

namespace lqcs_b200 {

namespace {

constexpr int F = kCostFeatures;
constexpr int Hd = kCostHidden;
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + Hd * F;
constexpr int OFF_W2 = OFF_B1 + Hd;
constexpr int OFF_B2 = OFF_W2 + Hd * Hd;
constexpr int OFF_W3 = OFF_B2 + Hd;
constexpr int OFF_B3 = OFF_W3 + Hd;

void check_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string("CUDA launch failed in ") + what + ": " +
                                 cudaGetErrorString(e));
    }
    count_launch();
}

// Forward, one thread per sample: keeps pre-activations for the backward pass.
__global__ void k_mlp_forward(const float* __restrict__ x, const float* __restrict__ w,
                              uint32_t n, float* __restrict__ a1, float* __restrict__ a2,
                              float* __restrict__ y) {
    __shared__ float sw[kCostParams];
    for (int i = threadIdx.x; i < kCostParams; i += blockDim.x) sw[i] = w[i];
    __syncthreads();
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float xi[F];
#pragma unroll
    for (int f = 0; f < F; ++f) xi[f] = x[s * F + f];
    float h1[Hd];
#pragma unroll
    for (int j = 0; j < Hd; ++j) {
        float acc = sw[OFF_B1 + j];
#pragma unroll
        for (int f = 0; f < F; ++f) acc = fmaf(sw[OFF_W1 + j * F + f], xi[f], acc);
        if (a1) a1[static_cast<uint64_t>(s) * Hd + j] = acc;
        h1[j] = fmaxf(acc, 0.0f);
    }
    float out = sw[OFF_B3];
    for (int j = 0; j < Hd; ++j) {
        float acc = sw[OFF_B2 + j];
#pragma unroll
        for (int i = 0; i < Hd; ++i) acc = fmaf(sw[OFF_W2 + j * Hd + i], h1[i], acc);
        if (a2) a2[static_cast<uint64_t>(s) * Hd + j] = acc;
        out = fmaf(sw[OFF_W3 + j], fmaxf(acc, 0.0f), out);
    }
    y[s] = out;
}

// Backward through the output and hidden layers, one thread per sample:
// g2[s][j] = dL/d(pre-activation of layer 2), g1[s][i] = dL/d(pre-activation of layer 1).
// Loss = mean((y - t)^2).
__global__ void k_mlp_backward_samples(const float* __restrict__ w, const float* __restrict__ y,
                                       const float* __restrict__ t, const float* __restrict__ a1,
                                       const float* __restrict__ a2, uint32_t n,
                                       float* __restrict__ dy, float* __restrict__ g1,
                                       float* __restrict__ g2) {
    __shared__ float sw[kCostParams];
    for (int i = threadIdx.x; i < kCostParams; i += blockDim.x) sw[i] = w[i];
    __syncthreads();
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float d = 2.0f * (y[s] - t[s]) / static_cast<float>(n);
    dy[s] = d;
    float gg2[Hd];
#pragma unroll
    for (int j = 0; j < Hd; ++j) {
        const float pre = a2[static_cast<uint64_t>(s) * Hd + j];
        gg2[j] = pre > 0.0f ? d * sw[OFF_W3 + j] : 0.0f;
        g2[static_cast<uint64_t>(s) * Hd + j] = gg2[j];
    }
    for (int i = 0; i < Hd; ++i) {
        const float pre = a1[static_cast<uint64_t>(s) * Hd + i];
        float acc = 0.0f;
        if (pre > 0.0f) {
#pragma unroll
            for (int j = 0; j < Hd; ++j) acc = fmaf(gg2[j], sw[OFF_W2 + j * Hd + i], acc);
        }
        g1[static_cast<uint64_t>(s) * Hd + i] = acc;
    }
}

// One thread per parameter: the gradient summed over the samples in sample order.
__global__ void k_mlp_param_grads(const float* __restrict__ x, const float* __restrict__ a1,
                                  const float* __restrict__ a2, const float* __restrict__ dy,
                                  const float* __restrict__ g1, const float* __restrict__ g2,
                                  uint32_t n, float* __restrict__ grad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kCostParams) return;
    float acc = 0.0f;
    if (p < OFF_B1) {                       // W1[j][f]
        const int j = (p - OFF_W1) / F, f = (p - OFF_W1) % F;
        for (uint32_t s = 0; s < n; ++s) acc = fmaf(g1[static_cast<uint64_t>(s) * Hd + j], x[s * F + f], acc);
    } else if (p < OFF_W2) {                // b1[j]
        const int j = p - OFF_B1;
        for (uint32_t s = 0; s < n; ++s) acc += g1[static_cast<uint64_t>(s) * Hd + j];
    } else if (p < OFF_B2) {                // W2[j][i]
        const int j = (p - OFF_W2) / Hd, i = (p - OFF_W2) % Hd;
        for (uint32_t s = 0; s < n; ++s)
            acc = fmaf(g2[static_cast<uint64_t>(s) * Hd + j],
                       fmaxf(a1[static_cast<uint64_t>(s) * Hd + i], 0.0f), acc);
    } else if (p < OFF_W3) {                // b2[j]
        const int j = p - OFF_B2;
        for (uint32_t s = 0; s < n; ++s) acc += g2[static_cast<uint64_t>(s) * Hd + j];
    } else if (p < OFF_B3) {                // W3[j]
        const int j = p - OFF_W3;
        for (uint32_t s = 0; s < n; ++s)
            acc = fmaf(dy[s], fmaxf(a2[static_cast<uint64_t>(s) * Hd + j], 0.0f), acc);
    } else {                                // b3
        for (uint32_t s = 0; s < n; ++s) acc += dy[s];
    }
    grad[p] = acc;
}

// Adam step (bias-corrected), one thread per parameter.
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1t, float b2t) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kCostParams) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    m[p] = b1 * m[p] + (1.0f - b1) * g[p];
    v[p] = b2 * v[p] + (1.0f - b2) * g[p] * g[p];
    const float mh = m[p] / (1.0f - b1t), vh = v[p] / (1.0f - b2t);
    w[p] -= lr * mh / (sqrtf(vh) + eps);
}

// Mean squared error of y against t, one block, fixed order.
__global__ void k_mse(const float* __restrict__ y, const float* __restrict__ t, uint32_t n,
                      float* __restrict__ out) {
    __shared__ float sh[256];
    float acc = 0.0f;
    for (uint32_t s = threadIdx.x; s < n; s += blockDim.x) {
        const float d = y[s] - t[s];
        acc = fmaf(d, d, acc);
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float tot = 0.0f;
        for (int i = 0; i < 256; ++i) tot += sh[i];
        out[0] = tot / static_cast<float>(n);
    }
}

struct Model {
    std::vector<float> w;   // host copy of the trained parameters
    bool trained = false;
    uint64_t version = 0;   // bumped whenever the weights change
};
std::mutex g_mu;
Model g_model;

struct Buffers {
    DeviceBuffer x, t, y, a1, a2, dy, g1, g2, w, grad, m, v, loss;
    void ensure(uint32_t n) {
        x.ensure(sizeof(float) * n * F);
        t.ensure(sizeof(float) * n);
        y.ensure(sizeof(float) * n);
        a1.ensure(sizeof(float) * n * Hd);
        a2.ensure(sizeof(float) * n * Hd);
        dy.ensure(sizeof(float) * n);
        g1.ensure(sizeof(float) * n * Hd);
        g2.ensure(sizeof(float) * n * Hd);
        w.ensure(sizeof(float) * kCostParams);
        grad.ensure(sizeof(float) * kCostParams);
        m.ensure(sizeof(float) * kCostParams);
        v.ensure(sizeof(float) * kCostParams);
        loss.ensure(sizeof(float));
    }
};

std::vector<float> init_weights(uint64_t seed) {
    std::mt19937_64 eng(seed);
    std::normal_distribution<float> nd(0.0f, 1.0f);
    std::vector<float> w(kCostParams, 0.0f);
    const float s1 = std::sqrt(2.0f / F), s2 = std::sqrt(2.0f / Hd), s3 = std::sqrt(1.0f / Hd);
    for (int i = 0; i < Hd * F; ++i) w[OFF_W1 + i] = nd(eng) * s1;
    for (int i = 0; i < Hd * Hd; ++i) w[OFF_W2 + i] = nd(eng) * s2;
    for (int i = 0; i < Hd; ++i) w[OFF_W3 + i] = nd(eng) * s3;
    return w;
}

void forward_backward(Buffers& b, uint32_t n, const LaunchCtx& ctx) {
    const uint32_t blocks = (n + 127) / 128;
    k_mlp_forward<<<blocks, 128, 0, ctx.stream>>>(b.x.as<float>(), b.w.as<float>(), n,
                                                  b.a1.as<float>(), b.a2.as<float>(), b.y.as<float>());
    check_launch("mlp_forward");
    k_mlp_backward_samples<<<blocks, 128, 0, ctx.stream>>>(b.w.as<float>(), b.y.as<float>(),
                                                           b.t.as<float>(), b.a1.as<float>(),
                                                           b.a2.as<float>(), n, b.dy.as<float>(),
                                                           b.g1.as<float>(), b.g2.as<float>());
    check_launch("mlp_backward");
    k_mlp_param_grads<<<(kCostParams + 255) / 256, 256, 0, ctx.stream>>>(
        b.x.as<float>(), b.a1.as<float>(), b.a2.as<float>(), b.dy.as<float>(), b.g1.as<float>(),
        b.g2.as<float>(), n, b.grad.as<float>());
    check_launch("mlp_param_grads");
}

}  // namespace

float costmodel_train(const float* features, const float* targets, uint64_t n, uint32_t epochs,
                      float lr, uint64_t seed) {
    if (n == 0) invalid("costmodel_train: no samples");
    if (n > (uint64_t{1} << 24)) invalid("costmodel_train: too many samples");
    const LaunchCtx ctx = make_ctx(nullptr);
    Buffers b;
    b.ensure(static_cast<uint32_t>(n));
    cuda_check(cudaMemcpy(b.x.ptr, features, sizeof(float) * n * F, cudaMemcpyHostToDevice), "H2D");
    cuda_check(cudaMemcpy(b.t.ptr, targets, sizeof(float) * n, cudaMemcpyHostToDevice), "H2D");
    const std::vector<float> w0 = init_weights(seed);
    cuda_check(cudaMemcpy(b.w.ptr, w0.data(), sizeof(float) * kCostParams, cudaMemcpyHostToDevice), "H2D");
    cuda_check(cudaMemset(b.m.ptr, 0, sizeof(float) * kCostParams), "memset");
    cuda_check(cudaMemset(b.v.ptr, 0, sizeof(float) * kCostParams), "memset");
    float b1t = 1.0f, b2t = 1.0f;
    for (uint32_t e = 0; e < epochs; ++e) {
        forward_backward(b, static_cast<uint32_t>(n), ctx);
        b1t *= 0.9f;
        b2t *= 0.999f;
        k_adam<<<(kCostParams + 255) / 256, 256, 0, ctx.stream>>>(b.w.as<float>(), b.grad.as<float>(),
                                                                 b.m.as<float>(), b.v.as<float>(),
                                                                 lr, b1t, b2t);
        check_launch("adam");
    }
    // final loss with the trained weights
    k_mlp_forward<<<(static_cast<uint32_t>(n) + 127) / 128, 128, 0, ctx.stream>>>(
        b.x.as<float>(), b.w.as<float>(), static_cast<uint32_t>(n), nullptr, nullptr, b.y.as<float>());
    check_launch("mlp_forward");
    k_mse<<<1, 256, 0, ctx.stream>>>(b.y.as<float>(), b.t.as<float>(), static_cast<uint32_t>(n),
                                     b.loss.as<float>());
    check_launch("mse");
    float loss = 0.0f;
    std::vector<float> w(kCostParams);
    cuda_check(cudaMemcpy(&loss, b.loss.ptr, sizeof(float), cudaMemcpyDeviceToHost), "D2H");
    cuda_check(cudaMemcpy(w.data(), b.w.ptr, sizeof(float) * kCostParams, cudaMemcpyDeviceToHost), "D2H");
    std::lock_guard<std::mutex> lk(g_mu);
    g_model.w = std::move(w);
    g_model.trained = true;
    ++g_model.version;
    return loss;
}

void costmodel_predict(const float* features, uint64_t n, float* out) {
    std::vector<float> w;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_model.trained) invalid("costmodel: no trained weights (train or set them first)");
        w = g_model.w;
    }
    if (n == 0) return;
    const LaunchCtx ctx = make_ctx(nullptr);
    DeviceBuffer dx, dw, dy;
    dx.ensure(sizeof(float) * n * F);
    dw.ensure(sizeof(float) * kCostParams);
    dy.ensure(sizeof(float) * n);
    cuda_check(cudaMemcpy(dx.ptr, features, sizeof(float) * n * F, cudaMemcpyHostToDevice), "H2D");
    cuda_check(cudaMemcpy(dw.ptr, w.data(), sizeof(float) * kCostParams, cudaMemcpyHostToDevice), "H2D");
    k_mlp_forward<<<(static_cast<uint32_t>(n) + 127) / 128, 128, 0, ctx.stream>>>(
        dx.as<float>(), dw.as<float>(), static_cast<uint32_t>(n), nullptr, nullptr, dy.as<float>());
    check_launch("mlp_forward");
    cuda_check(cudaMemcpy(out, dy.ptr, sizeof(float) * n, cudaMemcpyDeviceToHost), "D2H");
}

float costmodel_grad(const float* features, const float* targets, uint64_t n, float* grad_out) {
    std::vector<float> w;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_model.trained) invalid("costmodel: no trained weights (train or set them first)");
        w = g_model.w;
    }
    const LaunchCtx ctx = make_ctx(nullptr);
    Buffers b;
    b.ensure(static_cast<uint32_t>(n));
    cuda_check(cudaMemcpy(b.x.ptr, features, sizeof(float) * n * F, cudaMemcpyHostToDevice), "H2D");
    cuda_check(cudaMemcpy(b.t.ptr, targets, sizeof(float) * n, cudaMemcpyHostToDevice), "H2D");
    cuda_check(cudaMemcpy(b.w.ptr, w.data(), sizeof(float) * kCostParams, cudaMemcpyHostToDevice), "H2D");
    forward_backward(b, static_cast<uint32_t>(n), ctx);
    k_mse<<<1, 256, 0, ctx.stream>>>(b.y.as<float>(), b.t.as<float>(), static_cast<uint32_t>(n),
                                     b.loss.as<float>());
    check_launch("mse");
    float loss = 0.0f;
    cuda_check(cudaMemcpy(&loss, b.loss.ptr, sizeof(float), cudaMemcpyDeviceToHost), "D2H");
    cuda_check(cudaMemcpy(grad_out, b.grad.ptr, sizeof(float) * kCostParams, cudaMemcpyDeviceToHost), "D2H");
    return loss;
}

std::vector<float> costmodel_weights() {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_model.trained) invalid("costmodel: no trained weights");
    return g_model.w;
}

void costmodel_set_weights(const float* w, uint64_t n) {
    if (n != static_cast<uint64_t>(kCostParams)) invalid("costmodel: expected " + std::to_string(kCostParams) + " weights");
    std::lock_guard<std::mutex> lk(g_mu);
    g_model.w.assign(w, w + n);
    g_model.trained = true;
    ++g_model.version;
}

std::array<float, kCostFeatures> op_features(uint32_t kind, uint32_t width, uint32_t min_target,
                                             uint32_t max_target, uint32_t gates, uint32_t n,
                                             double flops_per_amp) {
    return {static_cast<float>(kind) / 6.0f, static_cast<float>(width) / 8.0f,
            static_cast<float>(min_target) / 32.0f, static_cast<float>(max_target) / 32.0f,
            std::log2(1.0f + static_cast<float>(gates)) / 8.0f, static_cast<float>(n) / 32.0f,
            static_cast<float>(std::log2(1.0 + std::max(0.0, flops_per_amp))) / 10.0f};
}

std::array<float, kCostFeatures> op_features(const DevOp& op, uint32_t n) {
    uint64_t mask = op.cmask | op.phase_mask | op.x | op.zy;
    for (uint32_t t : op.targets) mask |= uint64_t{1} << t;
    const uint32_t lo = mask ? static_cast<uint32_t>(__builtin_ctzll(mask)) : 0;
    const uint32_t hi = mask ? 63u - static_cast<uint32_t>(__builtin_clzll(mask)) : 0;
    return op_features(profile_kind(op), op.k, lo, hi, op.src_gates, n, op_flops_per_amp(op));
}

double predict_ops_ms(const std::vector<DevOp>& ops, uint32_t n) {
    if (ops.empty()) return 0.0;
    std::vector<float> x;
    x.reserve(ops.size() * kCostFeatures);
    for (const DevOp& op : ops) {
        const auto f = op_features(op, n);
        x.insert(x.end(), f.begin(), f.end());
    }
    std::vector<float> y(ops.size());
    costmodel_predict(x.data(), ops.size(), y.data());
    double ms = 0.0;
    for (float v : y) ms += std::exp(static_cast<double>(v));
    return ms * std::ldexp(1.0, static_cast<int>(n) - 24);
}

bool costmodel_trained() {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_model.trained;
}

void costmodel_clear() {
    std::lock_guard<std::mutex> lk(g_mu);
    g_model.w.clear();
    g_model.trained = false;
    ++g_model.version;
}

uint64_t costmodel_version() {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_model.version;
}

}  // namespace lqcs_b200
