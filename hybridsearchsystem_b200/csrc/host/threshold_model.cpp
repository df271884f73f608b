// threshold_model.cpp -- ThresholdModel: the learned K-th-score predictor's parameters, optimiser
// state and activations on one GPU, driven by the kernels of mlp.cu.
//
// Parameters are one flat FP32 vector: W1 [din][H], b1 [H], W2 [H][H], b2 [H], w3 [H], b3 [1].
// The network predicts a standardised target; `scale` and `shift` map it back to a score.
#include <cmath>
#include <cstring>
#include <random>

#include "../hss_kernels.h"
#include "hss_host.h"

namespace hss {

ThresholdModel::ThresholdModel(int32_t deviceId, uint32_t din, uint32_t hidden, uint64_t seed)
    : m_deviceId(deviceId), m_din(din), m_h(hidden) {
    if (din == 0 || hidden == 0 || din > (1u << 16) || hidden > 4096) {
        m_err = "bad model shape";
        return;
    }
    if (cudaSetDevice(deviceId) != cudaSuccess) {
        m_err = "cudaSetDevice";
        return;
    }
    m_np = static_cast<size_t>(din) * hidden + hidden + static_cast<size_t>(hidden) * hidden + hidden + hidden + 1;
    float** bufs[] = {&m_dP, &m_dG, &m_dM, &m_dV};
    for (float** b : bufs) {
        if (cudaMalloc(b, m_np * sizeof(float)) != cudaSuccess) {
            m_err = "cudaMalloc model parameters";
            return;
        }
    }
    if (cudaMemset(m_dM, 0, m_np * sizeof(float)) != cudaSuccess ||
        cudaMemset(m_dV, 0, m_np * sizeof(float)) != cudaSuccess) {
        m_err = "cudaMemset optimiser state";
        return;
    }
    // He-style uniform initialisation (GELU), zero biases
    std::vector<float> p(m_np, 0.0f);
    std::mt19937_64 rng(seed);
    auto fill = [&](size_t off, size_t n, uint32_t fanIn) {
        const float a = std::sqrt(6.0f / static_cast<float>(fanIn));
        std::uniform_real_distribution<float> u(-a, a);
        for (size_t i = 0; i < n; ++i) p[off + i] = u(rng);
    };
    fill(OffW1(), static_cast<size_t>(din) * hidden, din);
    fill(OffW2(), static_cast<size_t>(hidden) * hidden, hidden);
    fill(OffW3(), hidden, hidden);
    if (cudaMemcpy(m_dP, p.data(), m_np * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        m_err = "upload model parameters";
        return;
    }
    m_ok = true;
}

ThresholdModel::~ThresholdModel() {
    cudaSetDevice(m_deviceId);
    float* bufs[] = {m_dP, m_dG, m_dM, m_dV, m_dZ1, m_dA1, m_dZ2, m_dA2, m_dY, m_dDy, m_dD1, m_dD2, m_dSq};
    for (float* b : bufs)
        if (b) cudaFree(b);
}

bool ThresholdModel::Reserve(uint32_t batch) {
    if (batch <= m_cap) return true;
    float** acts[] = {&m_dZ1, &m_dA1, &m_dZ2, &m_dA2, &m_dD1, &m_dD2};
    float** vecs[] = {&m_dY, &m_dDy, &m_dSq};
    for (float** a : acts) {
        if (*a) cudaFree(*a);
        *a = nullptr;
    }
    for (float** a : vecs) {
        if (*a) cudaFree(*a);
        *a = nullptr;
    }
    m_cap = 0;
    for (float** a : acts)
        if (cudaMalloc(a, static_cast<size_t>(batch) * m_h * sizeof(float)) != cudaSuccess) {
            m_err = "cudaMalloc model activations";
            return false;
        }
    for (float** a : vecs)
        if (cudaMalloc(a, static_cast<size_t>(batch) * sizeof(float)) != cudaSuccess) {
            m_err = "cudaMalloc model activations";
            return false;
        }
    m_cap = batch;
    return true;
}

cudaError_t ThresholdModel::ForwardInto(const float* dX, uint32_t B, cudaStream_t s) {
    const int H = static_cast<int>(m_h), D = static_cast<int>(m_din), n = static_cast<int>(B);
    cudaError_t e =
        launch_gemm(false, false, dX, m_dP + OffW1(), m_dA1, n, H, D, D, H, H, m_dP + OffB1(), 1, m_dZ1, false, s);
    if (e == cudaSuccess)
        e = launch_gemm(false, false, m_dA1, m_dP + OffW2(), m_dA2, n, H, H, H, H, H, m_dP + OffB2(), 1, m_dZ2, false,
                        s);
    if (e == cudaSuccess)
        e = launch_gemm(false, false, m_dA2, m_dP + OffW3(), m_dY, n, 1, H, H, 1, 1, m_dP + OffB3(), 0, nullptr, false,
                        s);
    return e;
}

// Gradients of the loss (mean squared error, or the pinball loss of the tau-quantile) after
// ForwardInto, into m_dG (same layout as the parameters).
cudaError_t ThresholdModel::Backward(const float* dX, const float* dT, uint32_t B, cudaStream_t s) {
    const int H = static_cast<int>(m_h), D = static_cast<int>(m_din), n = static_cast<int>(B);
    cudaError_t e = launch_loss_grad(m_dY, dT, n, m_tau, m_dDy, m_dSq, s);
    // output layer: dw3 = A2^T dy, db3 = sum dy, dA2 = dy w3^T
    if (e == cudaSuccess)
        e = launch_gemm(true, false, m_dA2, m_dDy, m_dG + OffW3(), H, 1, n, H, 1, 1, nullptr, 0, nullptr, false, s);
    if (e == cudaSuccess) e = launch_colsum(m_dDy, n, 1, 1, m_dG + OffB3(), s);
    if (e == cudaSuccess)
        e = launch_gemm(false, true, m_dDy, m_dP + OffW3(), m_dD2, n, H, 1, 1, 1, H, nullptr, 0, nullptr, false, s);
    // hidden 2: dZ2 = dA2 * gelu'(Z2); dW2 = A1^T dZ2; db2 = colsum; dA1 = dZ2 W2^T
    if (e == cudaSuccess) e = launch_gelu_backward(m_dD2, m_dZ2, static_cast<int64_t>(n) * H, s);
    if (e == cudaSuccess)
        e = launch_gemm(true, false, m_dA1, m_dD2, m_dG + OffW2(), H, H, n, H, H, H, nullptr, 0, nullptr, false, s);
    if (e == cudaSuccess) e = launch_colsum(m_dD2, n, H, H, m_dG + OffB2(), s);
    if (e == cudaSuccess)
        e = launch_gemm(false, true, m_dD2, m_dP + OffW2(), m_dD1, n, H, H, H, H, H, nullptr, 0, nullptr, false, s);
    // hidden 1: dZ1 = dA1 * gelu'(Z1); dW1 = X^T dZ1; db1 = colsum
    if (e == cudaSuccess) e = launch_gelu_backward(m_dD1, m_dZ1, static_cast<int64_t>(n) * H, s);
    if (e == cudaSuccess)
        e = launch_gemm(true, false, dX, m_dD1, m_dG + OffW1(), D, H, n, D, H, H, nullptr, 0, nullptr, false, s);
    if (e == cudaSuccess) e = launch_colsum(m_dD1, n, H, H, m_dG + OffB1(), s);
    return e;
}

int ThresholdModel::Finish(cudaError_t e, float* hLoss, uint32_t B, cudaStream_t s) {
    std::vector<float> sq;
    if (e == cudaSuccess && hLoss) {
        sq.resize(B);
        e = cudaMemcpyAsync(sq.data(), m_dSq, B * sizeof(float), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        m_err = cudaGetErrorString(e);
        return -2;
    }
    if (hLoss) {
        double l = 0;
        for (float v : sq) l += v;
        *hLoss = static_cast<float>(l / B);
    }
    return 0;
}

int ThresholdModel::Forward(const float* dX, uint32_t B, float* dY, cudaStream_t s) {
    if (!m_ok) return -1;
    if (B == 0) return 0;
    if (cudaSetDevice(m_deviceId) != cudaSuccess) return -1;
    cudaError_t e = launch_mlp_forward(dX, static_cast<int>(B), static_cast<int>(m_din), static_cast<int>(m_h), m_dP,
                                       dY, s);
    if (e != cudaSuccess) {
        m_err = cudaGetErrorString(e);
        return -2;
    }
    return 0;
}

int ThresholdModel::Gradients(const float* dX, const float* dT, uint32_t B, float* hGrad, float* hLoss,
                              cudaStream_t s) {
    if (!m_ok || B == 0) return -1;
    if (cudaSetDevice(m_deviceId) != cudaSuccess || !Reserve(B)) return -1;
    cudaError_t e = ForwardInto(dX, B, s);
    if (e == cudaSuccess) e = Backward(dX, dT, B, s);
    if (e == cudaSuccess && hGrad) e = cudaMemcpyAsync(hGrad, m_dG, m_np * sizeof(float), cudaMemcpyDeviceToHost, s);
    return Finish(e, hLoss, B, s);
}

int ThresholdModel::TrainStep(const float* dX, const float* dT, uint32_t B, float lr, float* hLoss, cudaStream_t s) {
    if (!m_ok || B == 0) return -1;
    if (cudaSetDevice(m_deviceId) != cudaSuccess || !Reserve(B)) return -1;
    cudaError_t e = ForwardInto(dX, B, s);
    if (e == cudaSuccess) e = Backward(dX, dT, B, s);
    if (e == cudaSuccess)
        e = launch_adam(m_dP, m_dG, m_dM, m_dV, static_cast<int64_t>(m_np), lr, 0.9f, 0.999f, 1e-8f, ++m_step, s);
    return Finish(e, hLoss, B, s);
}

int ThresholdModel::SetQuantile(float tau) {
    if (!(tau >= 0.0f && tau < 1.0f)) {
        m_err = "quantile outside [0, 1)";
        return -1;
    }
    m_tau = tau;
    return 0;
}

int ThresholdModel::GetParams(float* h) const {
    if (!m_ok) return -1;
    cudaSetDevice(m_deviceId);
    return cudaMemcpy(h, m_dP, m_np * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -2;
}

int ThresholdModel::SetParams(const float* h) {
    if (!m_ok) return -1;
    cudaSetDevice(m_deviceId);
    return cudaMemcpy(m_dP, h, m_np * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess ? 0 : -2;
}

}  // namespace hss
