// mlp.cu -- the learned threshold predictor: a small MLP (features -> 2 hidden layers with GELU ->
// one output, the predicted K-th filtered score), trained and run by these kernels.
//
//   forward   Z1 = X W1 + b1, A1 = gelu(Z1), Z2 = A1 W2 + b2, A2 = gelu(Z2), y = A2 w3 + b3
//   backward  from dL/dy: the gradients of every parameter (GEMMs with transposed operands, GELU'
//             from the stored pre-activations, bias gradients as column sums)
//   adam      one Adam step over the flat parameter vector
// FP32 throughout. The GEMMs are small (batch x ~400 x 256): a shared-memory tiled SIMT GEMM with a
// fused bias + activation epilogue is enough; they are nowhere near the search's critical path.
#include <algorithm>

#include "hss_device.cuh"
#include "hss_kernels.h"

namespace hss {
namespace {

constexpr int kTM = 64, kTN = 64, kTK = 16;  // block tile
constexpr int kGT = 256;                     // threads: 16 x 16, 4 x 4 outputs each

__device__ inline float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ inline float gelu_grad(float z) {
    // d/dz [z Phi(z)] = Phi(z) + z phi(z)
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

// C = op(A) op(B) (+ C when accumulate) (+ bias[n]), then the activation; pre (if given) receives the
// value before the activation. op(A)(m, k) = TA ? A[k * lda + m] : A[m * lda + k], likewise B with
// (k, n). act: 0 identity, 1 GELU.
template <bool TA, bool TB>
__global__ void __launch_bounds__(kGT) gemm_kernel(const float* __restrict__ A, const float* __restrict__ B,
                                                  float* __restrict__ C, int M, int N, int K, int lda, int ldb,
                                                  int ldc, const float* __restrict__ bias, int act,
                                                  float* __restrict__ pre, int accumulate) {
    __shared__ float sA[kTK][kTM + 4];
    __shared__ float sB[kTK][kTN + 4];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int m0 = blockIdx.y * kTM, n0 = blockIdx.x * kTN;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += kTK) {
        for (int i = threadIdx.x; i < kTK * kTM; i += kGT) {
            const int kk = TA ? i / kTM : i % kTK;
            const int mm = TA ? i % kTM : i / kTK;
            const int m = m0 + mm, k = k0 + kk;
            sA[kk][mm] = (m < M && k < K) ? (TA ? A[static_cast<int64_t>(k) * lda + m]
                                                 : A[static_cast<int64_t>(m) * lda + k])
                                           : 0.0f;
        }
        for (int i = threadIdx.x; i < kTK * kTN; i += kGT) {
            const int kk = TB ? i % kTK : i / kTN;
            const int nn = TB ? i / kTK : i % kTN;
            const int n = n0 + nn, k = k0 + kk;
            sB[kk][nn] = (n < N && k < K) ? (TB ? B[static_cast<int64_t>(n) * ldb + k]
                                                 : B[static_cast<int64_t>(k) * ldb + n])
                                           : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kTK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                a[i] = sA[kk][ty * 4 + i];
                b[i] = sB[kk][tx * 4 + i];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + ty * 4 + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = n0 + tx * 4 + j;
            if (n >= N) continue;
            const int64_t at = static_cast<int64_t>(m) * ldc + n;
            float v = acc[i][j];
            if (accumulate) v += C[at];
            if (bias) v += bias[n];
            if (pre) pre[at] = v;
            C[at] = act == 1 ? gelu(v) : v;
        }
    }
}

// dZ = dA * gelu'(Z), in place on dA.
__global__ void gelu_backward_kernel(float* __restrict__ dA, const float* __restrict__ Z, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) dA[i] *= gelu_grad(Z[i]);
}

// out[n] = sum_m G[m * ld + n] (bias gradients), one thread per column.
__global__ void colsum_kernel(const float* __restrict__ G, int M, int N, int ld, float* __restrict__ out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.0f;
    for (int m = 0; m < M; ++m) s += G[static_cast<int64_t>(m) * ld + n];
    out[n] = s;
}

// The loss's gradient dL/dy and each row's loss term. tau = 0: mean squared error, dy = 2 (y - t) / B,
// term (y - t)^2. tau in (0, 1): the pinball loss of the tau-quantile, term tau (t - y) when t >= y and
// (1 - tau) (y - t) otherwise, dy = (y > t ? 1 - tau : -tau) / B (the network then predicts a
// conditional tau-quantile of the target).
__global__ void loss_grad_kernel(const float* __restrict__ y, const float* __restrict__ t, int B, float tau,
                                 float* __restrict__ dy, float* __restrict__ term) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B) return;
    const float d = y[i] - t[i];
    if (tau <= 0.0f) {
        dy[i] = 2.0f * d / static_cast<float>(B);
        if (term) term[i] = d * d;
    } else {
        dy[i] = (d > 0.0f ? 1.0f - tau : -tau) / static_cast<float>(B);
        if (term) term[i] = d > 0.0f ? (1.0f - tau) * d : -tau * d;
    }
}

// Inference forward pass fused into one launch: a CTA takes kFwdRows feature rows, thread j computes
// hidden unit j of both layers for all of them, and thread r < kFwdRows the output of row r. Every sum
// runs over k in ascending order with fmaf, the bias added after, as gemm_kernel does: the outputs equal
// the three-GEMM forward pass (ForwardInto) bit for bit.
constexpr int kFwdRows = 4;
constexpr int kFwdUnroll = 64;  // weight loads in flight per thread

__global__ void mlp_forward_kernel(const float* __restrict__ X, int B, int D, int H, const float* __restrict__ P,
                                   float* __restrict__ y) {
    extern __shared__ float fsm[];
    float* xs = fsm;                  // [kFwdRows][D]
    float* a1 = xs + kFwdRows * D;    // [kFwdRows][H]
    float* a2 = a1 + kFwdRows * H;    // [kFwdRows][H]
    const int r0 = blockIdx.x * kFwdRows;
    const int rows = min(kFwdRows, B - r0);
    for (int i = threadIdx.x; i < kFwdRows * D; i += blockDim.x) {
        const int r = i / D;
        xs[i] = r < rows ? X[static_cast<int64_t>(r0 + r) * D + i % D] : 0.0f;
    }
    __syncthreads();
    const float* W1 = P;
    const float* b1 = W1 + static_cast<int64_t>(D) * H;
    const float* W2 = b1 + H;
    const float* b2 = W2 + static_cast<int64_t>(H) * H;
    const float* w3 = b2 + H;
    const float* b3 = w3 + H;
    const int j = threadIdx.x;
    // acc[r] += in[r][k] * W[k][j] for k ascending; the weights of kFwdUnroll k's are loaded before
    // they are used, so that many loads are in flight (the loop is otherwise bound by load latency)
    // (the last block is partial: its loads and sums stop at K, a uniform condition)
    auto layer = [&](const float* __restrict__ W, const float* in, int K, float (&acc)[kFwdRows]) {
        for (int k = 0; k < K; k += kFwdUnroll) {
            float w[kFwdUnroll];
#pragma unroll
            for (int u = 0; u < kFwdUnroll; ++u) w[u] = k + u < K ? __ldg(W + static_cast<int64_t>(k + u) * H + j) : 0.0f;
#pragma unroll
            for (int u = 0; u < kFwdUnroll; ++u) {
                if (k + u < K) {
#pragma unroll
                    for (int r = 0; r < kFwdRows; ++r) acc[r] = fmaf(in[r * K + k + u], w[u], acc[r]);
                }
            }
        }
    };
    if (j < H) {
        float acc[kFwdRows] = {};
        layer(W1, xs, D, acc);
#pragma unroll
        for (int r = 0; r < kFwdRows; ++r) a1[r * H + j] = gelu(acc[r] + b1[j]);
    }
    __syncthreads();
    if (j < H) {
        float acc[kFwdRows] = {};
        layer(W2, a1, H, acc);
#pragma unroll
        for (int r = 0; r < kFwdRows; ++r) a2[r * H + j] = gelu(acc[r] + b2[j]);
    }
    __syncthreads();
    if (j < rows) {
        float acc = 0.0f;
        for (int k = 0; k < H; ++k) acc = fmaf(a2[j * H + k], w3[k], acc);
        y[r0 + j] = acc + b3[0];
    }
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Features of one query (row q of X, din columns): [ q * sqrt(dim) | per posting row: 1 + log10
// density / 4 for the rows of the query's filter, 0 elsewhere | log10 selectivity / 4 | log10 K / 3 |
// 1 | the doc sample's best score | its K-th best score (-2 when absent) | log10(filtered sample
// docs + 1) / 5 ].
__global__ void features_kernel(FeatureLaunch L) {
    const uint32_t q = blockIdx.x;
    float* x = L.x + static_cast<uint64_t>(q) * L.din;
    const float s = sqrtf(static_cast<float>(L.dim));
    for (uint32_t i = threadIdx.x; i < L.din; i += blockDim.x) {
        float v = 0.0f;
        if (i < L.dim) v = L.qry[static_cast<uint64_t>(q) * L.dim + i] * s;
        x[i] = v;
    }
    __syncthreads();
    const uint32_t o0 = L.opnd_off[q], o1 = L.opnd_off[q + 1];
    for (uint32_t j = o0 + threadIdx.x; j < o1; j += blockDim.x) {
        const uint32_t r = L.opnd_row[j];
        if (r < L.rows) x[L.dim + r] = 1.0f + log10f(fmaxf(L.row_density[r], 1e-9f)) * 0.25f;
    }
    if (threadIdx.x == 0) {
        const float sel = fmaxf(static_cast<float>(L.pass_count[q]), 1.0f) / static_cast<float>(L.doc_num);
        const float* st = L.stats + static_cast<uint64_t>(q) * kSampleStats;
        float* t = x + L.dim + L.rows;
        t[0] = log10f(sel) * 0.25f;
        t[1] = log10f(fmaxf(static_cast<float>(L.topk[q]), 1.0f)) / 3.0f;
        t[2] = 1.0f;
        for (uint32_t j = 0; j < kSampleRanks; ++j) t[3 + j] = st[j];
        t[3 + kSampleRanks] = st[kSampleRanks];
        t[4 + kSampleRanks] = log10f(st[kSampleRanks + 1] + 1.0f) * 0.2f;
    }
}

// theta[q] = max(proven threshold, predicted K-th score (y * scale + shift) minus the margin and the
// query's error bound), the proven one kept in theta_proven. A doc of the true top K then clears
// theta whenever the prediction minus the margin is at most the true K-th score. A query whose filter
// passes at most kLearnedMinPass * K docs keeps its proven threshold: its candidates are few whatever
// the threshold, and its K-th score is the hardest to predict. So does a query whose doc sample held
// fewer than kLearnedMinSample filtered docs (its sample rank features are missing). fmaxf drops a
// NaN prediction.
// theta_model may alias y (each thread reads, then writes, its own element).
__global__ void predict_theta_kernel(const float* y, const float* __restrict__ eps,
                                     const uint32_t* __restrict__ pass_count, const uint32_t* __restrict__ topk,
                                     const float* __restrict__ stats, uint32_t nq, float scale, float shift,
                                     float margin, float* theta, float* theta_proven, float* theta_model) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const float t1 = theta[q];
    const bool use = static_cast<uint64_t>(pass_count[q]) > static_cast<uint64_t>(kLearnedMinPass) * topk[q] &&
                     stats[static_cast<uint64_t>(q) * kSampleStats + kSampleRanks + 1] >= kLearnedMinSample;
    const float t = use ? fmaxf(t1, __fsub_rd(__fsub_rd(fmaf(y[q], scale, shift), margin), eps[q])) : t1;
    theta_proven[q] = t1;
    theta[q] = t;
    theta_model[q] = t;
}

}  // namespace

cudaError_t launch_gemm(bool ta, bool tb, const float* A, const float* B, float* C, int M, int N, int K, int lda,
                        int ldb, int ldc, const float* bias, int act, float* pre, bool accumulate,
                        cudaStream_t stream) {
    if (M <= 0 || N <= 0 || K <= 0) return cudaSuccess;
    const dim3 grid((N + kTN - 1) / kTN, (M + kTM - 1) / kTM);
    if (grid.y > 65535u) return cudaErrorInvalidValue;
    const int acc = accumulate ? 1 : 0;
    if (!ta && !tb)
        gemm_kernel<false, false><<<grid, kGT, 0, stream>>>(A, B, C, M, N, K, lda, ldb, ldc, bias, act, pre, acc);
    else if (ta && !tb)
        gemm_kernel<true, false><<<grid, kGT, 0, stream>>>(A, B, C, M, N, K, lda, ldb, ldc, bias, act, pre, acc);
    else if (!ta && tb)
        gemm_kernel<false, true><<<grid, kGT, 0, stream>>>(A, B, C, M, N, K, lda, ldb, ldc, bias, act, pre, acc);
    else
        gemm_kernel<true, true><<<grid, kGT, 0, stream>>>(A, B, C, M, N, K, lda, ldb, ldc, bias, act, pre, acc);
    return cudaGetLastError();
}

cudaError_t launch_gelu_backward(float* dA, const float* Z, int64_t n, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    gelu_backward_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(dA, Z, n);
    return cudaGetLastError();
}

cudaError_t launch_colsum(const float* G, int M, int N, int ld, float* out, cudaStream_t stream) {
    if (N <= 0) return cudaSuccess;
    colsum_kernel<<<(N + 127) / 128, 128, 0, stream>>>(G, M, N, ld, out);
    return cudaGetLastError();
}

cudaError_t launch_loss_grad(const float* y, const float* t, int B, float tau, float* dy, float* term,
                             cudaStream_t stream) {
    if (B <= 0) return cudaSuccess;
    if (!(tau >= 0.0f && tau < 1.0f)) return cudaErrorInvalidValue;
    loss_grad_kernel<<<(B + 255) / 256, 256, 0, stream>>>(y, t, B, tau, dy, term);
    return cudaGetLastError();
}

cudaError_t launch_mlp_forward(const float* X, int B, int D, int H, const float* P, float* y, cudaStream_t stream) {
    if (B <= 0) return cudaSuccess;
    const int threads = ((std::max(H, kFwdRows) + 31) / 32) * 32;
    const size_t smem = static_cast<size_t>(kFwdRows) * (D + 2 * H) * sizeof(float);
    if (threads > 1024 || smem > 48 * 1024) return cudaErrorInvalidValue;
    mlp_forward_kernel<<<(B + kFwdRows - 1) / kFwdRows, threads, smem, stream>>>(X, B, D, H, P, y);
    return cudaGetLastError();
}

cudaError_t launch_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2,
                        float eps, int step, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const float c1 = 1.0f - powf(b1, static_cast<float>(step));
    const float c2 = 1.0f - powf(b2, static_cast<float>(step));
    adam_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2);
    return cudaGetLastError();
}

cudaError_t launch_features(const FeatureLaunch& L, cudaStream_t stream) {
    if (L.nq == 0) return cudaSuccess;
    if (L.din < L.dim + L.rows + kFeatureTail || !L.stats) return cudaErrorInvalidValue;
    features_kernel<<<L.nq, 128, 0, stream>>>(L);
    return cudaGetLastError();
}

cudaError_t launch_predict_theta(const float* y, const float* eps, const uint32_t* pass_count, const uint32_t* topk,
                                 const float* stats, uint32_t nq, float scale, float shift, float margin,
                                 float* theta, float* theta_proven, float* theta_model, cudaStream_t stream) {
    if (nq == 0) return cudaSuccess;
    predict_theta_kernel<<<(nq + 127) / 128, 128, 0, stream>>>(y, eps, pass_count, topk, stats, nq, scale, shift,
                                                               margin, theta, theta_proven, theta_model);
    return cudaGetLastError();
}

}  // namespace hss
