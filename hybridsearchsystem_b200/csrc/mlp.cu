// mlp.cu -- the learned threshold predictor: a small MLP (features -> 2 hidden layers with GELU ->
// one output, the predicted K-th filtered score), trained and run by these kernels.
//
//   forward   Z1 = X W1 + b1, A1 = gelu(Z1), Z2 = A1 W2 + b2, A2 = gelu(Z2), y = A2 w3 + b3
//   backward  from dL/dy: the gradients of every parameter (GEMMs with transposed operands, GELU'
//             from the stored pre-activations, bias gradients as column sums)
//   adam      one Adam step over the flat parameter vector
// FP32 throughout. The GEMMs are small (batch x ~400 x 256): a shared-memory tiled SIMT GEMM with a
// fused bias + activation epilogue is enough; they are nowhere near the search's critical path.
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

// dy = 2 (y - t) / B for the mean squared error; sq[i] = (y - t)^2.
__global__ void mse_grad_kernel(const float* __restrict__ y, const float* __restrict__ t, int B, float* __restrict__ dy,
                                float* __restrict__ sq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B) return;
    const float d = y[i] - t[i];
    dy[i] = 2.0f * d / static_cast<float>(B);
    if (sq) sq[i] = d * d;
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

// theta_a[q] = max(proven threshold, predicted K-th score (y * scale + shift) minus the margin). fmaxf
// drops a NaN prediction. theta_a may alias y (each thread reads, then writes, its own element).
__global__ void predict_theta_kernel(const float* y, const float* __restrict__ theta, uint32_t nq, float scale,
                                     float shift, float margin, float* theta_a) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    theta_a[q] = fmaxf(theta[q], __fsub_rd(fmaf(y[q], scale, shift), margin));
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

cudaError_t launch_mse_grad(const float* y, const float* t, int B, float* dy, float* sq, cudaStream_t stream) {
    if (B <= 0) return cudaSuccess;
    mse_grad_kernel<<<(B + 255) / 256, 256, 0, stream>>>(y, t, B, dy, sq);
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

cudaError_t launch_predict_theta(const float* y, const float* theta, uint32_t nq, float scale, float shift,
                                 float margin, float* theta_a, cudaStream_t stream) {
    if (nq == 0) return cudaSuccess;
    predict_theta_kernel<<<(nq + 127) / 128, 128, 0, stream>>>(y, theta, nq, scale, shift, margin, theta_a);
    return cudaGetLastError();
}

}  // namespace hss
