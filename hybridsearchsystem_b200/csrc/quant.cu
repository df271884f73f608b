// quant.cu -- corpus copies and query staging for the tensor-core candidate pass, and the error bound
// that keeps the pass exact.
//
// For a doc v and a query q, the pass computes s~ from quantised vectors v~ = v + dv, q~ = q + dq
// (TF32: the tensor core drops the low 13 mantissa bits, |dv_i| < 2^-10 |v_i|; BF16: round to
// nearest; E4M3: per-vector scale then round to nearest) with FP32 accumulation in the tensor core.
// Against the ground truth's own FP32 score s (sequential over d):
//   |s~ - s| <= gamma_d |q||v| + acc (|q|+|dq|)(|v|+|dv|) + |q||dv| + |dq||v| + |dq||dv|
// (Cauchy-Schwarz on each term; gamma_d = d u / (1 - d u), u = 2^-24, is the ground truth's own
// rounding; acc bounds the tensor core's accumulation and the final scale multiply). The per-query
// bound E_q takes the corpus maxima of |v| and |dv|, which are measured exactly here in FP64.
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include "hss_device.cuh"
#include "hss_kernels.h"

namespace hss {
namespace {

constexpr float kE4M3Max = 448.0f;

__device__ inline double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ inline float warp_max_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Quantise one row (a warp); returns (||x||^2, ||x~ - x||^2) in FP64. TF32 writes nothing and bounds
// the truncation error by 2^-10 per element.
__device__ inline void quantize_row(const float* x, uint32_t dim, int format, void* out_row, float* scale_out,
                                    double* nrm2, double* err2) {
    const uint32_t lane = threadIdx.x & 31;
    double n2 = 0.0, e2 = 0.0;
    float s = 1.0f;
    if (format == kTcE4M3) {
        float m = 0.0f;
        for (uint32_t i = lane; i < dim; i += 32) m = fmaxf(m, fabsf(x[i]));
        m = warp_max_f(m);
        s = m > 0.0f ? m / kE4M3Max : 1.0f;
        if (!(s > 0.0f) || isinf(s)) s = 1.0f;
    }
    for (uint32_t i = lane; i < dim; i += 32) {
        const float v = x[i];
        double dq;
        if (format == kTcBF16) {
            const __nv_bfloat16 b = __float2bfloat16_rn(v);
            reinterpret_cast<__nv_bfloat16*>(out_row)[i] = b;
            dq = static_cast<double>(__bfloat162float(b));
        } else if (format == kTcE4M3) {
            const __nv_fp8_storage_t f = __nv_cvt_float_to_fp8(v / s, __NV_SATFINITE, __NV_E4M3);
            reinterpret_cast<uint8_t*>(out_row)[i] = f;
            const __half_raw hr = __nv_cvt_fp8_to_halfraw(f, __NV_E4M3);
            dq = static_cast<double>(__half2float(__half(hr))) * static_cast<double>(s);
        } else {
            dq = static_cast<double>(v);
        }
        const double dv = static_cast<double>(v);
        n2 += dv * dv;
        e2 += (dq - dv) * (dq - dv);
    }
    n2 = warp_sum_d(n2);
    e2 = warp_sum_d(e2);
    if (format == kTcTF32) e2 = n2 * 0x1p-20;  // (2^-10 |x|)^2
    *nrm2 = n2;
    *err2 = e2;
    if (scale_out) *scale_out = s;
}

__global__ void quantize_docs_kernel(const float* __restrict__ vec, uint64_t rows, uint64_t valid_rows, uint32_t dim,
                                     int format, void* out, float* scale, float* norm, float* err_norm) {
    const uint64_t r = static_cast<uint64_t>(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (r >= rows) return;
    const uint32_t elem = format == kTcBF16 ? 2u : (format == kTcE4M3 ? 1u : 4u);
    void* row = out ? static_cast<void*>(static_cast<uint8_t*>(out) + r * dim * elem) : nullptr;
    if (r >= valid_rows) {
        if (row)
            for (uint32_t i = threadIdx.x & 31; i < dim * elem; i += 32) static_cast<uint8_t*>(row)[i] = 0;
        if ((threadIdx.x & 31) == 0) {
            if (scale) scale[r] = 1.0f;
            if (norm) norm[r] = 0.0f;
            if (err_norm) err_norm[r] = 0.0f;
        }
        return;
    }
    double n2, e2;
    float s = 1.0f;
    quantize_row(vec + r * dim, dim, format, row, &s, &n2, &e2);
    if ((threadIdx.x & 31) == 0) {
        if (scale) scale[r] = s;
        if (norm) norm[r] = __double2float_ru(sqrt(n2) * (1.0 + 1e-12));
        if (err_norm) err_norm[r] = __double2float_ru(sqrt(e2) * (1.0 + 1e-12));
    }
}

__global__ void tile_minmax_kernel(const float* __restrict__ scale, uint64_t tiles, float2* __restrict__ out) {
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (t >= tiles) return;
    const uint32_t lane = threadIdx.x & 31;
    float lo = INFINITY, hi = 0.0f;
    for (uint32_t i = lane; i < 128; i += 32) {
        const float s = scale[t * 128 + i];
        lo = fminf(lo, s);
        hi = fmaxf(hi, s);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) out[t] = make_float2(lo, hi);
}

__global__ void stage_queries_kernel(StageQueriesLaunch L) {
    const uint32_t r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (r >= L.rows_alloc) return;
    const uint32_t elem = L.format == kTcBF16 ? 2u : (L.format == kTcE4M3 ? 1u : 4u);
    uint8_t* row = static_cast<uint8_t*>(L.staged) + static_cast<uint64_t>(r) * L.dim * elem;
    const uint32_t lane = threadIdx.x & 31;
    if (r >= L.nq_rows) {
        for (uint32_t i = lane; i < L.dim * elem; i += 32) row[i] = 0;
        if (lane == 0 && L.q_scale) L.q_scale[r] = 1.0f;
        return;
    }
    const uint32_t qi = L.qlist ? L.qlist[r] : r;
    const float* x = L.qry + static_cast<uint64_t>(qi) * L.dim;
    double n2, e2;
    float s = 1.0f;
    if (L.format == kTcTF32)
        for (uint32_t i = lane; i < L.dim; i += 32) reinterpret_cast<float*>(row)[i] = x[i];
    quantize_row(x, L.dim, L.format, L.format == kTcTF32 ? nullptr : row, &s, &n2, &e2);
    if (lane == 0) {
        if (L.q_scale) L.q_scale[r] = s;
        const double nq = sqrt(n2), dq = sqrt(e2);
        const double V = L.doc_norm_max, DV = L.doc_err_max;
        const double u = 0x1p-24, d = static_cast<double>(L.dim);
        const double gamma = d * u / (1.0 - d * u);
        const double e = gamma * nq * V + L.acc_rel * (nq + dq) * (V + DV) + nq * DV + dq * V + dq * DV;
        const float ef = __double2float_ru(e * (1.0 + 1e-6) + 1e-30);
        L.eps_main[qi] = ef;
        L.eps_sample[qi] = ef;
    }
}

}  // namespace

cudaError_t launch_quantize_docs(const float* vec, uint64_t rows, uint64_t valid_rows, uint32_t dim, int format,
                                 void* out, float* scale, float* norm, float* err_norm, cudaStream_t stream) {
    if (rows == 0) return cudaSuccess;
    const uint64_t blocks = (rows + 7) / 8;
    quantize_docs_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(vec, rows, valid_rows, dim, format, out,
                                                                           scale, norm, err_norm);
    return cudaGetLastError();
}

cudaError_t launch_tile_scale_minmax(const float* scale, uint64_t tiles, float2* out, cudaStream_t stream) {
    if (tiles == 0) return cudaSuccess;
    tile_minmax_kernel<<<static_cast<unsigned>((tiles + 7) / 8), 256, 0, stream>>>(scale, tiles, out);
    return cudaGetLastError();
}

cudaError_t launch_stage_queries(const StageQueriesLaunch& L, cudaStream_t stream) {
    if (L.rows_alloc == 0) return cudaSuccess;
    stage_queries_kernel<<<(L.rows_alloc + 7) / 8, 256, 0, stream>>>(L);
    return cudaGetLastError();
}

}  // namespace hss
