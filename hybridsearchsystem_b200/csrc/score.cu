// score.cu -- scoring kernels.
//
//  * exact_score_kernel: the materialised score matrix C[m x n] = Q . D^T of the reference's
//    kernel_vector_mmad (kernel_vector_mmad_op.cpp:3-11), computed in the ground truth's own
//    arithmetic (FP32, sequential over d, separate multiply and add), so every entry is bit-identical
//    to the CPU oracle's score. Used by the operator-level API and the parity tests.
//  * cand_simt_kernel: the bulk candidate pass on FP32 SIMT cores. Scores a 128-doc x 64-query tile
//    with FFMA (any summation order, error <= gamma_d * sum|q_i v_i|), tests the filter bit and the
//    per-query threshold in the epilogue and appends survivors to per-query candidate lists. The
//    B x N score matrix is never written.
#include "hss_device.cuh"
#include "hss_kernels.h"

namespace hss {
namespace {

// ---------------------------------------------------------------------------------------------
// Exact materialised scorer. One thread per doc; the CTA holds kExactQ query rows in shared memory.
// ---------------------------------------------------------------------------------------------
constexpr int kExactDocs = 128;
constexpr int kExactQ = 8;

__global__ void __launch_bounds__(kExactDocs) exact_score_kernel(const float* __restrict__ qry,
                                                                 const float* __restrict__ docs,
                                                                 float* __restrict__ out, uint32_t m, uint32_t n,
                                                                 uint32_t dim, uint64_t ldc) {
    extern __shared__ float sq[];  // [kExactQ][dim]
    const uint32_t q0 = blockIdx.y * kExactQ;
    const uint32_t nq = min(static_cast<uint32_t>(kExactQ), m - q0);
    for (uint32_t i = threadIdx.x; i < nq * dim; i += blockDim.x) sq[i] = qry[static_cast<uint64_t>(q0) * dim + i];
    __syncthreads();
    const uint64_t doc = static_cast<uint64_t>(blockIdx.x) * kExactDocs + threadIdx.x;
    if (doc >= n) return;
    const float* v = docs + doc * dim;
    for (uint32_t j = 0; j < nq; ++j) out[(q0 + j) * ldc + doc] = exact_dot(sq + j * dim, v, dim);
}

// ---------------------------------------------------------------------------------------------
// SIMT candidate pass.
// 256 threads = 32 doc groups (4 docs each) x 8 query groups (8 queries each); a warp is one query
// group, so the epilogue's per-query ballots are warp-uniform.
// ---------------------------------------------------------------------------------------------
constexpr int kCT = 256;
constexpr int kCQ = 64;   // queries per chunk
constexpr int kCK = 32;   // dims per smem stage
constexpr int kDPad = kDocTile + 4;
constexpr int kQPad = kCQ + 4;

__global__ void __launch_bounds__(kCT) cand_simt_kernel(CandLaunch L) {
    extern __shared__ uint32_t sCount[];  // [nq_list] candidates this CTA found per query
    __shared__ __align__(16) float sD[kCK][kDPad];
    __shared__ __align__(16) float sQ[kCK][kQPad];
    __shared__ uint64_t sBits[kCQ][2];
    __shared__ float sTheta[kCQ];
    __shared__ uint32_t sQi[kCQ];

    const uint32_t tid = threadIdx.x;
    const uint32_t dg = tid & 31;  // lane
    const uint32_t qg = tid >> 5;  // warp
    const uint32_t nchunks = (L.nq_list + kCQ - 1) / kCQ;
    const uint32_t kchunks = (L.dim + kCK - 1) / kCK;
    for (uint32_t i = tid; i < L.nq_list; i += kCT) sCount[i] = 0;

    TileWalk walk(L.tile_begin, L.tile_step, L.tile_skip, blockIdx.x, gridDim.x);
    for (uint64_t it = blockIdx.x; it < L.tile_count; it += gridDim.x, walk.advance()) {
        const uint64_t tile = walk.tile();
        const uint64_t doc0 = tile * kDocTile;
        for (uint32_t chunk = 0; chunk < nchunks; ++chunk) {
            float acc[4][8];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[r][j] = 0.0f;

            for (uint32_t kc = 0; kc < kchunks; ++kc) {
                __syncthreads();
                const uint32_t k0 = kc * kCK;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const uint32_t f = tid + kCT * i;
                    const uint32_t doc = f >> 3, part = f & 7;
                    const uint32_t k = k0 + part * 4;
                    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (k < L.dim) v = *reinterpret_cast<const float4*>(L.vec + (doc0 + doc) * L.dim + k);
                    sD[part * 4 + 0][doc] = v.x;
                    sD[part * 4 + 1][doc] = v.y;
                    sD[part * 4 + 2][doc] = v.z;
                    sD[part * 4 + 3][doc] = v.w;
                }
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const uint32_t f = tid + kCT * i;
                    const uint32_t qq = f >> 3, part = f & 7;
                    const uint32_t k = k0 + part * 4;
                    const uint32_t li = chunk * kCQ + qq;
                    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (li < L.nq_list && k < L.dim) {
                        const uint32_t qi = L.qlist ? L.qlist[li] : li;
                        v = *reinterpret_cast<const float4*>(L.qry + static_cast<uint64_t>(qi) * L.dim + k);
                    }
                    sQ[part * 4 + 0][qq] = v.x;
                    sQ[part * 4 + 1][qq] = v.y;
                    sQ[part * 4 + 2][qq] = v.z;
                    sQ[part * 4 + 3][qq] = v.w;
                }
                if (kc == 0 && tid < kCQ) {
                    const uint32_t li = chunk * kCQ + tid;
                    uint64_t b0 = 0, b1 = 0;
                    float th = INFINITY;
                    uint32_t qi = 0xffffffffu;
                    if (li < L.nq_list) {
                        qi = L.qlist ? L.qlist[li] : li;
                        const uint64_t* brow = L.bits + static_cast<uint64_t>(qi) * L.bits_stride + tile * 2;
                        b0 = brow[0];
                        b1 = brow[1];
                        th = L.theta[qi];
                    }
                    sBits[tid][0] = b0;
                    sBits[tid][1] = b1;
                    sTheta[tid] = th;
                    sQi[tid] = qi;
                }
                __syncthreads();
#pragma unroll 8
                for (int k = 0; k < kCK; ++k) {
                    const float4 d4 = *reinterpret_cast<const float4*>(&sD[k][dg * 4]);
                    const float4 qa = *reinterpret_cast<const float4*>(&sQ[k][qg * 8]);
                    const float4 qb = *reinterpret_cast<const float4*>(&sQ[k][qg * 8 + 4]);
                    const float dv[4] = {d4.x, d4.y, d4.z, d4.w};
                    const float qv[8] = {qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z, qb.w};
#pragma unroll
                    for (int r = 0; r < 4; ++r)
#pragma unroll
                        for (int j = 0; j < 8; ++j) acc[r][j] = fmaf(dv[r], qv[j], acc[r][j]);
                }
            }

            // Epilogue: filter bit && score >= theta -> append (score, location) to this CTA's segment
            // of the query's list (a shared-memory count per query; no global atomics).
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint32_t qq = qg * 8 + j;
                const uint32_t qi = sQi[qq];
                if (qi == 0xffffffffu) continue;  // warp-uniform
                const float th = sTheta[qq];
                const uint64_t w0 = sBits[qq][0], w1 = sBits[qq][1];
                const uint64_t seg =
                    static_cast<uint64_t>(qi) * L.cap + static_cast<uint64_t>(L.seg_base + blockIdx.x) * L.seg_cap;
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const uint32_t dl = dg * 4 + r;
                    const uint64_t w = dl < 64 ? w0 : w1;
                    const bool pred = ((w >> (dl & 63)) & 1ull) && acc[r][j] >= th;
                    const uint32_t mask = __ballot_sync(0xffffffffu, pred);
                    if (mask == 0) continue;
                    uint32_t base = 0;
                    const uint32_t leader = __ffs(mask) - 1;
                    if (dg == leader) base = atomicAdd(&sCount[chunk * kCQ + qq], __popc(mask));
                    base = __shfl_sync(0xffffffffu, base, leader);
                    if (pred) {
                        const uint32_t idx = base + __popc(mask & ((1u << dg) - 1u));
                        if (idx < L.seg_cap) {
                            L.cand_score[seg + idx] = acc[r][j];
                            L.cand_loc[seg + idx] = static_cast<uint32_t>(doc0 + dl);
                        }
                    }
                }
            }
        }
    }
    __syncthreads();
    for (uint32_t i = tid; i < L.nq_list; i += kCT) {
        const uint32_t qi = L.qlist ? L.qlist[i] : i;
        L.cand_count[static_cast<uint64_t>(qi) * kMaxCandSegs + L.seg_base + blockIdx.x] = sCount[i];
    }
}

}  // namespace

cudaError_t launch_exact_score(const float* qry, const float* docs, float* out, uint32_t m, uint32_t n, uint32_t dim,
                               uint64_t ldc, cudaStream_t stream) {
    if (m == 0 || n == 0) return cudaSuccess;
    const size_t smem = static_cast<size_t>(kExactQ) * dim * sizeof(float);
    if (smem > 48 * 1024) {
        // one ceiling for every caller (concurrent callers with other dimensions launch it too)
        constexpr size_t kCeiling = 200 * 1024;
        if (smem > kCeiling) return cudaErrorInvalidValue;
        cudaError_t e = cudaFuncSetAttribute(exact_score_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(kCeiling));
        if (e != cudaSuccess) return e;
    }
    dim3 grid((n + kExactDocs - 1) / kExactDocs, (m + kExactQ - 1) / kExactQ);
    if (grid.y > 65535u) return cudaErrorInvalidValue;
    exact_score_kernel<<<grid, kExactDocs, smem, stream>>>(qry, docs, out, m, n, dim, ldc);
    return cudaGetLastError();
}

uint32_t cand_simt_segments(uint64_t tile_count, int num_sms, uint32_t cap) {
    uint64_t g = static_cast<uint64_t>(num_sms) * 3;
    g = tile_count < g ? tile_count : g;
    g = g < kMaxCandSegs / 2 ? g : kMaxCandSegs / 2;  // one segment per CTA, room for two passes
    const uint64_t by_cap = cap / (2 * kMinSegCap) > 0 ? cap / (2 * kMinSegCap) : 1;
    return static_cast<uint32_t>(g < by_cap ? g : by_cap);
}

cudaError_t launch_cand_simt(const CandLaunch& L, int num_sms, cudaStream_t stream) {
    if (L.tile_count == 0 || L.nq_list == 0) return cudaSuccess;
    const uint64_t seg_end = static_cast<uint64_t>(L.seg_base) + L.segs;
    if (L.segs != cand_simt_segments(L.tile_count, num_sms, L.cap) || L.seg_cap == 0 || seg_end > kMaxCandSegs ||
        seg_end * L.seg_cap > L.cap || L.nq_list > kMaxSimtBatch ||
        !tile_walk_fits(L.tile_begin, L.tile_step, L.tile_skip, L.tile_count, L.segs))
        return cudaErrorInvalidValue;
    const size_t smem = static_cast<size_t>(L.nq_list) * sizeof(uint32_t);
    cand_simt_kernel<<<L.segs, kCT, smem, stream>>>(L);
    return cudaGetLastError();
}

}  // namespace hss
