// hss_device.cuh -- device-side helpers shared by the filter, scoring and selection kernels.
#pragma once

#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

namespace hss {

// ---- limits (stated in include/hss.h as well) ----
constexpr int kMaxOperands = 64;     // postings one query's filter program may reference
constexpr int kMaxProgram = 512;     // u32 words in one postfix program
constexpr int kMaxStack = 16;        // evaluation stack depth of a program
constexpr int kMaxTopK = 4096;       // largest K a query may ask for
constexpr int kFilterTileWords = 256;  // u64 bitmap words one filter CTA produces
constexpr int kDocTile = 128;        // docs per scoring tile

// Filter operator codes (the reference's FilterOpType, query_node.h:17-22).
enum DeviceFilterOp : uint32_t { kOpConjunction = 0, kOpAnd = 1, kOpOr = 2, kOpNot = 3 };

// Posting layouts (the reference's PostingLayout, posting_layout.h:8).
enum Layout : uint32_t {
    kDenseBitmap = 0,
    kSparseBitmap = 1,
    kDenseBytemap = 2,
    kSparseIdList = 3,
    kSparsePacked = 4,
};

// Per-query status bits written by the kernels (0 = fine).
enum DeviceStatus : int32_t {
    kStatusBadProgram = 1,
    kStatusBadPosting = 2,
    kStatusOverflow = 4,
    kStatusTopKTooLarge = 8,
    // internal: the query's threshold was a prediction above its proven one and failed the select
    // step's check (the host re-runs it at a proven threshold; never reported as an error)
    kStatusThresholdMiss = 16,
};

// Order-preserving map float -> u32 (larger float -> larger key). -0.0 is folded onto +0.0 so the two
// compare equal, as they do for the float comparison in the ground truth.
__host__ __device__ inline uint32_t float_bits(float f) {
    uint32_t b;
    memcpy(&b, &f, sizeof(b));
    return b;
}
__host__ __device__ inline float bits_float(uint32_t b) {
    float f;
    memcpy(&f, &b, sizeof(f));
    return f;
}
__host__ __device__ inline uint32_t float_key(float f) {
    const uint32_t b = float_bits(f == 0.0f ? 0.0f : f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ inline float key_float(uint32_t k) {
    return bits_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// 64-bit result key: descending order of this key is (score descending, location ascending), the
// tie-break of the reference's Better comparator (recall_ref.cpp:19-25) with location == doc id.
__host__ __device__ inline uint64_t result_key(float s, uint32_t loc) {
    return (static_cast<uint64_t>(float_key(s)) << 32) | static_cast<uint64_t>(0xffffffffu - loc);
}
__host__ __device__ inline uint32_t result_key_loc(uint64_t k) { return 0xffffffffu - static_cast<uint32_t>(k); }
__host__ __device__ inline float result_key_score(uint64_t k) { return key_float(static_cast<uint32_t>(k >> 32)); }

__device__ inline uint32_t warp_sum(uint32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Exact inner product in the ground truth's order: s = 0; s += q[d] * v[d] for d ascending, each
// multiply and add rounded separately (no FMA contraction).
__device__ inline float exact_dot(const float* __restrict__ q, const float* __restrict__ v, uint32_t dim) {
    float s = 0.0f;
    uint32_t k = 0;
    if ((reinterpret_cast<uintptr_t>(v) & 15u) == 0) {
        for (; k + 4 <= dim; k += 4) {
            const float4 x = *reinterpret_cast<const float4*>(v + k);
            s = __fadd_rn(s, __fmul_rn(q[k + 0], x.x));
            s = __fadd_rn(s, __fmul_rn(q[k + 1], x.y));
            s = __fadd_rn(s, __fmul_rn(q[k + 2], x.z));
            s = __fadd_rn(s, __fmul_rn(q[k + 3], x.w));
        }
    }
    for (; k < dim; ++k) s = __fadd_rn(s, __fmul_rn(q[k], v[k]));
    return s;
}

// Tile of iteration `it` of a candidate pass: begin + it * step, or, with skip >= 2, the it-th tile
// that is not a multiple of skip.
__host__ __device__ inline uint64_t pass_tile(uint64_t begin, uint64_t step, uint32_t skip, uint64_t it) {
    return skip >= 2 ? it + it / (skip - 1) + 1 : begin + it * step;
}

// Launch-side guard for TileWalk: every `it` a CTA reaches (below count + stride) and every tile index
// of the pass fit in 32 bits.
__host__ __device__ inline bool tile_walk_fits(uint64_t begin, uint64_t step, uint32_t skip, uint64_t count,
                                               uint64_t stride) {
    if (count == 0) return true;
    if (count + stride >= (1ull << 32) || begin >= (1ull << 32) || step >= (1ull << 32)) return false;
    return pass_tile(begin, step, skip, count - 1) < (1ull << 32);
}

// pass_tile over it = it0, it0 + stride, it0 + 2 stride, ... without a division per step: the quotient
// and remainder of it / (skip - 1) are carried along (a division by a runtime divisor costs tens of
// instructions, and the candidate kernels step once per tile in every thread). 32-bit state: a pass
// has far fewer than 2^32 tiles (launchers check tile_walk_fits).
struct TileWalk {
    uint32_t begin, step, it, stride, q, dq, d, r, dr;  // d = skip - 1 (0: strided), it = q d + r, stride = dq d + dr
    __device__ TileWalk(uint64_t b, uint64_t s, uint32_t skip, uint64_t it0, uint64_t strd)
        : begin(static_cast<uint32_t>(b)), step(static_cast<uint32_t>(s)), it(static_cast<uint32_t>(it0)),
          stride(static_cast<uint32_t>(strd)), q(0), dq(0), d(skip >= 2 ? skip - 1 : 0), r(0), dr(0) {
        if (d) {
            q = it / d;
            r = it - q * d;
            dq = stride / d;
            dr = stride - dq * d;
        }
    }
    __device__ uint64_t tile() const {
        return d ? static_cast<uint64_t>(it) + q + 1 : static_cast<uint64_t>(begin) + static_cast<uint64_t>(it) * step;
    }
    __device__ void advance() {
        it += stride;
        if (d) {
            q += dq;
            r += dr;  // r, dr < d: one correction suffices
            if (r >= d) {
                r -= d;
                ++q;
            }
        }
    }
};

}  // namespace hss
