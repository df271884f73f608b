// score_tc.cu -- the candidate pass on the 5th-generation tensor cores (tcgen05 + TMA + TMEM).
//
// D[query, doc] = Q . D^T for a 128-doc tile and up to 256 staged queries per CTA iteration:
//   A = staged queries   (M = 128 per half, 1 or 2 halves), resident in shared memory
//   B = the corpus tile  (N = 128 docs), streamed by TMA through a ring of 16 KB k-block stages
//   D = FP32 accumulators in TMEM, double buffered (2 x halves x 128 columns)
// Operands are K-major with the 128-byte swizzle that TMA writes and UMMA reads. Formats: FP32 corpus
// read as TF32 (kind::tf32), BF16 (kind::f16) and FP8 E4M3 with per-vector scales (kind::f8f6f4).
//
// Warp roles (persistent CTA, one per SM): warp 0 issues TMA, warp 1 owns TMEM and issues MMAs
// (one elected lane), warps 2 .. 2+8*halves-1 drain the accumulators. Each epilogue thread owns one
// query (its TMEM lane) and one half of the tile's doc columns for the whole launch: it pulls its 64
// scores out of TMEM in one batch, releases the accumulator, tests a 32-doc chunk with one max
// reduction against the query's threshold, and only for a chunk that clears it applies the filter
// bits and appends the survivors to its own segment of the query's candidate list (a
// register-held count, no atomics).
//
// Every mbarrier wait is bounded (a clock budget); on expiry the CTA records an error, stops issuing
// and drains, releases TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "hss_device.cuh"
#include "hss_kernels.h"

namespace hss {
namespace {

constexpr int kStageBytes = 16384;        // one k-block of a 128-row tile: 128 rows x 128 bytes
constexpr int kRows = 128;
constexpr long long kWaitBudget = 4000000000ll;  // clock cycles (~2 s) before a wait gives up

struct TcShared {
    unsigned long long full[kMaxTcStages];
    unsigned long long empty[kMaxTcStages];
    unsigned long long acc_full[2];
    unsigned long long acc_empty[2];
    unsigned long long qbar;
    unsigned long long drain;
    uint32_t tmem_base;
    uint32_t n_issued, n_consumed;  // stage loads issued by TMA / waited for by the MMA issuer
    volatile int abort;
};

__device__ inline uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ inline void mbar_init(unsigned long long* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ inline void mbar_expect_tx(unsigned long long* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ inline void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ inline bool mbar_try(unsigned long long* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait that ignores the abort flag (draining copies and MMAs still in flight).
__device__ inline bool mbar_wait_drain(unsigned long long* bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try(bar, parity))
        if (clock64() - t0 > kWaitBudget) return false;
    return true;
}

// Bounded wait for the phase of `parity`; false (and the CTA marked aborted) when the budget runs out
// or another role already aborted.
__device__ inline bool mbar_wait(unsigned long long* bar, uint32_t parity, TcShared& S, int32_t* err, int code,
                                 long long budget = kWaitBudget) {
    if (mbar_try(bar, parity)) return true;  // no clock read when the phase is already complete
    const long long t0 = clock64();
    while (!mbar_try(bar, parity)) {
        if (S.abort) return false;
        if (clock64() - t0 > budget) {
            S.abort = 1;
            if (err) atomicOr(err, code);
            return false;
        }
    }
    return true;
}

__device__ inline void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// UMMA shared-memory descriptor: K-major operand with the 128-byte swizzle, 8-row groups 1024 bytes
// apart (stride byte offset), sm_100 descriptor version 1.
__device__ inline uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((addr >> 4) & 0x3fffu);
    d |= static_cast<uint64_t>(1u) << 16;            // leading byte offset (unused for this layout)
    d |= static_cast<uint64_t>(1024u >> 4) << 32;    // stride byte offset
    d |= static_cast<uint64_t>(1u) << 46;            // version
    d |= static_cast<uint64_t>(2u) << 61;            // SWIZZLE_128B
    return d;
}

template <int F>
struct Fmt;
template <>
struct Fmt<kTcTF32> {
    static constexpr int elem = 4;
    static constexpr uint32_t ab = 2;  // TF32
};
template <>
struct Fmt<kTcBF16> {
    static constexpr int elem = 2;
    static constexpr uint32_t ab = 1;  // BF16
};
template <>
struct Fmt<kTcE4M3> {
    static constexpr int elem = 1;
    static constexpr uint32_t ab = 0;  // E4M3
};

// Instruction descriptor: FP32 accumulate, A/B format, both K-major, N = 128, M = 128.
template <int F>
__device__ constexpr uint32_t instr_desc() {
    return (1u << 4) | (Fmt<F>::ab << 7) | (Fmt<F>::ab << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
}

template <int F>
__device__ inline void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    const uint32_t idesc = instr_desc<F>();
    if constexpr (F == kTcTF32) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
    } else if constexpr (F == kTcBF16) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
    }
}

__device__ inline void mma_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ inline void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ inline void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// ---- SM-pair (cta_group::2) primitives ----
__device__ inline uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// Address of the same shared-memory object in CTA `rank` of the cluster.
__device__ inline uint32_t peer_addr(const void* p, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
    return r;
}

// Arrive on a barrier of another CTA of the cluster. Release at CTA scope (the default): what it
// publishes are async-proxy results (TMA writes, completed TMEM reads) that are complete before the
// arrive executes; a cluster-scope release would also wait for this thread's unrelated loads.
__device__ inline void mbar_arrive_cluster(uint32_t cluster_addr) {
    asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}

__device__ inline void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Wait on a local barrier that other CTAs of the cluster arrive on (acquire at cluster scope).
__device__ inline bool mbar_try_cluster(unsigned long long* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Pair MMA: D (this CTA's 128 query rows x 256 doc columns, in each CTA's TMEM) += A (128 query rows in
// each CTA) x B (128 doc rows in each CTA), issued by the even CTA for both.
template <int F>
__device__ inline void mma_pair(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    if constexpr (F == kTcTF32) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
    } else if constexpr (F == kTcBF16) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
    }
}

// Arrives on `bar` (same offset) in both CTAs of the pair once the pair MMAs issued so far complete.
__device__ inline void mma_commit_pair(unsigned long long* bar) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            smem_u32(bar)),
        "h"(static_cast<unsigned short>(3))
        : "memory");
}

// Arrives on this CTA's `bar` once the pair MMAs issued so far complete.
__device__ inline void mma_commit_pair_local(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 32 lanes x 32 consecutive FP32 columns; thread i gets lane (base lane + i). The registers are
// written asynchronously: they are valid only after tmem_wait_ld() and a reg_fence() over them.
__device__ inline void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}

__device__ inline void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Ties 32 registers to this point of the program (after tmem_wait_ld), so no use of them -- and no
// copy the compiler might make -- is placed before the wait.
__device__ inline void reg_fence(uint32_t (&r)[32]) {
    asm volatile(""
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                   "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                   "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
                 :
                 : "memory");
}

// Three-input maximum (one instruction on sm_100).
__device__ inline float max3(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Maximum of a lane's 32 scores as a tree of three-input maxima (four dependent steps, not sixteen:
// the epilogue warps have little else to hide the latency behind).
__device__ inline float max32(const uint32_t (&r)[32]) {
    float a[11];
#pragma unroll
    for (int i = 0; i < 10; ++i)
        a[i] = max3(__uint_as_float(r[3 * i]), __uint_as_float(r[3 * i + 1]), __uint_as_float(r[3 * i + 2]));
    a[10] = fmaxf(__uint_as_float(r[30]), __uint_as_float(r[31]));
    const float b0 = max3(a[0], a[1], a[2]), b1 = max3(a[3], a[4], a[5]), b2 = max3(a[6], a[7], a[8]);
    const float b3 = fmaxf(a[9], a[10]);
    return fmaxf(max3(b0, b1, b2), b3);
}

// Maximum of the 8 scores v[8k .. 8k + 7] (three steps).
__device__ __forceinline__ float max8(const uint32_t (&v)[32], int k) {
    const float a = max3(__uint_as_float(v[8 * k]), __uint_as_float(v[8 * k + 1]), __uint_as_float(v[8 * k + 2]));
    const float b = max3(__uint_as_float(v[8 * k + 3]), __uint_as_float(v[8 * k + 4]), __uint_as_float(v[8 * k + 5]));
    return max3(a, b, fmaxf(__uint_as_float(v[8 * k + 6]), __uint_as_float(v[8 * k + 7])));
}

// v[8k + j] for a lane-varying j < 8, as a three-level select tree over registers (no local array).
__device__ __forceinline__ uint32_t pick8(const uint32_t (&v)[32], int k, uint32_t j) {
    uint32_t a[4], b[2];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = (j & 4u) ? v[8 * k + 4 + i] : v[8 * k + i];
#pragma unroll
    for (int i = 0; i < 2; ++i) b[i] = (j & 2u) ? a[2 + i] : a[i];
    return (j & 1u) ? b[1] : b[0];
}

// One 32-doc chunk of a thread's TF32 / BF16 scores (its query): the docs whose filter bit (m) is set
// and whose approximate score clears the threshold t go to the thread's list segment, in doc order.
// The epilogue runs on the ALU pipe (compares, maxima, selects), so the chunk is tested as four 8-doc
// groups: only a group whose maximum clears t builds a keep mask, and a kept doc is picked from its
// group's 8 registers. The loop runs once per kept doc (typically zero or one per chunk).
__device__ __forceinline__ void emit_lane(uint32_t m, const uint32_t (&v)[32], float t, uint64_t doc0,
                                          float* out_score, uint32_t* out_loc, uint32_t seg_cap, uint32_t& ncand) {
    if (m == 0u) return;
    float g[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) g[k] = max8(v, k);
    if (!(fmaxf(max3(g[0], g[1], g[2]), g[3]) >= t)) return;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t mk = (m >> (8 * k)) & 0xffu;
        if (mk == 0u || !(g[k] >= t)) continue;
        uint32_t pass = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) pass |= (__uint_as_float(v[8 * k + j]) >= t ? 1u : 0u) << j;
        pass &= mk;
        while (pass != 0u) {
            const uint32_t j = static_cast<uint32_t>(__ffs(pass) - 1);
            pass &= pass - 1u;
            if (ncand < seg_cap) {
                out_score[ncand] = __uint_as_float(pick8(v, k, j));
                out_loc[ncand] = static_cast<uint32_t>(doc0 + 8u * k + j);
            }
            ++ncand;
        }
    }
}

// Threshold on a tile's raw E4M3 accumulators: every doc of the tile whose dequantised score
// acc * qs * ds (ds in [mm.x, mm.y], both positive) reaches theta has acc >= the returned value.
// The two divisions round to nearest; the result is then lowered by a relative 2^-20 (plus a tiny
// absolute step) whatever its sign, so it stays below the exact quotient. NaN (no query) gives -inf.
__device__ __forceinline__ float e4m3_tile_threshold(float theta, float qs, float2 mm) {
    const float tq = theta / qs;
    float t = tq > 0.0f ? tq / mm.y : tq / mm.x;
    if (!(t == t)) return -INFINITY;
    return __fsub_rd(t, __fmaf_ru(fabsf(t), 0x1p-20f, 1e-30f));
}

// One 32-doc chunk of a thread's E4M3 scores (its query, raw accumulators v): the docs whose filter
// bit (m) is set and whose dequantised score clears the threshold go to the thread's list segment.
// Warp-collective: the warp leaves at once when no lane's chunk clears its tile threshold t, and the
// emission loop visits only doc positions that some lane keeps (E4M3's wide bound lets many chunks
// through; for TF32 / BF16 the per-lane form in the kernels measured faster).
template <int F>
__device__ __forceinline__ void emit_chunk(bool live, uint32_t m, const uint32_t (&v)[32], float t, float theta,
                                           float qs, const float* doc_scale, uint64_t doc0, float* out_score,
                                           uint32_t* out_loc, uint32_t seg_cap, uint32_t& ncand) {
    const bool hot = live && m != 0u && max32(v) >= t;
    if (!__any_sync(0xffffffffu, hot)) return;
    uint32_t pass = 0;
    if (hot) {
#pragma unroll
        for (int j = 0; j < 32; ++j) pass |= (__uint_as_float(v[j]) >= t ? 1u : 0u) << j;
        pass &= m;
        if (F == kTcE4M3) {  // the tile threshold is conservative: apply the doc's own scale
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (((pass >> j) & 1u) && !(__uint_as_float(v[j]) * qs * doc_scale[doc0 + j] >= theta))
                    pass &= ~(1u << j);
        }
    }
    const uint32_t any = __reduce_or_sync(0xffffffffu, pass);
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        if (!((any >> j) & 1u)) continue;  // warp-uniform
        if ((pass >> j) & 1u) {
            float sc = __uint_as_float(v[j]);
            if (F == kTcE4M3) sc = sc * qs * doc_scale[doc0 + j];
            if (ncand < seg_cap) {
                out_score[ncand] = sc;
                out_loc[ncand] = static_cast<uint32_t>(doc0 + j);
            }
            ++ncand;
        }
    }
}

template <int F, int H>
__global__ void __launch_bounds__(64 + 256 * H, 1) tc_cand_kernel(const __grid_constant__ CUtensorMap doc_map,
                                                                  const __grid_constant__ CUtensorMap qry_map,
                                                                  TcCandLaunch L) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte aligned operand region: queries [H][kb][16 KB], then the stage ring
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t kb_n = L.kblocks;
    const uint32_t G = L.group;                           // k-blocks per stage
    const uint32_t sg_n = kb_n / G;                       // stages per tile
    const size_t stage_bytes = static_cast<size_t>(G) * kStageBytes;
    unsigned char* qsm = base;
    unsigned char* ring = base + static_cast<size_t>(H) * kb_n * kStageBytes;
    TcShared& S = *reinterpret_cast<TcShared*>(ring + static_cast<size_t>(L.stages) * stage_bytes);

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t stages = L.stages;

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < stages; ++s) {
            mbar_init(&S.full[s], 1);
            mbar_init(&S.empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&S.acc_full[b], 1);
            mbar_init(&S.acc_empty[b], 8 * H);  // one arrival per epilogue warp
        }
        mbar_init(&S.qbar, 1);
        mbar_init(&S.drain, 1);
        S.abort = 0;
        S.n_issued = 0;
        S.n_consumed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                     "r"(static_cast<uint32_t>(256 * H)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    fence_after();
    const uint32_t tmem = S.tmem_base;
    const uint64_t ntiles = L.tile_count;
    const long long budget = L.wait_budget > 0 ? L.wait_budget : kWaitBudget;

    if (warp == 0) {
        if (lane == 0) {
            // queries once
            mbar_expect_tx(&S.qbar, static_cast<uint32_t>(H) * kb_n * kStageBytes);
            for (int h = 0; h < H; ++h)
                for (uint32_t kb = 0; kb < kb_n; ++kb)
                    tma_load_2d(qsm + (static_cast<size_t>(h) * kb_n + kb) * kStageBytes, &qry_map,
                                static_cast<int>(kb * (128 / Fmt<F>::elem)), h * kRows, &S.qbar);
            uint32_t n = 0;
            bool held = false;
            TileWalk walk(L.tile_begin, L.tile_step, L.tile_skip, blockIdx.x, gridDim.x);
            for (uint64_t it = blockIdx.x; it < ntiles && !S.abort && !held; it += gridDim.x, walk.advance()) {
                const int y = static_cast<int>(walk.tile() * kRows);
                for (uint32_t g = 0; g < sg_n; ++g, ++n) {
                    const uint32_t s = n % stages, ph = (n / stages) & 1u;
                    if (L.hold_load && n + 1 >= L.hold_load) {  // pipeline test: stop issuing here
                        held = true;
                        break;
                    }
                    if (!mbar_wait(&S.empty[s], ph ^ 1u, S, L.error, 1, budget)) break;
                    mbar_expect_tx(&S.full[s], static_cast<uint32_t>(stage_bytes));
                    for (uint32_t j = 0; j < G; ++j)
                        tma_load_2d(ring + s * stage_bytes + j * kStageBytes, &doc_map,
                                    static_cast<int>((g * G + j) * (128 / Fmt<F>::elem)), y, &S.full[s]);
                }
            }
            S.n_issued = n;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            uint32_t n = 0, iter = 0;
            if (!mbar_wait(&S.qbar, 0, S, L.error, 2, budget)) iter = 0xffffffffu;  // nothing to issue
            for (uint64_t it = blockIdx.x; iter != 0xffffffffu && it < ntiles && !S.abort; it += gridDim.x, ++iter) {
                const uint32_t buf = iter & 1u;
                if (!mbar_wait(&S.acc_empty[buf], ((iter >> 1) & 1u) ^ 1u, S, L.error, 4, budget)) break;
                fence_after();
                bool ok = true;
                for (uint32_t g = 0; g < sg_n; ++g, ++n) {
                    const uint32_t s = n % stages, ph = (n / stages) & 1u;
                    if (!mbar_wait(&S.full[s], ph, S, L.error, 8, budget)) {
                        ok = false;
                        break;
                    }
                    fence_after();
                    for (uint32_t j = 0; j < G; ++j) {
                        const uint32_t kb = g * G + j;
                        const uint64_t bdesc = smem_desc(smem_u32(ring + s * stage_bytes + j * kStageBytes));
#pragma unroll
                        for (uint32_t ks = 0; ks < 4; ++ks) {  // 32 bytes of K per instruction
#pragma unroll
                            for (int h = 0; h < H; ++h) {
                                const uint64_t adesc =
                                    smem_desc(smem_u32(qsm + (static_cast<size_t>(h) * kb_n + kb) * kStageBytes));
                                mma<F>(tmem + (buf * H + h) * 128u, adesc + ks * 2u, bdesc + ks * 2u, (kb | ks) != 0);
                            }
                        }
                    }
                    mma_commit(&S.empty[s]);  // frees the stage once these MMAs have read it
                }
                if (!ok) break;
                mma_commit(&S.acc_full[buf]);
            }
            S.n_consumed = n;
            // every MMA this thread issued has completed before TMEM and the stages are released
            mma_commit(&S.drain);
            if (!mbar_wait_drain(&S.drain, 0) && L.error) atomicOr(L.error, 32);
        }
    } else {
        // Epilogue: 8 warps per accumulator half. Warp w may only touch TMEM lanes 32 * (w % 4) ..
        // +31, so the warps of group g = (w - 2) / 4 cover the four lane quarters of half g / 2, and
        // the two groups of a half split its 128 doc columns (64 each). A thread owns one staged query
        // row and one column half for the whole launch: its candidate count lives in a register and
        // its candidates go to its own segment (2 per CTA) of the query's list, no atomics.
        const uint32_t g = (warp - 2) / 4;
        const uint32_t half = g / 2;
        const uint32_t colh = g % 2;
        const uint32_t sub = warp & 3u;
        const uint32_t row = half * 128u + sub * 32u + lane;
        const bool valid = row < L.nq_rows;
        const uint32_t qi = valid ? (L.qlist ? L.qlist[row] : row) : 0u;
        const float theta = valid ? L.theta[qi] : INFINITY;
        const float qs = (F == kTcE4M3 && valid) ? L.q_scale[row] : 1.0f;
        const uint64_t* brow = L.bits + static_cast<uint64_t>(qi) * L.bits_stride;
        const uint32_t segment = L.seg_base + 2u * blockIdx.x + colh;
        const uint64_t seg = static_cast<uint64_t>(qi) * L.cap + static_cast<uint64_t>(segment) * L.seg_cap;
        float* out_score = L.cand_score + seg;
        uint32_t* out_loc = L.cand_loc + seg;
        const uint32_t seg_cap = L.seg_cap;
        uint32_t ncand = 0;
        uint32_t iter = 0;
        // the query's filter bits of this thread's 64 docs, loaded one tile ahead so the (uncoalesced)
        // load is in flight during the previous tile's work
        TileWalk walk(L.tile_begin, L.tile_step, L.tile_skip, blockIdx.x, gridDim.x);
        uint64_t tile_next = walk.tile();
        uint64_t fw_next = 0;
        if (valid && blockIdx.x < ntiles) fw_next = brow[tile_next * 2 + colh];
        for (uint64_t it = blockIdx.x; it < ntiles; it += gridDim.x, ++iter) {
            const uint32_t buf = iter & 1u;
            const uint64_t tile = tile_next;
            const uint64_t fw = fw_next;
            walk.advance();
            tile_next = walk.tile();
            if (valid && it + gridDim.x < ntiles) fw_next = brow[tile_next * 2 + colh];
            // threshold on the raw accumulator: acc * qs * ds >= theta
            const float t = F == kTcE4M3 ? e4m3_tile_threshold(theta, qs, L.tile_scale[tile]) : theta;
            const uint32_t m[2] = {static_cast<uint32_t>(fw), static_cast<uint32_t>(fw >> 32)};
            // 32-doc chunks that no query of the warp lets through are not read from TMEM at all
            bool live[2];
#pragma unroll
            for (int c = 0; c < 2; ++c) live[c] = __any_sync(0xffffffffu, m[c] != 0u);
            // every lane waits; the warp leaves together if any lane gave up (the warp collectives
            // below need all 32 lanes)
            const bool ready = mbar_wait(&S.acc_full[buf], (iter >> 1) & 1u, S, L.error, 16, budget);
            if (!__all_sync(0xffffffffu, ready)) break;
            fence_after();
            const uint32_t tbase = tmem + ((sub * 32u) << 16) + (buf * H + half) * 128u + colh * 64u;
            uint32_t v[2][32];
#pragma unroll
            for (int c = 0; c < 2; ++c)
                if (live[c]) tmem_ld32(tbase + c * 32u, v[c]);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < 2; ++c) reg_fence(v[c]);
            // the accumulator is in registers: hand the TMEM buffer back to the MMA issuer now
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&S.acc_empty[buf]);
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const uint64_t doc0 = tile * kRows + colh * 64u + c * 32u;
                if constexpr (F == kTcE4M3) {
                    emit_chunk<F>(live[c], m[c], v[c], t, theta, qs, L.doc_scale, doc0, out_score, out_loc, seg_cap,
                                  ncand);
                } else if (live[c]) {
                    emit_lane(m[c], v[c], t, doc0, out_score, out_loc, seg_cap, ncand);
                }
            }
        }
        if (valid) L.cand_count[static_cast<uint64_t>(qi) * kMaxCandSegs + segment] = ncand;
    }
    __syncthreads();
    if (threadIdx.x == 0 && S.n_consumed < S.n_issued) {
        // aborted: wait (bounded) for the copies still landing in the stage ring
        for (uint32_t k = S.n_consumed; k < S.n_issued; ++k)
            if (!mbar_wait_drain(&S.full[k % stages], (k / stages) & 1u)) break;
    }
    if (threadIdx.x == 0 && !mbar_try(&S.qbar, 0)) mbar_wait_drain(&S.qbar, 0);
    __syncthreads();
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(static_cast<uint32_t>(256 * H)));
    }
}

// ---------------------------------------------------------------------------------------------
// SM-pair candidate pass (rows 129..256). A cluster of two CTAs on two SMs computes D[256 queries,
// 256 docs] per tile with one cta_group::2 MMA per 32 bytes of K: CTA r holds queries
// [128 r, 128 r + 128) (A) and streams docs [256 t + 128 r, +128) of tile t (B); each CTA's TMEM holds
// its 128 query rows x 256 doc columns. Per MMA each SM reads 8 KB of shared memory for 128 x 256
// outputs -- half the operand traffic per output of the single-SM form, which saturates shared
// memory bandwidth before the tensor pipe.
//
// Each CTA's TMA loads complete on its own barriers; warp 1 of the odd CTA forwards each completed
// stage (and the queries) to the even CTA with a remote arrive on the even CTA's barrier of the same
// stage, which therefore takes two arrivals (its own producer's and the forwarded one): the MMA
// issuer waits on one barrier per stage, and each CTA can always drain its own copies. The even
// CTA's warp 1 issues the MMAs and commits them to both CTAs' barriers. Epilogue warps of both CTAs
// return an accumulator buffer with a remote arrive on the even CTA's acc_empty. (Every wait in the
// issuer's loop costs MMA issue slots: the issuing thread does not overlap a barrier wait with the
// MMAs it has queued, so one wait per stage and stages of two k-blocks keep their number low.)
struct PairShared {
    unsigned long long full[kMaxTcStages];   // stage loaded (TMA; even CTA: also the odd CTA's, forwarded)
    unsigned long long empty[kMaxTcStages];  // stage free (pair MMA commit, both CTAs)
    unsigned long long acc_full[2];          // accumulator buffer ready (pair MMA commit, both CTAs)
    unsigned long long acc_empty[2];         // even CTA: buffer drained by the epilogue warps of both CTAs
    unsigned long long qbar;                 // queries loaded (even CTA: also the odd CTA's, forwarded)
    unsigned long long drain;
    uint32_t tmem_base;
    uint32_t n_issued, n_consumed;  // stage loads issued by TMA / waited for by the MMA issuer or forwarder
    volatile int abort;
};

// shared-memory bytes the barriers take ahead of the 1024-byte aligned query tile
constexpr size_t kPairSharedBytes = (sizeof(PairShared) + 1023) & ~static_cast<size_t>(1023);

constexpr int kPairEpiWarps = 16;  // 4 column groups x 4 TMEM lane quarters
constexpr int kPairThreads = 64 + 32 * kPairEpiWarps;

template <int F>
__device__ inline bool pair_wait(unsigned long long* bar, uint32_t parity, PairShared& S, int32_t* err, int code,
                                 bool cluster_scope) {
    // no clock read when the phase is already complete
    if (cluster_scope ? mbar_try_cluster(bar, parity) : mbar_try(bar, parity)) return true;
    const long long t0 = clock64();
    while (!(cluster_scope ? mbar_try_cluster(bar, parity) : mbar_try(bar, parity))) {
        if (S.abort) return false;
        if (clock64() - t0 > kWaitBudget) {
            S.abort = 1;
            if (err) atomicOr(err, code);
            return false;
        }
    }
    return true;
}

// SQ (streamed queries, long vectors): no resident query tile; each stage holds the query k-block
// (16 KB, from the L2-resident staged queries) followed by the doc k-block, loaded together.
template <int F, bool SQ, bool WIDE>
__global__ void __launch_bounds__(kPairThreads, 1) tc2_cand_kernel(const __grid_constant__ CUtensorMap doc_map,
                                                                  const __grid_constant__ CUtensorMap qry_map,
                                                                  TcCandLaunch L) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t kb_n = L.kblocks;
    const uint32_t G = SQ ? 1u : L.group;  // corpus k-blocks per stage
    const uint32_t sg_n = kb_n / G;        // stages per tile
    // bytes of one ring stage: G doc k-blocks, or (streamed queries) a query k-block and a doc k-block
    const size_t kStage = SQ ? 2 * kStageBytes : static_cast<size_t>(G) * kStageBytes;
    // barriers first (a fixed offset, so the epilogue keeps no pointer to them in registers), then
    // the resident query tile and the ring, both 1024-byte aligned for the 128-byte swizzle
    PairShared& S = *reinterpret_cast<PairShared*>(base);
    unsigned char* qsm = base + kPairSharedBytes;
    unsigned char* ring = qsm + (SQ ? 0 : static_cast<size_t>(kb_n) * kStageBytes);

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t stages = L.stages;
    const uint32_t rank = cluster_rank();
    const uint32_t pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < stages; ++s) {
            mbar_init(&S.full[s], rank == 0 ? 2 : 1);  // even CTA: own load + the odd CTA's, forwarded
            mbar_init(&S.empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&S.acc_full[b], 1);
            mbar_init(&S.acc_empty[b], 2 * kPairEpiWarps);
        }
        mbar_init(&S.qbar, (rank == 0 && !SQ) ? 2 : 1);
        mbar_init(&S.drain, 1);
        S.abort = 0;
        S.n_issued = 0;
        S.n_consumed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                     "r"(512u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    cluster_sync();  // both CTAs' barriers are initialised before any remote arrive
    fence_after();
    const uint32_t tmem = S.tmem_base;
    const uint64_t ntiles = L.tile_count;

    if (warp == 0) {
        if (lane == 0) {
            if (!SQ) {
                mbar_expect_tx(&S.qbar, kb_n * kStageBytes);
                for (uint32_t kb = 0; kb < kb_n; ++kb)
                    tma_load_2d(qsm + static_cast<size_t>(kb) * kStageBytes, &qry_map,
                                static_cast<int>(kb * (128 / Fmt<F>::elem)), static_cast<int>(rank * kRows), &S.qbar);
            }
            uint32_t n = 0, s = 0, ph = 0;  // stages issued; ring slot and phase of the next
            TileWalk walk(L.tile_begin, L.tile_step, L.tile_skip, pair, npairs);
            for (uint64_t it = pair; it < ntiles && !S.abort; it += npairs, walk.advance()) {
                const int y = static_cast<int>(walk.tile() * 2 * kRows + rank * kRows);
                for (uint32_t g = 0; g < sg_n; ++g, ++n, s = s + 1 == stages ? 0 : s + 1, ph ^= s == 0 ? 1u : 0u) {
                    if (!pair_wait<F>(&S.empty[s], ph ^ 1u, S, L.error, 1, false)) break;
                    unsigned char* st = ring + static_cast<size_t>(s) * kStage;
                    mbar_expect_tx(&S.full[s], static_cast<uint32_t>(kStage));
                    if (SQ) {
                        tma_load_2d(st, &qry_map, static_cast<int>(g * (128 / Fmt<F>::elem)),
                                    static_cast<int>(rank * kRows), &S.full[s]);
                        tma_load_2d(st + kStageBytes, &doc_map, static_cast<int>(g * (128 / Fmt<F>::elem)), y,
                                    &S.full[s]);
                    } else {
                        for (uint32_t j = 0; j < G; ++j)
                            tma_load_2d(st + j * kStageBytes, &doc_map,
                                        static_cast<int>((g * G + j) * (128 / Fmt<F>::elem)), y, &S.full[s]);
                    }
                }
            }
            S.n_issued = n;
        }
    } else if (warp == 1) {
        if (lane == 0 && rank == 1) {
            // forwarder: the even CTA's MMAs read this CTA's queries and stages; tell it when they land
            uint32_t n = 0, s = 0, ph = 0;
            if (SQ || pair_wait<F>(&S.qbar, 0, S, L.error, 2, false)) {
                if (!SQ) mbar_arrive_cluster(peer_addr(&S.qbar, 0));
                for (uint64_t it = pair; it < ntiles && !S.abort; it += npairs) {
                    bool ok = true;
                    for (uint32_t g = 0; g < sg_n; ++g, ++n, s = s + 1 == stages ? 0 : s + 1, ph ^= s == 0 ? 1u : 0u) {
                        if (!pair_wait<F>(&S.full[s], ph, S, L.error, 8, false)) {
                            ok = false;
                            break;
                        }
                        mbar_arrive_cluster(peer_addr(&S.full[s], 0));
                    }
                    if (!ok) break;
                }
            }
            S.n_consumed = n;
        } else if (lane == 0) {
            // MMA issuer of the pair
            constexpr uint32_t idesc =
                (1u << 4) | (Fmt<F>::ab << 7) | (Fmt<F>::ab << 10) | ((256u >> 3) << 17) | ((256u >> 4) << 24);
            uint32_t n = 0, iter = 0, s = 0, ph = 0;
            // the even CTA's query barrier completes with both CTAs' query tiles (one forwarded); a
            // one-time wait, acquired at cluster scope
            bool ok = SQ || pair_wait<F>(&S.qbar, 0, S, L.error, 2, true);
            for (uint64_t it = pair; ok && it < ntiles && !S.abort; it += npairs, ++iter) {
                const uint32_t buf = iter & 1u;
                // CTA-scope waits on the barriers the odd CTA arrives on remotely (as its arrives are
                // CTA-scope): a cluster-scope acquire on every stage cost the TF32 pass about 4 %
                if (!pair_wait<F>(&S.acc_empty[buf], ((iter >> 1) & 1u) ^ 1u, S, L.error, 4, false)) break;
                fence_after();
                for (uint32_t g = 0; g < sg_n; ++g, ++n, s = s + 1 == stages ? 0 : s + 1, ph ^= s == 0 ? 1u : 0u) {
                    // both CTAs' halves of the stage: this CTA's load and the odd CTA's, forwarded
                    if (!pair_wait<F>(&S.full[s], ph, S, L.error, 8, false)) {
                        ok = false;
                        break;
                    }
                    fence_after();
                    unsigned char* st = ring + static_cast<size_t>(s) * kStage;
                    for (uint32_t j = 0; j < G; ++j) {
                        const uint32_t kb = g * G + j;
                        const uint64_t adesc =
                            smem_desc(smem_u32(SQ ? st : qsm + static_cast<size_t>(kb) * kStageBytes));
                        const uint64_t bdesc = smem_desc(smem_u32(st + (SQ ? kStageBytes : j * kStageBytes)));
#pragma unroll
                        for (uint32_t ks = 0; ks < 4; ++ks)  // 32 bytes of K per instruction
                            mma_pair<F>(tmem + buf * 256u, adesc + ks * 2u, bdesc + ks * 2u, idesc, (kb | ks) != 0);
                    }
                    mma_commit_pair(&S.empty[s]);  // frees the stage in both CTAs once read
                }
                if (!ok) break;
                mma_commit_pair(&S.acc_full[buf]);
            }
            S.n_consumed = n;
            mma_commit_pair_local(&S.drain);  // every pair MMA issued has completed
            if (!mbar_wait_drain(&S.drain, 0) && L.error) atomicOr(L.error, 32);
        }
    } else {
        // Epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (query rows) and doc columns
        // [64 g, 64 g + 64) of the 256, g = (w - 2) / 4. A thread owns one query row and one 64-doc
        // column group for the whole launch: candidates go to its own list segment, no atomics.
        const uint32_t g = (warp - 2) / 4;
        const uint32_t sub = warp & 3u;
        const uint32_t row = rank * 128u + sub * 32u + lane;
        const bool valid = row < L.nq_rows;
        const uint32_t qi = valid ? (L.qlist ? L.qlist[row] : row) : 0u;
        const float theta = valid ? L.theta[qi] : INFINITY;
        const float qs = (F == kTcE4M3 && valid) ? L.q_scale[row] : 1.0f;
        const uint64_t* brow = L.bits + static_cast<uint64_t>(qi) * L.bits_stride;
        const uint32_t segment = L.seg_base + 4u * pair + g;
        const uint64_t seg = static_cast<uint64_t>(qi) * L.cap + static_cast<uint64_t>(segment) * L.seg_cap;
        float* out_score = L.cand_score + seg;
        uint32_t* out_loc = L.cand_loc + seg;
        const uint32_t seg_cap = L.seg_cap;
        const uint32_t acc_empty_addr0 = peer_addr(&S.acc_empty[0], 0);
        const uint32_t acc_empty_addr1 = peer_addr(&S.acc_empty[1], 0);
        uint32_t ncand = 0;
        uint32_t iter = 0;
        // filter word of this thread's 64 docs of a tile (past the bitmap: none pass)
        auto word_of = [&](uint64_t tile) -> uint64_t {
            const uint64_t w = tile * 4 + g;
            return (valid && w < L.bits_stride) ? brow[w] : 0ull;
        };
        // 32-bit tile counters (the launcher checks tile_walk_fits): registers are tight at 576 threads
        TileWalk walk(L.tile_begin, L.tile_step, L.tile_skip, pair, npairs);
        const uint32_t nt = static_cast<uint32_t>(ntiles);
        uint32_t tile_next = static_cast<uint32_t>(walk.tile());
        uint64_t fw_next = pair < nt ? word_of(tile_next) : 0ull;
        for (uint32_t it = pair; it < nt; it += npairs, ++iter) {
            const uint32_t buf = iter & 1u;
            const uint64_t tile = tile_next;
            const uint64_t fw = fw_next;
            walk.advance();
            tile_next = static_cast<uint32_t>(walk.tile());
            if (it + npairs < nt) fw_next = word_of(tile_next);
            float t = theta;
            if (F == kTcE4M3) {
                uint64_t ts = tile * 2 + g / 2;  // 128-doc tile holding this thread's docs
                ts = ts < L.tiles128 ? ts : L.tiles128 - 1;
                t = e4m3_tile_threshold(theta, qs, L.tile_scale[ts]);
            }
            const uint32_t m[2] = {static_cast<uint32_t>(fw), static_cast<uint32_t>(fw >> 32)};
            bool live[2];
#pragma unroll
            for (int c = 0; c < 2; ++c) live[c] = __any_sync(0xffffffffu, m[c] != 0u);
            const bool ready = pair_wait<F>(&S.acc_full[buf], (iter >> 1) & 1u, S, L.error, 16, false);
            if (!__all_sync(0xffffffffu, ready)) break;
            fence_after();
            const uint32_t tbase = tmem + ((sub * 32u) << 16) + buf * 256u + g * 64u;
            if constexpr (WIDE) {
                // a pass that keeps most docs (the doc sample): both chunks in registers, the buffer
                // back to the issuer before the long emission (spills a little at 96 registers)
                uint32_t v[2][32];
#pragma unroll
                for (int c = 0; c < 2; ++c)
                    if (live[c]) tmem_ld32(tbase + c * 32u, v[c]);
                tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < 2; ++c) reg_fence(v[c]);
                fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_cluster(buf ? acc_empty_addr1 : acc_empty_addr0);
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const uint64_t doc0 = tile * 256u + g * 64u + c * 32u;
                    if constexpr (F == kTcE4M3) {
                        emit_chunk<F>(live[c], m[c], v[c], t, theta, qs, L.doc_scale, doc0, out_score, out_loc,
                                      seg_cap, ncand);
                    } else if (live[c]) {
                        emit_lane(m[c], v[c], t, doc0, out_score, out_loc, seg_cap, ncand);
                    }
                }
            } else {
                // one 32-doc chunk in registers at a time (79 registers, where both chunks at once
                // spilled at the 96-register ceiling); the buffer goes back to the issuer once the
                // second is loaded
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    uint32_t v[32];
                    if (live[c]) tmem_ld32(tbase + c * 32u, v);
                    tmem_wait_ld();
                    reg_fence(v);
                    if (c == 1) {
                        fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive_cluster(buf ? acc_empty_addr1 : acc_empty_addr0);
                    }
                    const uint64_t doc0 = tile * 256u + g * 64u + c * 32u;
                    if constexpr (F == kTcE4M3) {
                        emit_chunk<F>(live[c], m[c], v, t, theta, qs, L.doc_scale, doc0, out_score, out_loc, seg_cap,
                                      ncand);
                    } else if (live[c]) {
                        emit_lane(m[c], v, t, doc0, out_score, out_loc, seg_cap, ncand);
                    }
                }
            }
        }
        if (valid) L.cand_count[static_cast<uint64_t>(qi) * kMaxCandSegs + segment] = ncand;
    }
    __syncthreads();
    if (threadIdx.x == 0 && S.n_consumed < S.n_issued) {
        // aborted: wait (bounded) for this CTA's copies still landing in its stage ring
        for (uint32_t k = S.n_consumed; k < S.n_issued; ++k)
            if (!mbar_wait_drain(&S.full[k % stages], (k / stages) & 1u)) break;
    }
    if (!SQ && threadIdx.x == 0 && !mbar_try(&S.qbar, 0)) mbar_wait_drain(&S.qbar, 0);
    __syncthreads();
    // neither CTA leaves (or frees TMEM) while the pair's MMAs or the other CTA's remote arrives may
    // still touch its shared memory
    cluster_sync();
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u));
    }
}

constexpr size_t kTcSmemCeiling = 232448;  // dynamic shared memory of one CTA (the launchers check smem <= it)

template <int F, bool SQ>
cudaError_t launch_tc2_typed(const TcCandLaunch& L, const CUtensorMap& dmap, const CUtensorMap& qmap,
                             cudaStream_t stream) {
    const size_t smem = tc_pair_smem_bytes(L.kblocks, L.stages, L.group);
    auto kernel = L.emit_all ? tc2_cand_kernel<F, SQ, true> : tc2_cand_kernel<F, SQ, false>;
    // the ceiling, not this launch's size: searchers of other tables launch it concurrently
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kTcSmemCeiling));
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(L.ctas, 1, 1);
    cfg.blockDim = dim3(kPairThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, dmap, qmap, L);
}

template <int F>
cudaError_t launch_tc1_typed(const TcCandLaunch& L, const CUtensorMap& dmap, const CUtensorMap& qmap,
                             cudaStream_t stream) {
    const size_t smem = tc_smem_bytes(1, L.kblocks, L.stages, L.group);
    cudaError_t e = cudaFuncSetAttribute(tc_cand_kernel<F, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kTcSmemCeiling));
    if (e != cudaSuccess) return e;
    tc_cand_kernel<F, 1><<<L.ctas, 64 + 256, smem, stream>>>(dmap, qmap, L);
    return cudaGetLastError();
}

constexpr size_t kSmemBudget = 232448;  // dynamic shared memory of one CTA

}  // namespace

bool tc_stream_queries(uint32_t kblocks) {
    return 1024 + kPairSharedBytes + (static_cast<size_t>(kblocks) + 4) * kStageBytes > kSmemBudget;
}

uint32_t tc_tile_docs(uint32_t rows, uint32_t kblocks) {
    return rows > 128 || tc_stream_queries(kblocks) ? 256u : 128u;
}

uint32_t tc_cand_ctas(uint32_t rows, uint32_t kblocks, uint64_t tile_count, int num_sms, uint32_t cap) {
    // every CTA fills two list segments; two passes' segments must fit kMaxCandSegs with at least
    // kMinSegCap entries each
    const uint64_t unit = tc_tile_docs(rows, kblocks) == 256u ? 2 : 1;  // CTAs per tile group
    uint64_t g = static_cast<uint64_t>(num_sms) / unit;
    g = tile_count < g ? tile_count : g;
    const uint64_t by_segs = kMaxCandSegs / (4 * unit);
    g = g < by_segs ? g : by_segs;
    uint64_t by_cap = cap / (4 * unit * kMinSegCap);
    by_cap = by_cap > 0 ? by_cap : 1;
    g = g < by_cap ? g : by_cap;
    return static_cast<uint32_t>(g * unit);
}

size_t tc_smem_bytes(int halves, uint32_t kblocks, uint32_t stages, uint32_t group) {
    return 1024 + static_cast<size_t>(halves) * kblocks * kStageBytes +
           static_cast<size_t>(stages) * group * kStageBytes + sizeof(TcShared);
}

size_t tc_pair_smem_bytes(uint32_t kblocks, uint32_t stages, uint32_t group) {
    if (tc_stream_queries(kblocks))  // no resident queries; a stage holds a query and a doc k-block
        return 1024 + kPairSharedBytes + static_cast<size_t>(stages) * 2 * kStageBytes;
    return 1024 + kPairSharedBytes + static_cast<size_t>(kblocks) * kStageBytes +
           static_cast<size_t>(stages) * group * kStageBytes;
}

uint32_t tc_group(uint32_t kblocks, bool pair) {
    if (kblocks % 2 != 0 || (pair && tc_stream_queries(kblocks))) return 1;
    const size_t fixed = pair ? tc_pair_smem_bytes(kblocks, 0, 2) : tc_smem_bytes(1, kblocks, 0, 2);
    return fixed + 3 * 2 * static_cast<size_t>(kStageBytes) <= kSmemBudget ? 2u : 1u;
}

cudaError_t launch_tc_cand(const TcCandLaunch& Lin, const CUtensorMap& doc_map, const CUtensorMap& qry_map, int sms,
                           cudaStream_t stream) {
    if (Lin.tile_count == 0 || Lin.nq_rows == 0) return cudaSuccess;
    if (Lin.kblocks == 0 || Lin.nq_rows > 256 || Lin.tiles128 == 0 ||
        !tile_walk_fits(Lin.tile_begin, Lin.tile_step, Lin.tile_skip, Lin.tile_count, Lin.ctas))
        return cudaErrorInvalidValue;
    TcCandLaunch L = Lin;
    const bool sq = tc_stream_queries(L.kblocks);
    const bool pair = tc_tile_docs(L.nq_rows, L.kblocks) == 256u;
    // as many stages as shared memory holds next to the resident queries (or, streamed, as many
    // query + doc stage pairs as it holds); a stage holds `group` doc k-blocks
    L.group = tc_group(L.kblocks, pair);
    const size_t stage = sq ? 2 * kStageBytes : static_cast<size_t>(L.group) * kStageBytes;
    const size_t fixed = pair ? tc_pair_smem_bytes(L.kblocks, 0, L.group) : tc_smem_bytes(1, L.kblocks, 0, L.group);
    if (fixed + 2 * stage > kSmemBudget) return cudaErrorInvalidValue;
    const size_t st = (kSmemBudget - fixed) / stage;
    L.stages = static_cast<uint32_t>(st < static_cast<size_t>(kMaxTcStages) ? st : kMaxTcStages);
    // every CTA writes segments seg_base + 2 b and seg_base + 2 b + 1 (pair: 4 per pair)
    const uint64_t seg_end = static_cast<uint64_t>(L.seg_base) + 2ull * L.ctas;
    if (L.ctas != tc_cand_ctas(L.nq_rows, L.kblocks, L.tile_count, sms, L.cap) || L.seg_cap == 0 || seg_end > kMaxCandSegs ||
        seg_end * L.seg_cap > L.cap)
        return cudaErrorInvalidValue;
    switch (L.format) {
        case kTcTF32: return sq ? launch_tc2_typed<kTcTF32, true>(L, doc_map, qry_map, stream)
                                : pair ? launch_tc2_typed<kTcTF32, false>(L, doc_map, qry_map, stream)
                                       : launch_tc1_typed<kTcTF32>(L, doc_map, qry_map, stream);
        case kTcBF16: return sq ? launch_tc2_typed<kTcBF16, true>(L, doc_map, qry_map, stream)
                                : pair ? launch_tc2_typed<kTcBF16, false>(L, doc_map, qry_map, stream)
                                       : launch_tc1_typed<kTcBF16>(L, doc_map, qry_map, stream);
        case kTcE4M3: return sq ? launch_tc2_typed<kTcE4M3, true>(L, doc_map, qry_map, stream)
                                : pair ? launch_tc2_typed<kTcE4M3, false>(L, doc_map, qry_map, stream)
                                       : launch_tc1_typed<kTcE4M3>(L, doc_map, qry_map, stream);
    }
    return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------------------------
// Tensor maps (cuTensorMapEncodeTiled through the runtime's driver entry point; no libcuda link).
namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}
}  // namespace

bool make_tc_map(CUtensorMap* map, int format, const void* base, uint64_t rows, uint32_t dim) {
    auto fn = encode_fn();
    if (!fn) return false;
    const uint32_t elem = format == kTcTF32 ? 4 : (format == kTcBF16 ? 2 : 1);
    const CUtensorMapDataType dt = format == kTcTF32   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : format == kTcBF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                       : CU_TENSOR_MAP_DATA_TYPE_UINT8;
    if ((reinterpret_cast<uintptr_t>(base) & 15u) || (static_cast<uint64_t>(dim) * elem) % 128 != 0) return false;
    cuuint64_t gdim[2] = {dim, rows};
    cuuint64_t gstride[1] = {static_cast<cuuint64_t>(dim) * elem};
    cuuint32_t box[2] = {128u / elem, 128u};
    cuuint32_t estride[2] = {1, 1};
    const CUresult r = fn(map, dt, 2, const_cast<void*>(base), gdim, gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace hss
