// select.cu -- selection kernels.
//
//  * sample_threshold_kernel: per query, the K-th best approximate score of a doc sample, lowered by
//    the error bounds into a threshold that every true top-K doc is guaranteed to clear.
//  * select_topk_kernel: per query, from the candidate list: the K-th best approximate score, the
//    set of candidates that can still reach the top K, their exact FP32 rescoring in the ground
//    truth's order, and the final deterministic top K (score desc, doc id asc).
//  * aggregate_* kernels: stable compaction of (score, location) by the filter bitmap -- the
//    reference's Aggregator operator (kernel_aggregator.h:18-206) without the host count round trip.
//  * topk_op_kernel: exact top K of a compacted (score, location) list -- the reference's TOPK
//    operator (kernel_topk.h:27-419), which there is only a pivot pre-select followed by a host sort.
#include "hss_device.cuh"
#include "hss_kernels.h"

namespace hss {
namespace {

constexpr int kST = 1024;             // threads of the selection CTAs
constexpr int kHist = 16;             // radix histograms per CTA (warp w adds to hist[w % kHist])
// candidate scores a select CTA holds in shared memory: kSelFast, or kSelFastLarge for batches whose
// lists run long (large K). The larger buffer leaves less of the SM's memory to L1, which costs the
// short lists' select step (K = 100: 0.098 -> 0.112 ms at 10M), so it is taken only where asked.
constexpr uint32_t kSelFast = 12288;
constexpr uint32_t kSelFastLarge = 32768;

struct SelectSmem {
    uint32_t hist[kHist][256];                  // radix histograms
    unsigned long long sortbuf[kMaxTopK];       // bitonic sort buffer
    uint32_t segn[kMaxCandSegs];                // stored entries of each candidate segment
    uint32_t segoff[kMaxCandSegs];              // their exclusive prefix sum (scan_segments)
    uint32_t bcast[4];
    uint32_t counter;
    uint32_t total;                             // stored entries (load_segments)
    uint32_t wsum[kST / 32];
};

// Merges the histograms into hist[0] and picks, from the top, the digit holding the k-th
// largest key. Returns the digit and updates *krem to the rank inside that digit.
__device__ inline uint32_t pick_digit(SelectSmem& S, uint32_t* krem) {
    const uint32_t tid = threadIdx.x;
    if (tid < 256) {
        uint32_t s = 0;
        for (int w = 0; w < kHist; ++w) s += S.hist[w][tid];
        S.hist[0][tid] = s;
    }
    __syncthreads();
    if (tid < 32) {
        // warp 0 scans the 256 digits from the top: lane l owns digits 255 - 8l .. 248 - 8l
        const uint32_t lane = tid;
        const uint32_t kr = *krem;
        uint32_t h[8], local = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            h[i] = S.hist[0][255 - 8 * lane - i];
            local += h[i];
        }
        uint32_t incl = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= static_cast<uint32_t>(o)) incl += y;
        }
        const uint32_t excl = incl - local;
        // the first lane whose digits bring the running count to kr holds the k-th largest key
        const uint32_t hit = __ballot_sync(0xffffffffu, excl < kr && incl >= kr);
        if (hit && lane == static_cast<uint32_t>(__ffs(hit) - 1)) {
            uint32_t cum = excl;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (cum + h[i] >= kr) {
                    S.bcast[0] = 255 - 8 * lane - i;
                    S.bcast[1] = kr - cum;
                    break;
                }
                cum += h[i];
            }
        }
    }
    __syncthreads();
    const uint32_t chosen = S.bcast[0];
    *krem = S.bcast[1];
    __syncthreads();
    return chosen;
}

// Counts digit d (< 256; 256 = nothing) of each calling lane into hist_row. Lanes holding the same
// digit add once, together: candidate scores cluster (a query's nearest cluster scores within a few
// hundredths), so most of a warp's keys share their leading digits and 32 increments of one
// shared-memory word would serialise.
__device__ __forceinline__ void hist_add(uint32_t* hist_row, uint32_t d) {
    const uint32_t active = __activemask();
    const uint32_t grp = __match_any_sync(active, d);
    if (d < 256u && (threadIdx.x & 31u) == static_cast<uint32_t>(__ffs(grp) - 1))
        atomicAdd(&hist_row[d], static_cast<uint32_t>(__popc(grp)));
}

__device__ inline void clear_hist(SelectSmem& S) {
    for (uint32_t i = threadIdx.x; i < kHist * 256; i += blockDim.x) (&S.hist[0][0])[i] = 0;
    __syncthreads();
}

// k-th largest (1-based, k <= the number of keys) of the u32 keys that visit(fn) hands to fn.
template <class Visit>
__device__ uint32_t kth_largest_u32_visit(Visit visit, uint32_t k, SelectSmem& S) {
    uint32_t prefix = 0, mask = 0, krem = k;
    const uint32_t warp = threadIdx.x >> 5;
    for (int shift = 24; shift >= 0; shift -= 8) {
        clear_hist(S);
        visit([&](uint32_t v) {
            hist_add(S.hist[warp % kHist], (v & mask) == prefix ? ((v >> shift) & 255u) : 256u);
        });
        __syncthreads();
        const uint32_t d = pick_digit(S, &krem);
        prefix |= d << shift;
        mask |= 255u << shift;
    }
    return prefix;
}

// Picks, from the top of a 4096-bin histogram, the bin holding the k-th largest key (blockDim.x ==
// kST: thread t owns bins 4095 - 4t .. 4092 - 4t). Returns the bin; *krem becomes the rank inside it.
__device__ inline uint32_t pick_digit4096(const uint32_t* hist, uint32_t* krem, SelectSmem& S) {
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t kr = *krem;
    uint32_t h[4], local = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        h[j] = hist[4095 - 4 * t - j];
        local += h[j];
    }
    uint32_t x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= static_cast<uint32_t>(o)) x += y;
    }
    if (lane == 31) S.wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = S.wsum[lane];
        uint32_t z = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= static_cast<uint32_t>(o)) z += y;
        }
        S.wsum[lane] = z - w;  // exclusive over warps
    }
    __syncthreads();
    const uint32_t incl = S.wsum[warp] + x, excl = incl - local;
    if (excl < kr && incl >= kr) {  // exactly one thread
        uint32_t cum = excl;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (cum + h[j] >= kr) {
                S.bcast[0] = 4095 - 4 * t - j;
                S.bcast[1] = kr - cum;
                break;
            }
            cum += h[j];
        }
    }
    __syncthreads();
    const uint32_t d = S.bcast[0];
    *krem = S.bcast[1];
    __syncthreads();
    return d;
}

// A lower bound of the k-th largest (1-based, k <= the number of keys) of the u32 keys that visit(fn)
// hands to fn: the k-th largest key's top 24 bits with the low 8 bits cleared. Every key sharing that
// prefix is >= the result, so at least k keys are >= it -- all a proven threshold or a rescoring cut
// needs -- and as an order-preserving float key it is at most 2^-15 (relative) below the k-th
// largest. Two passes of 12-bit digits over one 4096-bin histogram; each thread merges runs of equal
// digits before adding them (keys of one query cluster, so consecutive keys mostly share a digit).
template <class Visit>
__device__ uint32_t kth_lower_bound_u32_visit(Visit visit, uint32_t k, SelectSmem& S) {
    uint32_t* hist = &S.hist[0][0];
    static_assert(sizeof(S.hist) / sizeof(uint32_t) >= 4096, "4096-bin histogram");
    uint32_t prefix = 0, mask = 0, krem = k;
    for (int pass = 0; pass < 2; ++pass) {
        const int shift = pass == 0 ? 20 : 8;
        for (uint32_t i = threadIdx.x; i < 4096; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        uint32_t cur = 0, cnt = 0;
        visit([&](uint32_t v) {
            if ((v & mask) != prefix) return;
            const uint32_t d = (v >> shift) & 4095u;
            if (d != cur) {
                if (cnt) atomicAdd(&hist[cur], cnt);
                cur = d;
                cnt = 0;
            }
            ++cnt;
        });
        if (cnt) atomicAdd(&hist[cur], cnt);
        __syncthreads();
        const uint32_t d = pick_digit4096(hist, &krem, S);
        prefix |= d << shift;
        mask |= 4095u << shift;
    }
    return prefix;
}

// k-th largest (1-based, k <= n) of n u32 keys produced by key(i).
template <class KeyFn>
__device__ uint32_t kth_largest_u32(KeyFn key, uint32_t n, uint32_t k, SelectSmem& S) {
    return kth_largest_u32_visit(
        [&](auto fn) {
            for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) fn(key(i));
        },
        k, S);
}

// S.segoff[g] = entries stored in segments before g (exclusive prefix sum of S.segn[0..segs)).
// segs <= kMaxCandSegs = blockDim.x.
__device__ inline void scan_segments(SelectSmem& S, uint32_t segs) {
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t v = t < segs ? S.segn[t] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= static_cast<uint32_t>(o)) x += y;
    }
    if (lane == 31) S.wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < (blockDim.x >> 5) ? S.wsum[lane] : 0u;
        uint32_t z = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= static_cast<uint32_t>(o)) z += y;
        }
        S.wsum[lane] = z - w;  // exclusive over warps
    }
    __syncthreads();
    if (t < segs) S.segoff[t] = S.wsum[warp] + x - v;
    __syncthreads();
}

// Loads the per-segment counts of one query's segmented candidate list (kMaxCandSegs layout) into
// S.segn (clamped to seg_cap) and their prefix sums into S.segoff. Returns the stored total (also in
// S.total); *overflow = some segment lost entries. segs <= blockDim.x.
__device__ uint32_t load_segments(SelectSmem& S, const uint32_t* counts, uint32_t segs, uint32_t seg_cap,
                                  bool* overflow) {
    if (threadIdx.x == 0) {
        S.bcast[2] = 0;
        S.bcast[3] = 0;
    }
    __syncthreads();
    for (uint32_t g = threadIdx.x; g < segs; g += blockDim.x) {
        const uint32_t c = counts[g];
        const uint32_t st = min(c, seg_cap);
        S.segn[g] = st;
        if (st) atomicAdd(&S.bcast[2], st);
        if (c > seg_cap) atomicOr(&S.bcast[3], 1u);
    }
    __syncthreads();
    const uint32_t n = S.bcast[2];
    *overflow = S.bcast[3] != 0;
    if (threadIdx.x == 0) S.total = n;
    scan_segments(S, segs);  // synchronises
    return n;
}

// Storage index of the idx-th stored entry (idx < S.total) of a segmented list: the last segment
// starting at or before idx, by binary search over S.segoff (empty segments share their successor's
// start, so the last such segment is the non-empty one holding idx).
__device__ __forceinline__ uint64_t segment_entry(const SelectSmem& S, uint32_t segs, uint32_t seg_cap, uint32_t idx) {
    uint32_t lo = 0, hi = segs;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (S.segoff[mid] <= idx) lo = mid;
        else hi = mid;
    }
    return static_cast<uint64_t>(lo) * seg_cap + (idx - S.segoff[lo]);
}

// Calls fn(index, valid, score) for every stored entry of a segmented list of scores src (after
// load_segments). Short segments (a candidate list's: a few entries each): a warp takes 4 x 32
// consecutive entries of the flattened list per round: lanes read consecutive entries (coalesced
// within a segment), and each lane's 4 segment lookups and loads are independent, so a thread keeps 4
// loads in flight instead of one dependent chain per entry. Long segments: walked segment by segment.
// Every call is made by a full warp (valid = false past the end), so fn may use warp collectives.
template <class Fn>
__device__ inline void for_each_segment_entry(const SelectSmem& S, uint32_t segs, uint32_t seg_cap,
                                              const float* src, Fn fn) {
    constexpr uint32_t U = 4;
    const uint32_t n = S.total, lane = threadIdx.x & 31;
    if (n >= 32u * segs) {
        // long segments (a doc sample's lists): warp w walks segments w, w + 32, ..., 4 x 32 entries
        // a round, with no per-entry segment lookup
        for (uint32_t g = threadIdx.x >> 5; g < segs; g += blockDim.x >> 5) {
            const uint32_t cnt = S.segn[g];
            const uint64_t base = static_cast<uint64_t>(g) * seg_cap;
            for (uint32_t o = 0; o < cnt; o += 32u * U) {
                bool ok[U];
                float v[U];
#pragma unroll
                for (uint32_t u = 0; u < U; ++u) {
                    const uint32_t e = o + 32u * u + lane;
                    ok[u] = e < cnt;
                    v[u] = ok[u] ? src[base + e] : 0.0f;
                }
#pragma unroll
                for (uint32_t u = 0; u < U; ++u) fn(static_cast<uint32_t>(base + o + 32u * u + lane), ok[u], v[u]);
            }
        }
        return;
    }
    for (uint32_t b = (threadIdx.x >> 5) * 32u * U; b < n; b += blockDim.x * U) {
        uint64_t i[U];
        bool ok[U];
        float v[U];
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) {
            const uint32_t idx = b + 32u * u + lane;
            ok[u] = idx < n;
            i[u] = ok[u] ? segment_entry(S, segs, seg_cap, idx) : 0ull;
        }
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) v[u] = ok[u] ? src[i[u]] : 0.0f;
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) fn(static_cast<uint32_t>(i[u]), ok[u], v[u]);
    }
}

template <class KeyFn>
__device__ uint64_t kth_largest_u64(KeyFn key, uint32_t n, uint32_t k, SelectSmem& S) {
    uint64_t prefix = 0, mask = 0;
    uint32_t krem = k;
    const uint32_t warp = threadIdx.x >> 5;
    for (int shift = 56; shift >= 0; shift -= 8) {
        clear_hist(S);
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t v = key(i);
            hist_add(S.hist[warp % kHist], (v & mask) == prefix ? static_cast<uint32_t>((v >> shift) & 255u) : 256u);
        }
        __syncthreads();
        const uint64_t d = pick_digit(S, &krem);
        prefix |= d << shift;
        mask |= 255ull << shift;
    }
    return prefix;
}

// Sorts S.sortbuf[0..m) descending; m is a power of two <= kMaxTopK.
__device__ void bitonic_desc(SelectSmem& S, uint32_t m) {
    for (uint32_t k = 2; k <= m; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long a = S.sortbuf[i], b = S.sortbuf[ixj];
                    const bool desc = (i & k) == 0;
                    if (desc ? (a < b) : (a > b)) {
                        S.sortbuf[i] = b;
                        S.sortbuf[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
}

__device__ inline uint32_t pow2_at_least(uint32_t x) {
    uint32_t m = 1;
    while (m < x) m <<= 1;
    return m;
}

// Top `kq` (<= kMaxTopK) of n distinct u64 keys key(i), sorted descending into S.sortbuf[0..kq).
template <class KeyFn>
__device__ void top_keys(KeyFn key, uint32_t n, uint32_t kq, SelectSmem& S) {
    if (n <= static_cast<uint32_t>(kMaxTopK) && n > 2 * kq) {
        // keep only keys whose score half is at least a lower bound of the kq-th best score (it keeps
        // the top kq and at most the few keys sharing the kq-th's 24-bit prefix beyond them), then
        // sort those: a bitonic sort over about kq keys instead of n
        const uint32_t lb = kth_lower_bound_u32_visit(
            [&](auto fn) {
                for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) fn(static_cast<uint32_t>(key(i) >> 32));
            },
            kq, S);
        if (threadIdx.x == 0) S.counter = 0;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t v = key(i);
            if (static_cast<uint32_t>(v >> 32) >= lb) S.sortbuf[atomicAdd(&S.counter, 1u)] = v;
        }
        __syncthreads();
        const uint32_t got = S.counter;  // >= kq, <= n
        const uint32_t m = pow2_at_least(got);
        for (uint32_t i = got + threadIdx.x; i < m; i += blockDim.x) S.sortbuf[i] = 0ull;
        __syncthreads();
        bitonic_desc(S, m);
        return;
    }
    if (n <= static_cast<uint32_t>(kMaxTopK)) {
        const uint32_t m = pow2_at_least(n);
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) S.sortbuf[i] = i < n ? key(i) : 0ull;
        __syncthreads();
        bitonic_desc(S, m);
        return;
    }
    const uint64_t kth = kth_largest_u64(key, n, kq, S);
    if (threadIdx.x == 0) S.counter = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint64_t v = key(i);
        if (v >= kth) {
            const uint32_t pos = atomicAdd(&S.counter, 1u);
            if (pos < static_cast<uint32_t>(kMaxTopK)) S.sortbuf[pos] = v;
        }
    }
    __syncthreads();
    const uint32_t got = min(S.counter, static_cast<uint32_t>(kMaxTopK));
    const uint32_t m = pow2_at_least(got);
    for (uint32_t i = got + threadIdx.x; i < m; i += blockDim.x) S.sortbuf[i] = 0ull;
    __syncthreads();
    bitonic_desc(S, m);
}

// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kST) sample_threshold_kernel(SampleThresholdLaunch L) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SelectSmem& S = *reinterpret_cast<SelectSmem*>(smem_raw);
    const uint32_t qi = L.qlist ? L.qlist[blockIdx.x] : blockIdx.x;
    const uint32_t k = L.topk[qi];
    bool lost = false;  // a sample segment that overflowed only lowers the sample's K-th best
    const uint32_t n = load_segments(S, L.count + static_cast<uint64_t>(qi) * kMaxCandSegs, L.segs, L.seg_cap, &lost);
    float theta = L.raise_only ? L.theta[qi] : -INFINITY;
    if (L.stats) {
        // the sample's best scores at ranks 1, 2, 4, ..., 64: a lower bound of the key at rank
        // r = min(64, n) (its 24-bit prefix, two walks of the list), then the (fewer than r) keys above
        // that prefix's bucket, each placed by counting the keys that precede it; a rank inside the
        // bucket gets the bound (at most 2^-15 relative below the score)
        float* st = L.stats + static_cast<uint64_t>(qi) * kSampleStats;
        const float* sc = L.score + static_cast<uint64_t>(qi) * L.cap;
        const uint32_t r = min(n, 64u);
        uint32_t key_r = 0;
        if (r > 0)
            key_r = kth_lower_bound_u32_visit(
                [&](auto fn) {
                    for_each_segment_entry(S, L.segs, L.seg_cap, sc, [&](uint32_t, bool ok, float v) {
                        if (ok) fn(float_key(v));
                    });
                },
                r, S);
        const uint32_t bucket_top = key_r | 0xFFu;
        if (threadIdx.x == 0) S.counter = 0;
        __syncthreads();
        if (r > 0)
            for_each_segment_entry(S, L.segs, L.seg_cap, sc, [&](uint32_t, bool ok, float v) {
                const uint32_t key = ok ? float_key(v) : 0u;
                if (ok && key > bucket_top) {
                    const uint32_t slot = atomicAdd(&S.counter, 1u);
                    if (slot < 64u) S.sortbuf[slot] = key;
                }
            });
        __syncthreads();
        const uint32_t c = min(S.counter, 64u);  // < r unless keys were lost
        if (threadIdx.x < c) {
            const unsigned long long key = S.sortbuf[threadIdx.x];
            uint32_t rank = 0;
            for (uint32_t j = 0; j < c; ++j) {
                const unsigned long long o = S.sortbuf[j];
                rank += (o > key || (o == key && j < threadIdx.x)) ? 1u : 0u;
            }
            S.sortbuf[64 + rank] = key;
        }
        __syncthreads();
        if (threadIdx.x < kSampleRanks) {
            const uint32_t rho = 1u << threadIdx.x;
            float v = -2.0f;
            if (rho <= r) v = key_float(rho <= c ? static_cast<uint32_t>(S.sortbuf[64 + rho - 1]) : key_r);
            st[threadIdx.x] = v;
        } else if (threadIdx.x == kSampleRanks) {
            st[kSampleRanks] = -2.0f;  // the K-th best, set below when the sample holds K docs
            st[kSampleRanks + 1] = static_cast<float>(n);
            for (uint32_t j = kSampleRanks + 2; j < kSampleStats; ++j) st[j] = 0.0f;
        }
        __syncthreads();
    }
    if (k > 0 && n >= k) {
        const float* sc = L.score + static_cast<uint64_t>(qi) * L.cap;
        // a lower bound of the K-th best serves the proof below as well as the K-th best itself
        const uint32_t kk = kth_lower_bound_u32_visit(
            [&](auto fn) {
                for_each_segment_entry(S, L.segs, L.seg_cap, sc, [&](uint32_t, bool ok, float v) {
                    if (ok) fn(float_key(v));
                });
            },
            k, S);
        // k sample docs score >= t approximately, so the true K-th best exact score is >= t - eps_s;
        // a true top-K doc therefore scores >= t - eps_s - eps_m under the main pass's arithmetic.
        const float t = __fsub_rd(__fsub_rd(key_float(kk), L.eps_sample[qi]), L.eps_main[qi]);
        theta = L.raise_only ? fmaxf(theta, t) : t;
        if (L.stats && threadIdx.x == 0) L.stats[static_cast<uint64_t>(qi) * kSampleStats + kSampleRanks] = key_float(kk);
        if (L.theta_also && L.raise_only && threadIdx.x == 0) L.theta_also[qi] = fmaxf(L.theta_also[qi], t);
    }
    __syncthreads();  // every thread has read the old theta
    if (threadIdx.x == 0) {
        L.theta[qi] = theta;
        if (L.theta_also && !L.raise_only) L.theta_also[qi] = theta;
    }
}

// Byte offset of the shared-memory candidate arrays of select_topk_kernel: after SelectSmem and the
// query (dim floats), 16-byte aligned.
__host__ __device__ inline size_t select_cand_offset(uint32_t dim) {
    return (sizeof(SelectSmem) + static_cast<size_t>(dim) * sizeof(float) + 15) & ~static_cast<size_t>(15);
}

// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kST) select_topk_kernel(SelectLaunch L) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SelectSmem& S = *reinterpret_cast<SelectSmem*>(smem_raw);
    float* sq = reinterpret_cast<float*>(smem_raw + sizeof(SelectSmem));
    const uint32_t qi = L.qlist ? L.qlist[blockIdx.x] : blockIdx.x;
    const uint32_t tid = threadIdx.x;
    const uint32_t k = L.topk[qi];
    const uint64_t row = static_cast<uint64_t>(qi) * L.cap;
    if (k > static_cast<uint32_t>(kMaxTopK)) {
        if (tid == 0) {
            L.out_count[qi] = 0;
            atomicOr(L.status + qi, kStatusTopKTooLarge);
        }
        return;
    }
    bool overflow = false;
    const uint32_t n =
        load_segments(S, L.cand_count + static_cast<uint64_t>(qi) * kMaxCandSegs, L.segs, L.seg_cap, &overflow);
    const float* sc = L.cand_score + row;
    const uint32_t* lc = L.cand_loc + row;
    const float eps = L.eps_main[qi];
    auto visit_scores = [&](auto fn) {
        for_each_segment_entry(S, L.segs, L.seg_cap, sc, [&](uint32_t, bool ok, float v) {
            if (ok) fn(float_key(v));
        });
    };
    // A threshold above the proven one (a prediction) has to be checked: the list holds every doc
    // with s~ >= theta, so a doc left out scores s < theta + eps, and the K best candidates are the
    // K best docs when their K-th exact score s_K >= theta + eps. A query that fails goes back to a
    // proven threshold: the larger of its proven one and s_K - eps (every true top-K doc scores at
    // least s_K, the candidates' K-th best, hence s~ >= s_K - eps).
    const float theta_q = L.theta[qi];
    const bool unproven = L.theta_proven != nullptr && theta_q > L.theta_proven[qi];
    auto threshold_miss = [&](float raised) {
        if (tid == 0) {
            const float t = fmaxf(L.theta_proven[qi], raised);
            L.theta[qi] = t;
            L.theta_proven[qi] = t;
            L.out_count[qi] = 0;
            atomicOr(L.status + qi, kStatusOverflow | kStatusThresholdMiss);
        }
    };
    if (overflow) {
        // The stored candidates are a subset of the qualifying docs, so their K-th best still bounds
        // the true K-th best from below: raise the threshold and let the host re-run this query.
        float theta = unproven ? L.theta_proven[qi] : theta_q;
        if (n >= k && k > 0) {
            const uint32_t kk = kth_lower_bound_u32_visit(visit_scores, k, S);
            theta = fmaxf(theta, __fsub_rd(key_float(kk), 2.0f * eps));
        }
        if (tid == 0) {
            L.theta[qi] = theta;
            if (L.theta_proven) L.theta_proven[qi] = theta;
            L.out_count[qi] = 0;
            atomicOr(L.status + qi, kStatusOverflow);
        }
        return;
    }
    if (n == 0 || k == 0) {
        if (unproven && k > 0) {
            threshold_miss(-INFINITY);
            return;
        }
        if (tid == 0) L.out_count[qi] = 0;
        return;
    }
    const uint32_t kq = min(k, n);
    for (uint32_t i = tid; i < L.dim; i += blockDim.x) sq[i] = L.qry[static_cast<uint64_t>(qi) * L.dim + i];
    // A list that fits is gathered into shared memory once (scores only: the few rescored entries
    // look their location up again); the selection and rescoring passes then read shared memory
    // instead of walking the segments again.
    const bool fast = n <= (L.fast_large ? kSelFastLarge : kSelFast);
    float* cs = reinterpret_cast<float*>(smem_raw + select_cand_offset(L.dim));
    if (fast) {
        for (uint32_t idx = tid; idx < n; idx += blockDim.x) cs[idx] = sc[segment_entry(S, L.segs, L.seg_cap, idx)];
        __syncthreads();
    }
    float thr = -INFINITY;
    if (n > kq) {
        // a lower bound of the K-th best approximate score only widens the rescoring cut
        const uint32_t kk = fast ? kth_lower_bound_u32_visit(
                                       [&](auto fn) {
                                           for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) fn(float_key(cs[i]));
                                       },
                                       kq, S)
                                 : kth_lower_bound_u32_visit(visit_scores, kq, S);
        thr = __fsub_rd(key_float(kk), 2.0f * eps);
    }
    if (tid == 0) S.counter = 0;
    __syncthreads();
    unsigned long long* ws = L.work + row;
    // rescoring of one entry (score s, location loc; warp-collective): kept entries are appended to ws
    auto rescore = [&](bool ok, float s, uint32_t loc) {
        bool take = false;
        unsigned long long key = 0;
        if (ok && s >= thr) {
            const float e = exact_dot(sq, L.vec + static_cast<uint64_t>(loc) * L.dim, L.dim);
            key = result_key(e, loc);
            take = true;
        }
        const uint32_t mask = __ballot_sync(0xffffffffu, take);
        if (mask) {
            const uint32_t lane = tid & 31;
            const uint32_t leader = __ffs(mask) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(&S.counter, __popc(mask));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (take) ws[base + __popc(mask & ((1u << lane) - 1u))] = key;
        }
    };
    if (fast) {
        for (uint32_t b = tid & ~31u; b < n; b += blockDim.x) {  // warp-uniform bounds
            const uint32_t idx = b + (tid & 31);
            const bool ok = idx < n;
            const float v = ok ? cs[idx] : 0.0f;
            rescore(ok, v, ok && v >= thr ? lc[segment_entry(S, L.segs, L.seg_cap, idx)] : 0u);
        }
    } else {
        for_each_segment_entry(S, L.segs, L.seg_cap, sc, [&](uint32_t i, bool ok, float v) {
            rescore(ok, v, ok && v >= thr ? lc[i] : 0u);
        });
    }
    __syncthreads();
    const uint32_t nf = S.counter;
    __syncthreads();
    top_keys([&](uint32_t i) { return static_cast<uint64_t>(ws[i]); }, nf, kq, S);
    if (unproven) {
        const float lo = kq == k ? __fsub_rd(result_key_score(S.sortbuf[kq - 1]), eps) : -INFINITY;
        if (!(lo >= theta_q)) {
            threshold_miss(lo);
            return;
        }
    }
    const uint64_t orow = static_cast<uint64_t>(qi) * L.out_stride;
    for (uint32_t i = tid; i < kq; i += blockDim.x) {
        const uint64_t key = S.sortbuf[i];
        const uint32_t loc = result_key_loc(key);
        L.out_score[orow + i] = result_key_score(key);
        L.out_id[orow + i] = L.gdocid ? L.gdocid[loc] : static_cast<int64_t>(loc);
    }
    if (tid == 0) L.out_count[qi] = kq;
}

// ---------------------------------------------------------------------------------------------
// Aggregator: stable compaction in three launches (count per block, scan, scatter).
constexpr int kAggT = 1024;  // docs per aggregation block (one per thread)

__global__ void __launch_bounds__(kAggT) aggregate_count_kernel(const uint64_t* __restrict__ bits, uint32_t n,
                                                                 uint32_t* __restrict__ block_count) {
    __shared__ uint32_t part[kAggT / 32];
    const uint32_t doc = blockIdx.x * kAggT + threadIdx.x;
    const bool hit = doc < n && ((bits[doc >> 6] >> (doc & 63)) & 1ull);
    const uint32_t c = __popc(__ballot_sync(0xffffffffu, hit));
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t v = part[threadIdx.x];
        v = warp_sum(v);
        if (threadIdx.x == 0) block_count[blockIdx.x] = v;
    }
}

// Exclusive scan of nb block counts in place (one CTA); writes the total to *total.
__global__ void __launch_bounds__(1024) aggregate_scan_kernel(uint32_t* __restrict__ block_count, uint32_t nb,
                                                              uint32_t* __restrict__ total) {
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t b0 = 0; b0 < nb; b0 += blockDim.x) {
        const uint32_t i = b0 + threadIdx.x;
        const uint32_t v = i < nb ? block_count[i] : 0;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= static_cast<uint32_t>(o)) x += y;
        }
        if (lane == 31) warp_tot[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t t = warp_tot[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= static_cast<uint32_t>(o)) t += y;
            }
            warp_tot[lane] = t;  // inclusive over warps
        }
        __syncthreads();
        const uint32_t warp_excl = warp ? warp_tot[warp - 1] : 0;
        const uint32_t excl = carry + warp_excl + x - v;
        if (i < nb) block_count[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kAggT) aggregate_scatter_kernel(const uint64_t* __restrict__ bits,
                                                                  const float* __restrict__ scores,
                                                                  const uint32_t* __restrict__ loc_in, uint32_t n,
                                                                  const uint32_t* __restrict__ block_off,
                                                                  float* __restrict__ out_scores,
                                                                  uint32_t* __restrict__ out_loc) {
    __shared__ uint32_t woff[kAggT / 32];
    const uint32_t doc = blockIdx.x * kAggT + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool hit = doc < n && ((bits[doc >> 6] >> (doc & 63)) & 1ull);
    const uint32_t m = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) woff[warp] = __popc(m);
    __syncthreads();
    if (warp == 0) {
        uint32_t v = woff[lane], x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= static_cast<uint32_t>(o)) x += y;
        }
        woff[lane] = x - v;
    }
    __syncthreads();
    if (hit) {
        const uint32_t pos = block_off[blockIdx.x] + woff[warp] + __popc(m & ((1u << lane) - 1u));
        out_scores[pos] = scores[doc];
        out_loc[pos] = loc_in ? loc_in[doc] : doc;
    }
}

// ---------------------------------------------------------------------------------------------
// TOPK operator: exact top K of one compacted list, one CTA.
__global__ void __launch_bounds__(kST) topk_op_kernel(const float* __restrict__ scores,
                                                      const uint32_t* __restrict__ locs,
                                                      const uint32_t* __restrict__ count, uint32_t k,
                                                      float* __restrict__ out_scores, uint32_t* __restrict__ out_locs,
                                                      uint32_t* __restrict__ out_count) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SelectSmem& S = *reinterpret_cast<SelectSmem*>(smem_raw);
    const uint32_t n = *count;
    const uint32_t kq = min(k, n);
    if (kq == 0) {
        if (threadIdx.x == 0) *out_count = 0;
        return;
    }
    top_keys([&](uint32_t i) { return result_key(scores[i], locs[i]); }, n, kq, S);
    for (uint32_t i = threadIdx.x; i < kq; i += blockDim.x) {
        const uint64_t key = S.sortbuf[i];
        out_scores[i] = result_key_score(key);
        out_locs[i] = result_key_loc(key);
    }
    if (threadIdx.x == 0) *out_count = kq;
}

// Per-query error bounds: eps = c * ||q||_2 * max_doc ||v||_2 (Cauchy-Schwarz on sum |q_i v_i|),
// computed in double and rounded up to float.
// Bounds of queries qlist[0..nq) (or 0..nq-1 when qlist is null), written at the query's own index.
__global__ void query_eps_kernel(const float* __restrict__ qry, const uint32_t* __restrict__ qlist, uint32_t nq,
                                 uint32_t dim, float max_norm, double c_main, double c_sample,
                                 float* __restrict__ eps_main, float* __restrict__ eps_sample) {
    const uint32_t r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31;
    if (r >= nq) return;
    const uint32_t q = qlist ? qlist[r] : r;
    double s = 0.0;
    for (uint32_t d = lane; d < dim; d += 32) {
        const double x = qry[static_cast<uint64_t>(q) * dim + d];
        s += x * x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        const double base = sqrt(s) * (1.0 + 1e-12) * static_cast<double>(max_norm);
        eps_main[q] = __double2float_ru(c_main * base + 1e-30);
        eps_sample[q] = __double2float_ru(c_sample * base + 1e-30);
    }
}

// Opts a kernel into more than 48 KB of dynamic shared memory, always to the same ceiling: searchers
// on other threads launch the same kernel concurrently with their own sizes, and a per-call value
// could drop below another caller's launch.
template <class K>
cudaError_t set_smem(K kernel, size_t bytes) {
    constexpr size_t kCeiling = 200 * 1024;
    if (bytes <= 48 * 1024) return cudaSuccess;
    if (bytes > kCeiling) return cudaErrorInvalidValue;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kCeiling));
}

}  // namespace

namespace {
bool bad_segments(uint32_t segs, uint32_t seg_cap, uint32_t cap) {
    return segs == 0 || segs > kMaxCandSegs || seg_cap == 0 || static_cast<uint64_t>(segs) * seg_cap > cap;
}
}  // namespace

cudaError_t launch_sample_threshold(const SampleThresholdLaunch& L, cudaStream_t stream) {
    if (L.nq_list == 0) return cudaSuccess;
    if (bad_segments(L.segs, L.seg_cap, L.cap)) return cudaErrorInvalidValue;
    const size_t smem = sizeof(SelectSmem);
    cudaError_t e = set_smem(sample_threshold_kernel, smem);
    if (e != cudaSuccess) return e;
    sample_threshold_kernel<<<L.nq_list, kST, smem, stream>>>(L);
    return cudaGetLastError();
}

cudaError_t launch_select_topk(const SelectLaunch& L, cudaStream_t stream) {
    if (L.nq_list == 0) return cudaSuccess;
    if (bad_segments(L.segs, L.seg_cap, L.cap) || L.segs > static_cast<uint32_t>(kST)) return cudaErrorInvalidValue;
    const size_t smem = select_cand_offset(L.dim) + (L.fast_large ? kSelFastLarge : kSelFast) * sizeof(float);
    cudaError_t e = set_smem(select_topk_kernel, smem);
    if (e != cudaSuccess) return e;
    select_topk_kernel<<<L.nq_list, kST, smem, stream>>>(L);
    return cudaGetLastError();
}

cudaError_t launch_query_eps(const float* qry, const uint32_t* qlist, uint32_t nq, uint32_t dim, float max_norm,
                             double c_main, double c_sample, float* eps_main, float* eps_sample, cudaStream_t stream) {
    if (nq == 0) return cudaSuccess;
    query_eps_kernel<<<(nq + 7) / 8, 256, 0, stream>>>(qry, qlist, nq, dim, max_norm, c_main, c_sample, eps_main,
                                                       eps_sample);
    return cudaGetLastError();
}

size_t aggregate_workspace_bytes(uint32_t n) {
    const size_t nb = (static_cast<size_t>(n) + kAggT - 1) / kAggT;
    return (nb > 0 ? nb : 1) * sizeof(uint32_t);
}

cudaError_t launch_aggregate(const uint64_t* bits, const float* scores, const uint32_t* loc_in, uint32_t n,
                             float* out_scores, uint32_t* out_loc, uint32_t* total, uint32_t* workspace,
                             cudaStream_t stream) {
    const uint32_t nb = (n + kAggT - 1) / kAggT;
    if (nb == 0) return cudaMemsetAsync(total, 0, sizeof(uint32_t), stream);
    aggregate_count_kernel<<<nb, kAggT, 0, stream>>>(bits, n, workspace);
    aggregate_scan_kernel<<<1, 1024, 0, stream>>>(workspace, nb, total);
    aggregate_scatter_kernel<<<nb, kAggT, 0, stream>>>(bits, scores, loc_in, n, workspace, out_scores, out_loc);
    return cudaGetLastError();
}

// Scratch of the allocation-free aggregator: one block count per kAggT docs, kAggStaticBlocks of
// them (64 KB, docNumber <= 16,777,216). Module-scope, so it exists once per device for the life of
// the process and every call on that device shares it. The count kernel writes every entry a call
// reads before the scan reads it, so a call never sees an earlier call's contents and nothing has to
// be cleared; two calls that overlap on the GPU (different streams, no ordering) do race on it.
static __device__ __align__(256) uint32_t g_aggregate_scratch[kAggStaticBlocks];
static_assert(kAggStaticMaxDocs == kAggStaticBlocks * static_cast<uint32_t>(kAggT), "one block count per kAggT docs");

cudaError_t aggregate_static_scratch(uint32_t** scratch) {
    return cudaGetSymbolAddress(reinterpret_cast<void**>(scratch), g_aggregate_scratch);
}

cudaError_t launch_topk_op(const float* scores, const uint32_t* locs, const uint32_t* count, uint32_t k,
                           float* out_scores, uint32_t* out_locs, uint32_t* out_count, cudaStream_t stream) {
    if (k > static_cast<uint32_t>(kMaxTopK)) return cudaErrorInvalidValue;
    const size_t smem = sizeof(SelectSmem);
    cudaError_t e = set_smem(topk_op_kernel, smem);
    if (e != cudaSuccess) return e;
    topk_op_kernel<<<1, kST, smem, stream>>>(scores, locs, count, k, out_scores, out_locs, out_count);
    return cudaGetLastError();
}


// ---------------------------------------------------------------------------------------------
// Cross-shard merge (the reference's k-way merge of per-shard results, run_context.cpp:86-118 and
// 237-270): the shards' sorted lists are merged by score descending, equal scores taking the lower
// shard first (within a shard, list order). Every entry finds its output position directly: its
// index in its own list plus, for every other shard, how many of that shard's entries precede it
// (a binary search on the score), so one thread places one entry and no thread waits on another.
namespace {
// Entries of a list sorted by score descending that come before score x: those with score > x, or
// with score >= x when `ties_first` (a lower shard).
__device__ inline uint32_t preceding(const float* sc, uint32_t n, float x, bool ties_first) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const float v = sc[mid];
        if (ties_first ? (v >= x) : (v > x))
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(256) merge_shards_kernel(const __grid_constant__ ShardMergeLaunch L) {
    const uint32_t q = blockIdx.x;
    __shared__ uint32_t s_n[kMaxShards], s_off[kMaxShards + 1];
    if (threadIdx.x == 0) {
        uint32_t total = 0;
        for (uint32_t s = 0; s < L.shards; ++s) {
            uint32_t c = L.counts[s][q];
            c = min(c, min(L.in_stride, L.topk));
            s_n[s] = c;
            s_off[s] = total;
            total += c;
        }
        s_off[L.shards] = total;
        L.out_count[q] = min(total, L.topk);
    }
    __syncthreads();
    const uint32_t total = s_off[L.shards];
    for (uint32_t e = threadIdx.x; e < total; e += blockDim.x) {
        uint32_t s = 0;
        while (e >= s_off[s + 1]) ++s;
        const uint32_t i = e - s_off[s];
        const uint64_t row = static_cast<uint64_t>(q) * L.in_stride;
        const float x = L.scores[s][row + i];
        uint32_t pos = i;
        for (uint32_t t = 0; t < L.shards && pos < L.topk; ++t)
            if (t != s) pos += preceding(L.scores[t] + row, s_n[t], x, t < s);
        if (pos < L.topk) {
            const uint64_t o = static_cast<uint64_t>(q) * L.out_stride + pos;
            L.out_score[o] = x;
            L.out_id[o] = L.ids[s][row + i];
        }
    }
}
}  // namespace

cudaError_t launch_merge_shards(const ShardMergeLaunch& L, cudaStream_t stream) {
    if (L.nq == 0) return cudaSuccess;
    if (L.shards == 0 || L.shards > kMaxShards || L.topk > static_cast<uint32_t>(kMaxTopK) || L.topk > L.out_stride ||
        !L.out_score || !L.out_id || !L.out_count)
        return cudaErrorInvalidValue;
    for (uint32_t s = 0; s < L.shards; ++s)
        if (!L.scores[s] || !L.ids[s] || !L.counts[s]) return cudaErrorInvalidValue;
    merge_shards_kernel<<<L.nq, 256, 0, stream>>>(L);
    return cudaGetLastError();
}

}  // namespace hss
