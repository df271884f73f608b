// filter.cu -- the posting filter: decodes all five posting layouts and evaluates each query's
// postfix filter program into a per-query doc bitmap, for a whole batch of queries in one launch.
//
// Replaces the reference's per-query BitmapTextFilter launches plus the PostingBitListToSet
// conversion pass (kernel_bitmap_text_filter.cpp:18-119, filter_{and,or,not,conjunction}_op.h,
// bitlist_to_set.h): sparse postings are decoded straight into shared memory instead of being
// expanded into 16 KB scratch bitsets in global memory, and the stack lives in registers.
//
// Output layout: one row per query, one bit per doc, bit b of u64 word w = doc 64w+b. Read as bytes
// this is exactly the reference's filter result (segNum x docNumPerSegment/8 bytes of u16 units,
// bit i of unit u = doc 16u+i, posting_serializer.cpp:46-55).
#include "hss_device.cuh"
#include "hss_kernels.h"

namespace hss {
namespace {

constexpr int kTile = kFilterTileWords;  // == blockDim.x
// the operand slots' shared memory at most: one 256-word tile of kMaxOperands operands
constexpr size_t kFilterSmemCeiling = static_cast<size_t>(kFilterTileWords) * kMaxOperands * sizeof(uint64_t);

// Operand descriptor for one (operand, segment) pair, resolved once per CTA.
struct OperandInfo {
    const uint8_t* addr;
    uint32_t layout;  // kEmpty for an all-zero or absent posting
    uint32_t plen;    // payload bytes (clamped to what the layout can legally hold)
    uint32_t k;       // sparse entries
    int32_t lo, hi;   // sparse entries whose unit falls in this tile
};
constexpr uint32_t kEmpty = 0xffu;

__device__ inline uint32_t ld32(const uint8_t* p) { return __ldg(reinterpret_cast<const uint32_t*>(p)); }
__device__ inline uint16_t ld16(const uint8_t* p) { return __ldg(reinterpret_cast<const unsigned short*>(p)); }

// 8 bytes at a 4-byte aligned address.
__device__ inline uint64_t ld64(const uint8_t* p) {
    if ((reinterpret_cast<uintptr_t>(p) & 7u) == 0) return __ldg(reinterpret_cast<const unsigned long long*>(p));
    return static_cast<uint64_t>(ld32(p)) | (static_cast<uint64_t>(ld32(p + 4)) << 32);
}

// Dense word j (64 docs) of a DENSE_BITMAP payload, bytes past plen masked off.
__device__ inline uint64_t dense_word(const OperandInfo& o, uint32_t j) {
    const uint32_t b0 = j * 8u;
    if (b0 >= o.plen) return 0;
    uint64_t v = ld64(o.addr + 8 + b0);
    const uint32_t valid = o.plen - b0;
    if (valid < 8) v &= (1ull << (valid * 8)) - 1;
    return v;
}

// Dense word j of a DENSE_BYTEMAP payload: 64 bytes, non-zero byte = hit.
__device__ inline uint64_t bytemap_word(const OperandInfo& o, uint32_t j) {
    const uint32_t b0 = j * 64u;
    if (b0 >= o.plen) return 0;
    const uint32_t valid = min(64u, o.plen - b0);
    uint64_t v = 0;
    const uint8_t* p = o.addr + 8 + b0;
#pragma unroll 4
    for (uint32_t i = 0; i < 16; ++i) {
        if (i * 4 >= valid) break;
        uint32_t x = ld32(p + 4 * i);
        const uint32_t nz = __vcmpne4(x, 0u) & 0x01010101u;
        const uint64_t nib = (nz * 0x01020408u) >> 24;
        v |= nib << (4 * i);
    }
    if (valid < 64) v &= (1ull << valid) - 1;
    return v;
}

// Largest payload a legal posting of `layout` can have for a segment of seg_docs docs; a longer
// length word can only come from a corrupt posting and is clamped so no read leaves the posting.
__device__ inline uint32_t max_payload(uint32_t layout, uint32_t seg_docs) {
    const uint32_t units = (seg_docs + 15) / 16;
    switch (layout) {
        case kDenseBitmap: return units * 2;
        case kSparseBitmap: return units * 6;
        case kDenseBytemap: return seg_docs;
        case kSparseIdList: return seg_docs * 4;
        case kSparsePacked: return units * 4;
    }
    return 0;
}

// First sparse entry whose unit index is >= u (entries are sorted by unit, posting_serializer.cpp).
__device__ inline int32_t sparse_lower_bound(const OperandInfo& o, uint32_t u) {
    int32_t lo = 0, hi = static_cast<int32_t>(o.k);
    while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        const uint32_t unit = o.layout == kSparseBitmap ? ld32(o.addr + 8 + 4u * mid) / 2u
                                                          : ld32(o.addr + 8 + 4u * mid) >> 16;
        if (unit < u)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__device__ inline void resolve_operand(OperandInfo& o, const uint8_t* addr, uint32_t seg_docs, uint32_t unit_lo,
                                       uint32_t unit_hi, int* bad) {
    o.addr = addr;
    o.layout = kEmpty;
    o.plen = 0;
    o.k = 0;
    o.lo = o.hi = 0;
    if (addr == nullptr) return;
    const uint32_t head = ld32(addr);
    const uint32_t hits = head & 0x0fffffffu;
    const uint32_t layout = head >> 28;
    if (layout > kSparsePacked) {
        *bad = 1;
        return;
    }
    if (hits == 0) return;  // all-zero posting: identity of OR, annihilator of AND
    o.layout = layout;
    o.plen = min(ld32(addr + 4), max_payload(layout, seg_docs));
    if (layout == kSparseBitmap) o.k = o.plen / 6;
    if (layout == kSparsePacked) o.k = o.plen / 4;
    if (layout == kSparseIdList) o.k = o.plen / 4;
    if (layout == kSparseBitmap || layout == kSparsePacked) {
        // a tile spanning the whole segment needs every entry: no search (each step of it is a
        // dependent global load)
        const uint32_t units = (seg_docs + 15) / 16;
        o.lo = unit_lo == 0 ? 0 : sparse_lower_bound(o, unit_lo);
        o.hi = unit_hi >= units ? static_cast<int32_t>(o.k) : sparse_lower_bound(o, unit_hi);
    }
}

__device__ inline uint64_t tail_mask(uint64_t gw, uint64_t doc_num) {
    const uint64_t d0 = gw * 64;
    if (d0 >= doc_num) return 0;
    const uint64_t valid = doc_num - d0;
    return valid >= 64 ? ~0ull : ((1ull << valid) - 1);
}

// Postfix evaluation of W words at once (words w0 + k * step, k < W), the reference's interpretation
// of the program (kernel_bitmap_text_filter.cpp:52-119): [AND|OR|NOT, postingNum, stackNum] combines
// the next postingNum operands with stackNum popped results, [CONJUNCTION, parts, n_1..n_parts] ANDs
// the ORs of consecutive operand groups. Every op is decoded and checked once and applied to all W
// words, so the per-op decode cost is shared. Returns false for a malformed program.
template <int W>
__device__ inline bool eval_words(const uint32_t* prog, uint32_t plen, const uint64_t* slots, uint32_t slot_stride,
                                  uint32_t w0, uint32_t step, uint32_t nop, uint64_t (&result)[W]) {
    uint64_t st[kMaxStack][W];
    uint32_t sp = 0, next = 0, pc = 0;
    while (pc < plen) {
        const uint32_t op = prog[pc];
        uint64_t acc[W];
        if (op == kOpAnd || op == kOpOr || op == kOpNot) {
            if (pc + 2 >= plen) return false;
            const uint32_t pn = prog[pc + 1], sn = prog[pc + 2];
            pc += 3;
            // comparisons written so that no u32 sum can wrap (the program may come straight from a
            // caller's device buffer): next <= nop always holds
            const bool ok = op == kOpNot ? ((pn == 1 && sn == 0) || (pn == 0 && sn == 1)) : (pn != 0 || sn != 0);
            if (!ok || pn > nop - next || sn > sp) return false;
            const uint64_t* row = slots + static_cast<uint64_t>(next) * slot_stride + w0;
            if (op == kOpNot) {
                if (pn) {
#pragma unroll
                    for (int k = 0; k < W; ++k) acc[k] = ~row[k * step];
                } else {
                    --sp;
#pragma unroll
                    for (int k = 0; k < W; ++k) acc[k] = ~st[sp][k];
                }
            } else if (op == kOpAnd) {
#pragma unroll
                for (int k = 0; k < W; ++k) acc[k] = ~0ull;
                for (uint32_t j = 0; j < pn; ++j, row += slot_stride)
#pragma unroll
                    for (int k = 0; k < W; ++k) acc[k] &= row[k * step];
                for (uint32_t j = 0; j < sn; ++j) {
                    --sp;
#pragma unroll
                    for (int k = 0; k < W; ++k) acc[k] &= st[sp][k];
                }
            } else {
#pragma unroll
                for (int k = 0; k < W; ++k) acc[k] = 0ull;
                for (uint32_t j = 0; j < pn; ++j, row += slot_stride)
#pragma unroll
                    for (int k = 0; k < W; ++k) acc[k] |= row[k * step];
                for (uint32_t j = 0; j < sn; ++j) {
                    --sp;
#pragma unroll
                    for (int k = 0; k < W; ++k) acc[k] |= st[sp][k];
                }
            }
            next += pn;
        } else if (op == kOpConjunction) {
            if (pc + 1 >= plen) return false;
            const uint32_t parts = prog[pc + 1];
            if (parts == 0 || parts > plen - pc - 2) return false;
#pragma unroll
            for (int k = 0; k < W; ++k) acc[k] = ~0ull;
            for (uint32_t p = 0; p < parts; ++p) {
                const uint32_t pn = prog[pc + 2 + p];
                if (pn == 0 || pn > nop - next) return false;
                uint64_t o[W];
#pragma unroll
                for (int k = 0; k < W; ++k) o[k] = 0ull;
                const uint64_t* row = slots + static_cast<uint64_t>(next) * slot_stride + w0;
                for (uint32_t j = 0; j < pn; ++j, row += slot_stride)
#pragma unroll
                    for (int k = 0; k < W; ++k) o[k] |= row[k * step];
#pragma unroll
                for (int k = 0; k < W; ++k) acc[k] &= o[k];
                next += pn;
            }
            pc += 2 + parts;
        } else {
            return false;
        }
        if (sp >= static_cast<uint32_t>(kMaxStack)) return false;
#pragma unroll
        for (int k = 0; k < W; ++k) st[sp][k] = acc[k];
        ++sp;
    }
    if (sp != 1 || next != nop) return false;
#pragma unroll
    for (int k = 0; k < W; ++k) result[k] = st[0][k];
    return true;
}

// One CTA per (query, segment tile of WPT * 256 words). Operands are decoded into shared-memory
// slots of the tile (dense: each thread its own words; sparse: zeroed, then scattered), then every
// word is run through the program. Grid: x = query (fastest, so all queries of a tile share the
// tile's postings in L2), y = segment tile.
template <int WPT>
__global__ void __launch_bounds__(kTile) filter_batch_kernel(FilterLaunch L) {
    constexpr uint32_t TW = kTile * WPT;  // words per CTA
    extern __shared__ uint64_t slots[];   // [nop][TW]
    __shared__ OperandInfo s_op[kMaxOperands];
    __shared__ uint32_t s_prog[kMaxProgram];
    __shared__ int s_bad;

    const uint32_t q = blockIdx.x;
    const uint32_t t = threadIdx.x;
    const uint32_t seg_words = L.docs_per_seg / 64;
    const uint32_t tiles = (seg_words + TW - 1) / TW;
    const uint32_t seg = blockIdx.y / tiles;
    const uint32_t w0 = (blockIdx.y % tiles) * TW;
    const uint32_t nw = min(TW, seg_words - w0);
    const uint64_t seg_doc0 = static_cast<uint64_t>(seg) * L.docs_per_seg;
    const uint32_t seg_docs = static_cast<uint32_t>(min(static_cast<uint64_t>(L.docs_per_seg), L.doc_num - seg_doc0));
    const uint64_t gw0 = static_cast<uint64_t>(seg) * seg_words + w0;
    uint64_t* out_row = L.out + static_cast<uint64_t>(q) * L.out_stride;

    const uint32_t p0 = L.prog_off ? L.prog_off[q] : 0u;
    const uint32_t p1 = L.prog_off ? L.prog_off[q + 1] : L.single_prog_len;
    const uint32_t o0 = L.opnd_off ? L.opnd_off[q] : 0u;
    const uint32_t o1 = L.opnd_off ? L.opnd_off[q + 1] : L.single_nop;
    const uint32_t nop = o1 - o0;
    const uint32_t plen = p1 - p0;

    if (plen == 0) {  // empty program: match all (the reference memsets 0xff, text_filter.cpp:553-559)
        uint32_t c = 0;
#pragma unroll
        for (int k = 0; k < WPT; ++k) {
            const uint32_t w = k * kTile + t;
            if (w < nw) {
                const uint64_t v = tail_mask(gw0 + w, L.doc_num);
                out_row[gw0 + w] = v;
                c += __popcll(v);
            }
        }
        if (L.pass_count) {
            c = warp_sum(c);
            if ((t & 31) == 0 && c) atomicAdd(L.pass_count + q, c);
        }
        return;
    }
    if (nop > L.max_opnd || nop > static_cast<uint32_t>(kMaxOperands) || plen > static_cast<uint32_t>(kMaxProgram)) {
        for (uint32_t w = t; w < nw; w += kTile) out_row[gw0 + w] = 0;
        if (t == 0 && L.status) atomicOr(L.status + q, kStatusBadProgram);
        return;
    }

    if (t == 0) s_bad = 0;
    for (uint32_t i = t; i < plen; i += kTile) s_prog[i] = L.prog[p0 + i];
    __syncthreads();
    if (t < nop) {
        const uint64_t row = L.opnd_row ? L.opnd_row[o0 + t] : t;
        const uint64_t a = L.table[row * L.row_stride + static_cast<uint64_t>(seg) * L.seg_stride];
        if (!L.ref_table) {
            resolve_operand(s_op[t], reinterpret_cast<const uint8_t*>(a), seg_docs, w0 * 4u, (w0 + nw) * 4u, &s_bad);
        } else if (a == 2u || a == 0u) {  // EMPTY_OPERAND_TAG
            resolve_operand(s_op[t], nullptr, seg_docs, 0u, 0u, &s_bad);
        } else if (a & 1u) {  // SPARSE_OPERAND_TAG: the sparse posting's head
            resolve_operand(s_op[t], reinterpret_cast<const uint8_t*>(a & ~1ull), seg_docs, w0 * 4u, (w0 + nw) * 4u,
                            &s_bad);
        } else {  // a dense bitset: the payload of a DENSE_BITMAP posting, no head
            OperandInfo& o = s_op[t];
            o.addr = reinterpret_cast<const uint8_t*>(a) - 8;
            o.layout = kDenseBitmap;
            o.plen = L.docs_per_seg / 8;
            o.k = 0;
            o.lo = o.hi = 0;
        }
    }
    __syncthreads();

    // Dense operands: each thread its own words (coalesced). Sparse ones: zero, then scatter below.
    for (uint32_t i = 0; i < nop; ++i) {
        const OperandInfo& o = s_op[i];
#pragma unroll
        for (int k = 0; k < WPT; ++k) {
            const uint32_t w = k * kTile + t;
            uint64_t v = 0;
            if (w < nw) {
                if (o.layout == kDenseBitmap) v = dense_word(o, w0 + w);
                else if (o.layout == kDenseBytemap) v = bytemap_word(o, w0 + w);
            }
            slots[i * TW + w] = v;
        }
    }
    __syncthreads();
    for (uint32_t i = 0; i < nop; ++i) {
        const OperandInfo& o = s_op[i];
        if (o.layout == kSparseBitmap || o.layout == kSparsePacked) {
            uint16_t* units = reinterpret_cast<uint16_t*>(slots + i * TW);
            for (int32_t e = o.lo + static_cast<int32_t>(t); e < o.hi; e += kTile) {
                uint32_t unit, mask;
                if (o.layout == kSparseBitmap) {
                    unit = ld32(o.addr + 8 + 4u * e) / 2u;
                    mask = ld16(o.addr + 8 + 4u * o.k + 2u * e);
                } else {
                    const uint32_t w = ld32(o.addr + 8 + 4u * e);
                    unit = w >> 16;
                    mask = w & 0xffffu;
                }
                const uint32_t rel = unit - w0 * 4u;
                if (rel < nw * 4u) units[rel] = static_cast<uint16_t>(mask);
            }
        } else if (o.layout == kSparseIdList) {
            uint32_t* bits = reinterpret_cast<uint32_t*>(slots + i * TW);
            for (uint32_t e = t; e < o.k; e += kTile) {
                const uint32_t id = ld32(o.addr + 8 + 4u * e);
                const uint32_t rel = id - w0 * 64u;
                if (id < seg_docs && rel < nw * 64u) atomicOr(bits + rel / 32, 1u << (rel % 32));
            }
        }
    }
    __syncthreads();

    const bool bad_posting = s_bad != 0;
    uint64_t res[WPT];
    const bool bad = bad_posting || !eval_words<WPT>(s_prog, plen, slots, TW, t, kTile, nop, res);
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < WPT; ++k) {
        const uint32_t w = k * kTile + t;
        if (w >= nw) continue;
        const uint64_t r = bad ? 0ull : res[k] & tail_mask(gw0 + w, L.doc_num);
        out_row[gw0 + w] = r;
        c += __popcll(r);
    }
    if (L.pass_count) {
        c = warp_sum(c);
        if ((t & 31) == 0 && c) atomicAdd(L.pass_count + q, c);
    }
    if (L.status && bad && t < nw) atomicOr(L.status + q, bad_posting ? kStatusBadPosting : kStatusBadProgram);
}

// ---------------------------------------------------------------------------------------------
// Batch filter over the dense posting matrix (every posting pre-expanded, DataTable::
// EnableDensePostings): operand words need no decoding and no dependent loads, so a CTA copies its
// operands' words for a tile straight into shared memory (cp.async, 16 bytes per thread per
// operand), then runs every word through the program. Small tiles keep many CTAs resident per SM.
__device__ inline void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
                 "l"(gmem)
                 : "memory");
}
__device__ inline void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

constexpr int kDenseT = 256;  // threads of a dense-filter CTA

template <int WPT>
__global__ void __launch_bounds__(kDenseT) filter_dense_kernel(DenseFilterLaunch L) {
    constexpr uint32_t TW = kDenseT * WPT;  // words per CTA
    extern __shared__ __align__(16) uint64_t dslots[];  // [nop][TW]
    __shared__ uint32_t s_prog[kMaxProgram];
    __shared__ uint32_t s_row[kMaxOperands];

    const uint32_t q = blockIdx.x;
    const uint32_t t = threadIdx.x;
    const uint32_t seg_words = L.seg_words;
    const uint32_t tiles = (seg_words + TW - 1) / TW;
    const uint32_t seg = blockIdx.y / tiles;
    const uint32_t w0 = (blockIdx.y % tiles) * TW;
    const uint32_t nw = min(TW, seg_words - w0);
    const uint64_t gw0 = static_cast<uint64_t>(seg) * seg_words + w0;
    uint64_t* out_row = L.out + static_cast<uint64_t>(q) * L.out_stride;

    const uint32_t p0 = L.prog_off[q], p1 = L.prog_off[q + 1];
    const uint32_t o0 = L.opnd_off[q], o1 = L.opnd_off[q + 1];
    const uint32_t nop = o1 - o0;
    const uint32_t plen = p1 - p0;
    if (plen == 0) {  // empty program: match all (text_filter.cpp:553-559)
        uint32_t c = 0;
#pragma unroll
        for (int k = 0; k < WPT; ++k) {
            const uint32_t w = k * kDenseT + t;
            if (w < nw) {
                const uint64_t v = tail_mask(gw0 + w, L.doc_num);
                out_row[gw0 + w] = v;
                c += __popcll(v);
            }
        }
        if (L.pass_count) {
            c = warp_sum(c);
            if ((t & 31) == 0 && c) atomicAdd(L.pass_count + q, c);
        }
        return;
    }
    if (nop > L.max_opnd || nop > static_cast<uint32_t>(kMaxOperands) || plen > static_cast<uint32_t>(kMaxProgram)) {
        for (uint32_t w = t; w < nw; w += kDenseT) out_row[gw0 + w] = 0;
        if (t == 0 && L.status) atomicOr(L.status + q, kStatusBadProgram);
        return;
    }
    for (uint32_t i = t; i < plen; i += kDenseT) s_prog[i] = L.prog[p0 + i];
    if (t < nop) {
        const uint32_t r = L.opnd_row[o0 + t];
        s_row[t] = r < L.rows ? r : L.rows - 1;  // a row past the table reads the all-zero row
    }
    __syncthreads();
    // nw is even (segments hold a multiple of 128 docs): 16-byte pieces, one per thread per operand
    for (uint32_t i = 0; i < nop; ++i) {
        const uint64_t* src = L.dense + (static_cast<uint64_t>(s_row[i]) * L.seg_num + seg) * seg_words + w0;
        for (uint32_t c = t; c < nw / 2; c += kDenseT) cp_async16(dslots + i * TW + 2 * c, src + 2 * c);
    }
    cp_async_wait_all();
    __syncthreads();
    uint64_t res[WPT];
    const bool bad = !eval_words<WPT>(s_prog, plen, dslots, TW, t, kDenseT, nop, res);
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < WPT; ++k) {
        const uint32_t w = k * kDenseT + t;
        if (w >= nw) continue;
        const uint64_t r = bad ? 0ull : res[k] & tail_mask(gw0 + w, L.doc_num);
        out_row[gw0 + w] = r;
        c += __popcll(r);
    }
    if (L.pass_count) {
        c = warp_sum(c);
        if ((t & 31) == 0 && c) atomicAdd(L.pass_count + q, c);
    }
    if (L.status && bad) atomicOr(L.status + q, kStatusBadProgram);
}

template <int WPT>
cudaError_t launch_filter_dense_wpt(const DenseFilterLaunch& L, cudaStream_t stream) {
    constexpr uint32_t TW = kDenseT * WPT;
    const uint32_t tiles = (L.seg_words + TW - 1) / TW;
    const uint64_t gy = static_cast<uint64_t>(L.seg_num) * tiles;
    if (gy > 65535u) return cudaErrorInvalidValue;
    const size_t smem = static_cast<size_t>(L.max_opnd > 0 ? L.max_opnd : 1) * TW * sizeof(uint64_t);
    // opt in always (static plus dynamic shared memory may pass 48 KB even when the dynamic part does
    // not), to the one ceiling every caller sets: searchers on other threads launch it concurrently
    if (smem > kFilterSmemCeiling) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(filter_dense_kernel<WPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kFilterSmemCeiling));
    if (e != cudaSuccess) return e;
    filter_dense_kernel<WPT><<<dim3(L.nq, static_cast<uint32_t>(gy)), kDenseT, smem, stream>>>(L);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// The dense filter for programs of at most kWideMaxOpnd operands. A CTA takes tiles_per_cta (1, 2 or
// 4) consecutive word tiles of one query's bitmap, across segment boundaries; 128 threads each own 4
// of a tile's 512 words (2 adjacent words in each of 2 groups of 256), so the per-op decode is
// shared by 4 words, and 10 CTAs per SM keep many operand loads in flight.
// Operands are read straight from the dense posting matrix as 16-byte read-only loads:
// the batch's queries share rows, so most reads hit L2, and without staging buffers sized for the
// batch's largest program the SM holds as many CTAs as registers allow. One thread checks the program
// (check_program: eval_words' acceptance rules), so the evaluation carries no checks. The top of the
// evaluation stack stays in registers; only entries under it (a sibling subtree still waiting for its
// parent) go to a local array.
constexpr int kWideT = 128;
constexpr int kWideW = 4;
constexpr uint32_t kWideTW = kWideT * kWideW;  // words per tile
constexpr uint32_t kWideGS = 2 * kWideT;       // words between a thread's word pairs
constexpr uint32_t kWideMaxTilesPerCta = 4;    // word tiles per CTA at most (consecutive, across segments)
constexpr uint32_t kWideCtasPerSm = 10;        // resident CTAs per SM (__launch_bounds__ below; 48 registers)
constexpr uint32_t kWideMaxOpnd = 8;          // operand rows held in shared memory

// True exactly when eval_words would accept the program (same rules, no evaluation).
__device__ inline bool check_program(const uint32_t* prog, uint32_t plen, uint32_t nop) {
    uint32_t sp = 0, next = 0, pc = 0;
    while (pc < plen) {
        const uint32_t op = prog[pc];
        if (op == kOpAnd || op == kOpOr || op == kOpNot) {
            if (pc + 2 >= plen) return false;
            const uint32_t pn = prog[pc + 1], sn = prog[pc + 2];
            pc += 3;
            const bool ok = op == kOpNot ? ((pn == 1 && sn == 0) || (pn == 0 && sn == 1)) : (pn != 0 || sn != 0);
            if (!ok || pn > nop - next || sn > sp) return false;
            sp -= sn;
            next += pn;
        } else if (op == kOpConjunction) {
            if (pc + 1 >= plen) return false;
            const uint32_t parts = prog[pc + 1];
            if (parts == 0 || parts > plen - pc - 2) return false;
            for (uint32_t p = 0; p < parts; ++p) {
                const uint32_t pn = prog[pc + 2 + p];
                if (pn == 0 || pn > nop - next) return false;
                next += pn;
            }
            pc += 2 + parts;
        } else {
            return false;
        }
        if (sp >= static_cast<uint32_t>(kMaxStack)) return false;
        ++sp;
    }
    return sp == 1 && next == nop;
}

// This thread's kWideW words of operand i: words off[g] + {0, 1} of the operand's row in the segment.
__device__ __forceinline__ void wide_load(const uint64_t* const* base, uint32_t i, const uint32_t (&off)[kWideW / 2],
                                          uint64_t (&o)[kWideW]) {
    const uint64_t* p = base[i];
#pragma unroll
    for (int g = 0; g < kWideW / 2; ++g) {
        const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(p + off[g]));
        o[2 * g] = v.x;
        o[2 * g + 1] = v.y;
    }
}

// Evaluates a checked program (check_program) over this thread's kWideW words of the operand rows
// at base[i] + off[g] into res.
__device__ __forceinline__ void eval_wide(const uint32_t* s_prog, uint32_t plen, const uint64_t* const* s_base,
                                          const uint32_t (&off)[kWideW / 2], uint64_t (&res)[kWideW]) {
    uint64_t top[kWideW];
    uint64_t deep[kMaxStack][kWideW];  // entries under the top
    uint32_t depth = 0, next = 0, pc = 0;
    bool has_top = false;
    auto pop_into = [&](uint64_t (&acc)[kWideW], bool is_and) {
        if (has_top) {
            has_top = false;
#pragma unroll
            for (int k = 0; k < kWideW; ++k) acc[k] = is_and ? (acc[k] & top[k]) : (acc[k] | top[k]);
        } else {
            --depth;
#pragma unroll
            for (int k = 0; k < kWideW; ++k)
                acc[k] = is_and ? (acc[k] & deep[depth][k]) : (acc[k] | deep[depth][k]);
        }
    };
    while (pc < plen) {
        const uint32_t op = s_prog[pc];
        uint64_t acc[kWideW], o[kWideW];
        if (op == kOpConjunction) {
            const uint32_t parts = s_prog[pc + 1];
#pragma unroll
            for (int k = 0; k < kWideW; ++k) acc[k] = ~0ull;
            for (uint32_t p = 0; p < parts; ++p) {
                const uint32_t pn = s_prog[pc + 2 + p];
                uint64_t u[kWideW];
                wide_load(s_base, next, off, u);
                // two operands' loads in flight at a time (the pass waits on L2 latency)
#pragma unroll 2
                for (uint32_t j = 1; j < pn; ++j) {
                    wide_load(s_base, next + j, off, o);
#pragma unroll
                    for (int k = 0; k < kWideW; ++k) u[k] |= o[k];
                }
#pragma unroll
                for (int k = 0; k < kWideW; ++k) acc[k] &= u[k];
                next += pn;
            }
            pc += 2 + parts;
        } else {
            const uint32_t pn = s_prog[pc + 1], sn = s_prog[pc + 2];
            pc += 3;
            if (op == kOpNot) {
                if (pn) {
                    wide_load(s_base, next, off, acc);
                } else {
#pragma unroll
                    for (int k = 0; k < kWideW; ++k) acc[k] = 0ull;
                    pop_into(acc, false);
                }
#pragma unroll
                for (int k = 0; k < kWideW; ++k) acc[k] = ~acc[k];
            } else {
                const bool is_and = op == kOpAnd;
#pragma unroll
                for (int k = 0; k < kWideW; ++k) acc[k] = is_and ? ~0ull : 0ull;
#pragma unroll 2  // two operands' loads in flight, as above
                for (uint32_t j = 0; j < pn; ++j) {
                    wide_load(s_base, next + j, off, o);
#pragma unroll
                    for (int k = 0; k < kWideW; ++k) acc[k] = is_and ? (acc[k] & o[k]) : (acc[k] | o[k]);
                }
                for (uint32_t j = 0; j < sn; ++j) pop_into(acc, is_and);
            }
            next += pn;
        }
        // push: the old top (if any) moves under the new one
        if (has_top) {
#pragma unroll
            for (int k = 0; k < kWideW; ++k) deep[depth][k] = top[k];
            ++depth;
        }
#pragma unroll
        for (int k = 0; k < kWideW; ++k) top[k] = acc[k];
        has_top = true;
    }
#pragma unroll
    for (int k = 0; k < kWideW; ++k) res[k] = top[k];
}

__global__ void __launch_bounds__(kWideT, kWideCtasPerSm) filter_dense_wide_kernel(DenseFilterLaunch L,
                                                                                    uint32_t tiles_per_cta) {
    __shared__ uint32_t s_prog[kMaxProgram];
    __shared__ const uint64_t* s_base[kWideMaxOpnd];
    __shared__ int s_ok;

    const uint32_t q = blockIdx.x;
    const uint32_t t = threadIdx.x;
    const uint32_t seg_words = L.seg_words;
    const uint32_t tiles = (seg_words + kWideTW - 1) / kWideTW;  // word tiles of a segment
    const uint32_t total = L.seg_num * tiles;                    // word tiles of a query's bitmap
    const uint32_t tile0 = blockIdx.y * tiles_per_cta;
    const uint32_t tile1 = min(total, tile0 + tiles_per_cta);
    uint64_t* out_row = L.out + static_cast<uint64_t>(q) * L.out_stride;

    const uint32_t p0 = L.prog_off[q], p1 = L.prog_off[q + 1];
    const uint32_t o0 = L.opnd_off[q], o1 = L.opnd_off[q + 1];
    const uint32_t nop = o1 - o0;
    const uint32_t plen = p1 - p0;
    const bool empty = plen == 0;  // match all (text_filter.cpp:553-559)
    const bool fits = nop <= L.max_opnd && nop <= kWideMaxOpnd && plen <= static_cast<uint32_t>(kMaxProgram);
    if (!empty && fits) {
        for (uint32_t i = t; i < plen; i += kWideT) s_prog[i] = L.prog[p0 + i];
        if (t < nop) {
            uint32_t r = L.opnd_row[o0 + t];
            r = r < L.rows ? r : L.rows - 1;  // a row past the table reads the all-zero row
            s_base[t] = L.dense + static_cast<uint64_t>(r) * L.seg_num * seg_words;  // the row's first segment
        }
        __syncthreads();
        if (t == 0) s_ok = check_program(s_prog, plen, nop);
    } else if (t == 0) {
        s_ok = empty;
    }
    __syncthreads();
    const bool ok = s_ok != 0;
    uint32_t c = 0;
    // the program's setup (load, check) is shared by the CTA's word tiles, which may span segments
    for (uint32_t gt = tile0; gt < tile1; ++gt) {
        const uint32_t seg = gt / tiles;
        const uint32_t w0 = (gt % tiles) * kWideTW;
        const uint32_t nw = min(kWideTW, seg_words - w0);  // even
        const uint32_t seg_w0 = seg * seg_words;           // < 2^32: a row's words
        // word offsets (from the row's start) of this thread's pairs; a pair past a partial tile reads
        // the tile's first pair instead (in bounds; not stored)
        uint32_t off[kWideW / 2];
#pragma unroll
        for (int g = 0; g < kWideW / 2; ++g)
            off[g] = seg_w0 + w0 + (kWideGS * g + 2u * t < nw ? kWideGS * g + 2u * t : 0u);
        uint64_t res[kWideW];
        if (empty || !ok) {
#pragma unroll
            for (int k = 0; k < kWideW; ++k) res[k] = empty ? ~0ull : 0ull;
        } else {
            eval_wide(s_prog, plen, s_base, off, res);
        }
        // only a tile reaching past the last doc needs the per-word tail mask (uniform per CTA)
        const bool tail = (static_cast<uint64_t>(seg_w0) + w0 + nw) * 64 > L.doc_num;
#pragma unroll
        for (int g = 0; g < kWideW / 2; ++g) {
            const uint32_t w = kWideGS * g + 2u * t;
            if (w >= nw) continue;
            const uint64_t gw = static_cast<uint64_t>(seg_w0) + w0 + w;
            uint64_t a = res[2 * g], b = res[2 * g + 1];
            if (tail) {
                a &= tail_mask(gw, L.doc_num);
                b &= tail_mask(gw + 1, L.doc_num);
            }
            *reinterpret_cast<ulonglong2*>(out_row + gw) = make_ulonglong2(a, b);
            c += __popcll(a) + __popcll(b);
        }
    }
    if (L.pass_count) {
        c = warp_sum(c);
        if ((t & 31) == 0 && c) atomicAdd(L.pass_count + q, c);
    }
    if (t == 0 && L.status && !empty && !ok) atomicOr(L.status + q, kStatusBadProgram);
}

// One CTA per posting: expand `src[i]` (any layout) into the dense bitset `dst[i]` of
// byte_size bytes (the PostingBitListToSet operator, bitlist_to_set.h:6-155).
__global__ void __launch_bounds__(256) posting_expand_kernel(const uint64_t* src, const uint64_t* dst, uint32_t count,
                                                             uint32_t byte_size, uint32_t seg_docs, int32_t* status) {
    const uint32_t i = blockIdx.x;
    if (i >= count) return;
    const uint8_t* addr = reinterpret_cast<const uint8_t*>(src[i]);
    uint8_t* out = reinterpret_cast<uint8_t*>(dst[i]);
    __shared__ OperandInfo o;
    __shared__ int bad;
    if (threadIdx.x == 0) {
        bad = 0;
        resolve_operand(o, addr, seg_docs, 0u, 0xffffffffu, &bad);
        if (o.layout == kSparseBitmap || o.layout == kSparsePacked) {
            o.lo = 0;
            o.hi = static_cast<int32_t>(o.k);
        }
    }
    __syncthreads();
    if (bad && threadIdx.x == 0 && status) atomicOr(status, kStatusBadPosting);
    // byte_size is a multiple of 8 (checked on the host), dst 8-byte aligned.
    uint64_t* words = reinterpret_cast<uint64_t*>(out);
    const uint32_t nwords = byte_size / 8;
    for (uint32_t w = threadIdx.x; w < nwords; w += blockDim.x) {
        uint64_t v = 0;
        if (o.layout == kDenseBitmap) v = dense_word(o, w);
        else if (o.layout == kDenseBytemap) v = bytemap_word(o, w);
        words[w] = v;
    }
    __syncthreads();
    if (o.layout == kSparseBitmap || o.layout == kSparsePacked) {
        uint16_t* units = reinterpret_cast<uint16_t*>(out);
        for (int32_t e = threadIdx.x; e < o.hi; e += blockDim.x) {
            uint32_t unit, mask;
            if (o.layout == kSparseBitmap) {
                unit = ld32(o.addr + 8 + 4u * e) / 2u;
                mask = ld16(o.addr + 8 + 4u * o.k + 2u * e);
            } else {
                const uint32_t w = ld32(o.addr + 8 + 4u * e);
                unit = w >> 16;
                mask = w & 0xffffu;
            }
            if (unit < byte_size / 2) units[unit] = static_cast<uint16_t>(mask);
        }
    } else if (o.layout == kSparseIdList) {
        uint32_t* bits = reinterpret_cast<uint32_t*>(out);
        for (uint32_t e = threadIdx.x; e < o.k; e += blockDim.x) {
            const uint32_t id = ld32(o.addr + 8 + 4u * e);
            if (id < seg_docs && id < byte_size * 8u) atomicOr(bits + id / 32, 1u << (id % 32));
        }
    }
}


template <int WPT>
cudaError_t launch_filter_wpt(const FilterLaunch& L, cudaStream_t stream) {
    constexpr uint32_t TW = kTile * WPT;
    const uint32_t seg_words = L.docs_per_seg / 64;
    const uint32_t tiles = (seg_words + TW - 1) / TW;
    const uint64_t gy = static_cast<uint64_t>(L.seg_num) * tiles;
    if (gy > 65535u) return cudaErrorInvalidValue;
    const size_t smem = static_cast<size_t>(L.max_opnd > 0 ? L.max_opnd : 1) * TW * sizeof(uint64_t);
    // opt in always (static plus dynamic shared memory may pass 48 KB even when the dynamic part does
    // not), to the one ceiling every caller sets: searchers on other threads launch it concurrently
    if (smem > kFilterSmemCeiling) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(filter_batch_kernel<WPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kFilterSmemCeiling));
    if (e != cudaSuccess) return e;
    dim3 grid(L.nq, static_cast<uint32_t>(gy));
    filter_batch_kernel<WPT><<<grid, kTile, smem, stream>>>(L);
    return cudaGetLastError();
}

}  // namespace

// The tile is as wide as the segment allows (up to 2048 words = 131072 docs) while the operand slots
// stay within 96 KB of shared memory.
cudaError_t launch_filter_batch(const FilterLaunch& L, cudaStream_t stream) {
    if (L.nq == 0 || L.seg_num == 0) return cudaSuccess;
    if (L.max_opnd > static_cast<uint32_t>(kMaxOperands)) return cudaErrorInvalidValue;
    const uint32_t seg_words = L.docs_per_seg / 64;
    const size_t per_word = static_cast<size_t>(L.max_opnd > 0 ? L.max_opnd : 1) * sizeof(uint64_t);
    int wpt = 8;
    while (wpt > 1 && (static_cast<size_t>(wpt) * kTile * per_word > 96 * 1024 || static_cast<uint32_t>(wpt / 2) * kTile >= seg_words))
        wpt /= 2;
    switch (wpt) {
        case 8: return launch_filter_wpt<8>(L, stream);
        case 4: return launch_filter_wpt<4>(L, stream);
        case 2: return launch_filter_wpt<2>(L, stream);
        default: return launch_filter_wpt<1>(L, stream);
    }
}

// Four words per thread (8 KB of each operand per CTA) while the operand slots fit 48 KB, then two,
// then one (an evaluation's decode cost is shared by a thread's words).
cudaError_t launch_filter_dense(const DenseFilterLaunch& L, cudaStream_t stream) {
    if (L.nq == 0 || L.seg_num == 0) return cudaSuccess;
    if (L.max_opnd > static_cast<uint32_t>(kMaxOperands) || L.rows == 0 || L.seg_words == 0 || (L.seg_words & 1u) ||
        (reinterpret_cast<uintptr_t>(L.dense) & 15u))
        return cudaErrorInvalidValue;
    if (L.max_opnd <= kWideMaxOpnd && (L.out_stride & 1u) == 0 && (reinterpret_cast<uintptr_t>(L.out) & 15u) == 0) {
        const uint32_t tiles = (L.seg_words + kWideTW - 1) / kWideTW;
        const uint64_t total = static_cast<uint64_t>(L.seg_num) * tiles;
        // More tiles per CTA share its program setup over more words, fewer leave more CTAs: take the
        // most (4, 2, 1) that still leaves 4 waves of resident CTAs (small batches and tables take 1),
        // but no fewer than the grid's height limit needs.
        const uint64_t want = 4ull * kWideCtasPerSm * (L.sm_count ? L.sm_count : 148u);
        uint32_t tpc = kWideMaxTilesPerCta;
        while (tpc > 1 && static_cast<uint64_t>(L.nq) * ((total + tpc - 1) / tpc) < want &&
               (total + tpc / 2 - 1) / (tpc / 2) <= 65535u)
            tpc >>= 1;
        const uint64_t gy = (total + tpc - 1) / tpc;
        if (gy <= 65535u && static_cast<uint64_t>(L.seg_num) * L.seg_words < (1ull << 32)) {
            filter_dense_wide_kernel<<<dim3(L.nq, static_cast<uint32_t>(gy)), kWideT, 0, stream>>>(L, tpc);
            return cudaGetLastError();
        }
    }
    const size_t per_word = static_cast<size_t>(L.max_opnd > 0 ? L.max_opnd : 1) * sizeof(uint64_t);
    if (4 * kDenseT * per_word <= 48 * 1024 && L.seg_words >= 2 * kDenseT) return launch_filter_dense_wpt<4>(L, stream);
    if (2 * kDenseT * per_word <= 48 * 1024) return launch_filter_dense_wpt<2>(L, stream);
    return launch_filter_dense_wpt<1>(L, stream);
}

cudaError_t launch_posting_expand(const uint64_t* src, const uint64_t* dst, uint32_t count, uint32_t byte_size,
                                  uint32_t seg_docs, int32_t* status, cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    posting_expand_kernel<<<count, 256, 0, stream>>>(src, dst, count, byte_size, seg_docs, status);
    return cudaGetLastError();
}

}  // namespace hss
