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
        o.lo = sparse_lower_bound(o, unit_lo);
        o.hi = sparse_lower_bound(o, unit_hi);
    }
}

__device__ inline uint64_t tail_mask(uint64_t gw, uint64_t doc_num) {
    const uint64_t d0 = gw * 64;
    if (d0 >= doc_num) return 0;
    const uint64_t valid = doc_num - d0;
    return valid >= 64 ? ~0ull : ((1ull << valid) - 1);
}

__global__ void __launch_bounds__(kTile) filter_batch_kernel(FilterLaunch L) {
    extern __shared__ uint64_t slots[];  // [nop][kTile]
    __shared__ OperandInfo s_op[kMaxOperands];
    __shared__ uint32_t s_prog[kMaxProgram];
    __shared__ int s_bad;

    const uint32_t q = blockIdx.x;
    const uint32_t t = threadIdx.x;
    const uint32_t seg_words = L.docs_per_seg / 64;
    const uint32_t tiles = (seg_words + kTile - 1) / kTile;
    const uint32_t seg = blockIdx.y / tiles;
    const uint32_t w0 = (blockIdx.y % tiles) * kTile;
    const uint32_t nw = min(static_cast<uint32_t>(kTile), seg_words - w0);
    const uint64_t seg_doc0 = static_cast<uint64_t>(seg) * L.docs_per_seg;
    const uint32_t seg_docs = static_cast<uint32_t>(min(static_cast<uint64_t>(L.docs_per_seg), L.doc_num - seg_doc0));
    const uint64_t gw = static_cast<uint64_t>(seg) * seg_words + w0 + t;
    uint64_t* out_row = L.out + static_cast<uint64_t>(q) * L.out_stride;

    const uint32_t p0 = L.prog_off ? L.prog_off[q] : 0u;
    const uint32_t p1 = L.prog_off ? L.prog_off[q + 1] : L.single_prog_len;
    const uint32_t o0 = L.opnd_off ? L.opnd_off[q] : 0u;
    const uint32_t o1 = L.opnd_off ? L.opnd_off[q + 1] : L.single_nop;
    const uint32_t nop = o1 - o0;
    const uint32_t plen = p1 - p0;

    if (plen == 0) {  // empty program: match all (the reference memsets 0xff, text_filter.cpp:553-559)
        const uint64_t v = t < nw ? tail_mask(gw, L.doc_num) : 0ull;
        if (t < nw) out_row[gw] = v;
        if (L.pass_count) {
            const uint32_t c = warp_sum(__popcll(v));
            if ((t & 31) == 0 && c) atomicAdd(L.pass_count + q, c);
        }
        return;
    }
    if (nop > L.max_opnd || nop > static_cast<uint32_t>(kMaxOperands) || plen > static_cast<uint32_t>(kMaxProgram)) {
        if (t < nw) out_row[gw] = 0;
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

    // Dense operands: each thread its own word. Sparse ones: zero, then scatter below.
    for (uint32_t i = 0; i < nop; ++i) {
        const OperandInfo& o = s_op[i];
        uint64_t v = 0;
        if (t < nw) {
            if (o.layout == kDenseBitmap) v = dense_word(o, w0 + t);
            else if (o.layout == kDenseBytemap) v = bytemap_word(o, w0 + t);
        }
        slots[i * kTile + t] = v;
    }
    __syncthreads();
    for (uint32_t i = 0; i < nop; ++i) {
        const OperandInfo& o = s_op[i];
        if (o.layout == kSparseBitmap || o.layout == kSparsePacked) {
            uint16_t* units = reinterpret_cast<uint16_t*>(slots + i * kTile);
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
            uint32_t* bits = reinterpret_cast<uint32_t*>(slots + i * kTile);
            for (uint32_t e = t; e < o.k; e += kTile) {
                const uint32_t id = ld32(o.addr + 8 + 4u * e);
                const uint32_t rel = id - w0 * 64u;
                if (id < seg_docs && rel < nw * 64u) atomicOr(bits + rel / 32, 1u << (rel % 32));
            }
        }
    }
    __syncthreads();

    bool bad = s_bad != 0;
    uint64_t result = 0;
    if (t < nw && !bad) {
        uint64_t st[kMaxStack];
        int sp = 0;
        uint32_t next = 0;
        uint32_t pc = 0;
        while (pc < plen && !bad) {
            const uint32_t op = s_prog[pc];
            if (op == kOpAnd || op == kOpOr || op == kOpNot) {
                if (pc + 2 >= plen) { bad = true; break; }
                const uint32_t pn = s_prog[pc + 1], sn = s_prog[pc + 2];
                pc += 3;
                const bool ok = op == kOpNot ? (pn + sn == 1) : (pn + sn > 0);
                if (!ok || next + pn > nop || sn > static_cast<uint32_t>(sp)) { bad = true; break; }
                uint64_t acc = op == kOpAnd ? ~0ull : 0ull;
                if (op == kOpNot) {
                    acc = pn ? ~slots[next * kTile + t] : ~st[--sp];
                } else {
                    for (uint32_t k = 0; k < pn; ++k) {
                        const uint64_t v = slots[(next + k) * kTile + t];
                        acc = op == kOpAnd ? (acc & v) : (acc | v);
                    }
                    for (uint32_t k = 0; k < sn; ++k) {
                        const uint64_t v = st[--sp];
                        acc = op == kOpAnd ? (acc & v) : (acc | v);
                    }
                }
                next += pn;
                if (sp >= kMaxStack) { bad = true; break; }
                st[sp++] = acc;
            } else if (op == kOpConjunction) {
                if (pc + 1 >= plen) { bad = true; break; }
                const uint32_t parts = s_prog[pc + 1];
                if (parts == 0 || pc + 2 + parts > plen) { bad = true; break; }
                uint64_t acc = ~0ull;
                for (uint32_t p = 0; p < parts && !bad; ++p) {
                    const uint32_t pn = s_prog[pc + 2 + p];
                    if (pn == 0 || next + pn > nop) { bad = true; break; }
                    uint64_t o = 0;
                    for (uint32_t k = 0; k < pn; ++k) o |= slots[(next + k) * kTile + t];
                    acc &= o;
                    next += pn;
                }
                pc += 2 + parts;
                if (bad || sp >= kMaxStack) { bad = true; break; }
                st[sp++] = acc;
            } else {
                bad = true;
            }
        }
        if (!bad && (sp != 1 || next != nop)) bad = true;
        if (!bad) result = st[0];
    }
    if (t < nw) {
        result &= tail_mask(gw, L.doc_num);
        out_row[gw] = result;
    }
    if (L.pass_count) {
        const uint32_t c = warp_sum(t < nw ? __popcll(result) : 0u);
        if ((t & 31) == 0 && c) atomicAdd(L.pass_count + q, c);
    }
    if (L.status && t < nw && bad) {
        atomicOr(L.status + q, s_bad ? kStatusBadPosting : kStatusBadProgram);
    }
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

}  // namespace

cudaError_t launch_filter_batch(const FilterLaunch& L, cudaStream_t stream) {
    if (L.nq == 0 || L.seg_num == 0) return cudaSuccess;
    const uint32_t seg_words = L.docs_per_seg / 64;
    const uint32_t tiles = (seg_words + kTile - 1) / kTile;
    const uint64_t gy = static_cast<uint64_t>(L.seg_num) * tiles;
    if (gy > 65535u || L.max_opnd > static_cast<uint32_t>(kMaxOperands)) return cudaErrorInvalidValue;
    const size_t smem = static_cast<size_t>(L.max_opnd > 0 ? L.max_opnd : 1) * kTile * sizeof(uint64_t);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(filter_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    dim3 grid(L.nq, static_cast<uint32_t>(gy));
    filter_batch_kernel<<<grid, kTile, smem, stream>>>(L);
    return cudaGetLastError();
}

cudaError_t launch_posting_expand(const uint64_t* src, const uint64_t* dst, uint32_t count, uint32_t byte_size,
                                  uint32_t seg_docs, int32_t* status, cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    posting_expand_kernel<<<count, 256, 0, stream>>>(src, dst, count, byte_size, seg_docs, status);
    return cudaGetLastError();
}

}  // namespace hss
