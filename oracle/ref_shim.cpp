// ref_shim.cpp -- extern "C" entry points over the reference's OWN CPU code, compiled unchanged
// from the reference sources by oracle/Makefile into oracle/_ref/libref.so.
//
// TEST INFRASTRUCTURE ONLY: it pins the C restatement (oracle.c) and, as the "reference" kind of
// CPU baseline, times the reference's ground-truth scan. The product never loads it.
//
// Reference functions called (paths relative to the reference project root):
//   npur_harness::ParseFilter / EvalFilterBitmap      src/harness/query/filter_expr.h:164-232
//   npur_harness::CpuTopK / CpuTopKBatch               10.13/load/src/harness/recall/recall_ref.cpp:33-142
//   NpuRetrieval::PostingSerializer::Serialize         src/engine/format/posting_serializer.cpp:81-101
//   NpuRetrieval::Hash64                               src/engine/core/hash/hash.cpp:10-16
//   NpuRetrieval::Float32ToFloat16 / Float16ToFloat32  src/engine/core/number/trans_number.cpp:38-105
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

#include "harness/query/filter_expr.h"
#include "harness/recall/recall_ref.h"
#include "io/dataset_hw.h"
#include "src/full_recall/core/hash/hash.h"
#include "src/full_recall/core/number/trans_number.h"
#include "src/full_recall/format/posting_serializer.h"

namespace {
// A HwDataset over caller-owned arrays, filled the way test_recall_ref.cpp's FakeCorpus does.
void FillHw(npur_port::HwDataset& hw, const float* vectors, const uint64_t* bitmaps, uint32_t dim, uint32_t tag_num,
            uint64_t doc_num) {
    hw.vectors = vectors;
    hw.bitmaps = bitmaps;
    hw.dim = dim;
    hw.tag_num = tag_num;
    hw.stride = (tag_num + 63u) / 64u;
    hw.doc_num = doc_num;
}
}  // namespace

extern "C" {

uint64_t ref_hash64(const char* data, uint32_t len) { return NpuRetrieval::Hash64(data, len); }

uint16_t ref_f32_to_f16(float f) { return NpuRetrieval::Float32ToFloat16(f); }
float ref_f16_to_f32(uint16_t h) { return NpuRetrieval::Float16ToFloat32(h); }

// Returns the serialized length, -1 on failure, -2 when `cap` is too small.
int64_t ref_posting_serialize(const uint32_t* ids, uint32_t n, uint32_t doc_num, int is_matrix, float threshold,
                              uint8_t* out, uint64_t cap) {
    std::unordered_set<uint32_t> set(ids, ids + n);
    std::string buf;
    NpuRetrieval::PostingSerializer ser;
    if (!ser.Serialize(set, doc_num, is_matrix != 0, threshold, buf)) return -1;
    if (buf.size() > cap) return -2;
    std::memcpy(out, buf.data(), buf.size());
    return static_cast<int64_t>(buf.size());
}

// 1 when the expression parses (an empty one included), 0 on a parse error.
int ref_parse_ok(const char* expr) {
    bool ok = true;
    auto n = npur_harness::ParseFilter(expr, ok);
    (void)n;
    return ok ? 1 : 0;
}

// EvalFilterBitmap of one doc bitmap; -1 on a parse error.
int ref_eval_bitmap(const char* expr, const uint64_t* bm, uint32_t words) {
    bool ok = true;
    auto n = npur_harness::ParseFilter(expr, ok);
    if (!ok) return -1;
    return npur_harness::EvalFilterBitmap(n.get(), bm, words) ? 1 : 0;
}

// CpuTopK for one query. Writes the (unordered) id set, sorted ascending, and returns its size;
// -1 on a parse error, -2 when cap is too small.
int ref_cpu_topk(const float* query, uint32_t dim, const char* filter, const float* vectors, const uint64_t* bitmaps,
                 uint32_t tag_num, uint64_t doc_num, uint64_t doc_offset, int topk, int fp32, int64_t* out_ids,
                 int cap) {
    bool ok = true;
    auto ast = npur_harness::ParseFilter(filter, ok);
    if (!ok) return -1;
    npur_port::HwDataset hw;
    FillHw(hw, vectors, bitmaps, dim, tag_num, doc_offset + doc_num);
    std::vector<float> q(query, query + dim);
    auto set = npur_harness::CpuTopK(q, ast.get(), hw, doc_num, topk, doc_offset, fp32 != 0);
    std::vector<int64_t> ids(set.begin(), set.end());
    std::sort(ids.begin(), ids.end());
    hw.vectors = nullptr;  // caller-owned; HwDataset's destructor only unmaps its own mapping
    if (static_cast<int>(ids.size()) > cap) return -2;
    std::copy(ids.begin(), ids.end(), out_ids);
    return static_cast<int>(ids.size());
}

// CpuTopKBatch over `threads` query slices, each slice one corpus pass -- the reference's batched
// ground truth, as the CPU baseline times it. Row q of out_ids (stride out_stride) gets the sorted
// id set, out_counts[q] its size. Returns 0, or -1 on a parse error.
int ref_cpu_topk_batch(const float* queries, uint32_t nq, uint32_t dim, const char* const* filters,
                       const int32_t* topks, const float* vectors, const uint64_t* bitmaps, uint32_t tag_num,
                       uint64_t doc_num, uint64_t doc_offset, int fp32, int threads, int32_t out_stride,
                       int64_t* out_ids, int32_t* out_counts) {
    std::vector<std::unique_ptr<npur_harness::FilterNode>> asts(nq);
    for (uint32_t q = 0; q < nq; ++q) {
        bool ok = true;
        asts[q] = npur_harness::ParseFilter(filters[q], ok);
        if (!ok) return -1;
    }
    std::vector<std::vector<float>> qv(nq);
    for (uint32_t q = 0; q < nq; ++q) qv[q].assign(queries + static_cast<size_t>(q) * dim, queries + (q + 1ull) * dim);
    npur_port::HwDataset hw;
    FillHw(hw, vectors, bitmaps, dim, tag_num, doc_offset + doc_num);
    const auto quantized = npur_harness::QuantizeCorpus(hw, doc_num, doc_offset, fp32 != 0,
                                                        static_cast<unsigned>(std::max(1, threads)));
    std::vector<std::unordered_set<int64_t>> out(nq);
    const uint32_t t = std::max<uint32_t>(1, std::min<uint32_t>(static_cast<uint32_t>(std::max(1, threads)), nq));
    const uint32_t per = (nq + t - 1) / t;
    std::vector<std::thread> pool;
    for (uint32_t i = 0; i < t; ++i) {
        const uint32_t q0 = std::min(nq, i * per), q1 = std::min(nq, q0 + per);
        pool.emplace_back([&, q0, q1]() {
            std::vector<npur_harness::RecallRefJob> jobs;
            for (uint32_t q = q0; q < q1; ++q) jobs.push_back({&qv[q], asts[q].get(), topks[q], q});
            npur_harness::CpuTopKBatch(jobs, hw, quantized, doc_num, doc_offset, fp32 != 0, out);
        });
    }
    for (auto& th : pool) th.join();
    for (uint32_t q = 0; q < nq; ++q) {
        std::vector<int64_t> ids(out[q].begin(), out[q].end());
        std::sort(ids.begin(), ids.end());
        const int32_t n = std::min<int32_t>(static_cast<int32_t>(ids.size()), out_stride);
        std::copy(ids.begin(), ids.begin() + n, out_ids + static_cast<size_t>(q) * out_stride);
        out_counts[q] = static_cast<int32_t>(ids.size());
    }
    hw.vectors = nullptr;
    return 0;
}

}  // extern "C"
