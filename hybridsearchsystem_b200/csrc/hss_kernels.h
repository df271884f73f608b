// hss_kernels.h -- launch descriptors and host-side launchers of the CUDA kernels (internal to
// libhss.so; the public C-ABI is include/hss.h).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace hss {

// Batched postfix filter (filter.cu). Operand i of query q at segment s is the posting at device
// address table[row * row_stride + s * seg_stride], row = opnd_row[opnd_off[q] + i] (or i when
// opnd_row is null). An address of 0 is an all-zero posting.
struct FilterLaunch {
    const uint32_t* prog;      // concatenated postfix programs
    const uint32_t* prog_off;  // [nq + 1]
    const uint32_t* opnd_row;  // concatenated operand rows, or null
    const uint32_t* opnd_off;  // [nq + 1]
    const uint64_t* table;     // posting address table
    uint64_t row_stride;
    uint64_t seg_stride;
    uint64_t* out;             // [nq][out_stride] bitmap words
    uint64_t out_stride;
    uint32_t* pass_count;      // [nq] docs passing, accumulated (zeroed by the caller), or null
    int32_t* status;           // [nq] error bits, or null
    uint32_t nq;
    uint32_t seg_num;
    uint32_t docs_per_seg;     // multiple of 128
    uint64_t doc_num;
    uint32_t max_opnd;         // largest operand count of any query in the batch (<= 64)
    // Single-query form: when prog_off is null, query 0's program is prog[0..single_prog_len) over
    // single_nop operands.
    uint32_t single_prog_len;
    uint32_t single_nop;
    // Table entries follow the reference's convention (untagged = dense bitset address, bit 0 =
    // sparse posting head, 2 = empty) instead of being posting head addresses.
    int ref_table;
};

// Batched filter over the dense posting matrix (filter.cu): operand i of query q at segment s is
// dense[(opnd_row[opnd_off[q] + i] * seg_num + s) * seg_words ...], already decoded.
struct DenseFilterLaunch {
    const uint32_t* prog;      // concatenated postfix programs
    const uint32_t* prog_off;  // [nq + 1]
    const uint32_t* opnd_row;  // concatenated operand rows
    const uint32_t* opnd_off;  // [nq + 1]
    const uint64_t* dense;     // [rows][seg_num][seg_words], 16-byte aligned
    uint32_t rows;
    uint32_t seg_words;        // docs per segment / 64 (even)
    uint64_t* out;             // [nq][out_stride] bitmap words
    uint64_t out_stride;
    uint32_t* pass_count;      // [nq] docs passing, accumulated (zeroed by the caller), or null
    int32_t* status;           // [nq] error bits, or null
    uint32_t nq;
    uint32_t seg_num;
    uint64_t doc_num;
    uint32_t max_opnd;         // largest operand count of any query in the batch (<= 64)
    uint32_t sm_count;         // SMs of the device (sizes the grid; 0: 148)
};
cudaError_t launch_filter_dense(const DenseFilterLaunch& L, cudaStream_t stream);


// Candidate lists are segmented so that no producer needs a global atomic: query q's region
// [q * cap, (q + 1) * cap) is cut into segments of seg_cap entries; segment g (at g * seg_cap) is
// written by exactly one producer thread group, and counts[q * kMaxCandSegs + g] is how many
// candidates it found for q (more than seg_cap means the segment overflowed; only seg_cap are
// stored). A pass writes the segments [seg_base, seg_base + its segments): a SIMT pass one per CTA,
// a tensor-core pass two per CTA. Each producer writes its count for every query it serves, so the
// counts need no clearing. Tiles of a pass: tile_begin + i * tile_step, or, when tile_skip >= 2,
// every tile that is not a multiple of tile_skip (the complement of a step-tile_skip pass).
constexpr uint32_t kMaxCandSegs = 1024;

// Bulk candidate pass (score.cu). Processes tiles tile_begin + i * tile_step, i < tile_count, of
// 128 docs each, for the queries qlist[0..nq_list) (or 0..nq_list-1 when qlist is null), with
// `segs` CTAs (one candidate segment each).
struct CandLaunch {
    const float* vec;          // [tiles * 128][dim] FP32 corpus, rows 16-byte aligned
    const float* qry;          // [nq][dim]
    const uint64_t* bits;      // [nq][bits_stride] filter bitmaps
    uint64_t bits_stride;
    const float* theta;        // [nq] candidate thresholds
    const uint32_t* qlist;
    uint32_t nq_list;
    float* cand_score;         // [nq][cap], segmented
    uint32_t* cand_loc;        // [nq][cap], segmented
    uint32_t* cand_count;      // [nq][kMaxCandSegs] per-segment counts
    uint32_t cap;
    uint32_t segs, seg_cap;    // CTAs of the launch (cand_simt_segments) and entries per segment
    uint32_t seg_base;         // first segment this pass writes
    uint32_t dim;              // multiple of 4
    uint64_t tile_begin, tile_step, tile_count;
    uint32_t tile_skip;
};
// Largest query count of one SIMT candidate pass (its per-query counts live in shared memory).
constexpr uint32_t kMaxSimtBatch = 4096;
// CTAs of a SIMT candidate pass over tile_count tiles into lists of `cap` entries (one list segment
// each): the kernel's natural grid, but few enough that two passes' segments fit kMaxCandSegs with
// at least kMinSegCap entries each (a small list split too finely would overflow on uneven segments).
constexpr uint32_t kMinSegCap = 256;
uint32_t cand_simt_segments(uint64_t tile_count, int num_sms, uint32_t cap);

// Threshold from the K-th best approximate score of a segmented list (segments [0, segs)):
// theta = kth - eps_sample - eps_main. With raise_only the result is max(old theta, that), and a list
// with fewer than K entries keeps the old theta.
// Doc-sample statistics for the threshold predictor's features, floats per query: [0, kSampleRanks)
// the sample's best approximate scores at ranks 1, 2, 4, ..., 64 (-2 past the sample's size), then
// the K-th best (-2 when the sample holds fewer than K), then the number of filtered sample docs,
// then zeros.
constexpr uint32_t kSampleRanks = 7;
constexpr uint32_t kSampleStats = 12;
// Features past the query vector and the per-row block: log selectivity, log K, a constant, the
// sample's rank scores, its K-th best and its log size.
constexpr uint32_t kFeatureTail = 3 + kSampleRanks + 2;

struct SampleThresholdLaunch {
    const float* score;        // [nq][cap] sample scores, segmented
    const uint32_t* count;     // [nq][kMaxCandSegs]
    uint32_t cap;
    uint32_t segs, seg_cap;
    int raise_only;
    const uint32_t* topk;      // [nq]
    const float* eps_sample;   // [nq] error bound of the sample pass
    const float* eps_main;     // [nq] error bound of the main pass
    float* theta;              // [nq] out
    float* theta_also;         // [nq] or null: raised with theta (raise_only launches), else a copy of it
    const uint32_t* qlist;
    uint32_t nq_list;
    float* stats;              // [nq][kSampleStats] or null (layout at kSampleStats)
};

struct SelectLaunch {
    const float* vec;
    const float* qry;
    uint32_t dim;
    const float* cand_score;   // segmented lists (see kMaxCandSegs)
    const uint32_t* cand_loc;
    const uint32_t* cand_count;  // [nq][kMaxCandSegs]
    uint32_t cap;
    uint32_t segs, seg_cap;    // segments [0, segs) hold the candidates
    unsigned long long* work;  // [nq][cap]
    const uint32_t* topk;
    const float* eps_main;
    float* theta;              // raised on overflow
    // [nq] proven thresholds, or null when every theta is proven. A query whose theta is above its
    // proven one (a predicted threshold) has its result checked; when the check fails both are set to
    // a proven threshold and the query is flagged for a re-run.
    float* theta_proven;
    const int64_t* gdocid;     // location -> global doc id, or null (identity)
    float* out_score;          // [nq][out_stride]
    int64_t* out_id;
    uint32_t* out_count;       // [nq]
    uint32_t out_stride;
    int32_t* status;
    const uint32_t* qlist;
    uint32_t nq_list;
    int fast_large;            // hold up to 32,768 candidate scores in shared memory (else 12,288)
};

// Tensor-core candidate pass (score_tc.cu).
enum TcFormat : int { kTcTF32 = 0, kTcBF16 = 1, kTcE4M3 = 2 };
constexpr int kMaxTcStages = 12;

struct TcCandLaunch {
    int format;                // TcFormat of both the corpus copy and the staged queries
    uint32_t kblocks;          // dim * element bytes / 128
    uint32_t stages;           // stages in the TMA ring (set by launch_tc_cand)
    uint32_t group;            // corpus k-blocks per ring stage (set by launch_tc_cand; 1 or 2)
    int emit_all;              // every row's threshold is -inf (the doc sample): most docs are kept
    const float* doc_scale;    // E4M3: per-doc dequantisation scale
    const float2* tile_scale;  // E4M3: per 128-doc tile (min, max) of doc_scale
    const float* q_scale;      // E4M3: per staged query row
    const uint64_t* bits;      // [nq][bits_stride] filter bitmaps
    uint64_t bits_stride;
    const float* theta;        // [nq]
    const uint32_t* qlist;     // staged row r is query qlist[r] (or r)
    uint32_t nq_rows;          // staged rows in use (<= 256)
    float* cand_score;         // segmented lists (see kMaxCandSegs)
    uint32_t* cand_loc;
    uint32_t* cand_count;      // [nq][kMaxCandSegs]
    uint32_t cap;
    uint32_t ctas, seg_cap;    // CTAs of the launch (tc_cand_ctas); entries per list segment
    uint32_t seg_base;         // first segment this pass writes (it writes 2 per CTA)
    uint64_t tile_begin, tile_step, tile_count;  // tiles of tc_tile_docs(nq_rows, kblocks) docs
    uint32_t tile_skip;
    uint64_t tiles128;         // 128-doc tiles of the corpus (rows of the tensor map / 128)
    int32_t* error;            // device error bits (bounded waits that expired)
    // Pipeline test knobs (single-SM kernel): wait_budget > 0 replaces the clock budget of the waits
    // that can abort the pass; hold_load > 0 makes the producer stop before issuing its
    // (hold_load)-th corpus stage, so the MMA issuer's wait for it runs out.
    long long wait_budget;
    uint32_t hold_load;
};

// Whether a tensor-core pass over rows of `kblocks` 128-byte k-blocks streams the queries' k-blocks
// through its stage ring with the docs' (an SM pair per tile, any batch size) instead of keeping them
// resident: when fewer than four stages would fit next to the resident queries (long vectors).
bool tc_stream_queries(uint32_t kblocks);
// Docs per tile of a tensor-core pass over `rows` staged queries: 128 (one SM per tile, rows <= 128)
// or 256 (an SM pair per tile, cta_group::2: rows 129..256, or streamed queries).
uint32_t tc_tile_docs(uint32_t rows, uint32_t kblocks);
// CTAs of a tensor-core pass over tile_count such tiles into lists of `cap` entries; it writes two
// list segments per CTA.
uint32_t tc_cand_ctas(uint32_t rows, uint32_t kblocks, uint64_t tile_count, int num_sms, uint32_t cap);
// Corpus k-blocks per ring stage of a pass over `kblocks` k-blocks (single SM or SM pair): two when
// they divide the row and three such stages still fit beside the resident queries, else one. A
// stage is one TMA barrier: the fewer stages per tile, the fewer waits in the MMA issuer's loop.
uint32_t tc_group(uint32_t kblocks, bool pair);
size_t tc_smem_bytes(int halves, uint32_t kblocks, uint32_t stages, uint32_t group);
size_t tc_pair_smem_bytes(uint32_t kblocks, uint32_t stages, uint32_t group);
cudaError_t launch_tc_cand(const TcCandLaunch& L, const CUtensorMap& doc_map, const CUtensorMap& qry_map, int sms,
                           cudaStream_t stream);
// 2D tensor map over [rows][dim] elements of `format`, 128-byte swizzle, box {128 bytes, 128 rows}.
bool make_tc_map(CUtensorMap* map, int format, const void* base, uint64_t rows, uint32_t dim);

// Quantised copies of the corpus for the tensor-core formats (quant.cu): bf16 / e4m3 rows with
// per-doc scale (e4m3), per-doc norm and quantisation-error norm (FP64, rounded up to float).
cudaError_t launch_quantize_docs(const float* vec, uint64_t rows, uint64_t valid_rows, uint32_t dim, int format,
                                 void* out, float* scale, float* norm, float* err_norm, cudaStream_t stream);
cudaError_t launch_tile_scale_minmax(const float* scale, uint64_t tiles, float2* out, cudaStream_t stream);
// Stage a batch of queries in a tensor-core format (rows past nq zero) and compute the per-query error
// bounds of the candidate pass (see score_tc.cu / searcher.cpp).
struct StageQueriesLaunch {
    const float* qry;      // [nq][dim]
    const uint32_t* qlist; // staged row r = query qlist[r], or r
    uint32_t nq_rows, rows_alloc, dim;
    int format;
    void* staged;          // [rows_alloc][dim] in `format`
    float* q_scale;        // E4M3
    float* eps_main;       // [nq] (indexed by query)
    float* eps_sample;
    double doc_norm_max, doc_err_max;  // corpus-wide max ||v|| and max ||quantised v - v||
    double acc_rel;        // relative accumulation bound of the tensor-core dot products
};
cudaError_t launch_stage_queries(const StageQueriesLaunch& L, cudaStream_t stream);

cudaError_t launch_filter_batch(const FilterLaunch& L, cudaStream_t stream);
cudaError_t launch_posting_expand(const uint64_t* src, const uint64_t* dst, uint32_t count, uint32_t byte_size,
                                  uint32_t seg_docs, int32_t* status, cudaStream_t stream);
cudaError_t launch_exact_score(const float* qry, const float* docs, float* out, uint32_t m, uint32_t n, uint32_t dim,
                               uint64_t ldc, cudaStream_t stream);
cudaError_t launch_cand_simt(const CandLaunch& L, int num_sms, cudaStream_t stream);
cudaError_t launch_sample_threshold(const SampleThresholdLaunch& L, cudaStream_t stream);
cudaError_t launch_select_topk(const SelectLaunch& L, cudaStream_t stream);
// Error bounds of the SIMT pass for queries qlist[0..nq) (all of 0..nq-1 when qlist is null).
cudaError_t launch_query_eps(const float* qry, const uint32_t* qlist, uint32_t nq, uint32_t dim, float max_norm,
                             double c_main, double c_sample, float* eps_main, float* eps_sample, cudaStream_t stream);
size_t aggregate_workspace_bytes(uint32_t n);
// Allocation-free aggregator scratch: kAggStaticBlocks block counts in a module-scope device array;
// aggregate_static_scratch returns its address on the current device (the runtime may load the
// module on the first call on a device).
constexpr uint32_t kAggStaticBlocks = 16384;
constexpr uint32_t kAggStaticMaxDocs = kAggStaticBlocks * 1024u;
cudaError_t aggregate_static_scratch(uint32_t** scratch);
cudaError_t launch_aggregate(const uint64_t* bits, const float* scores, const uint32_t* loc_in, uint32_t n,
                             float* out_scores, uint32_t* out_loc, uint32_t* total, uint32_t* workspace,
                             cudaStream_t stream);
// Learned threshold predictor (mlp.cu).
// C = op(A) op(B) (+ C) (+ bias), then act (0 identity, 1 GELU); pre receives the value before act.
cudaError_t launch_gemm(bool ta, bool tb, const float* A, const float* B, float* C, int M, int N, int K, int lda,
                        int ldb, int ldc, const float* bias, int act, float* pre, bool accumulate,
                        cudaStream_t stream);
cudaError_t launch_gelu_backward(float* dA, const float* Z, int64_t n, cudaStream_t stream);
cudaError_t launch_colsum(const float* G, int M, int N, int ld, float* out, cudaStream_t stream);
// dL/dy and the per-row loss terms: squared error (tau = 0) or the pinball loss of the tau-quantile.
cudaError_t launch_loss_grad(const float* y, const float* t, int B, float tau, float* dy, float* term,
                             cudaStream_t stream);
// The whole inference forward pass of the MLP (parameters P in ThresholdModel's layout) in one launch;
// bit-identical to the three-GEMM pass. H <= 1024, 4 (D + 2H) floats of shared memory <= 48 KB.
cudaError_t launch_mlp_forward(const float* X, int B, int D, int H, const float* P, float* y, cudaStream_t stream);
cudaError_t launch_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2,
                        float eps, int step, cudaStream_t stream);
struct FeatureLaunch {
    const float* qry;           // [nq][dim]
    const float* stats;         // [nq][kSampleStats] doc-sample statistics (sample_threshold_kernel)
    const uint32_t* opnd_row;   // concatenated filter operand rows
    const uint32_t* opnd_off;   // [nq + 1]
    const uint32_t* pass_count; // [nq] docs the filter lets through
    const uint32_t* topk;       // [nq]
    const float* row_density;   // [rows] fraction of docs holding each posting row's token
    float* x;                   // [nq][din] out
    uint32_t nq, dim, rows, din;
    uint64_t doc_num;
};
cudaError_t launch_features(const FeatureLaunch& L, cudaStream_t stream);
// The learned threshold of each query: theta_proven[q] = theta[q] (the proven one), then
// theta[q] = max(theta[q], y[q] * scale + shift - margin - eps[q]) where the filter passes more than
// kLearnedMinPass * topk[q] docs and the doc sample (stats [nq][kSampleStats]) held at least
// kLearnedMinSample of them; theta_model[q] gets the new theta (it may alias y).
constexpr uint32_t kLearnedMinPass = 4;
constexpr float kLearnedMinSample = 64.0f;  // every sample rank feature (1, 2, 4, ..., 64) present
cudaError_t launch_predict_theta(const float* y, const float* eps, const uint32_t* pass_count, const uint32_t* topk,
                                 const float* stats, uint32_t nq, float scale, float shift, float margin,
                                 float* theta, float* theta_proven, float* theta_model, cudaStream_t stream);

// Cross-shard merge of sorted per-shard top-K lists (select.cu).
constexpr uint32_t kMaxShards = 64;
struct ShardMergeLaunch {
    const float* scores[kMaxShards];    // shard s: [nq][in_stride], score descending
    const int64_t* ids[kMaxShards];     // shard s: [nq][in_stride]
    const uint32_t* counts[kMaxShards]; // shard s: [nq]
    uint32_t shards, nq, in_stride, topk;
    float* out_score;                   // [nq][out_stride]
    int64_t* out_id;
    uint32_t* out_count;                // [nq]
    uint32_t out_stride;
};
cudaError_t launch_merge_shards(const ShardMergeLaunch& L, cudaStream_t stream);

cudaError_t launch_topk_op(const float* scores, const uint32_t* locs, const uint32_t* count, uint32_t k,
                           float* out_scores, uint32_t* out_locs, uint32_t* out_count, cudaStream_t stream);

}  // namespace hss
