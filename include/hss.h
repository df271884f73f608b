/*
 * hss.h -- C-ABI of libhss.so, the B200 implementation of the filtered full-recall path.
 *
 * Two layers:
 *   1. Operator entry points: drop-ins for the reference's device operators, which its host code
 *      launches through the generated aclrtlaunch_* headers (ACLRT_LAUNCH_KERNEL(name)(blockDim, stream,
 *      args...)). Each takes device pointers plus a cudaStream_t in place of the ACL stream and
 *      returns a status code instead of having none.
 *   2. Index and searcher handles: DataTable load / build and the FullRecallSearcher batch call.
 *
 * Paths in citations are relative to the reference project root. All sizes are in elements unless
 * named *Bytes. No function allocates device memory on the calling thread's behalf except the
 * table/searcher constructors, which allocate their whole arena once.
 */
#ifndef HSS_H
#define HSS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* cudaStream_t without pulling in the CUDA headers */
typedef struct CUstream_st* hss_stream_t;

/* ---- status codes ---- */
#define HSS_OK 0
#define HSS_ERR_INVALID (-1) /* bad argument */
#define HSS_ERR_CUDA (-2)    /* CUDA runtime error (message in hss_last_error) */
#define HSS_ERR_PARSE (-3)   /* filter expression does not parse */
#define HSS_ERR_PROGRAM (-4) /* malformed postfix filter program */
#define HSS_ERR_LIMIT (-5)   /* a size beyond one of the limits below */
#define HSS_ERR_INDEX (-6)   /* index build / load failure */
#define HSS_ERR_QUERY (-7)   /* some queries of the batch failed: see hss_searcher_last_status */

/* ---- limits ---- */
#define HSS_MAX_TOPK 4096       /* largest K per query */
#define HSS_MAX_OPERANDS 64     /* postings one filter program reads */
#define HSS_MAX_PROGRAM 512     /* u32 words of one postfix program */
#define HSS_MAX_STACK 16        /* evaluation stack depth of one program */

/* per-query status bits (hss_searcher_last_status) */
#define HSS_QSTATUS_BAD_PROGRAM 1
#define HSS_QSTATUS_BAD_POSTING 2
#define HSS_QSTATUS_OVERFLOW 4   /* candidate list still over capacity after all re-runs */
#define HSS_QSTATUS_TOPK_TOO_LARGE 8

/* TextFilterContextData (src/engine/retrieval/device/device_common_external.h:17-25). */
typedef struct hss_filter_context {
    uint32_t postingNum;    /* operands (postings) of the program */
    uint32_t segmentNum;
    uint32_t segmentLength; /* u16 bitset units per segment = docNumPerSegment / 16; a multiple of 8 */
    uint32_t tileNum;       /* ignored: one pass per segment tile */
    uint32_t exprLen;       /* u32 words of postOrderExpr */
    uint32_t opNum;         /* operators in postOrderExpr */
    uint32_t flags;         /* HSS_FILTER_HEAD_ADDRESSES, other bits ignored */
} hss_filter_context;

/* postings[] holds posting head addresses (the 8-byte [layout:4|hits:28][payloadLen] head), any of
 * the five layouts, 0 = all-zero posting. Without this flag the reference's convention applies
 * (text_filter.cpp:720-745): an untagged entry is a dense bitset address (head + 8), an entry with
 * bit 0 set (SPARSE_OPERAND_TAG) is a sparse posting's head, and EMPTY_OPERAND_TAG (2) an all-zero
 * operand. */
#define HSS_FILTER_HEAD_ADDRESSES 0x80000000u

/* Replaces kernel_vector_mmad (scorer/kernel_vector_mmad_op.cpp:3-11, launched by
 * VectorScorerMmad::BatchComputeLaunch, vector_scorer_mmad.cpp:32-168):
 *   resultMatrix[i * ldResult + j] = sum_d queryMatrix[i][d] * docMatrix[j][d]
 * for i < m, j < n. FP32 in and out, row-major contiguous docMatrix (not the zN tiling), computed in
 * the ground truth's order (sequential over d, multiply then add, no FMA), so every entry equals the
 * CPU oracle's score bit for bit. k % 4 == 0, k <= 4096. */
int hss_vector_score_launch(const float* queryMatrix, const float* docMatrix, float* resultMatrix, uint32_t m,
                            uint32_t n, uint32_t k, uint64_t ldResult, hss_stream_t stream);

/* Replaces BitmapTextFilter (filter/kernel_bitmap_text_filter.cpp:52-119, launched by
 * TextFilter::BitmapTextFilter, text_filter.cpp:1071-1129): evaluates one postfix program
 * (query_node_imp.cpp form: [AND|OR|NOT, postingNum, stackNum] / [CONJUNCTION, parts, n_1..n_parts])
 * over postings[segment * postingNum + i] for every segment, writing segmentNum * segmentLength u16
 * units of result bits (bit i of unit u = doc 16u+i). All five posting layouts are decoded in place,
 * so the PostingBitListToSet pre-pass is not needed. resultStack is unused (the stack lives on chip)
 * and may be NULL. status (device int32, may be NULL) gets HSS_QSTATUS_* bits. result must be
 * 8-byte aligned. */
int hss_bitmap_text_filter_launch(const uint64_t* postings, const uint32_t* postOrderExpr, void* resultStack,
                                  hss_filter_context context, uint8_t* result, int32_t* status,
                                  hss_stream_t stream);

/* Replaces PostingBitListToSet (filter/kernel_bitmap_text_filter.cpp:18-43, bitlist_to_set.h): expands
 * the posting at postings[i] (head address, any layout) into the dense bitset resultPostings[i] of
 * byteSizePerSegment bytes, for i < count. The reference's core-split arguments (former/tail) and
 * ablation switches have no counterpart. byteSizePerSegment % 8 == 0. */
int hss_posting_bitlist_to_set_launch(const uint64_t* postings, uint32_t byteSizePerSegment,
                                      const uint64_t* resultPostings, uint32_t count, int32_t* status,
                                      hss_stream_t stream);

/* Replaces Aggregator (aggregator/kernel_aggregator.cpp:4-13, kernel_aggregator.h:18-206, launched by
 * ResultAggregator::Aggregator, result_aggregator.cpp:1054-1147): keeps (docScores[i],
 * docLocationConst[i]) for every i < docNumber whose filter bit is set, in order, and writes the
 * total to effectiveCount[0] on the device (no per-core count slots, no host round trip).
 * docLocationConst may be NULL (identity). The outputs must not alias the inputs. `workspace` is
 * device scratch of hss_aggregator_workspace_size(docNumber) bytes. */
size_t hss_aggregator_workspace_size(uint32_t docNumber);
int hss_aggregator_launch(const uint8_t* filterResult, const float* docScores, const uint32_t* docLocationConst,
                          float* outScores, uint32_t* outLocations, uint32_t* effectiveCount, uint32_t docNumber,
                          void* workspace, size_t workspaceBytes, hss_stream_t stream);

/* Allocation-free aggregator. NO COUNTERPART IN THE REFERENCE (whose Aggregator always takes
 * pool-allocated scratch). Same arguments and results as hss_aggregator_launch minus the workspace:
 * for callers that must not allocate device memory per call or hold a workspace of their own --
 * a request handler running under a fixed device-memory budget that another allocator owns, or a
 * latency-critical loop that cannot afford cudaFree, which waits for the whole device to go idle.
 * Its scratch is a 64 KB array compiled into the library, one per device, so docNumber <=
 * HSS_AGGREGATOR_NOALLOC_MAX_DOCS (else HSS_ERR_LIMIT, nothing launched). It calls no allocator.
 * The first call on each device looks the array's address up (cudaGetSymbolAddress, with that
 * device current); make that first call before any stream capture. The address is cached per device
 * together with the id of the CUDA context it belongs to, so the first call after the device's
 * context was replaced (cudaDeviceReset) looks it up again. Every call on a device shares
 * the one array: calls that can overlap on the GPU (different streams without ordering between
 * them) race and must not be made; calls ordered on one stream are safe, since each call rewrites
 * all the scratch it reads. */
#define HSS_AGGREGATOR_NOALLOC_MAX_DOCS 16777216u
int hss_aggregator_launch_noalloc(const uint8_t* filterResult, const float* docScores,
                                  const uint32_t* docLocationConst, float* outScores, uint32_t* outLocations,
                                  uint32_t* effectiveCount, uint32_t docNumber, hss_stream_t stream);

/* Replaces TOPK (topk/kernel_topk.cpp:4-13, launched by ResultAggregator::TopK,
 * result_aggregator.cpp:1180-1252) and the host nth_element + sort after it
 * (AggregatorResultFillExtract, :846-1032): the exact top min(topK, *count) of the compacted list,
 * ordered by score descending then location ascending. count / outCount are device pointers.
 * topK <= HSS_MAX_TOPK. */
int hss_topk_launch(const float* scores, const uint32_t* locations, const uint32_t* count, uint32_t topK,
                    float* outScores, uint32_t* outLocations, uint32_t* outCount, hss_stream_t stream);

/* Replaces the reference's cross-shard merge of per-shard results (RunContext::FoldShardIntoAcc and
 * the k-way merge, src/harness/run/run_context.cpp:86-118,237-270): shard s's results for query q are
 * shardScores[s][q * inStride + i], shardIds[s][...] (i < shardCounts[s][q], score descending, as the
 * searcher returns them); the merged top min(topK, sum of counts) go to outScores / outIds
 * [q * outStride + j] and outCounts[q], by score descending, equal scores to the lower shard first
 * (then list order). With shards holding ascending doc ranges this is the ground truth's (score
 * descending, doc id ascending) order. The pointer arrays are host arrays of device pointers on the
 * current device (gather other GPUs' results there first). shards <= HSS_MAX_SHARDS. */
#define HSS_MAX_SHARDS 64
int hss_merge_shards_launch(const float* const* shardScores, const int64_t* const* shardIds,
                            const uint32_t* const* shardCounts, uint32_t shards, uint32_t nq, uint32_t inStride,
                            uint32_t topK, float* outScores, int64_t* outIds, uint32_t* outCounts, uint32_t outStride,
                            hss_stream_t stream);

/* ---- index (DataTable, src/engine/index/data_table.h:10-92) ---- */
typedef struct hss_table hss_table;

typedef struct hss_index_config {
    uint32_t docNumPerSegment; /* multiple of 128 (the reference needs a multiple of 8) */
    float densityThreshold;    /* posting is sparse below this density (1/64 in the configs) */
    int32_t matrixPosting;     /* 1: DENSE_BYTEMAP / SPARSE_IDLIST layouts */
    int32_t sparsePacked;      /* 1: SPARSE_PACKED instead of SPARSE_BITMAP (NPUR_SPARSE_PACKED) */
    uint64_t docOffset;        /* global doc id of the first doc */
} hss_index_config;

/* Offline build (fr_converter + fr_builder) from HYDSET2-shaped host arrays: vectors [docNum][dim]
 * float32 and tag bitmaps [docNum][ceil(tagNum/64)] uint64; tag t is indexed as the token
 * Hash64(decimal string of t). The result is resident on deviceId. */
int hss_table_build(int32_t deviceId, const float* vectors, const uint64_t* tagBits, uint64_t docNum, uint32_t dim,
                    uint32_t tagNum, const hss_index_config* cfg, hss_table** out);
/* The same build from vectors already resident on deviceId: dVectors is device memory of that
 * device ([docNum][dim] float32, copied into the table's own allocation, so the caller may free it
 * afterwards); tagBits stays a host array. For corpora too large to stage through host memory (the
 * reference's builder writes its .vector files from host records, vector_builder.cpp:34-176). */
int hss_table_build_device(int32_t deviceId, const float* dVectors, const uint64_t* tagBits, uint64_t docNum,
                           uint32_t dim, uint32_t tagNum, const hss_index_config* cfg, hss_table** out);
/* DataTable::LoadData(deviceId, dir) (data_table.cpp:35-124) over a directory hss_table_save wrote. */
int hss_table_load(int32_t deviceId, const char* dir, hss_table** out);
int hss_table_save(const hss_table* table, const char* dir);
/* DataTable::LoadData over the REFERENCE's own index directory, as its fr_builder writes it
 * (data_table.cpp:35-124,147-186): poissonengine_<ver>.meta (IndexMeta, protobuf JSON form),
 * id/poissonengine_<ver>_<seg>.idm (64-bit global ids; string ids are rejected),
 * <vectorField>/poissonengine_<ver>_<seg>_<vectorField>.vector (FP16 in blocks of splitDocNumZn docs,
 * vector_builder.cpp:34-176; loaded as the exact FP32 values) and the posting files of the first
 * posting field. docNumPerSegment must be a multiple of 128 here. */
int hss_table_load_reference(int32_t deviceId, const char* dir, hss_table** out);
/* Writes a table in that layout (meta, id mapping, FP16 vectors rounded as the reference's
 * Float32ToFloat16 rounds, trans_number.cpp:38-83, and the posting files); splitDocNumZn docs per
 * vector block (the reference's loader needs dim * splitDocNumZn <= 16384). */
int hss_table_save_reference(const hss_table* table, const char* dir, uint32_t splitDocNumZn);
/* Where the table's load spent its time, ms: meta, posting files read, vector rows read / decoded
 * (host, on `threads` threads), vectors to the device (reading and pinned, double-buffered copies
 * overlapped; the whole phase), postings to the device, total; bytes of vectors and posting files.
 * Zero for a built table. Replaces the reference's [Load] line (data_table.cpp:105-112). */
int hss_table_load_times(const hss_table* table, double* ms6, uint64_t* vectorBytes, uint64_t* postingBytes,
                         uint32_t* threads);
void hss_table_free(hss_table* table);
int hss_table_info(const hss_table* table, uint64_t* docNum, uint32_t* dim, uint32_t* segmentNum,
                   uint32_t* docNumPerSegment, uint32_t* postingRows, float* maxNorm);
/* Host copy of a token's posting in one segment (len 0 and *data NULL when absent). */
int hss_table_posting(const hss_table* table, uint64_t token, uint32_t segment, const uint8_t** data, uint32_t* len);
/* Device arrays: vectors [ceil(docNum/128)*128][dim], posting table [postingRows][segmentNum] of
 * posting head addresses (last row: the all-zero posting), global doc ids [docNum]. */
int hss_table_device_ptrs(const hss_table* table, const float** vectors, const uint64_t** postingTable,
                          const int64_t** gdocids);

/* ---- searcher (FullRecallSearcher, full_recall_searcher.h:12-47) ---- */
typedef struct hss_searcher hss_searcher;
typedef struct hss_filters hss_filters; /* compiled filter programs of one batch */

typedef struct hss_searcher_config {
    uint32_t maxBatch;     /* queries per batch (default 256; at most 256 for the tensor-core methods,
                              4096 for SIMT: larger values are clamped) */
    uint32_t candidateCap; /* per-query candidate capacity (default 262144, >= HSS_MAX_TOPK) */
    uint32_t sampleDocs;   /* minimum doc sample for the candidate threshold (default 32768) */
    uint32_t maxRetries;   /* re-runs of a query whose candidates overflowed (default 4) */
    int32_t method;        /* candidate pass: 0 FP32 SIMT, 1 tensor cores TF32 over the FP32 rows,
                              2 tensor cores over a BF16 copy, 3 tensor cores over an FP8 E4M3 copy
                              with per-vector scales (every method returns the exact FP32 results).
                              The tensor-core methods need dim a multiple of 32 (TF32), 64 (BF16)
                              or 128 (E4M3), else hss_searcher_create fails; any dim up to 4096
                              otherwise (long vectors stream through the pass) */
    int32_t decodeInPlace; /* 0: filter over a dense bitmap of every posting, decoded once when the
                              searcher is created if it takes at most 40% of free device memory;
                              1: always decode the postings in place (no extra memory) */
} hss_searcher_config;

/* cfg may be NULL for the defaults. The searcher allocates its whole device arena here. */
int hss_searcher_create(hss_table* table, const hss_searcher_config* cfg, hss_searcher** out);

/* Caller-owned workspace (the reference's ownership model: the host owns every device block, the
 * library is given sizes; GmMemoryPool / GmMemoryManager, gm_memory_pool.h:40-181,
 * gm_memory_manager.cpp:9-47, named pools of full_recall_result.h:9-20).
 * hss_searcher_workspace_bytes: device bytes of one searcher's arena for this table and config --
 * filter bitmaps, candidate lists, select workspace, doc sample, per-batch staging, results and
 * model features; 0 for bad arguments. It grows with maxBatch x candidateCap.
 * hss_table_prepare: builds the table's resident data a searcher of this config reads (the dense
 * posting matrix unless decodeInPlace; the BF16 / E4M3 copy of the rows for methods 2 / 3), which
 * belongs to the table and is shared by all its searchers; call it at load time so that searcher
 * creation allocates no device memory.
 * hss_searcher_create_in: hss_searcher_create on a caller-owned device arena of at least
 * hss_searcher_workspace_bytes bytes, 256-byte aligned, on the table's device. The searcher keeps
 * every device buffer there, never frees it, and allocates only its pinned host staging (and, if
 * hss_table_prepare was not called, the table's resident data). The arena must outlive the searcher
 * and may not be shared with another searcher that runs at the same time. */
size_t hss_searcher_workspace_bytes(const hss_table* table, const hss_searcher_config* cfg);
int hss_table_prepare(hss_table* table, const hss_searcher_config* cfg);
int hss_searcher_create_in(hss_table* table, const hss_searcher_config* cfg, void* dWorkspace, size_t workspaceBytes,
                           hss_searcher** out);
void hss_searcher_free(hss_searcher* s);

/* FullRecallSearcher::AddQuery (full_recall_searcher.cpp:93-105): the filter is given as text in the
 * reference grammar (filter_expr.h: tag ids, AND / OR / NOT, parentheses; empty = match all). */
int hss_searcher_add_query(hss_searcher* s, const char* filterExpr, const float* vector, uint32_t dim,
                           uint32_t topK);
/* FullRecallSearcher::BatchSearch (full_recall_searcher.cpp:107-231) over the added queries, results
 * copied to host arrays of outStride entries per query: scores (descending) and global doc ids, ties
 * broken by ascending doc id. Clears the added queries. HSS_ERR_QUERY when some queries failed. */
int hss_searcher_batch_search(hss_searcher* s, float* outScores, int64_t* outIds, uint32_t* outCounts,
                              uint32_t outStride);

/* Compile a batch's filter texts once (TextFilter::PrepareExpr, text_filter.cpp:432-467). */
int hss_filters_compile(hss_searcher* s, const char* const* filterExprs, uint32_t n, hss_filters** out);
void hss_filters_free(hss_filters* f);
/* Device-resident batch: dQueries [nq][dim] and the outputs are device arrays; filters[i] is the
 * filter of query i. Synchronises `stream` once per batch (candidate-overflow check). */
int hss_searcher_search_device(hss_searcher* s, const float* dQueries, uint32_t nq, const hss_filters* filters,
                               const uint32_t* topks, float* dOutScores, int64_t* dOutIds, uint32_t* dOutCounts,
                               uint32_t outStride, hss_stream_t stream);

/* hss_searcher_search_device in two halves, so that the caller keeps the GPU busy while it waits.
 * The first enqueues the whole batch on `stream` (the filter programs are compiled into the
 * searcher's staging on the calling thread) and returns without waiting; the filters may be freed
 * after it returns, the queries and outputs must stay valid until the second returns. The second
 * waits for the batch's statuses, runs any candidate-overflow re-runs on the same stream and returns
 * what hss_searcher_search_device returns. A searcher takes no other batch in between: two
 * searchers of one table alternate (batch i on one while the host finishes batch i - 1 of the
 * other), so the GPU never idles between batches while the host waits. */
int hss_searcher_search_device_async(hss_searcher* s, const float* dQueries, uint32_t nq, const hss_filters* filters,
                                     const uint32_t* topks, float* dOutScores, int64_t* dOutIds, uint32_t* dOutCounts,
                                     uint32_t outStride, hss_stream_t stream);
int hss_searcher_finish(hss_searcher* s);

/* The filter stage alone (FullRecallSearcher::OneFilter, full_recall_searcher.cpp:233-262): row q of
 * dOutBits (outStrideWords u64 per row, >= segmentNum * docNumPerSegment / 64) gets query q's doc
 * bitmap (bit b of word w = doc 64w+b, docs past docNum cleared) and dPassCounts[q] (may be NULL) its
 * popcount. Synchronises `stream` once. */
int hss_searcher_filter_device(hss_searcher* s, const hss_filters* filters, uint32_t nq, uint64_t* dOutBits,
                               uint64_t outStrideWords, uint32_t* dPassCounts, hss_stream_t stream);

/* Per-query HSS_QSTATUS_* bits of the last batch. */
int hss_searcher_last_status(const hss_searcher* s, int32_t* status, uint32_t n);
/* Inspection of the last batch's approximate pass for one query (its batch row): up to `cap` of its
 * candidates (approximate scores, locations), the candidate count, the threshold theta the pass used
 * and the query's error bound eps (|approximate - exact FP32 score| <= eps for every doc). */
int hss_searcher_last_candidates(hss_searcher* s, uint32_t query, float* scores, uint32_t* locations, uint32_t cap,
                                 uint32_t* count, float* theta, float* eps);
/* Stage times of the last batch in ms (filter, sample, candidates, select, total; needs
 * hss_searcher_set_timing(s, 1)), candidate re-runs and kernel launches. */
int hss_searcher_set_timing(hss_searcher* s, int32_t on);
/* Test of the tensor-core pass's bounded waits (no counterpart in the reference, whose kernels
 * have no error channel). The next batch's first single-SM tensor-core candidate pass (<= 128
 * queries) stops issuing corpus loads before its holdLoad-th, so its MMA issuer's wait for that load
 * runs out after waitBudgetCycles clock cycles (0: the default, about 2 s). The pass records an
 * error bit, drains its copies and MMAs, frees its tensor memory and returns; the batch returns
 * HSS_ERR_CUDA ("timed out waiting on its pipeline"), and the searcher stays usable. */
int hss_searcher_set_pipeline_test(hss_searcher* s, uint32_t holdLoad, uint64_t waitBudgetCycles);
int hss_searcher_last_times(const hss_searcher* s, float* ms5, uint32_t* retries, uint32_t* launches);
/* CUDA-graph replay of each batch's first attempt (no counterpart in the reference, whose ACL
 * launches are issued per call). A batch shape -- rows rounded up to 1, 2, 4, 8, 16 or a multiple of
 * 16 (at most maxBatch), the largest K rounded up to a power of two (the K that plan alike as one),
 * the filters' largest operand count rounded up to a power of two, the threshold model, the query
 * and output pointers and outStride -- is captured
 * from the stream at its first batch and replayed for every later one, the graph copying in each
 * batch's filter programs; re-runs are launched directly. The rows past nq run as match-nothing
 * queries with K = 1: with graphs on, dQueries and the outputs of hss_searcher_search_device must
 * hold maxBatch rows, and the stream must not be the legacy default stream (it cannot be captured).
 * Results are the same as without. Off by default. */
int hss_searcher_set_graphs(hss_searcher* s, int32_t on);
/* Shapes captured and batches replayed so far, the host milliseconds spent capturing and
 * instantiating; *failed = 1 when a capture failed (graphs are then off for this searcher and its
 * batches launch directly). Any pointer may be NULL. */
int hss_searcher_graph_stats(const hss_searcher* s, uint64_t* captures, uint64_t* replays, double* captureMs,
                             int32_t* failed);

/* ---- learned threshold predictor ----
 * An MLP (feature row -> hidden -> hidden -> 1, GELU) that predicts a query's K-th filtered score,
 * trained and run on the GPU by this library's own kernels. With a model set, a searcher's candidate
 * passes prune at max(doc sample's proven threshold, prediction - margin - error bound) inside the
 * scoring epilogue, and its doc sample stays at sample_docs for every K. The select step checks each
 * query whose threshold came from the prediction: its K-th best exact score must clear that
 * threshold by the error bound, else the query is re-run at a proven threshold. A bad prediction
 * costs candidates or a re-run, never exactness. No counterpart in the reference (whose only
 * threshold is its TOPK pivot pre-select). */
typedef struct hss_model hss_model;

/* dim + posting rows + 12: the feature row width a model for this searcher must take. */
uint32_t hss_searcher_feature_dim(const hss_searcher* s);
/* Feature rows dX [nq][feature_dim] of a batch (device queries and output): query * sqrt(dim); per
 * posting row of the query's filter 1 + log10(row density) / 4 (0 elsewhere); log10(filter
 * selectivity) / 4; log10(K) / 3; 1; the doc sample's best scores at ranks 1, 2, 4, ..., 64 (-2
 * past the sample's size); its K-th best score (-2 when absent); log10(filtered sample docs + 1) / 5.
 * Runs the filter stage and the doc sample; synchronises `stream`. */
int hss_searcher_features(hss_searcher* s, const float* dQueries, uint32_t nq, const hss_filters* filters,
                          const uint32_t* topks, float* dX, hss_stream_t stream);
/* model NULL switches the learned threshold off. margin (score units) is subtracted from the
 * prediction. */
int hss_searcher_set_threshold_model(hss_searcher* s, hss_model* model, float margin);
/* Per query of the last batch: the doc sample's proven threshold and the threshold the model set
 * (-inf without a model); host arrays of n floats, either may be NULL. */
int hss_searcher_last_thresholds(const hss_searcher* s, float* sampleTheta, float* modelTheta, uint32_t n);

/* Per query of the last batch: the docs that cleared the threshold of its last candidate pass (the
 * list the select step read, counting any beyond the list's capacity). Call before the next batch. */
int hss_searcher_last_candidate_counts(hss_searcher* s, uint32_t* counts, uint32_t n);

/* Per query of the last batch: 1 when the model's threshold was too high for it (its K-th best exact
 * score did not clear the threshold by the error bound) and the query was re-run at a proven
 * threshold, else 0. Its results are exact either way. */
int hss_searcher_last_threshold_misses(const hss_searcher* s, uint8_t* miss, uint32_t n);

int hss_model_create(int32_t deviceId, uint32_t din, uint32_t hidden, uint64_t seed, hss_model** out);
void hss_model_free(hss_model* m);
/* din*hidden + hidden + hidden*hidden + hidden + hidden + 1: W1, b1, W2, b2, w3, b3 in this order. */
uint64_t hss_model_param_count(const hss_model* m);
int hss_model_get_params(const hss_model* m, float* params);
int hss_model_set_params(hss_model* m, const float* params);
/* The model predicts standardised scores: score = output * scale + shift. */
int hss_model_set_output_scale(hss_model* m, float scale, float shift);
/* Outputs dY [B] (standardised) of device features dX [B][din], in one launch (hidden <= 1024). */
int hss_model_forward(hss_model* m, const float* dX, uint32_t B, float* dY, hss_stream_t stream);
/* The training loss: tau = 0 (the default) the mean squared error, mean((y - t)^2); tau in (0, 1) the
 * pinball loss of the tau-quantile, mean(tau (t - y) where t >= y, (1 - tau) (y - t) elsewhere), so
 * the network predicts a conditional tau-quantile of the target. */
int hss_model_set_quantile(hss_model* m, float tau);
/* One Adam step (b1 0.9, b2 0.999, eps 1e-8) on the loss over device dX [B][din] and dT [B]
 * (standardised targets); *loss (may be NULL) = the batch loss before the step. Synchronises. */
int hss_model_train_step(hss_model* m, const float* dX, const float* dT, uint32_t B, float lr, float* loss,
                         hss_stream_t stream);
/* The gradient of the loss at the current parameters into a host array of param_count floats
 * (parameter order); *loss (may be NULL) = the loss. Synchronises `stream`. */
int hss_model_gradients(hss_model* m, const float* dX, const float* dT, uint32_t B, float* grad, float* loss,
                        hss_stream_t stream);

/* ---- serving loop ----
 * Continuous batching of single queries over one resident table: clients submit (vector, filter text,
 * K) at any time; `slots` workers, each with its own searcher arena and CUDA stream, take every
 * queued request (up to maxBatch, waiting at most maxWaitUs for more) as one batch, so batches of
 * different slots overlap on the GPU and requests arriving meanwhile join the next free slot's batch.
 * Slots are admitted by device memory (memoryBudget bytes of arenas). Replaces the reference's
 * RunContext / schedule_* drivers (run_context.cpp:121-274), which run pre-formed batches. */
typedef struct hss_server hss_server;
typedef struct hss_server_config {
    uint32_t slots;        /* concurrent batches on the GPU (default 2) */
    uint32_t maxBatch;     /* queries per batch (default 256) */
    uint32_t maxWaitUs;    /* longest wait for a fuller batch (default 200) */
    int32_t method;        /* as hss_searcher_config.method */
    uint64_t memoryBudget; /* bytes for the slots' arenas; 0 = half the free device memory */
    uint32_t candidateCap; /* as in hss_searcher_config; 0 = default */
    uint32_t sampleDocs;
    uint32_t graphs;       /* 1: the slots replay captured CUDA graphs per batch shape
                              (hss_searcher_set_graphs); default 0: every batch launched directly */
} hss_server_config;
typedef struct hss_server_stats {
    uint64_t completed, batches;
    uint32_t slots;
    double meanBatch, p50Ms, p99Ms, maxMs; /* latency from submission to results on the host */
    uint64_t graphCaptures, graphReplays;  /* over all slots */
    double graphCaptureMs;                 /* host time the slots spent capturing and instantiating */
} hss_server_stats;

int hss_server_create(hss_table* table, const hss_server_config* cfg, hss_server** out);
void hss_server_free(hss_server* s);
/* Compiles the filter on the calling thread and queues the query; *id identifies it. */
int hss_server_submit(hss_server* s, const float* vector, uint32_t dim, const char* filterExpr, uint32_t topK,
                      uint64_t* id);
/* Blocks up to timeoutMs (< 0: no limit) for query id; copies up to cap results (scores descending,
 * global doc ids), *count = its result count, *latencyMs, *status (HSS_QSTATUS_* bits, -2 when its
 * batch failed on the device). HSS_OK, 1 on timeout (the query stays pending), HSS_ERR_INVALID for an
 * unknown id. Each id is returned once. */
int hss_server_wait(hss_server* s, uint64_t id, float* scores, int64_t* ids, uint32_t cap, uint32_t* count,
                    double* latencyMs, int32_t* status, int32_t timeoutMs);
int hss_server_get_stats(const hss_server* s, hss_server_stats* out);
int hss_server_reset_stats(hss_server* s);
int hss_server_set_threshold_model(hss_server* s, hss_model* model, float margin);
/* Open-loop load test: query i (queries [n][dim], filterExprs[i], topks[i]) arrives at Poisson times
 * of rate rateQps; per-request latencies into latencyMs[n]. Returns HSS_OK, or HSS_ERR_QUERY when
 * some queries failed; *offeredQps = the arrival rate achieved, *wallSeconds = the whole run. */
int hss_server_run_poisson(hss_server* s, const float* queries, uint32_t n, const char* const* filterExprs,
                           const uint32_t* topks, double rateQps, uint64_t seed, double* latencyMs,
                           double* offeredQps, double* wallSeconds);

/* ---- host-side codec (the index format contract) ---- */
/* Hash64 (src/engine/core/hash/hash.cpp:10-16). */
uint64_t hss_hash64(const char* data, uint32_t len);
/* PostingSerializer::Serialize (src/engine/format/posting_serializer.cpp:81-101) of sorted local ids;
 * returns the byte length or a negative status. */
int64_t hss_posting_serialize(const uint32_t* ids, uint32_t n, uint32_t docNum, int32_t isMatrix,
                              float densityThreshold, int32_t sparsePacked, uint8_t* out, uint64_t cap);
/* The postfix program and operand rows of one filter text over a table (QueryNode lowering,
 * query_node_imp.cpp). *emptyTree = 1 for match-all. */
int hss_filter_compile(const hss_table* table, const char* filterExpr, uint32_t* prog, uint32_t progCap,
                       uint32_t* progLen, uint32_t* rows, uint32_t rowCap, uint32_t* rowLen, uint32_t* opNum,
                       int32_t* emptyTree);

/* Last error message of this thread ("" when none). */
const char* hss_last_error(void);
/* Number of visible CUDA devices (0 without a GPU). */
int hss_device_count(void);

#ifdef __cplusplus
}
#endif
#endif
