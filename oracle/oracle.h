/*
 * oracle.h -- CPU restatement of the reference's filtered full-recall path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker the parity tests, the smoke test and the
 * CPU-baseline leg of the benchmark compare the CUDA path against. Nothing in the product
 * (hybridsearchsystem_b200/, libhss.so) links, loads or calls it.
 *
 * Every function cites the reference file:line it restates (paths are relative to the reference
 * project root). The restatement is pinned by the golden fixtures under tests/golden/, which were
 * generated by the reference's own sources compiled by oracle/Makefile into oracle/_ref/.
 *
 * Build: `make -C oracle` -> oracle/liboracle.so (gcc -O2 -ffp-contract=off, so every score is a
 * sequential IEEE mul then add over d ascending, exactly like the reference's CpuTopK).
 */
#ifndef HSS_ORACLE_H
#define HSS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- filter AST (restates src/harness/query/filter_expr.h:19-177) ---- */
enum { ORC_TERM = 0, ORC_AND = 1, ORC_OR = 2, ORC_NOT = 3 };

typedef struct {
    int32_t op;     /* ORC_TERM / ORC_AND / ORC_OR / ORC_NOT */
    int32_t nkids;  /* number of children */
    int32_t kid0;   /* first child's slot in the kids[] array */
    int32_t pad;
    uint64_t tag;   /* valid when op == ORC_TERM */
} orc_node;

/* Parses `expr` with the reference grammar (NOT > AND > OR, n-ary AND/OR flattening).
 * Returns the node count (> 0) and sets *root; 0 for an empty/blank expression (match-all,
 * *root = -1); -1 on a parse error; -2 when a capacity is exceeded. */
int orc_parse(const char* expr, orc_node* nodes, int cap_nodes, int32_t* kids, int cap_kids, int* root);

/* EvalFilterBitmap (filter_expr.h:212-232): root < 0 means match-all. */
int orc_eval_bitmap(const orc_node* nodes, const int32_t* kids, int root, const uint64_t* bm, uint32_t words);

/* Per-doc evaluation over `doc_num` docs starting at `doc_offset`; packs the result one bit per doc
 * (bit i%64 of word i/64, i relative to doc_offset). out has ceil(doc_num/64) words. */
void orc_filter_bits(const orc_node* nodes, const int32_t* kids, int root, const uint64_t* bitmaps,
                     uint32_t stride, uint64_t doc_num, uint64_t doc_offset, uint64_t* out);

/* ---- ground truth top-K (restates 10.13/load/src/harness/recall/recall_ref.cpp:33-62,90-142) ----
 * Exact FP32 inner product, sequential over d, ties broken by (score desc, doc id asc) (the Better
 * comparator, recall_ref.cpp:19-25). Unlike the reference (which returns an unordered set) the
 * result is the ordered list, so the device output can be checked bit for bit and in order.
 * Returns the number of results (min(topk, filter hits)). */
int orc_topk(const float* query, uint32_t dim, const orc_node* nodes, const int32_t* kids, int root,
             const float* vectors, const uint64_t* bitmaps, uint32_t stride, uint64_t doc_num,
             uint64_t doc_offset, int32_t topk, float* out_scores, int64_t* out_ids);

/* The batched form: nq queries, each with its own filter (roots[q]; nodes/kids shared), its own
 * top-K (topks[q]) and output row q of stride out_stride. Queries are split over `threads` POSIX
 * threads; each thread makes one corpus pass for its slice (the CpuTopKBatch pattern). */
void orc_topk_batch(const float* queries, uint32_t nq, uint32_t dim, const orc_node* nodes,
                    const int32_t* kids, const int32_t* roots, const float* vectors,
                    const uint64_t* bitmaps, uint32_t stride, uint64_t doc_num, uint64_t doc_offset,
                    const int32_t* topks, int32_t out_stride, float* out_scores, int64_t* out_ids,
                    int32_t* out_counts, int threads);

/* FP64 inner products of one query against `n` listed docs (for the score-error report). */
void orc_score_f64(const float* query, uint32_t dim, const float* vectors, const int64_t* ids, int n,
                   double* out);

/* ---- posting codec (restates src/engine/format/posting_serializer.cpp:15-208) ----
 * Serialises one posting of a segment holding seg_docs docs. ids need not be sorted; duplicates are
 * ignored. packed != 0 selects SPARSE_PACKED for the sparse bitmap case (NPUR_SPARSE_PACKED).
 * SPARSE_IDLIST ids are written in ascending order. Returns the byte length (before the builder's
 * 4-byte padding) or -1 on error / insufficient capacity. */
int64_t orc_posting_serialize(const uint32_t* ids, uint32_t n, uint32_t seg_docs, int is_matrix,
                              float density_threshold, int packed, uint8_t* out, uint64_t cap);

/* Decodes any of the five layouts into a dense bitset of ceil(seg_docs/64) words. Returns the layout
 * code, or -1 when the posting is malformed. */
int orc_posting_decode(const uint8_t* posting, uint64_t len, uint32_t seg_docs, uint64_t* out_words);

/* Evaluates a postfix filter program (the [op, postingNum, stackNum] / [CONJ, parts, n_i...] form that
 * query_node_imp.cpp:8-47,65-96,295-342 emits and kernel_bitmap_text_filter.cpp:52-119 interprets)
 * over dense operand bitsets operands[i] (each `words` u64). Returns 0 and writes `out`, or -1 when
 * the program is malformed (CheckPostExpr rules, text_filter.cpp:1314-1352). */
int orc_eval_postfix(const uint32_t* prog, uint32_t prog_len, uint32_t op_count,
                     const uint64_t* const* operands, uint32_t n_operands, uint32_t words, uint64_t* out);

/* ---- token hash (restates src/engine/core/hash/hash.cpp:10-16 over MurmurHash3_x64_128) ---- */
uint64_t orc_hash64(const char* data, uint32_t len);

#ifdef __cplusplus
}
#endif
#endif
