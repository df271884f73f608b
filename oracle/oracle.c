/*
 * oracle.c -- CPU restatement of the reference's filtered full-recall path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path (see oracle.h). Compiled with
 * -O2 -ffp-contract=off so the inner product is a sequential IEEE multiply then add, d ascending,
 * which is how the reference's CpuTopK computes it on x86-64 (no FMA contraction).
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------------------
 * Filter grammar. Restates the tokenizer and recursive descent of src/harness/query/filter_expr.h:
 *   skipWs/peek/consume (filter_expr.h:28-69), ParseAtom (:73-97), ParseNot (:99-113),
 *   ParseAnd (:115-137), ParseOr (:139-161), ParseFilter (:164-177).
 * Keywords are the exact upper-case letter runs "AND"/"OR"/"NOT"; a number is a digit run whose
 * value wraps modulo 2^64 exactly as `v = v * 10 + digit` does in the reference.
 * ----------------------------------------------------------------------------------------------*/
typedef struct {
    const char* s;
    size_t n, i;
    orc_node* nodes;
    int cap_nodes, nn;
    int32_t* kids;
    int cap_kids, nk;
    int ok;      /* 0 once a parse error was seen */
    int overflow;
} parser;

enum { TK_EOF, TK_LP, TK_RP, TK_NUM, TK_WORD };

static void skip_ws(parser* p) {
    while (p->i < p->n && (p->s[p->i] == ' ' || p->s[p->i] == '\t' || p->s[p->i] == '\r' || p->s[p->i] == '\n'))
        p->i++;
}

/* Returns the token kind at the cursor without consuming it. For TK_WORD, *wlen is the letter-run
 * length (0 for a character that is neither a letter, a digit nor a parenthesis). */
static int peek(parser* p, uint64_t* num, size_t* wlen) {
    skip_ws(p);
    if (p->i >= p->n) return TK_EOF;
    char c = p->s[p->i];
    if (c == '(') return TK_LP;
    if (c == ')') return TK_RP;
    if (c >= '0' && c <= '9') {
        size_t j = p->i;
        uint64_t v = 0;
        while (j < p->n && p->s[j] >= '0' && p->s[j] <= '9') {
            v = v * 10u + (uint64_t)(p->s[j] - '0');
            j++;
        }
        *num = v;
        return TK_NUM;
    }
    size_t j = p->i;
    while (j < p->n && ((p->s[j] >= 'A' && p->s[j] <= 'Z') || (p->s[j] >= 'a' && p->s[j] <= 'z'))) j++;
    *wlen = j - p->i;
    return TK_WORD;
}

static int peek_is(parser* p, const char* kw) {
    uint64_t num = 0;
    size_t wlen = 0;
    int t = peek(p, &num, &wlen);
    size_t kl = strlen(kw);
    return t == TK_WORD && wlen == kl && memcmp(p->s + p->i, kw, kl) == 0;
}

static int new_node(parser* p, int op, uint64_t tag) {
    if (p->nn >= p->cap_nodes) {
        p->overflow = 1;
        p->ok = 0;
        return -1;
    }
    orc_node* nd = &p->nodes[p->nn];
    nd->op = op;
    nd->nkids = 0;
    nd->kid0 = 0;
    nd->pad = 0;
    nd->tag = tag;
    return p->nn++;
}

/* Child lists are collected on the C stack then copied into kids[] contiguously. */
#define ORC_MAX_ARITY 4096

static int parse_or(parser* p);

static int parse_atom(parser* p) {
    uint64_t num = 0;
    size_t wlen = 0;
    int t = peek(p, &num, &wlen);
    if (t == TK_LP) {
        p->i++;
        int node = parse_or(p);
        if (!p->ok) return -1;
        t = peek(p, &num, &wlen);
        if (t != TK_RP) {
            p->ok = 0;
            return -1;
        }
        p->i++;
        return node;
    }
    if (t == TK_NUM) {
        while (p->i < p->n && p->s[p->i] >= '0' && p->s[p->i] <= '9') p->i++;
        return new_node(p, ORC_TERM, num);
    }
    p->ok = 0;
    return -1;
}

static int parse_not(parser* p) {
    if (peek_is(p, "NOT")) {
        p->i += 3;
        int child = parse_not(p);
        if (!p->ok) return -1;
        int node = new_node(p, ORC_NOT, 0);
        if (node < 0) return -1;
        if (p->nk + 1 > p->cap_kids) {
            p->overflow = 1;
            p->ok = 0;
            return -1;
        }
        p->nodes[node].kid0 = p->nk;
        p->nodes[node].nkids = 1;
        p->kids[p->nk++] = child;
        return node;
    }
    return parse_atom(p);
}

static int finish_nary(parser* p, int op, const int32_t* parts, int nparts) {
    if (nparts == 1) return parts[0];
    int node = new_node(p, op, 0);
    if (node < 0) return -1;
    if (p->nk + nparts > p->cap_kids) {
        p->overflow = 1;
        p->ok = 0;
        return -1;
    }
    p->nodes[node].kid0 = p->nk;
    p->nodes[node].nkids = nparts;
    memcpy(p->kids + p->nk, parts, sizeof(int32_t) * (size_t)nparts);
    p->nk += nparts;
    return node;
}

static int parse_and(parser* p) {
    int32_t* parts = (int32_t*)malloc(sizeof(int32_t) * ORC_MAX_ARITY);
    int np = 0;
    int first = parse_not(p);
    if (!p->ok) {
        free(parts);
        return -1;
    }
    parts[np++] = first;
    while (peek_is(p, "AND")) {
        p->i += 3;
        int next = parse_not(p);
        if (!p->ok) {
            free(parts);
            return -1;
        }
        if (np >= ORC_MAX_ARITY) {
            p->overflow = 1;
            p->ok = 0;
            free(parts);
            return -1;
        }
        parts[np++] = next;
    }
    int r = finish_nary(p, ORC_AND, parts, np);
    free(parts);
    return r;
}

static int parse_or(parser* p) {
    int32_t* parts = (int32_t*)malloc(sizeof(int32_t) * ORC_MAX_ARITY);
    int np = 0;
    int first = parse_and(p);
    if (!p->ok) {
        free(parts);
        return -1;
    }
    parts[np++] = first;
    while (peek_is(p, "OR")) {
        p->i += 2;
        int next = parse_and(p);
        if (!p->ok) {
            free(parts);
            return -1;
        }
        if (np >= ORC_MAX_ARITY) {
            p->overflow = 1;
            p->ok = 0;
            free(parts);
            return -1;
        }
        parts[np++] = next;
    }
    int r = finish_nary(p, ORC_OR, parts, np);
    free(parts);
    return r;
}

int orc_parse(const char* expr, orc_node* nodes, int cap_nodes, int32_t* kids, int cap_kids, int* root) {
    parser p;
    memset(&p, 0, sizeof(p));
    p.s = expr;
    p.n = strlen(expr);
    p.nodes = nodes;
    p.cap_nodes = cap_nodes;
    p.kids = kids;
    p.cap_kids = cap_kids;
    p.ok = 1;
    *root = -1;
    skip_ws(&p);
    if (p.i >= p.n) return 0; /* empty -> match all (ParseFilter, filter_expr.h:167-168) */
    int r = parse_or(&p);
    if (!p.ok) return p.overflow ? -2 : -1;
    skip_ws(&p);
    if (p.i < p.n) return -1; /* trailing garbage (filter_expr.h:172-175) */
    *root = r;
    return p.nn;
}

/* ------------------------------------------------------------------------------------------------
 * Bitmap evaluation: EvalFilterBitmap and BitSet (filter_expr.h:204-232).
 * ----------------------------------------------------------------------------------------------*/
static int bit_set(const uint64_t* bm, uint32_t words, uint64_t tag) {
    uint32_t w = (uint32_t)(tag >> 6);
    if (w >= words) return 0;
    return (int)((bm[w] >> (tag & 63u)) & 1u);
}

static int eval_node(const orc_node* nodes, const int32_t* kids, int n, const uint64_t* bm, uint32_t words) {
    const orc_node* nd = &nodes[n];
    switch (nd->op) {
        case ORC_TERM:
            return bit_set(bm, words, nd->tag);
        case ORC_AND:
            for (int i = 0; i < nd->nkids; i++)
                if (!eval_node(nodes, kids, kids[nd->kid0 + i], bm, words)) return 0;
            return 1;
        case ORC_OR:
            for (int i = 0; i < nd->nkids; i++)
                if (eval_node(nodes, kids, kids[nd->kid0 + i], bm, words)) return 1;
            return 0;
        case ORC_NOT:
            return !eval_node(nodes, kids, kids[nd->kid0], bm, words);
    }
    return 1;
}

int orc_eval_bitmap(const orc_node* nodes, const int32_t* kids, int root, const uint64_t* bm, uint32_t words) {
    if (root < 0) return 1;
    return eval_node(nodes, kids, root, bm, words);
}

void orc_filter_bits(const orc_node* nodes, const int32_t* kids, int root, const uint64_t* bitmaps,
                     uint32_t stride, uint64_t doc_num, uint64_t doc_offset, uint64_t* out) {
    uint64_t nw = (doc_num + 63) / 64;
    memset(out, 0, sizeof(uint64_t) * nw);
    for (uint64_t i = 0; i < doc_num; i++) {
        const uint64_t* bm = bitmaps + (doc_offset + i) * stride;
        if (orc_eval_bitmap(nodes, kids, root, bm, stride)) out[i >> 6] |= 1ull << (i & 63);
    }
}

/* ------------------------------------------------------------------------------------------------
 * Ground-truth top-K. CpuTopK (recall_ref.cpp:33-62) in fp32 mode: q16[d] = query[d]; for every doc
 * passing the filter, s = 0; s += q[d] * v[d] for d ascending; keep the best by Better
 * (recall_ref.cpp:19-25): score descending, then doc id ascending. The reference returns the set;
 * this returns it sorted by the same comparator.
 * ----------------------------------------------------------------------------------------------*/
typedef struct {
    float s;
    int64_t id;
} scored;

/* a is better than b (Better, recall_ref.cpp:19-25) */
static int better(const scored* a, const scored* b) {
    if (a->s != b->s) return a->s > b->s;
    return a->id < b->id;
}

/* min-heap on Better: the root is the worst kept element */
static void heap_sift_down(scored* h, int n, int i) {
    for (;;) {
        int l = 2 * i + 1, r = l + 1, w = i;
        if (l < n && better(&h[w], &h[l])) w = l;
        if (r < n && better(&h[w], &h[r])) w = r;
        if (w == i) return;
        scored t = h[i];
        h[i] = h[w];
        h[w] = t;
        i = w;
    }
}

static void heap_sift_up(scored* h, int i) {
    while (i > 0) {
        int parent = (i - 1) / 2;
        if (better(&h[parent], &h[i])) {
            scored t = h[i];
            h[i] = h[parent];
            h[parent] = t;
            i = parent;
        } else {
            return;
        }
    }
}

static int cmp_better(const void* a, const void* b) {
    const scored* x = (const scored*)a;
    const scored* y = (const scored*)b;
    if (better(x, y)) return -1;
    if (better(y, x)) return 1;
    return 0;
}

static float dot_seq(const float* q, const float* v, uint32_t dim) {
    float s = 0.0f;
    for (uint32_t d = 0; d < dim; ++d) s += q[d] * v[d];
    return s;
}

typedef struct {
    scored* heap;
    int n, cap;
} topk_state;

static void topk_push(topk_state* st, float s, int64_t id) {
    scored c = {s, id};
    if (st->cap <= 0) return;
    if (st->n < st->cap) {
        st->heap[st->n] = c;
        heap_sift_up(st->heap, st->n);
        st->n++;
    } else if (better(&c, &st->heap[0])) {
        st->heap[0] = c;
        heap_sift_down(st->heap, st->n, 0);
    }
}

static int topk_finish(topk_state* st, float* out_scores, int64_t* out_ids) {
    qsort(st->heap, (size_t)st->n, sizeof(scored), cmp_better);
    for (int i = 0; i < st->n; i++) {
        out_scores[i] = st->heap[i].s;
        out_ids[i] = st->heap[i].id;
    }
    return st->n;
}

int orc_topk(const float* query, uint32_t dim, const orc_node* nodes, const int32_t* kids, int root,
             const float* vectors, const uint64_t* bitmaps, uint32_t stride, uint64_t doc_num,
             uint64_t doc_offset, int32_t topk, float* out_scores, int64_t* out_ids) {
    topk_state st;
    st.cap = topk > 0 ? topk : 0;
    st.n = 0;
    st.heap = (scored*)malloc(sizeof(scored) * (size_t)(st.cap > 0 ? st.cap : 1));
    for (uint64_t doc = doc_offset; doc < doc_offset + doc_num; ++doc) {
        if (!orc_eval_bitmap(nodes, kids, root, bitmaps + doc * stride, stride)) continue;
        float s = dot_seq(query, vectors + doc * dim, dim);
        topk_push(&st, s, (int64_t)doc);
    }
    int n = topk_finish(&st, out_scores, out_ids);
    free(st.heap);
    return n;
}

typedef struct {
    const float* queries;
    uint32_t q0, q1, dim;
    const orc_node* nodes;
    const int32_t* kids;
    const int32_t* roots;
    const float* vectors;
    const uint64_t* bitmaps;
    uint32_t stride;
    uint64_t doc_num, doc_offset;
    const int32_t* topks;
    int32_t out_stride;
    float* out_scores;
    int64_t* out_ids;
    int32_t* out_counts;
} batch_job;

/* One corpus pass for a slice of queries, as CpuTopKBatch does (recall_ref.cpp:90-142). */
static void* batch_worker(void* arg) {
    batch_job* j = (batch_job*)arg;
    uint32_t nq = j->q1 - j->q0;
    if (nq == 0) return NULL;
    topk_state* st = (topk_state*)calloc(nq, sizeof(topk_state));
    for (uint32_t k = 0; k < nq; k++) {
        int32_t kk = j->topks[j->q0 + k];
        st[k].cap = kk > 0 ? kk : 0;
        st[k].heap = (scored*)malloc(sizeof(scored) * (size_t)(st[k].cap > 0 ? st[k].cap : 1));
    }
    for (uint64_t doc = j->doc_offset; doc < j->doc_offset + j->doc_num; ++doc) {
        const uint64_t* bm = j->bitmaps + doc * j->stride;
        const float* v = j->vectors + doc * j->dim;
        for (uint32_t k = 0; k < nq; k++) {
            uint32_t q = j->q0 + k;
            if (!orc_eval_bitmap(j->nodes, j->kids, j->roots[q], bm, j->stride)) continue;
            float s = dot_seq(j->queries + (size_t)q * j->dim, v, j->dim);
            topk_push(&st[k], s, (int64_t)doc);
        }
    }
    for (uint32_t k = 0; k < nq; k++) {
        uint32_t q = j->q0 + k;
        j->out_counts[q] = topk_finish(&st[k], j->out_scores + (size_t)q * j->out_stride,
                                       j->out_ids + (size_t)q * j->out_stride);
        free(st[k].heap);
    }
    free(st);
    return NULL;
}

void orc_topk_batch(const float* queries, uint32_t nq, uint32_t dim, const orc_node* nodes,
                    const int32_t* kids, const int32_t* roots, const float* vectors,
                    const uint64_t* bitmaps, uint32_t stride, uint64_t doc_num, uint64_t doc_offset,
                    const int32_t* topks, int32_t out_stride, float* out_scores, int64_t* out_ids,
                    int32_t* out_counts, int threads) {
    if (threads < 1) threads = 1;
    if ((uint32_t)threads > nq) threads = (int)(nq > 0 ? nq : 1);
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
    batch_job* jobs = (batch_job*)malloc(sizeof(batch_job) * (size_t)threads);
    uint32_t per = (nq + (uint32_t)threads - 1) / (uint32_t)threads;
    for (int t = 0; t < threads; t++) {
        batch_job* j = &jobs[t];
        j->queries = queries;
        j->q0 = (uint32_t)t * per < nq ? (uint32_t)t * per : nq;
        j->q1 = j->q0 + per < nq ? j->q0 + per : nq;
        j->dim = dim;
        j->nodes = nodes;
        j->kids = kids;
        j->roots = roots;
        j->vectors = vectors;
        j->bitmaps = bitmaps;
        j->stride = stride;
        j->doc_num = doc_num;
        j->doc_offset = doc_offset;
        j->topks = topks;
        j->out_stride = out_stride;
        j->out_scores = out_scores;
        j->out_ids = out_ids;
        j->out_counts = out_counts;
        pthread_create(&th[t], NULL, batch_worker, j);
    }
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    free(th);
    free(jobs);
}

void orc_score_f64(const float* query, uint32_t dim, const float* vectors, const int64_t* ids, int n,
                   double* out) {
    for (int i = 0; i < n; i++) {
        const float* v = vectors + (size_t)ids[i] * dim;
        double s = 0.0;
        for (uint32_t d = 0; d < dim; d++) s += (double)query[d] * (double)v[d];
        out[i] = s;
    }
}

/* ------------------------------------------------------------------------------------------------
 * Posting codec. Head word [layout:4][hitCount:28] then payload byte length
 * (posting_serializer.cpp:15-39); layout chosen by density (:65-79): density = hits/docNum, sparse
 * iff density < threshold. Layouts (posting_layout.h:8): DENSE_BITMAP=0 (ceil(docNum/16) u16 units,
 * bit i of unit u = doc 16u+i, :46-55,103-120), SPARSE_BITMAP=1 (K u32 byte offsets then K u16
 * masks, :140-164), DENSE_BYTEMAP=2 (docNum bytes 0/1, :122-138), SPARSE_IDLIST=3 (hitCount u32 ids,
 * :194-208), SPARSE_PACKED=4 (K u32 [unit:16][mask:16], :166-192).
 * ----------------------------------------------------------------------------------------------*/
static void put32(uint8_t* p, uint32_t v) { memcpy(p, &v, 4); }
static void put16(uint8_t* p, uint16_t v) { memcpy(p, &v, 2); }
static uint32_t get32(const uint8_t* p) {
    uint32_t v;
    memcpy(&v, p, 4);
    return v;
}
static uint16_t get16(const uint8_t* p) {
    uint16_t v;
    memcpy(&v, p, 2);
    return v;
}

static int cmp_u32(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

int64_t orc_posting_serialize(const uint32_t* ids, uint32_t n, uint32_t seg_docs, int is_matrix,
                              float density_threshold, int packed, uint8_t* out, uint64_t cap) {
    if (seg_docs == 0) return -1;
    /* dedupe + sort (the reference builds an unordered_set; duplicates cannot occur) */
    uint32_t* s = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    memcpy(s, ids, sizeof(uint32_t) * (size_t)n);
    qsort(s, n, sizeof(uint32_t), cmp_u32);
    uint32_t m = 0;
    for (uint32_t i = 0; i < n; i++)
        if (m == 0 || s[m - 1] != s[i]) s[m++] = s[i];
    uint32_t hits = m;
    if (hits > 0x0FFFFFFFu) {
        free(s);
        return -1;
    }
    /* `float density = targetDocNum * 1.0 / docNum` converts the double quotient to float */
    float density = (float)((double)hits * 1.0 / (double)seg_docs);
    int sparse = density < density_threshold;
    int layout = sparse ? (is_matrix ? 3 : (packed ? 4 : 1)) : (is_matrix ? 2 : 0);
    uint32_t units = (seg_docs + 15) / 16;
    uint64_t need = 8;
    uint16_t* masks = NULL;
    uint32_t nz = 0;
    if (layout == 0 || layout == 1 || layout == 4) {
        masks = (uint16_t*)calloc(units, sizeof(uint16_t));
        for (uint32_t i = 0; i < m; i++)
            if (s[i] < units * 16u) masks[s[i] / 16] |= (uint16_t)(1u << (s[i] % 16));
        for (uint32_t u = 0; u < units; u++) nz += masks[u] != 0;
    }
    switch (layout) {
        case 0: need += (uint64_t)units * 2; break;
        case 1: need += (uint64_t)nz * 6; break;
        case 4: need += (uint64_t)nz * 4; break;
        case 2: need += seg_docs; break;
        case 3: need += (uint64_t)hits * 4; break;
    }
    if (need > cap || (layout == 4 && units > 0x10000u)) {
        free(s);
        free(masks);
        return -1;
    }
    put32(out, ((uint32_t)layout << 28) | hits);
    put32(out + 4, (uint32_t)(need - 8));
    uint8_t* p = out + 8;
    if (layout == 0) {
        for (uint32_t u = 0; u < units; u++) put16(p + 2 * u, masks[u]);
    } else if (layout == 1) {
        uint32_t k = 0;
        for (uint32_t u = 0; u < units; u++)
            if (masks[u]) {
                put32(p + 4 * k, u * 2u);
                put16(p + 4 * nz + 2 * k, masks[u]);
                k++;
            }
    } else if (layout == 4) {
        uint32_t k = 0;
        for (uint32_t u = 0; u < units; u++)
            if (masks[u]) put32(p + 4 * k++, (u << 16) | masks[u]);
    } else if (layout == 2) {
        memset(p, 0, seg_docs);
        for (uint32_t i = 0; i < m; i++)
            if (s[i] < seg_docs) p[s[i]] = 1;
    } else {
        for (uint32_t i = 0; i < m; i++) put32(p + 4 * i, s[i]);
    }
    free(s);
    free(masks);
    return (int64_t)need;
}

int orc_posting_decode(const uint8_t* posting, uint64_t len, uint32_t seg_docs, uint64_t* out_words) {
    uint32_t nw = (seg_docs + 63) / 64;
    memset(out_words, 0, sizeof(uint64_t) * nw);
    if (len < 8) return -1;
    uint32_t head = get32(posting);
    uint32_t plen = get32(posting + 4);
    int layout = (int)(head >> 28);
    if (8ull + plen > len) return -1;
    const uint8_t* p = posting + 8;
#define SETBIT(doc)                                                                 \
    do {                                                                            \
        uint32_t d_ = (doc);                                                        \
        if (d_ < seg_docs) out_words[d_ >> 6] |= 1ull << (d_ & 63);                \
    } while (0)
    switch (layout) {
        case 0:
            for (uint32_t u = 0; u < plen / 2; u++) {
                uint16_t m = get16(p + 2 * u);
                for (int b = 0; b < 16; b++)
                    if (m >> b & 1) SETBIT(u * 16 + (uint32_t)b);
            }
            return 0;
        case 1: {
            uint32_t k = plen / 6;
            for (uint32_t i = 0; i < k; i++) {
                uint32_t u = get32(p + 4 * i) / 2;
                uint16_t m = get16(p + 4 * k + 2 * i);
                for (int b = 0; b < 16; b++)
                    if (m >> b & 1) SETBIT(u * 16 + (uint32_t)b);
            }
            return 1;
        }
        case 4: {
            uint32_t k = plen / 4;
            for (uint32_t i = 0; i < k; i++) {
                uint32_t w = get32(p + 4 * i);
                uint32_t u = w >> 16;
                for (int b = 0; b < 16; b++)
                    if (w >> b & 1) SETBIT(u * 16 + (uint32_t)b);
            }
            return 4;
        }
        case 2:
            for (uint32_t i = 0; i < plen; i++)
                if (p[i]) SETBIT(i);
            return 2;
        case 3:
            for (uint32_t i = 0; i < plen / 4; i++) SETBIT(get32(p + 4 * i));
            return 3;
    }
#undef SETBIT
    return -1;
}

/* ------------------------------------------------------------------------------------------------
 * Postfix program evaluation: the interpretation kernel_bitmap_text_filter.cpp:52-119 gives the
 * program, with AND/OR (filter_and_op.h, filter_or_op.h: postings first, then stackNum entries popped
 * from the stack top), NOT (filter_not_op.h: exactly one posting or one stack entry) and CONJUNCTION
 * (filter_conjunction_op.h: AND over parts of the OR over each part's postings). Validation follows
 * CheckPostExpr (text_filter.cpp:1233-1352).
 * ----------------------------------------------------------------------------------------------*/
int orc_eval_postfix(const uint32_t* prog, uint32_t prog_len, uint32_t op_count,
                     const uint64_t* const* operands, uint32_t n_operands, uint32_t words, uint64_t* out) {
    (void)op_count;
    uint64_t** stack = (uint64_t**)calloc(prog_len + 1, sizeof(uint64_t*));
    uint64_t* acc = (uint64_t*)malloc(sizeof(uint64_t) * words);
    uint32_t sp = 0, next = 0;
    int rc = 0;
    for (uint32_t i = 0; i < prog_len && rc == 0; i++) {
        uint32_t op = prog[i];
        if (op == 1 || op == 2) {
            if (i + 2 >= prog_len) { rc = -1; break; }
            uint32_t pn = prog[i + 1], sn = prog[i + 2];
            if (pn + sn == 0 || next + pn > n_operands || sn > sp) { rc = -1; break; }
            for (uint32_t w = 0; w < words; w++) acc[w] = op == 1 ? ~0ull : 0ull;
            for (uint32_t k = 0; k < pn; k++)
                for (uint32_t w = 0; w < words; w++)
                    acc[w] = op == 1 ? (acc[w] & operands[next + k][w]) : (acc[w] | operands[next + k][w]);
            for (uint32_t k = 0; k < sn; k++) {
                uint64_t* e = stack[sp - 1 - k];
                for (uint32_t w = 0; w < words; w++) acc[w] = op == 1 ? (acc[w] & e[w]) : (acc[w] | e[w]);
                free(e);
            }
            next += pn;
            sp -= sn;
            i += 2;
        } else if (op == 3) {
            if (i + 2 >= prog_len) { rc = -1; break; }
            uint32_t pn = prog[i + 1], sn = prog[i + 2];
            if (pn + sn != 1 || next + pn > n_operands || sn > sp) { rc = -1; break; }
            if (pn == 1) {
                for (uint32_t w = 0; w < words; w++) acc[w] = ~operands[next][w];
                next++;
            } else {
                uint64_t* e = stack[--sp];
                for (uint32_t w = 0; w < words; w++) acc[w] = ~e[w];
                free(e);
            }
            i += 2;
        } else if (op == 0) {
            if (i + 1 >= prog_len) { rc = -1; break; }
            uint32_t parts = prog[i + 1];
            if (parts == 0 || i + 1 + parts >= prog_len) { rc = -1; break; }
            for (uint32_t w = 0; w < words; w++) acc[w] = ~0ull;
            for (uint32_t pidx = 0; pidx < parts; pidx++) {
                uint32_t pn = prog[i + 2 + pidx];
                if (pn == 0 || next + pn > n_operands) { rc = -1; break; }
                for (uint32_t w = 0; w < words; w++) {
                    uint64_t o = 0;
                    for (uint32_t k = 0; k < pn; k++) o |= operands[next + k][w];
                    acc[w] &= o;
                }
                next += pn;
            }
            i += 1 + parts;
        } else {
            rc = -1;
            break;
        }
        if (rc != 0) break;
        uint64_t* e = (uint64_t*)malloc(sizeof(uint64_t) * words);
        memcpy(e, acc, sizeof(uint64_t) * words);
        stack[sp++] = e;
    }
    if (rc == 0 && (sp != 1 || next != n_operands)) rc = -1;
    if (rc == 0) memcpy(out, stack[0], sizeof(uint64_t) * words);
    for (uint32_t k = 0; k < sp; k++) free(stack[k]);
    free(stack);
    free(acc);
    return rc;
}

/* ------------------------------------------------------------------------------------------------
 * Hash64 (hash.cpp:10-16): MurmurHash3_x64_128 with seed 0x20160713, result h1 ^ h2. The hash is
 * Austin Appleby's published, public-domain MurmurHash3 (x64, 128-bit variant), restated here from
 * its published description.
 * ----------------------------------------------------------------------------------------------*/
static uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
static uint64_t fmix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

uint64_t orc_hash64(const char* data, uint32_t len) {
    const uint8_t* d = (const uint8_t*)data;
    const uint64_t c1 = 0x87c37b91114253d5ull, c2 = 0x4cf5ad432745937full;
    uint64_t h1 = 0x20160713u, h2 = 0x20160713u;
    uint32_t nblocks = len / 16;
    for (uint32_t i = 0; i < nblocks; i++) {
        uint64_t k1, k2;
        memcpy(&k1, d + 16 * i, 8);
        memcpy(&k2, d + 16 * i + 8, 8);
        k1 *= c1; k1 = rotl64(k1, 31); k1 *= c2; h1 ^= k1;
        h1 = rotl64(h1, 27); h1 += h2; h1 = h1 * 5 + 0x52dce729;
        k2 *= c2; k2 = rotl64(k2, 33); k2 *= c1; h2 ^= k2;
        h2 = rotl64(h2, 31); h2 += h1; h2 = h2 * 5 + 0x38495ab5;
    }
    const uint8_t* tail = d + 16 * nblocks;
    uint64_t k1 = 0, k2 = 0;
    uint32_t rem = len & 15u;
    for (uint32_t i = rem; i > 8; i--) k2 ^= (uint64_t)tail[i - 1] << (8 * (i - 9));
    if (rem > 8) {
        k2 *= c2; k2 = rotl64(k2, 33); k2 *= c1; h2 ^= k2;
    }
    for (uint32_t i = rem < 8 ? rem : 8; i > 0; i--) k1 ^= (uint64_t)tail[i - 1] << (8 * (i - 1));
    if (rem > 0) {
        k1 *= c1; k1 = rotl64(k1, 31); k1 *= c2; h1 ^= k1;
    }
    h1 ^= len;
    h2 ^= len;
    h1 += h2;
    h2 += h1;
    h1 = fmix64(h1);
    h2 = fmix64(h2);
    h1 += h2;
    h2 += h1;
    return h1 ^ h2;
}
