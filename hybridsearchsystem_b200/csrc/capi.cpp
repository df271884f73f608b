// capi.cpp -- extern "C" entry points of libhss.so (declared in include/hss.h).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hss.h"
#include "hss_device.cuh"
#include "hss_kernels.h"
#include "host/hss_host.h"

namespace {
thread_local std::string g_lastError;

int SetError(int code, const std::string& msg) {
    g_lastError = msg;
    return code;
}

int FromCuda(cudaError_t e) {
    if (e == cudaSuccess) return HSS_OK;
    return SetError(HSS_ERR_CUDA, cudaGetErrorString(e));
}

cudaStream_t S(hss_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }
}  // namespace

struct hss_table {
    std::shared_ptr<hss::DataTable> t;
};

struct hss_searcher {
    std::unique_ptr<hss::FullRecallSearcher> s;
    std::shared_ptr<hss::DataTable> t;
    std::vector<std::unique_ptr<hss::QueryNode>> owned;  // trees of the added queries
};

struct hss_model {
    std::shared_ptr<hss::ThresholdModel> m;
};

struct hss_server {
    std::unique_ptr<hss::ServingLoop> s;
};

struct hss_filters {
    std::vector<hss::FilterExpr> exprs;
};

extern "C" {

const char* hss_last_error(void) { return g_lastError.c_str(); }

int hss_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// ---------------------------------------------------------------------------------------------
// operators

int hss_vector_score_launch(const float* queryMatrix, const float* docMatrix, float* resultMatrix, uint32_t m,
                            uint32_t n, uint32_t k, uint64_t ldResult, hss_stream_t stream) {
    if (!queryMatrix || !docMatrix || !resultMatrix || k == 0 || k % 4 || k > 4096 || ldResult < n)
        return SetError(HSS_ERR_INVALID, "hss_vector_score_launch: bad arguments");
    return FromCuda(hss::launch_exact_score(queryMatrix, docMatrix, resultMatrix, m, n, k, ldResult, S(stream)));
}

int hss_bitmap_text_filter_launch(const uint64_t* postings, const uint32_t* postOrderExpr, void* resultStack,
                                  hss_filter_context ctx, uint8_t* result, int32_t* status, hss_stream_t stream) {
    (void)resultStack;
    if (!postings || !postOrderExpr || !result || ctx.segmentNum == 0 || ctx.segmentLength == 0 ||
        ctx.segmentLength % 8 != 0 || (reinterpret_cast<uintptr_t>(result) & 7u))
        return SetError(HSS_ERR_INVALID, "hss_bitmap_text_filter_launch: bad arguments");
    if (ctx.postingNum > static_cast<uint32_t>(hss::kMaxOperands) || ctx.exprLen > static_cast<uint32_t>(hss::kMaxProgram))
        return SetError(HSS_ERR_LIMIT, "filter program beyond HSS_MAX_OPERANDS / HSS_MAX_PROGRAM");
    if (ctx.exprLen == 0) return SetError(HSS_ERR_PROGRAM, "empty filter program");
    hss::FilterLaunch F{};
    F.prog = postOrderExpr;
    F.prog_off = nullptr;
    F.opnd_off = nullptr;
    F.opnd_row = nullptr;
    F.single_prog_len = ctx.exprLen;
    F.single_nop = ctx.postingNum;
    F.table = postings;
    F.row_stride = 1;
    F.seg_stride = ctx.postingNum;
    F.out = reinterpret_cast<uint64_t*>(result);
    F.out_stride = 0;
    F.pass_count = nullptr;
    F.status = status;
    F.nq = 1;
    F.seg_num = ctx.segmentNum;
    F.docs_per_seg = ctx.segmentLength * 16u;
    F.doc_num = static_cast<uint64_t>(ctx.segmentNum) * F.docs_per_seg;
    F.max_opnd = ctx.postingNum;
    F.ref_table = (ctx.flags & HSS_FILTER_HEAD_ADDRESSES) ? 0 : 1;
    return FromCuda(hss::launch_filter_batch(F, S(stream)));
}

int hss_posting_bitlist_to_set_launch(const uint64_t* postings, uint32_t byteSizePerSegment,
                                      const uint64_t* resultPostings, uint32_t count, int32_t* status,
                                      hss_stream_t stream) {
    if ((count && (!postings || !resultPostings)) || byteSizePerSegment == 0 || byteSizePerSegment % 8)
        return SetError(HSS_ERR_INVALID, "hss_posting_bitlist_to_set_launch: bad arguments");
    return FromCuda(hss::launch_posting_expand(postings, resultPostings, count, byteSizePerSegment,
                                               byteSizePerSegment * 8u, status, S(stream)));
}

size_t hss_aggregator_workspace_size(uint32_t docNumber) { return hss::aggregate_workspace_bytes(docNumber); }

int hss_aggregator_launch(const uint8_t* filterResult, const float* docScores, const uint32_t* docLocationConst,
                          float* outScores, uint32_t* outLocations, uint32_t* effectiveCount, uint32_t docNumber,
                          void* workspace, size_t workspaceBytes, hss_stream_t stream) {
    if (!filterResult || !docScores || !outScores || !outLocations || !effectiveCount || !workspace ||
        (reinterpret_cast<uintptr_t>(filterResult) & 7u))
        return SetError(HSS_ERR_INVALID, "hss_aggregator_launch: bad arguments");
    if (workspaceBytes < hss::aggregate_workspace_bytes(docNumber))
        return SetError(HSS_ERR_INVALID, "hss_aggregator_launch: workspace too small");
    return FromCuda(hss::launch_aggregate(reinterpret_cast<const uint64_t*>(filterResult), docScores,
                                          docLocationConst, docNumber, outScores, outLocations, effectiveCount,
                                          static_cast<uint32_t*>(workspace), S(stream)));
}

namespace {
static_assert(HSS_AGGREGATOR_NOALLOC_MAX_DOCS == hss::kAggStaticMaxDocs,
              "the public allocation-free aggregator limit must equal the size of its scratch array");

// Address of the aggregator's module-scope scratch on each device, looked up (with that device
// current) on the first allocation-free call made there, and again whenever the device's CUDA context
// has changed since (cudaDeviceReset destroys the primary context; the module, and with it the array,
// is loaded anew in the next one, possibly at another address). The context is identified by its
// process-unique id (cuCtxGetId), not by its handle, which a new context may reuse.
constexpr int kMaxDevices = 64;
std::mutex g_staticScratchMu;
struct ScratchEntry {
    unsigned long long ctxId;
    uint32_t* ptr;
};
ScratchEntry g_staticScratch[kMaxDevices] = {};

// Id of the calling thread's current context; false when no context is current or the driver
// entry points are unavailable.
bool CurrentContextId(unsigned long long* id) {
    static PFN_cuCtxGetCurrent_v4000 getCurrent = nullptr;
    static PFN_cuCtxGetId_v12000 getId = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            getCurrent = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            getId = reinterpret_cast<PFN_cuCtxGetId_v12000>(p);
    });
    CUcontext ctx = nullptr;
    if (!getCurrent || !getId || getCurrent(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return getId(ctx, id) == CUDA_SUCCESS;
}

int StaticAggregateScratch(uint32_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return FromCuda(e);
    if (dev < 0 || dev >= kMaxDevices) return SetError(HSS_ERR_LIMIT, "hss_aggregator_launch_noalloc: device index");
    std::lock_guard<std::mutex> lock(g_staticScratchMu);
    ScratchEntry& ent = g_staticScratch[dev];
    unsigned long long ctx = 0;
    const bool known = CurrentContextId(&ctx);
    if (!ent.ptr || !known || ent.ctxId != ctx) {
        // the lookup also makes the device's primary context current if it was not yet
        uint32_t* p = nullptr;
        e = hss::aggregate_static_scratch(&p);
        if (e != cudaSuccess) return FromCuda(e);
        if (!p) return SetError(HSS_ERR_CUDA, "hss_aggregator_launch_noalloc: scratch symbol has no address");
        if (!CurrentContextId(&ctx)) {
            // without a context id the address cannot be cached safely: use it for this call only
            *out = p;
            ent = ScratchEntry{};
            return HSS_OK;
        }
        ent = ScratchEntry{ctx, p};
    }
    *out = ent.ptr;
    return HSS_OK;
}
}  // namespace

int hss_aggregator_launch_noalloc(const uint8_t* filterResult, const float* docScores,
                                  const uint32_t* docLocationConst, float* outScores, uint32_t* outLocations,
                                  uint32_t* effectiveCount, uint32_t docNumber, hss_stream_t stream) {
    if (!filterResult || !docScores || !outScores || !outLocations || !effectiveCount ||
        (reinterpret_cast<uintptr_t>(filterResult) & 7u))
        return SetError(HSS_ERR_INVALID, "hss_aggregator_launch_noalloc: bad arguments");
    if (docNumber > hss::kAggStaticMaxDocs)
        return SetError(HSS_ERR_LIMIT, "hss_aggregator_launch_noalloc: docNumber " + std::to_string(docNumber) +
                                           " exceeds HSS_AGGREGATOR_NOALLOC_MAX_DOCS (" +
                                           std::to_string(hss::kAggStaticMaxDocs) + ")");
    uint32_t* scratch = nullptr;
    const int rc = StaticAggregateScratch(&scratch);
    if (rc != HSS_OK) return rc;
    return FromCuda(hss::launch_aggregate(reinterpret_cast<const uint64_t*>(filterResult), docScores,
                                          docLocationConst, docNumber, outScores, outLocations, effectiveCount,
                                          scratch, S(stream)));
}

int hss_topk_launch(const float* scores, const uint32_t* locations, const uint32_t* count, uint32_t topK,
                    float* outScores, uint32_t* outLocations, uint32_t* outCount, hss_stream_t stream) {
    if (!scores || !locations || !count || !outScores || !outLocations || !outCount)
        return SetError(HSS_ERR_INVALID, "hss_topk_launch: bad arguments");
    if (topK > static_cast<uint32_t>(hss::kMaxTopK)) return SetError(HSS_ERR_LIMIT, "topK beyond HSS_MAX_TOPK");
    return FromCuda(hss::launch_topk_op(scores, locations, count, topK, outScores, outLocations, outCount, S(stream)));
}

int hss_merge_shards_launch(const float* const* shardScores, const int64_t* const* shardIds,
                            const uint32_t* const* shardCounts, uint32_t shards, uint32_t nq, uint32_t inStride,
                            uint32_t topK, float* outScores, int64_t* outIds, uint32_t* outCounts, uint32_t outStride,
                            hss_stream_t stream) {
    if (!shardScores || !shardIds || !shardCounts || !outScores || !outIds || !outCounts || shards == 0)
        return SetError(HSS_ERR_INVALID, "hss_merge_shards_launch: null argument");
    if (shards > hss::kMaxShards || topK > static_cast<uint32_t>(hss::kMaxTopK))
        return SetError(HSS_ERR_LIMIT, "shards beyond HSS_MAX_SHARDS or topK beyond HSS_MAX_TOPK");
    if (topK > outStride) return SetError(HSS_ERR_INVALID, "topK larger than the output stride");
    hss::ShardMergeLaunch L{};
    for (uint32_t s = 0; s < shards; ++s) {
        L.scores[s] = shardScores[s];
        L.ids[s] = shardIds[s];
        L.counts[s] = shardCounts[s];
    }
    L.shards = shards;
    L.nq = nq;
    L.in_stride = inStride;
    L.topk = topK;
    L.out_score = outScores;
    L.out_id = outIds;
    L.out_count = outCounts;
    L.out_stride = outStride;
    return FromCuda(hss::launch_merge_shards(L, S(stream)));
}

// ---------------------------------------------------------------------------------------------
// index

int hss_table_build(int32_t deviceId, const float* vectors, const uint64_t* tagBits, uint64_t docNum, uint32_t dim,
                    uint32_t tagNum, const hss_index_config* cfg, hss_table** out) {
    if (!vectors || !tagBits || !out) return SetError(HSS_ERR_INVALID, "hss_table_build: null argument");
    hss::IndexConfig c;
    if (cfg) {
        c.docNumPerSegment = cfg->docNumPerSegment;
        c.densityThreshold = cfg->densityThreshold;
        c.matrixPosting = cfg->matrixPosting != 0;
        c.sparsePacked = cfg->sparsePacked != 0;
        c.docOffset = cfg->docOffset;
    }
    auto t = std::make_shared<hss::DataTable>();
    std::string err;
    if (!t->Build(deviceId, vectors, tagBits, docNum, dim, tagNum, c, &err)) return SetError(HSS_ERR_INDEX, err);
    *out = new hss_table{t};
    return HSS_OK;
}

int hss_table_build_device(int32_t deviceId, const float* dVectors, const uint64_t* tagBits, uint64_t docNum,
                           uint32_t dim, uint32_t tagNum, const hss_index_config* cfg, hss_table** out) {
    if (!dVectors || !tagBits || !out) return SetError(HSS_ERR_INVALID, "hss_table_build_device: null argument");
    hss::IndexConfig c;
    if (cfg) {
        c.docNumPerSegment = cfg->docNumPerSegment;
        c.densityThreshold = cfg->densityThreshold;
        c.matrixPosting = cfg->matrixPosting != 0;
        c.sparsePacked = cfg->sparsePacked != 0;
        c.docOffset = cfg->docOffset;
    }
    auto t = std::make_shared<hss::DataTable>();
    std::string err;
    if (!t->BuildFromDevice(deviceId, dVectors, tagBits, docNum, dim, tagNum, c, &err))
        return SetError(HSS_ERR_INDEX, err);
    *out = new hss_table{t};
    return HSS_OK;
}

int hss_table_load(int32_t deviceId, const char* dir, hss_table** out) {
    if (!dir || !out) return SetError(HSS_ERR_INVALID, "hss_table_load: null argument");
    auto t = std::make_shared<hss::DataTable>();
    std::string err;
    if (!t->LoadData(deviceId, dir, &err)) return SetError(HSS_ERR_INDEX, err);
    *out = new hss_table{t};
    return HSS_OK;
}

int hss_table_load_reference(int32_t deviceId, const char* dir, hss_table** out) {
    if (!dir || !out) return SetError(HSS_ERR_INVALID, "hss_table_load_reference: null argument");
    auto t = std::make_shared<hss::DataTable>();
    std::string err;
    if (!t->LoadReferenceIndex(deviceId, dir, &err)) return SetError(HSS_ERR_INDEX, err);
    *out = new hss_table{t};
    return HSS_OK;
}

int hss_table_save_reference(const hss_table* table, const char* dir, uint32_t splitDocNumZn) {
    if (!table || !dir) return SetError(HSS_ERR_INVALID, "hss_table_save_reference: null argument");
    std::string err;
    if (!table->t->SaveReferenceIndex(dir, splitDocNumZn, &err)) return SetError(HSS_ERR_INDEX, err);
    return HSS_OK;
}

int hss_table_load_times(const hss_table* table, double* ms6, uint64_t* vectorBytes, uint64_t* postingBytes,
                         uint32_t* threads) {
    if (!table) return SetError(HSS_ERR_INVALID, "null table");
    const auto& t = table->t->GetLoadTimes();
    if (ms6) {
        ms6[0] = t.meta;
        ms6[1] = t.postingsRead;
        ms6[2] = t.vectorsRead;
        ms6[3] = t.vectorsH2D;
        ms6[4] = t.postingsH2D;
        ms6[5] = t.total;
    }
    if (vectorBytes) *vectorBytes = t.vectorBytes;
    if (postingBytes) *postingBytes = t.postingBytes;
    if (threads) *threads = t.threads;
    return HSS_OK;
}

int hss_table_save(const hss_table* table, const char* dir) {
    if (!table || !dir) return SetError(HSS_ERR_INVALID, "hss_table_save: null argument");
    std::string err;
    if (!table->t->Save(dir, &err)) return SetError(HSS_ERR_INDEX, err);
    return HSS_OK;
}

void hss_table_free(hss_table* table) { delete table; }

int hss_table_info(const hss_table* table, uint64_t* docNum, uint32_t* dim, uint32_t* segmentNum,
                   uint32_t* docNumPerSegment, uint32_t* postingRows, float* maxNorm) {
    if (!table) return SetError(HSS_ERR_INVALID, "null table");
    const hss::DataTable& t = *table->t;
    if (docNum) *docNum = t.GetDocNum();
    if (dim) *dim = t.GetDimension();
    if (segmentNum) *segmentNum = t.GetSegmentNum();
    if (docNumPerSegment) *docNumPerSegment = t.GetDocNumPerSegment();
    if (postingRows) *postingRows = t.PostingRows();
    if (maxNorm) *maxNorm = t.GetMaxNorm();
    return HSS_OK;
}

int hss_table_posting(const hss_table* table, uint64_t token, uint32_t segment, const uint8_t** data, uint32_t* len) {
    if (!table || !data || !len) return SetError(HSS_ERR_INVALID, "null argument");
    bool exist = false;
    const uint32_t row = table->t->TokenRow(token, exist);
    *data = exist ? table->t->HostPosting(row, segment, len) : nullptr;
    if (!*data) *len = 0;
    return HSS_OK;
}

int hss_table_device_ptrs(const hss_table* table, const float** vectors, const uint64_t** postingTable,
                          const int64_t** gdocids) {
    if (!table) return SetError(HSS_ERR_INVALID, "null table");
    if (vectors) *vectors = table->t->DeviceVectors();
    if (postingTable) *postingTable = table->t->DevicePostingTable();
    if (gdocids) *gdocids = table->t->DeviceGDocIds();
    return HSS_OK;
}

// ---------------------------------------------------------------------------------------------
// searcher

namespace {
bool ToSearcherConfig(const hss_searcher_config* cfg, hss::SearcherConfig& c) {
    if (cfg) {
        if (cfg->maxBatch) c.maxBatch = cfg->maxBatch;
        if (cfg->candidateCap) c.candidateCap = cfg->candidateCap;
        if (cfg->sampleDocs) c.sampleDocs = cfg->sampleDocs;
        c.maxRetries = cfg->maxRetries;
        if (cfg->method < 0 || cfg->method > 3) return false;
        c.method = static_cast<hss::ScoreMethod>(cfg->method);
        c.densePostings = cfg->decodeInPlace == 0;
    }
    return true;
}
}  // namespace

size_t hss_searcher_workspace_bytes(const hss_table* table, const hss_searcher_config* cfg) {
    hss::SearcherConfig c;
    if (!table || !ToSearcherConfig(cfg, c)) return 0;
    return hss::FullRecallSearcher::WorkspaceBytes(*table->t, c);
}

int hss_table_prepare(hss_table* table, const hss_searcher_config* cfg) {
    hss::SearcherConfig c;
    if (!table || !ToSearcherConfig(cfg, c)) return SetError(HSS_ERR_INVALID, "hss_table_prepare: bad arguments");
    if (table->t->GetDeviceId() < 0) return SetError(HSS_ERR_INVALID, "hss_table_prepare: host-only table");
    if (cudaSetDevice(table->t->GetDeviceId()) != cudaSuccess) return SetError(HSS_ERR_CUDA, "cudaSetDevice");
    std::string err;
    if (c.densePostings) {
        size_t freeB = 0, totalB = 0;
        if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess) return SetError(HSS_ERR_CUDA, "cudaMemGetInfo");
        if (!table->t->EnableDensePostings(static_cast<uint64_t>(freeB) / 5 * 2, &err)) return SetError(HSS_ERR_CUDA, err);
    }
    if (c.method != hss::ScoreMethod::SIMT_FP32 && !table->t->EnableFormat(static_cast<int>(c.method) - 1, &err))
        return SetError(HSS_ERR_INVALID, err);
    return HSS_OK;
}

int hss_searcher_create_in(hss_table* table, const hss_searcher_config* cfg, void* dWorkspace, size_t workspaceBytes,
                           hss_searcher** out) {
    if (!table || !out || !dWorkspace) return SetError(HSS_ERR_INVALID, "hss_searcher_create_in: null argument");
    hss::SearcherConfig c;
    if (!ToSearcherConfig(cfg, c)) return SetError(HSS_ERR_INVALID, "unknown scoring method");
    auto* s = new hss_searcher;
    s->t = table->t;
    s->s = std::make_unique<hss::FullRecallSearcher>(table->t->GetDeviceId(), table->t, c, dWorkspace, workspaceBytes);
    if (!s->s->Ok()) {
        const std::string e = s->s->Error();
        delete s;
        return SetError(HSS_ERR_INVALID, e);
    }
    *out = s;
    return HSS_OK;
}

int hss_searcher_create(hss_table* table, const hss_searcher_config* cfg, hss_searcher** out) {
    if (!table || !out) return SetError(HSS_ERR_INVALID, "hss_searcher_create: null argument");
    hss::SearcherConfig c;
    if (!ToSearcherConfig(cfg, c)) return SetError(HSS_ERR_INVALID, "unknown scoring method");
    auto* s = new hss_searcher;
    s->t = table->t;
    s->s = std::make_unique<hss::FullRecallSearcher>(table->t->GetDeviceId(), table->t, c);
    if (!s->s->Ok()) {
        const std::string e = s->s->Error();
        delete s;
        return SetError(HSS_ERR_CUDA, e);
    }
    *out = s;
    return HSS_OK;
}

void hss_searcher_free(hss_searcher* s) { delete s; }

int hss_searcher_add_query(hss_searcher* s, const char* filterExpr, const float* vector, uint32_t dim, uint32_t topK) {
    if (!s || !vector) return SetError(HSS_ERR_INVALID, "hss_searcher_add_query: null argument");
    if (dim != s->t->GetDimension()) return SetError(HSS_ERR_INVALID, "query dimension mismatch");
    bool ok = true;
    auto ast = hss::ParseFilter(filterExpr ? filterExpr : "", ok);
    if (!ok) return SetError(HSS_ERR_PARSE, std::string("filter does not parse: ") + (filterExpr ? filterExpr : ""));
    s->owned.push_back(hss::BuildQueryNode(ast.get(), s->t->GetConfig().postingField));
    s->s->AddQuery(s->owned.back().get(), std::vector<float>(vector, vector + dim), topK);
    return HSS_OK;
}

int hss_searcher_batch_search(hss_searcher* s, float* outScores, int64_t* outIds, uint32_t* outCounts,
                              uint32_t outStride) {
    if (!s || !outScores || !outIds || !outCounts) return SetError(HSS_ERR_INVALID, "null argument");
    std::vector<std::shared_ptr<hss::FullRecallResult>> res;
    const bool ok = s->s->BatchSearch(res, s->t->GetConfig().vectorField, false);
    s->owned.clear();
    if (!ok) return SetError(HSS_ERR_CUDA, s->s->Error());
    bool failed = false;
    for (size_t q = 0; q < res.size(); ++q) {
        const auto& r = *res[q];
        const uint32_t c = static_cast<uint32_t>(std::min<size_t>(r.docIds.size(), outStride));
        outCounts[q] = c;
        for (uint32_t i = 0; i < c; ++i) {
            outScores[q * static_cast<size_t>(outStride) + i] = r.scores[i];
            outIds[q * static_cast<size_t>(outStride) + i] = r.docIds[i];
        }
    }
    for (int32_t st : s->s->LastStatus()) failed |= st != 0;
    if (failed) return SetError(HSS_ERR_QUERY, "some queries failed (see hss_searcher_last_status)");
    return HSS_OK;
}

int hss_filters_compile(hss_searcher* s, const char* const* filterExprs, uint32_t n, hss_filters** out) {
    if (!s || !out || (n && !filterExprs)) return SetError(HSS_ERR_INVALID, "hss_filters_compile: null argument");
    auto f = std::make_unique<hss_filters>();
    f->exprs.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        bool ok = true;
        const char* e = filterExprs[i] ? filterExprs[i] : "";
        auto ast = hss::ParseFilter(e, ok);
        if (!ok) return SetError(HSS_ERR_PARSE, std::string("filter does not parse: ") + e);
        auto tree = hss::BuildQueryNode(ast.get(), s->t->GetConfig().postingField);
        std::string err;
        if (!hss::PrepareExpr(tree.get(), *s->t, f->exprs[i], &err)) return SetError(HSS_ERR_PROGRAM, err);
    }
    *out = f.release();
    return HSS_OK;
}

void hss_filters_free(hss_filters* f) { delete f; }

int hss_searcher_search_device(hss_searcher* s, const float* dQueries, uint32_t nq, const hss_filters* filters,
                               const uint32_t* topks, float* dOutScores, int64_t* dOutIds, uint32_t* dOutCounts,
                               uint32_t outStride, hss_stream_t stream) {
    if (!s || !filters || !topks || (nq && (!dQueries || !dOutScores || !dOutIds || !dOutCounts)))
        return SetError(HSS_ERR_INVALID, "hss_searcher_search_device: null argument");
    if (filters->exprs.size() < nq) return SetError(HSS_ERR_INVALID, "fewer filters than queries");
    std::vector<const hss::FilterExpr*> ptrs(nq);
    for (uint32_t i = 0; i < nq; ++i) ptrs[i] = &filters->exprs[i];
    const int rc = s->s->SearchDevice(dQueries, nq, ptrs.data(), topks, dOutScores, dOutIds, dOutCounts, outStride,
                                      S(stream));
    if (rc < 0) return SetError(rc == -1 ? HSS_ERR_INVALID : HSS_ERR_CUDA, s->s->Error());
    if (rc > 0) return SetError(HSS_ERR_QUERY, "some queries failed (see hss_searcher_last_status)");
    return HSS_OK;
}

int hss_searcher_search_device_async(hss_searcher* s, const float* dQueries, uint32_t nq, const hss_filters* filters,
                                     const uint32_t* topks, float* dOutScores, int64_t* dOutIds, uint32_t* dOutCounts,
                                     uint32_t outStride, hss_stream_t stream) {
    if (!s || !filters || !topks || (nq && (!dQueries || !dOutScores || !dOutIds || !dOutCounts)))
        return SetError(HSS_ERR_INVALID, "hss_searcher_search_device_async: null argument");
    if (filters->exprs.size() < nq) return SetError(HSS_ERR_INVALID, "fewer filters than queries");
    std::vector<const hss::FilterExpr*> ptrs(nq);
    for (uint32_t i = 0; i < nq; ++i) ptrs[i] = &filters->exprs[i];
    const int rc = s->s->SearchEnqueue(dQueries, nq, ptrs.data(), topks, dOutScores, dOutIds, dOutCounts, outStride,
                                       S(stream));
    if (rc < 0) return SetError(rc == -1 ? HSS_ERR_INVALID : HSS_ERR_CUDA, s->s->Error());
    return HSS_OK;
}

int hss_searcher_finish(hss_searcher* s) {
    if (!s) return SetError(HSS_ERR_INVALID, "hss_searcher_finish: null searcher");
    const int rc = s->s->SearchFinish();
    if (rc < 0) return SetError(HSS_ERR_CUDA, s->s->Error());
    if (rc > 0) return SetError(HSS_ERR_QUERY, "some queries failed (see hss_searcher_last_status)");
    return HSS_OK;
}

int hss_searcher_filter_device(hss_searcher* s, const hss_filters* filters, uint32_t nq, uint64_t* dOutBits,
                               uint64_t outStrideWords, uint32_t* dPassCounts, hss_stream_t stream) {
    if (!s || !filters || (nq && !dOutBits)) return SetError(HSS_ERR_INVALID, "hss_searcher_filter_device: null argument");
    if (filters->exprs.size() < nq) return SetError(HSS_ERR_INVALID, "fewer filters than queries");
    std::vector<const hss::FilterExpr*> ptrs(nq);
    for (uint32_t i = 0; i < nq; ++i) ptrs[i] = &filters->exprs[i];
    const int rc = s->s->FilterDevice(nq, ptrs.data(), dOutBits, outStrideWords, dPassCounts, S(stream));
    if (rc < 0) return SetError(rc == -1 ? HSS_ERR_INVALID : HSS_ERR_CUDA, s->s->Error());
    if (rc > 0) return SetError(HSS_ERR_QUERY, "some filters failed (see hss_searcher_last_status)");
    return HSS_OK;
}

int hss_searcher_last_status(const hss_searcher* s, int32_t* status, uint32_t n) {
    if (!s || (n && !status)) return SetError(HSS_ERR_INVALID, "null argument");
    const auto& st = s->s->LastStatus();
    for (uint32_t i = 0; i < n; ++i) status[i] = i < st.size() ? st[i] : 0;
    return HSS_OK;
}

int hss_searcher_last_candidates(hss_searcher* s, uint32_t query, float* scores, uint32_t* locations, uint32_t cap,
                                 uint32_t* count, float* theta, float* eps) {
    if (!s || !count || !theta || !eps || (cap && (!scores || !locations)))
        return SetError(HSS_ERR_INVALID, "hss_searcher_last_candidates: null argument");
    const int rc = s->s->LastCandidates(query, scores, locations, cap, count, theta, eps);
    if (rc < 0) return SetError(rc == -1 ? HSS_ERR_INVALID : HSS_ERR_CUDA, "hss_searcher_last_candidates");
    return HSS_OK;
}

int hss_searcher_set_pipeline_test(hss_searcher* s, uint32_t holdLoad, uint64_t waitBudgetCycles) {
    if (!s) return SetError(HSS_ERR_INVALID, "null searcher");
    if (waitBudgetCycles > (1ull << 40)) return SetError(HSS_ERR_LIMIT, "wait budget too large");
    s->s->SetPipelineTest(holdLoad, static_cast<long long>(waitBudgetCycles));
    return HSS_OK;
}

int hss_searcher_set_timing(hss_searcher* s, int32_t on) {
    if (!s) return SetError(HSS_ERR_INVALID, "null searcher");
    s->s->SetTiming(on != 0);
    return HSS_OK;
}

int hss_searcher_set_graphs(hss_searcher* s, int32_t on) {
    if (!s) return SetError(HSS_ERR_INVALID, "null searcher");
    s->s->SetGraphs(on != 0);
    return HSS_OK;
}

int hss_searcher_graph_stats(const hss_searcher* s, uint64_t* captures, uint64_t* replays, double* captureMs,
                             int32_t* failed) {
    if (!s) return SetError(HSS_ERR_INVALID, "null searcher");
    if (captures) *captures = s->s->GraphCaptures();
    if (replays) *replays = s->s->GraphReplays();
    if (captureMs) *captureMs = s->s->GraphCaptureMs();
    if (failed) *failed = s->s->GraphFailure().empty() ? 0 : 1;
    return HSS_OK;
}

int hss_searcher_last_times(const hss_searcher* s, float* ms5, uint32_t* retries, uint32_t* launches) {
    if (!s) return SetError(HSS_ERR_INVALID, "null searcher");
    const hss::StageTimes& t = s->s->LastTimes();
    if (ms5) {
        ms5[0] = t.filter;
        ms5[1] = t.sample;
        ms5[2] = t.candidates;
        ms5[3] = t.select;
        ms5[4] = t.total;
    }
    if (retries) *retries = t.retries;
    if (launches) *launches = t.launches;
    return HSS_OK;
}

// ---------------------------------------------------------------------------------------------
// codec

// ---------------------------------------------------------------------------------------------
// learned threshold predictor

uint32_t hss_searcher_feature_dim(const hss_searcher* s) { return s ? s->s->FeatureDim() : 0; }

int hss_searcher_features(hss_searcher* s, const float* dQueries, uint32_t nq, const hss_filters* filters,
                          const uint32_t* topks, float* dX, hss_stream_t stream) {
    if (!s || (nq && (!dQueries || !filters || !topks || !dX)) || (filters && filters->exprs.size() < nq))
        return SetError(HSS_ERR_INVALID, "hss_searcher_features: bad arguments");
    std::vector<const hss::FilterExpr*> ptrs(nq);
    for (uint32_t i = 0; i < nq; ++i) ptrs[i] = &filters->exprs[i];
    const int rc = s->s->Features(dQueries, nq, ptrs.data(), topks, dX, S(stream));
    if (rc == -1) return SetError(HSS_ERR_INVALID, s->s->Error());
    if (rc != 0) return SetError(rc < 0 ? HSS_ERR_CUDA : HSS_ERR_QUERY, s->s->Error());
    return HSS_OK;
}

int hss_searcher_set_threshold_model(hss_searcher* s, hss_model* model, float margin) {
    if (!s) return SetError(HSS_ERR_INVALID, "hss_searcher_set_threshold_model: null searcher");
    const int rc = s->s->SetThresholdModel(model ? model->m : nullptr, margin);
    if (rc == -1) return SetError(HSS_ERR_INVALID, s->s->Error());
    if (rc != 0) return SetError(HSS_ERR_CUDA, s->s->Error());
    return HSS_OK;
}

int hss_searcher_last_thresholds(const hss_searcher* s, float* sampleTheta, float* modelTheta, uint32_t n) {
    if (!s) return SetError(HSS_ERR_INVALID, "hss_searcher_last_thresholds: null searcher");
    const auto& t1 = s->s->LastSampleThreshold();
    const auto& ta = s->s->LastModelThreshold();
    for (uint32_t i = 0; i < n; ++i) {
        if (sampleTheta) sampleTheta[i] = i < t1.size() ? t1[i] : 0.0f;
        if (modelTheta) modelTheta[i] = i < ta.size() ? ta[i] : 0.0f;
    }
    return HSS_OK;
}

int hss_searcher_last_candidate_counts(hss_searcher* s, uint32_t* counts, uint32_t n) {
    if (!s || (n && !counts)) return SetError(HSS_ERR_INVALID, "hss_searcher_last_candidate_counts: bad arguments");
    const int rc = s->s->LastCandidateCounts(n, counts);
    if (rc == -1) return SetError(HSS_ERR_INVALID, "hss_searcher_last_candidate_counts: n beyond maxBatch");
    if (rc != 0) return SetError(HSS_ERR_CUDA, "hss_searcher_last_candidate_counts");
    return HSS_OK;
}

int hss_searcher_last_threshold_misses(const hss_searcher* s, uint8_t* miss, uint32_t n) {
    if (!s || (n && !miss)) return SetError(HSS_ERR_INVALID, "hss_searcher_last_threshold_misses: bad arguments");
    const auto& m = s->s->LastThresholdMisses();
    for (uint32_t i = 0; i < n; ++i) miss[i] = i < m.size() ? m[i] : 0;
    return HSS_OK;
}

int hss_model_create(int32_t deviceId, uint32_t din, uint32_t hidden, uint64_t seed, hss_model** out) {
    if (!out) return SetError(HSS_ERR_INVALID, "hss_model_create: null output");
    auto m = std::make_shared<hss::ThresholdModel>(deviceId, din, hidden, seed);
    if (!m->Ok()) return SetError(HSS_ERR_INVALID, m->Error());
    *out = new hss_model{m};
    return HSS_OK;
}

void hss_model_free(hss_model* m) { delete m; }

uint64_t hss_model_param_count(const hss_model* m) { return m ? m->m->ParamCount() : 0; }

int hss_model_get_params(const hss_model* m, float* params) {
    if (!m || !params) return SetError(HSS_ERR_INVALID, "hss_model_get_params: bad arguments");
    return m->m->GetParams(params) == 0 ? HSS_OK : SetError(HSS_ERR_CUDA, "hss_model_get_params");
}

int hss_model_set_params(hss_model* m, const float* params) {
    if (!m || !params) return SetError(HSS_ERR_INVALID, "hss_model_set_params: bad arguments");
    return m->m->SetParams(params) == 0 ? HSS_OK : SetError(HSS_ERR_CUDA, "hss_model_set_params");
}

int hss_model_set_output_scale(hss_model* m, float scale, float shift) {
    if (!m) return SetError(HSS_ERR_INVALID, "hss_model_set_output_scale: null model");
    m->m->scale = scale;
    m->m->shift = shift;
    return HSS_OK;
}

int hss_model_set_quantile(hss_model* m, float tau) {
    if (!m) return SetError(HSS_ERR_INVALID, "hss_model_set_quantile: null model");
    if (m->m->SetQuantile(tau) != 0) return SetError(HSS_ERR_INVALID, m->m->Error());
    return HSS_OK;
}

int hss_model_forward(hss_model* m, const float* dX, uint32_t B, float* dY, hss_stream_t stream) {
    if (!m || (B && (!dX || !dY))) return SetError(HSS_ERR_INVALID, "hss_model_forward: bad arguments");
    return m->m->Forward(dX, B, dY, S(stream)) == 0 ? HSS_OK : SetError(HSS_ERR_CUDA, m->m->Error());
}

int hss_model_train_step(hss_model* m, const float* dX, const float* dT, uint32_t B, float lr, float* loss,
                         hss_stream_t stream) {
    if (!m || B == 0 || !dX || !dT) return SetError(HSS_ERR_INVALID, "hss_model_train_step: bad arguments");
    return m->m->TrainStep(dX, dT, B, lr, loss, S(stream)) == 0 ? HSS_OK : SetError(HSS_ERR_CUDA, m->m->Error());
}

int hss_model_gradients(hss_model* m, const float* dX, const float* dT, uint32_t B, float* grad, float* loss,
                        hss_stream_t stream) {
    if (!m || B == 0 || !dX || !dT || !grad) return SetError(HSS_ERR_INVALID, "hss_model_gradients: bad arguments");
    return m->m->Gradients(dX, dT, B, grad, loss, S(stream)) == 0 ? HSS_OK : SetError(HSS_ERR_CUDA, m->m->Error());
}

// ---------------------------------------------------------------------------------------------
// serving loop

int hss_server_create(hss_table* table, const hss_server_config* cfg, hss_server** out) {
    if (!table || !out) return SetError(HSS_ERR_INVALID, "hss_server_create: null argument");
    hss::ServingConfig c;
    if (cfg) {
        if (cfg->slots) c.slots = cfg->slots;
        if (cfg->maxBatch) c.maxBatch = cfg->maxBatch;
        c.maxWaitUs = cfg->maxWaitUs;
        c.memoryBudget = cfg->memoryBudget;
        if (cfg->method < 0 || cfg->method > 3) return SetError(HSS_ERR_INVALID, "unknown scoring method");
        c.searcher.method = static_cast<hss::ScoreMethod>(cfg->method);
        if (cfg->candidateCap) c.searcher.candidateCap = cfg->candidateCap;
        if (cfg->sampleDocs) c.searcher.sampleDocs = cfg->sampleDocs;
        c.graphs = cfg->graphs != 0;
    }
    auto loop = std::make_unique<hss::ServingLoop>(table->t, c);
    if (!loop->Ok()) return SetError(HSS_ERR_CUDA, loop->Error());
    *out = new hss_server{std::move(loop)};
    return HSS_OK;
}

void hss_server_free(hss_server* s) { delete s; }

int hss_server_submit(hss_server* s, const float* vector, uint32_t dim, const char* filterExpr, uint32_t topK,
                      uint64_t* id) {
    if (!s) return SetError(HSS_ERR_INVALID, "hss_server_submit: null server");
    const int rc = s->s->Submit(vector, dim, filterExpr, topK, id);
    if (rc == -3) return SetError(HSS_ERR_PARSE, std::string("filter does not parse: ") + (filterExpr ? filterExpr : ""));
    if (rc == -4) return SetError(HSS_ERR_PROGRAM, "filter program rejected");
    if (rc != 0) return SetError(HSS_ERR_INVALID, "hss_server_submit: bad arguments");
    return HSS_OK;
}

int hss_server_wait(hss_server* s, uint64_t id, float* scores, int64_t* ids, uint32_t cap, uint32_t* count,
                    double* latencyMs, int32_t* status, int32_t timeoutMs) {
    if (!s) return SetError(HSS_ERR_INVALID, "hss_server_wait: null server");
    const int rc = s->s->Wait(id, scores, ids, cap, count, latencyMs, status, timeoutMs);
    if (rc < 0) return SetError(HSS_ERR_INVALID, "hss_server_wait: unknown request id");
    return rc;
}

int hss_server_get_stats(const hss_server* s, hss_server_stats* out) {
    if (!s || !out) return SetError(HSS_ERR_INVALID, "hss_server_get_stats: null argument");
    const hss::ServingStats st = s->s->Stats();
    out->completed = st.completed;
    out->batches = st.batches;
    out->slots = st.slots;
    out->meanBatch = st.meanBatch;
    out->p50Ms = st.p50Ms;
    out->p99Ms = st.p99Ms;
    out->maxMs = st.maxMs;
    out->graphCaptures = st.graphCaptures;
    out->graphReplays = st.graphReplays;
    out->graphCaptureMs = st.graphCaptureMs;
    return HSS_OK;
}

int hss_server_reset_stats(hss_server* s) {
    if (!s) return SetError(HSS_ERR_INVALID, "hss_server_reset_stats: null server");
    s->s->ResetStats();
    return HSS_OK;
}

int hss_server_set_threshold_model(hss_server* s, hss_model* model, float margin) {
    if (!s) return SetError(HSS_ERR_INVALID, "hss_server_set_threshold_model: null server");
    if (s->s->SetThresholdModel(model ? model->m : nullptr, margin) != 0)
        return SetError(HSS_ERR_INVALID, "threshold model does not fit this server's searchers");
    return HSS_OK;
}

int hss_server_run_poisson(hss_server* s, const float* queries, uint32_t n, const char* const* filterExprs,
                           const uint32_t* topks, double rateQps, uint64_t seed, double* latencyMs,
                           double* offeredQps, double* wallSeconds) {
    if (!s || !queries || !filterExprs || !topks || rateQps <= 0)
        return SetError(HSS_ERR_INVALID, "hss_server_run_poisson: bad arguments");
    const int bad = s->s->RunPoisson(queries, n, filterExprs, topks, rateQps, seed, latencyMs, offeredQps, wallSeconds);
    if (bad < 0) return SetError(HSS_ERR_INVALID, "hss_server_run_poisson: bad arguments");
    if (bad > 0) return SetError(HSS_ERR_QUERY, std::to_string(bad) + " queries failed");
    return HSS_OK;
}

uint64_t hss_hash64(const char* data, uint32_t len) { return hss::Hash64(data, len); }

int64_t hss_posting_serialize(const uint32_t* ids, uint32_t n, uint32_t docNum, int32_t isMatrix,
                              float densityThreshold, int32_t sparsePacked, uint8_t* out, uint64_t cap) {
    if ((n && !ids) || !out) return SetError(HSS_ERR_INVALID, "null argument");
    std::vector<uint32_t> v(ids, ids + n);
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    std::string buf;
    if (!hss::PostingSerializer::Serialize(v, docNum, isMatrix != 0, densityThreshold, sparsePacked != 0, buf))
        return SetError(HSS_ERR_INVALID, "posting cannot be serialised");
    if (buf.size() > cap) return SetError(HSS_ERR_LIMIT, "output buffer too small");
    std::memcpy(out, buf.data(), buf.size());
    return static_cast<int64_t>(buf.size());
}

int hss_filter_compile(const hss_table* table, const char* filterExpr, uint32_t* prog, uint32_t progCap,
                       uint32_t* progLen, uint32_t* rows, uint32_t rowCap, uint32_t* rowLen, uint32_t* opNum,
                       int32_t* emptyTree) {
    if (!table || !progLen || !rowLen) return SetError(HSS_ERR_INVALID, "null argument");
    bool ok = true;
    auto ast = hss::ParseFilter(filterExpr ? filterExpr : "", ok);
    if (!ok) return SetError(HSS_ERR_PARSE, "filter does not parse");
    auto tree = hss::BuildQueryNode(ast.get(), table->t->GetConfig().postingField);
    hss::FilterExpr e;
    std::string err;
    if (!hss::PrepareExpr(tree.get(), *table->t, e, &err)) return SetError(HSS_ERR_PROGRAM, err);
    *progLen = static_cast<uint32_t>(e.postExpr.size());
    *rowLen = static_cast<uint32_t>(e.postingRows.size());
    if (opNum) *opNum = e.opNum;
    if (emptyTree) *emptyTree = e.emptyTree ? 1 : 0;
    if (*progLen > progCap || *rowLen > rowCap) return SetError(HSS_ERR_LIMIT, "output buffers too small");
    if (prog) std::copy(e.postExpr.begin(), e.postExpr.end(), prog);
    if (rows) std::copy(e.postingRows.begin(), e.postingRows.end(), rows);
    return HSS_OK;
}

}  // extern "C"
