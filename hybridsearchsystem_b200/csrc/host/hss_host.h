// hss_host.h -- host-side C++ mirror of the reference's filtered full-recall interface:
//   Hash64                        (src/engine/core/hash/hash.h:15-20)
//   FilterNode / ParseFilter      (src/harness/query/filter_expr.h:19-177)
//   PostingLayout / serializer    (src/engine/format/posting_layout.h:8, posting_serializer.h)
//   QueryNode family              (src/engine/retrieval/query/query_node.h, query_node_imp.h)
//   DataTable                     (src/engine/index/data_table.h:10-92)
//   FullRecallSearcher / Result   (src/engine/retrieval/searcher/full_recall_searcher.h:12-47,
//                                  src/engine/core/full_recall_result.h:30-50)
// Names and argument meanings follow the reference; the device work goes to the CUDA kernels of
// libhss.so instead of the AscendC operators.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "../hss_kernels.h"

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace hss {

// ---------------------------------------------------------------------------------------------
// Token hash: MurmurHash3_x64_128(seed 0x20160713), h1 ^ h2 (hash.cpp:10-16).
uint64_t Hash64(const char* data, uint32_t len);
inline uint64_t Hash64(const std::string& s) { return Hash64(s.data(), static_cast<uint32_t>(s.size())); }

// ---------------------------------------------------------------------------------------------
// Filter expression AST and parser. Grammar, precedence NOT > AND > OR, n-ary AND/OR flattening
// and the empty-expression = match-all rule are the reference's (filter_expr.h:1-8,164-177).
enum class FilterOp { Term, And, Or, Not };

struct FilterNode {
    FilterOp op = FilterOp::Term;
    uint64_t tag = 0;  // valid when op == Term
    std::vector<std::unique_ptr<FilterNode>> children;
};

// nullptr with ok = true: empty expression (match all). nullptr with ok = false: parse error.
std::unique_ptr<FilterNode> ParseFilter(const std::string& expr, bool& ok);

// ---------------------------------------------------------------------------------------------
// Posting codec (on-disk format contract, posting_serializer.cpp:15-208).
enum class PostingLayout { DENSE_BITMAP = 0, SPARSE_BITMAP, DENSE_BYTEMAP, SPARSE_IDLIST, SPARSE_PACKED, UNKNOWN };

class PostingSerializer {
   public:
    // docIds: the segment-local ids of the hits, sorted ascending without duplicates. Appends the
    // posting (8-byte head + payload) to `buffer`. SPARSE_IDLIST ids are written ascending.
    static bool Serialize(const std::vector<uint32_t>& docIds, uint32_t docNum, bool isMatrixType,
                          float densityThreshold, bool sparsePacked, std::string& buffer);
    static PostingLayout SelectLayout(bool isMatrixType, uint32_t targetDocNum, uint32_t docNum,
                                      float densityThreshold, bool sparsePacked);
};

// Structural check of one posting for a segment of segDocs docs: known layout, payload inside the
// buffer and legal for the layout, sparse units sorted, strictly increasing and in range.
bool ValidatePosting(const uint8_t* p, size_t len, uint32_t segDocs, std::string* err);

// ---------------------------------------------------------------------------------------------
class DataTable;

enum class QueryNodeType { AndNode = 1, OrNode, NotNode, TermNode, TermsNode, OrTermsNode, ConjunctionNode };
enum FilterOpType : uint32_t { CONJUNCTION = 0, AND = 1, OR = 2, NOT = 3 };

// A compiled filter: the reference's postfix program (query_node_imp.cpp:8-47,65-96,295-342) plus,
// per operand, the posting row of the DataTable it reads.
struct FilterExpr {
    std::vector<uint32_t> postExpr;
    std::vector<uint32_t> postingRows;
    uint32_t opNum = 0;
    bool emptyTree = false;  // match all
};

class QueryNode {
   public:
    virtual ~QueryNode() = default;
    void AddChild(std::unique_ptr<QueryNode>& child);
    uint32_t GetChildrenNum() const { return static_cast<uint32_t>(m_children.size()); }
    virtual QueryNodeType GetNodeType() const = 0;
    virtual std::string GetName() const = 0;
    // Appends this subtree's postfix code; false when the subtree contributes nothing.
    virtual bool GetPostOrderExpression(const DataTable& table, FilterExpr& out) const = 0;

   protected:
    std::vector<std::unique_ptr<QueryNode>> m_children;
};

class QueryLeafNode : public QueryNode {
   public:
    virtual bool AppendPostings(const DataTable& table, FilterExpr& out) const = 0;
};

class AndNode : public QueryNode {
   public:
    QueryNodeType GetNodeType() const override { return QueryNodeType::AndNode; }
    std::string GetName() const override { return "and"; }
    bool GetPostOrderExpression(const DataTable& table, FilterExpr& out) const override;
};

class OrNode : public QueryNode {
   public:
    QueryNodeType GetNodeType() const override { return QueryNodeType::OrNode; }
    std::string GetName() const override { return "or"; }
    bool GetPostOrderExpression(const DataTable& table, FilterExpr& out) const override;
};

class NotNode : public QueryNode {
   public:
    QueryNodeType GetNodeType() const override { return QueryNodeType::NotNode; }
    std::string GetName() const override { return "not"; }
    bool GetPostOrderExpression(const DataTable& table, FilterExpr& out) const override;
};

class TermNode : public QueryLeafNode {
   public:
    TermNode(const std::string& fieldName, uint64_t token) : m_fieldName(fieldName), m_token(token) {}
    QueryNodeType GetNodeType() const override { return QueryNodeType::TermNode; }
    std::string GetName() const override { return "term:" + m_fieldName + ":" + std::to_string(m_token); }
    bool GetPostOrderExpression(const DataTable& table, FilterExpr& out) const override;
    bool AppendPostings(const DataTable& table, FilterExpr& out) const override;

   private:
    std::string m_fieldName;
    uint64_t m_token;
};

class TermsNode : public QueryLeafNode {
   public:
    TermsNode(const std::string& fieldName, std::vector<uint64_t> tokens)
        : m_fieldName(fieldName), m_tokens(std::move(tokens)) {}
    QueryNodeType GetNodeType() const override { return QueryNodeType::TermsNode; }
    std::string GetName() const override { return "terms:" + m_fieldName; }
    bool GetPostOrderExpression(const DataTable& table, FilterExpr& out) const override;
    bool AppendPostings(const DataTable& table, FilterExpr& out) const override;

   private:
    std::string m_fieldName;
    std::vector<uint64_t> m_tokens;
};

class OrTermsNode : public QueryLeafNode {
   public:
    QueryNodeType GetNodeType() const override { return QueryNodeType::OrTermsNode; }
    std::string GetName() const override { return "or_terms"; }
    bool GetPostOrderExpression(const DataTable& table, FilterExpr& out) const override;
    bool AppendPostings(const DataTable& table, FilterExpr& out) const override;
};

class ConjunctionNode : public QueryNode {
   public:
    QueryNodeType GetNodeType() const override { return QueryNodeType::ConjunctionNode; }
    std::string GetName() const override { return "conjunction"; }
    bool GetPostOrderExpression(const DataTable& table, FilterExpr& out) const override;
};

// Harness translation of a parsed filter (filter_setup.cpp:96-137): a Term becomes a TermNode on
// Hash64(decimal tag); a null AST becomes an empty AndNode (match all).
std::unique_ptr<QueryNode> BuildQueryNode(const FilterNode* n, const std::string& field);

// Builds the postfix program (TextFilter::PrepareExpr, text_filter.cpp:432-467) and validates it
// (CheckPostExpr, :1314-1352). Returns false on an invalid program.
bool PrepareExpr(const QueryNode* tree, const DataTable& table, FilterExpr& out, std::string* err);
bool CheckPostExpr(const std::vector<uint32_t>& postExpr, uint32_t postingNums);

// ---------------------------------------------------------------------------------------------
struct IndexConfig {
    uint32_t docNumPerSegment = 131072;  // multiple of 128
    float densityThreshold = 1.0f / 64.0f;
    bool matrixPosting = false;  // DENSE_BYTEMAP / SPARSE_IDLIST instead of the bitmap layouts
    bool sparsePacked = false;   // SPARSE_PACKED instead of SPARSE_BITMAP
    uint64_t docOffset = 0;      // global doc id of location 0
    std::string postingField = "content";
    std::string vectorField = "content";
};

// Index residency on one GPU. Device layout:
//   vectors    FP32 [tiles*128][dim] row-major, rows past docNum zero
//   postings   one arena; every posting copied to a 16-byte aligned slot, zero-padded
//   postingTable u64 [rows][segments]: device address of token row r's posting in segment s (the
//              all-zero posting where the token is absent); the last row is the all-zero token
//   gdocids    int64 [docNum], location -> global doc id
class DataTable {
   public:
    DataTable() = default;
    ~DataTable();
    DataTable(const DataTable&) = delete;
    DataTable& operator=(const DataTable&) = delete;

    // Offline build (fr_converter + fr_builder) from HYDSET2-style arrays: vectors [docNum][dim] and
    // per-doc tag bitmaps [docNum][ceil(tagNum/64)]; tag t is the token Hash64(to_string(t)).
    // deviceId < 0 keeps the table on the host only (index build, filter compilation, Save).
    bool Build(int32_t deviceId, const float* vectors, const uint64_t* tagBits, uint64_t docNum, uint32_t dim,
               uint32_t tagNum, const IndexConfig& cfg, std::string* err);
    // The same build from vectors already resident on deviceId (dVectors, [docNum][dim] device
    // memory, copied into the table's own allocation): corpora too large to stage through the host.
    // The tag bitmaps are host arrays (the postings are built on the host).
    bool BuildFromDevice(int32_t deviceId, const float* dVectors, const uint64_t* tagBits, uint64_t docNum,
                         uint32_t dim, uint32_t tagNum, const IndexConfig& cfg, std::string* err);
    // DataTable::LoadData (data_table.cpp:35-124) over the index directory Save() writes.
    bool LoadData(int32_t deviceId, const std::string& dataDir, std::string* err);
    bool Save(const std::string& dataDir, std::string* err) const;
    // The reference's own index directory (what its fr_builder writes, read as its
    // DataTable::LoadData does, data_table.cpp:35-124,147-186): poissonengine_<ver>.meta (IndexMeta
    // as protobuf JSON), id/poissonengine_<ver>_<seg>.idm (u64 global ids), per vector field
    // <field>/poissonengine_<ver>_<seg>_<field>.vector (FP16 in Zn blocks, vector_builder.cpp:34-176)
    // and per posting field the posting files. The first vector and posting fields of the schema are
    // loaded; the FP16 vectors become FP32 rows (exactly).
    bool LoadReferenceIndex(int32_t deviceId, const std::string& dataDir, std::string* err);
    // Writes that directory (the reference's builder output format; vectors rounded to FP16 as its
    // Float32ToFloat16 rounds them, Zn = splitDocNumZn docs per block).
    bool SaveReferenceIndex(const std::string& dataDir, uint32_t splitDocNumZn, std::string* err) const;
    // Where the last LoadData / LoadReferenceIndex spent its time (ms) and moved its bytes.
    struct LoadTimes {
        double meta = 0, postingsRead = 0, vectorsRead = 0, vectorsH2D = 0, postingsH2D = 0, total = 0;
        uint64_t vectorBytes = 0, postingBytes = 0;
        uint32_t threads = 0;
    };
    const LoadTimes& GetLoadTimes() const { return m_loadTimes; }

    int32_t GetDeviceId() const { return m_deviceId; }
    uint64_t GetDocNum() const { return m_docNum; }
    uint32_t GetDimension() const { return m_dim; }
    uint32_t GetSegmentNum() const { return m_segmentNum; }
    uint32_t GetDocNumPerSegment() const { return m_cfg.docNumPerSegment; }
    uint32_t GetSegmentLength() const { return m_cfg.docNumPerSegment / 16; }
    uint32_t GetSegmentByteSize() const { return m_cfg.docNumPerSegment / 8; }
    uint64_t GetTileNum() const { return (m_docNum + 127) / 128; }
    uint64_t GetBitmapWords() const { return static_cast<uint64_t>(m_segmentNum) * (m_cfg.docNumPerSegment / 64); }
    const IndexConfig& GetConfig() const { return m_cfg; }
    float GetMaxNorm() const { return m_maxNorm; }
    const std::unordered_set<std::string>& GetPostingFields() const { return m_postingFields; }

    const float* DeviceVectors() const { return m_dVectors; }
    const uint64_t* DevicePostingTable() const { return m_dPostingTable; }
    const int64_t* DeviceGDocIds() const { return m_dGDocIds; }
    uint32_t PostingRows() const { return m_rows; }

    // Row of the posting table for a token; the all-zero row when the token is absent
    // (PostingFieldData::GetData, posting_field_data.cpp:487-495). tokenExist reports which.
    uint32_t TokenRow(uint64_t token, bool& tokenExist) const;
    // Tensor-core scoring formats (TcFormat: 0 TF32 over the FP32 rows, 1 BF16 copy, 2 E4M3 copy with
    // per-vector scales). Builds the copy on the device and measures max ||v|| and max ||v~ - v||.
    bool EnableFormat(int format, std::string* err);
    bool HasFormat(int format) const { return format >= 0 && format < 3 && m_fmtReady[format]; }
    const void* DeviceRows(int format) const { return format == 0 ? static_cast<const void*>(m_dVectors) : m_dQuant[format]; }
    const float* DeviceDocScale() const { return m_dDocScale; }
    const float2* DeviceTileScale() const { return m_dTileScale; }
    double NormMax(int format) const { return m_fmtNormMax[format]; }
    double ErrMax(int format) const { return m_fmtErrMax[format]; }

    // Every posting of the table expanded into a dense bitmap (all five layouts decoded once):
    // u64 [rows][segments][docNumPerSegment / 64], 16-byte aligned rows, when its size fits
    // budgetBytes (else nothing is built and batches decode the postings in place). A malformed
    // posting also leaves it unbuilt, so the in-place path reports it per query.
    bool EnableDensePostings(uint64_t budgetBytes, std::string* err);
    const uint64_t* DeviceDensePostings() const { return m_dDense; }
    // Fraction of the docs that hold each posting row's token (float [rows], device).
    const float* DeviceRowDensity() const { return m_dRowDensity; }
    // Host copy of segment s's posting of a token row (for tests / save); null if absent.
    const uint8_t* HostPosting(uint32_t row, uint32_t seg, uint32_t* len) const;
    // Layout code of each posting of a row (PostingFieldData::GetPostingTypes).
    std::vector<uint8_t> PostingTypes(uint32_t row) const;

   private:
    bool Upload(std::string* err);
    bool WritePostingFiles(const std::string& dir, std::string* err) const;
    // Posting files of one field (version `ver` in their names) into the host posting tables.
    bool ReadPostingFiles(const std::string& dir, const std::string& field, uint32_t ver, std::string* err);
    // The table's FP32 rows, produced by fill(r0, r1, dst) (rows [r0, r1) into dst, called from
    // several threads on disjoint ranges), to the device through two pinned staging chunks (filling
    // one while the other is copied), then the norm bound, the postings and the doc ids. With
    // deviceId < 0 the rows are kept on the host.
    bool FinishRows(int32_t deviceId, const std::function<void(uint64_t, uint64_t, float*)>& fill, std::string* err);
    bool BuildImpl(int32_t deviceId, const float* vectors, bool onDevice, const uint64_t* tagBits, uint64_t docNum,
                   uint32_t dim, uint32_t tagNum, const IndexConfig& cfg, std::string* err);
    void Release();

    int32_t m_deviceId = -1;
    IndexConfig m_cfg;
    uint64_t m_docNum = 0;
    uint32_t m_dim = 0;
    uint32_t m_segmentNum = 0;
    uint32_t m_rows = 0;  // token rows + 1 (the all-zero row)
    float m_maxNorm = 0.0f;
    std::unordered_set<std::string> m_postingFields;
    LoadTimes m_loadTimes;

    // host side
    std::vector<float> m_vectors;            // [docNum][dim]
    std::vector<int64_t> m_gdocids;          // [docNum]
    std::vector<uint64_t> m_tokens;          // row -> token hash
    std::vector<std::string> m_tokenText;    // row -> token literal
    std::unordered_map<uint64_t, uint32_t> m_tokenRow;
    std::vector<std::string> m_segPostings;  // per segment: concatenated postings (4-byte padded)
    std::vector<std::vector<int64_t>> m_rowSegOffset;  // [row][seg] offset into m_segPostings[seg], -1 absent
    std::vector<std::vector<uint32_t>> m_rowSegLen;

    // device side
    float* m_dVectors = nullptr;
    void* m_dQuant[3] = {nullptr, nullptr, nullptr};
    float* m_dDocScale = nullptr;
    float2* m_dTileScale = nullptr;
    bool m_fmtReady[3] = {false, false, false};
    double m_fmtNormMax[3] = {0, 0, 0};
    double m_fmtErrMax[3] = {0, 0, 0};
    uint8_t* m_dArena = nullptr;
    uint64_t* m_dPostingTable = nullptr;
    int64_t* m_dGDocIds = nullptr;
    uint64_t* m_dDense = nullptr;  // EnableDensePostings
    float* m_dRowDensity = nullptr;  // [rows] fraction of docs holding each row's token
};

// ---------------------------------------------------------------------------------------------
struct ScoreWithIndex {
    float score;
    uint32_t index;
    uint64_t id{0};
    ScoreWithIndex(float s, uint32_t i) : score(s), index(i) {}
};

struct FullRecallResult {
    bool isMultiShard = false;
    std::vector<ScoreWithIndex> scoreWithIndexes;  // multi-shard form (unsorted merge input)
    std::vector<float> scores;                     // single-shard form, (score desc, doc id asc)
    std::vector<int64_t> docIds;
};

// Scoring method of the bulk candidate pass: FP32 FFMA on the SIMT cores, or the tensor cores over
// the FP32 rows (TF32), a BF16 copy or an FP8 E4M3 copy of the corpus. Every method is followed by
// the same exact FP32 rescoring, so all return the ground truth's results.
enum class ScoreMethod : int32_t { SIMT_FP32 = 0, TC_TF32 = 1, TC_BF16 = 2, TC_E4M3 = 3 };

struct SearcherConfig {
    uint32_t maxBatch = 256;
    uint32_t candidateCap = 1u << 18;  // per-query candidate list capacity (>= 4096)
    uint32_t sampleDocs = 32768;       // minimum doc sample for the candidate threshold
    uint32_t maxRetries = 4;           // candidate-overflow re-runs before a query fails
    ScoreMethod method = ScoreMethod::SIMT_FP32;
    bool densePostings = true;         // filter batches over the table's dense posting matrix
};

// Timing of the stages of the last batch (CUDA events, milliseconds).
struct StageTimes {
    float filter = 0, sample = 0, candidates = 0, select = 0, total = 0;
    uint32_t retries = 0;
    uint32_t launches = 0;
};

// The learned threshold predictor: an MLP (features -> H -> H -> 1, GELU) on one GPU, trained and
// run by the kernels of mlp.cu. It predicts a standardised K-th filtered score; scale / shift map the
// output back to a score. Parameters: one flat FP32 vector W1 [din][H], b1, W2 [H][H], b2, w3 [H], b3.
class ThresholdModel {
   public:
    ThresholdModel(int32_t deviceId, uint32_t din, uint32_t hidden, uint64_t seed);
    ~ThresholdModel();
    ThresholdModel(const ThresholdModel&) = delete;
    ThresholdModel& operator=(const ThresholdModel&) = delete;

    bool Ok() const { return m_ok; }
    const std::string& Error() const { return m_err; }
    int32_t DeviceId() const { return m_deviceId; }
    uint32_t Din() const { return m_din; }
    uint32_t Hidden() const { return m_h; }
    size_t ParamCount() const { return m_np; }

    // y[B] (standardised) of device features dX [B][din], in one launch.
    int Forward(const float* dX, uint32_t B, float* dY, cudaStream_t s);
    // The training loss: 0 (the default) the mean squared error, tau in (0, 1) the pinball loss of the
    // tau-quantile (the network then predicts a conditional tau-quantile of the target).
    int SetQuantile(float tau);
    float Quantile() const { return m_tau; }
    // One Adam step on the loss over a batch of device features / standardised targets.
    int TrainStep(const float* dX, const float* dT, uint32_t B, float lr, float* hLoss, cudaStream_t s);
    // The gradient of the loss at the current parameters, into a host vector of ParamCount().
    int Gradients(const float* dX, const float* dT, uint32_t B, float* hGrad, float* hLoss, cudaStream_t s);
    int GetParams(float* h) const;
    int SetParams(const float* h);

    float scale = 1.0f, shift = 0.0f;  // score = y * scale + shift

   private:
    size_t OffW1() const { return 0; }
    size_t OffB1() const { return static_cast<size_t>(m_din) * m_h; }
    size_t OffW2() const { return OffB1() + m_h; }
    size_t OffB2() const { return OffW2() + static_cast<size_t>(m_h) * m_h; }
    size_t OffW3() const { return OffB2() + m_h; }
    size_t OffB3() const { return OffW3() + m_h; }
    bool Reserve(uint32_t batch);
    cudaError_t ForwardInto(const float* dX, uint32_t B, cudaStream_t s);
    cudaError_t Backward(const float* dX, const float* dT, uint32_t B, cudaStream_t s);
    int Finish(cudaError_t e, float* hLoss, uint32_t B, cudaStream_t s);

    int32_t m_deviceId;
    uint32_t m_din, m_h;
    float m_tau = 0.0f;
    size_t m_np = 0;
    bool m_ok = false;
    std::string m_err;
    int m_step = 0;
    uint32_t m_cap = 0;
    float *m_dP = nullptr, *m_dG = nullptr, *m_dM = nullptr, *m_dV = nullptr;
    float *m_dZ1 = nullptr, *m_dA1 = nullptr, *m_dZ2 = nullptr, *m_dA2 = nullptr;
    float *m_dY = nullptr, *m_dDy = nullptr, *m_dD1 = nullptr, *m_dD2 = nullptr, *m_dSq = nullptr;
};

class FullRecallSearcher {
   public:
    // dArena: a caller-owned device arena of at least WorkspaceBytes(table, cfg) bytes (256-byte
    // aligned, on the table's device) that holds every device buffer of the searcher and is never
    // freed by it; null: the searcher allocates that arena itself (one cudaMalloc).
    FullRecallSearcher(int32_t deviceId, std::shared_ptr<DataTable> dataTable, const SearcherConfig& cfg = {},
                       void* dArena = nullptr, size_t arenaBytes = 0);
    ~FullRecallSearcher();
    // Device bytes of a searcher's arena for this table and configuration: the filter bitmaps,
    // candidate lists, select workspace, doc sample, staging, results and model features (the
    // reference's named pools hold the same kinds of blocks, gm_memory_manager.cpp:9-47).
    static size_t WorkspaceBytes(const DataTable& table, const SearcherConfig& cfg);
    FullRecallSearcher(const FullRecallSearcher&) = delete;
    FullRecallSearcher& operator=(const FullRecallSearcher&) = delete;

    bool Ok() const { return m_ok; }
    const std::string& Error() const { return m_err; }

    // FullRecallSearcher::AddQuery (full_recall_searcher.cpp:93-105); queries stay FP32.
    void AddQuery(QueryNode* queryTree, const std::vector<float>& queryVector, uint32_t topK);
    void ClearQueries();
    // FullRecallSearcher::BatchSearch (full_recall_searcher.cpp:107-231): runs every added query,
    // fills one result per query, clears the added queries.
    bool BatchSearch(std::vector<std::shared_ptr<FullRecallResult>>& results, const std::string& vectorFieldName,
                     bool isMultiShard);

    // Device-resident batch: queries [nq][dim] and results live in device memory; the filters were
    // compiled by PrepareExpr. Synchronises `stream` once (to read the overflow status). Returns the
    // number of failed queries, or a negative status.
    int SearchDevice(const float* dQueries, uint32_t nq, const FilterExpr* const* exprs, const uint32_t* topks,
                     float* dOutScores, int64_t* dOutIds, uint32_t* dOutCounts, uint32_t outStride,
                     cudaStream_t stream);
    // SearchDevice in two halves, so that a caller can keep the GPU busy while it waits: the first
    // enqueues the whole batch on `stream` (its host work -- filter compilation into the staging
    // buffer, launch planning -- done) and returns without waiting; the second waits for the batch's
    // statuses, runs any candidate-overflow re-runs (enqueued on the same stream, then waited for) and
    // returns what SearchDevice returns. The queries and outputs must stay valid until it returns; the
    // searcher takes no other batch in between (two searchers alternate to overlap batches).
    int SearchEnqueue(const float* dQueries, uint32_t nq, const FilterExpr* const* exprs, const uint32_t* topks,
                      float* dOutScores, int64_t* dOutIds, uint32_t* dOutCounts, uint32_t outStride,
                      cudaStream_t stream);
    int SearchFinish();
    bool Pending() const { return m_b.pending; }

    // Filter stage alone (FullRecallSearcher::OneFilter, full_recall_searcher.cpp:233-262): the
    // per-query doc bitmaps [nq][outStrideWords] and pass counts; synchronises `stream` once.
    int FilterDevice(uint32_t nq, const FilterExpr* const* exprs, uint64_t* dOutBits, uint64_t outStrideWords,
                     uint32_t* dPassCounts, cudaStream_t stream);

    // The last batch's candidate list of query q (approximate scores, locations), its threshold and
    // error bound; for checking the approximate pass against the exact scores.
    int LastCandidates(uint32_t q, float* scores, uint32_t* locs, uint32_t cap, uint32_t* count, float* theta,
                       float* eps);

    // Learned threshold: with a model set, the doc sample stays at sampleDocs whatever K (it feeds the
    // model's features and gives the proven threshold theta_1), and the passes run at
    // max(theta_1, prediction - margin - eps). That threshold is not proven: the select step checks,
    // per query, that the K-th best exact score clears it by eps; a query that fails (a "miss") is
    // re-run at a proven threshold. A bad prediction costs candidates or a re-run, never exactness.
    // nullptr switches the model off.
    int SetThresholdModel(std::shared_ptr<ThresholdModel> model, float margin);
    // Width of a query's feature row: dim + posting rows + 12.
    uint32_t FeatureDim() const;
    // Feature rows [nq][FeatureDim()] of a batch (runs the filter stage and the doc sample).
    int Features(const float* dQueries, uint32_t nq, const FilterExpr* const* exprs, const uint32_t* topks,
                 float* dX, cudaStream_t stream);
    // Per query of the last batch: the doc sample's proven threshold theta_1, and the threshold the
    // model set (-inf without a model).
    const std::vector<float>& LastSampleThreshold() const { return m_lastTheta1; }
    const std::vector<float>& LastModelThreshold() const { return m_lastThetaA; }
    // Per query of the last batch: 1 when the model's threshold failed the check and the query was
    // re-run at a proven one.
    const std::vector<uint8_t>& LastThresholdMisses() const { return m_lastMiss; }
    // Per query of the last batch: the docs that cleared the threshold of its last candidate pass
    // (those the select step read, plus any beyond the list's capacity). Reads the device; call before
    // the next batch.
    int LastCandidateCounts(uint32_t n, uint32_t* counts);

    static constexpr uint32_t kRerunSplit = 16;  // a tensor-core re-run's first part: every 16th tile

    // Pipeline test: the next batch's first single-SM tensor-core pass stops issuing corpus loads
    // before its holdLoad-th, with waitBudget clock cycles (0: the default) for its waits; the pass
    // then aborts through its bounded-wait path and the batch reports the error.
    void SetPipelineTest(uint32_t holdLoad, long long waitBudget) {
        m_testHold = holdLoad;
        m_testBudget = waitBudget;
    }
    // CUDA-graph replay of a batch's first attempt (filter, bounds, doc sample, model, both candidate
    // passes, select and the status copies). The launches of one batch shape are captured from the
    // stream once and replayed for every later batch of that shape, the graph copying in each
    // batch's own filter programs. A shape is: the rows, rounded up to 1, 2, 4, 8, 16 or a multiple
    // of 16 (at most maxBatch); the largest K, rounded up to a power of two (every K that plans
    // like K = 1 -- the same doc sample and select variant -- counting as one); the largest operand
    // count, rounded up to a power of two; the model; the query and output buffers and the output
    // stride. Rows past nq run as match-nothing queries with K = 1, so with graphs on, dQueries and
    // the outputs must hold maxBatch rows. Re-runs are launched directly. Off by default; batches
    // with timing on, Features and the pipeline test launch directly. At most kGraphCacheSize
    // shapes are kept (least recently used dropped).
    void SetGraphs(bool on);
    uint64_t GraphCaptures() const { return m_graphCaptures; }
    uint64_t GraphReplays() const { return m_graphReplays; }
    double GraphCaptureMs() const { return m_graphCaptureMs; }  // host time in captures and instantiation
    // Why a capture failed (graphs then stay off for this searcher); empty when none did.
    const std::string& GraphFailure() const { return m_graphFailure; }
    static constexpr size_t kGraphCacheSize = 128;
    // The rows a batch runs with under graph replay; K and operand counts rounded up to powers of two.
    static uint32_t GraphRows(uint32_t nq, uint32_t maxBatch);
    static uint32_t GraphTopK(uint32_t maxK);
    static uint32_t GraphOperands(uint32_t maxOpnd);
    // The K a batch's launch plan is made for under graph replay.
    uint32_t PlanTopK(uint32_t maxK) const;

    const StageTimes& LastTimes() const { return m_times; }
    void SetTiming(bool on) { m_timing = on; }
    const SearcherConfig& Config() const { return m_cfg; }
    // Per-query device status bits of the last batch (kStatus* values).
    const std::vector<int32_t>& LastStatus() const { return m_lastStatus; }

   private:
    struct ArenaLayout {
        size_t bits, candScore, candLoc, work, sampScore, sampLoc, stage, queries, outScore, outId, outCount, stats,
            features, predictions, staged, qScale, error, total;
        size_t stageBytes;
        uint32_t sampCap;
    };
    static ArenaLayout Layout(const DataTable& table, const SearcherConfig& cfg);
    bool Allocate(void* dArena, size_t arenaBytes);
    // The batch between SearchEnqueue and SearchFinish.
    struct Batch {
        const float* dQueries = nullptr;
        uint32_t nq = 0;
        cudaStream_t stream = nullptr;
        SelectLaunch se{};
        uint32_t launches = 0;
        uint64_t want = 0;        // doc-sample size of the batch
        uint64_t wantRerun = 0;   // doc-sample size of a SIMT re-run (grows with K, model or not)
        bool pending = false, learned = false;
        cudaError_t ce = cudaSuccess;
    };
    void Ck(cudaError_t e) {
        if (m_b.ce == cudaSuccess && e != cudaSuccess) m_b.ce = e;
    }
    // Launch planning of the candidate passes (see SearchEnqueue).
    bool UseSimt(bool simt) const { return m_tcFormat < 0 || simt; }
    uint32_t UnitOf(uint32_t rows, bool simt) const;
    uint64_t TilesOf(uint32_t unit) const;
    uint32_t CtasOf(uint32_t rows, uint64_t countTiles, uint32_t cap, bool simt) const;
    uint32_t SegsOf(uint32_t rows, uint64_t countTiles, uint32_t cap, bool simt) const;
    uint32_t SegCapOf(uint32_t rows, uint64_t countTiles, uint32_t cap, uint32_t segs, bool simt) const;
    void Stage(const uint32_t* dList, uint32_t rows);
    void Cand(const float* theta, float* score, uint32_t* loc, uint32_t* count, uint32_t cap, uint32_t segBase,
              uint32_t segCap, uint64_t begin, uint64_t step, uint32_t skip, uint64_t countTiles, const uint32_t* dList,
              uint32_t rows, bool simt);
    // The doc sample of m_b.want docs and its threshold (raised, with raiseOnly); the pass keeps the
    // filtered docs at or above emitTheta (null: every filtered doc).
    uint64_t Sample(const uint32_t* dList, uint32_t rows, bool simt, bool raiseOnly = false, float* stats = nullptr,
                    float* thetaCopy = nullptr, const float* emitTheta = nullptr);
    void SampleTiles(uint64_t want, uint32_t rows, bool simt, uint64_t* count, uint64_t* step) const;
    // A batch's small inputs in the pinned staging buffer: per-query program and operand offsets, K,
    // the programs and then their operands (operand offsets count from the program array's start);
    // rows [nq, rows) as match-nothing queries with K = padK.
    struct BatchInputs {
        uint32_t maxK = 0, maxOpnd = 0, np = 0, no = 0;
    };
    BatchInputs PrepareInputs(uint32_t nq, uint32_t rows, const FilterExpr* const* exprs, const uint32_t* topks,
                              uint32_t padK);
    // Bytes of the batch's one host-to-device input copy.
    size_t InputBytes(const BatchInputs& in) const;
    // Their copy to the device and the filter launch over `rows` queries.
    int EnqueueFilter(uint32_t rows, const BatchInputs& in, uint64_t* dBits, uint64_t bitsStride, cudaStream_t stream);
    // The first attempt of the batch in m_b over `rows` queries (directly or under capture). Returns
    // 1 when the batch ended early (Features), else 0.
    int EnqueueAttempt(uint32_t rows, const BatchInputs& in, float* dOutScores, int64_t* dOutIds,
                       uint32_t* dOutCounts, uint32_t outStride);
    struct GraphKey {
        uint32_t rows = 0, maxK = 0, maxOpnd = 0, outStride = 0;
        const void* model = nullptr;
        float scale = 0, shift = 0;
        const float* dQueries = nullptr;
        const void* dOutScores = nullptr;
        const void* dOutIds = nullptr;
        const void* dOutCounts = nullptr;
        bool operator==(const GraphKey& o) const {
            return rows == o.rows && maxK == o.maxK && maxOpnd == o.maxOpnd && outStride == o.outStride &&
                   model == o.model && scale == o.scale && shift == o.shift && dQueries == o.dQueries &&
                   dOutScores == o.dOutScores && dOutIds == o.dOutIds && dOutCounts == o.dOutCounts;
        }
    };
    struct GraphEntry {
        GraphKey key;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaGraphNode_t inputCopy = nullptr;  // the batch's inputs (its size follows the programs)
        Batch batch;  // the launch plan the capture made (segments, select parameters, counts)
        uint64_t used = 0;
    };
    // Replays (capturing first when new) the first attempt of a batch shape; 0 or a negative status.
    int EnqueueGraph(const GraphKey& key, uint32_t rows, const BatchInputs& in, float* dOutScores, int64_t* dOutIds,
                     uint32_t* dOutCounts, uint32_t outStride);
    void DropGraphs();
    uint64_t SampleWant(uint32_t maxK) const;

    int32_t m_deviceId;
    std::shared_ptr<DataTable> m_table;
    SearcherConfig m_cfg;
    bool m_ok = false;
    std::string m_err;
    int m_numSms = 148;

    std::vector<QueryNode*> m_queries;
    std::vector<float> m_queryVectors;
    std::vector<uint32_t> m_topKs;

    // device workspace: one arena (the caller's, or owned), carved by Layout()
    uint8_t* m_dArena = nullptr;
    bool m_arenaOwned = false;
    uint64_t* m_dBits = nullptr;
    float* m_dCandScore = nullptr;
    uint32_t* m_dCandLoc = nullptr;
    unsigned long long* m_dWork = nullptr;
    float* m_dSampScore = nullptr;
    uint32_t* m_dSampLoc = nullptr;
    uint32_t m_sampCap = 0;
    uint8_t* m_dStage = nullptr;  // packed per-batch inputs (programs, topk, eps) + counters
    size_t m_stageBytes = 0;
    uint8_t* m_hStage = nullptr;  // pinned host copy
    float* m_dQueries = nullptr;  // for BatchSearch
    float* m_dOutScore = nullptr;
    int64_t* m_dOutId = nullptr;
    uint32_t* m_dOutCount = nullptr;
    float* m_hOutScore = nullptr;
    int64_t* m_hOutId = nullptr;
    uint32_t* m_hOutCount = nullptr;
    // tensor-core pass
    int m_tcFormat = -1;  // TcFormat, or -1 for the SIMT pass
    uint32_t m_tcKblocks = 0;
    CUtensorMap m_docMap{};
    CUtensorMap m_qryMap{};
    void* m_dStaged = nullptr;  // [256][dim] staged queries in the pass's format
    float* m_dQScale = nullptr;
    int32_t* m_dError = nullptr;
    cudaEvent_t m_ev[6] = {};
    cudaEvent_t m_evStatus = nullptr;  // the batch's statuses are on the host
    Batch m_b;
    bool m_timing = false;
    StageTimes m_times;
    std::vector<int32_t> m_lastStatus;
    std::vector<std::pair<uint32_t, uint32_t>> m_lastSegs;  // per query: (segments, entries per segment)
    std::shared_ptr<ThresholdModel> m_model;
    float m_margin = 0.0f;
    float* m_dX = nullptr;           // [maxBatch][FeatureDim()] model features
    float* m_dYp = nullptr;          // [maxBatch] model outputs, then pass A's thresholds
    float* m_dStats = nullptr;       // [maxBatch][4] doc-sample statistics
    float* m_hThetaA = nullptr;      // pinned copy of pass A's thresholds
    float* m_featuresOut = nullptr;  // Features(): stop after writing the feature rows here
    std::vector<float> m_lastTheta1, m_lastThetaA;
    std::vector<uint8_t> m_lastMiss;
    uint32_t m_testHold = 0;
    long long m_testBudget = 0;
    bool m_graphs = false;
    std::vector<GraphEntry> m_graphCache;
    uint64_t m_graphCaptures = 0, m_graphReplays = 0, m_graphClock = 0;
    double m_graphCaptureMs = 0;
    std::string m_graphFailure;
};

// ---------------------------------------------------------------------------------------------
// Serving loop: continuous batching of single queries over one resident table.
//
// Clients submit (vector, filter text, K) at any time; the filter is compiled on the submitting
// thread. `slots` workers each own a FullRecallSearcher (its whole device arena) and a CUDA stream.
// A free worker takes every queued request up to maxBatch -- waiting at most maxWaitUs for more when
// fewer are queued -- and runs them as one batch, so requests that arrive while other batches are on
// the GPU join the next batch of the next free slot, and the slots' batches overlap on the device.
// The slot count is admitted by device memory: at most what `memoryBudget` bytes of searcher arenas
// allow. Each request's latency runs from its submission to its result being on the host.
struct ServingConfig {
    uint32_t slots = 2;
    uint32_t maxBatch = 256;
    uint32_t maxWaitUs = 200;
    uint64_t memoryBudget = 0;  // bytes for the slots' arenas; 0 = half of the free device memory
    SearcherConfig searcher;    // maxBatch is taken from above
    // Replay each batch shape's captured CUDA graph (FullRecallSearcher::SetGraphs); the device
    // rows of every batch then hold kMaxTopK entries. Off by default: measured no faster than direct
    // launches here, and a capture now and then takes tens of ms of host time.
    bool graphs = false;
};

struct ServingStats {
    uint64_t completed = 0, batches = 0;
    uint32_t slots = 0;
    double meanBatch = 0, p50Ms = 0, p99Ms = 0, maxMs = 0;
    uint64_t graphCaptures = 0, graphReplays = 0;  // over all slots
    double graphCaptureMs = 0;                     // host time the slots spent capturing
};

class ServingLoop {
   public:
    ServingLoop(std::shared_ptr<DataTable> table, const ServingConfig& cfg);
    ~ServingLoop();
    ServingLoop(const ServingLoop&) = delete;
    ServingLoop& operator=(const ServingLoop&) = delete;
    bool Ok() const { return m_ok; }
    const std::string& Error() const { return m_err; }

    // 0 and *id on success; HSS-style negative codes: -3 the filter does not parse, -4 bad program,
    // -1 bad arguments.
    int Submit(const float* vec, uint32_t dim, const char* filter, uint32_t topK, uint64_t* id);
    // Blocks (up to timeoutMs, < 0 = forever) for request `id`, copies its results (scores desc,
    // global ids) into cap-entry arrays and forgets it. 0 done, 1 timed out, -1 unknown id. *status
    // gets the query's status bits (HSS_QSTATUS_*), or -2 when its batch failed on the device.
    int Wait(uint64_t id, float* scores, int64_t* ids, uint32_t cap, uint32_t* count, double* latencyMs,
             int32_t* status, int timeoutMs);
    ServingStats Stats() const;
    void ResetStats();
    // Open-loop load: n queries (row i of queries [n][dim], filters[i], topks[i]) submitted at Poisson
    // arrival times of rate rateQps, each waited for; per-request latency into latencyMs[n]. Returns
    // the number of failed requests; *offeredQps = the arrival rate actually achieved.
    int RunPoisson(const float* queries, uint32_t n, const char* const* filters, const uint32_t* topks, double rateQps,
                   uint64_t seed, double* latencyMs, double* offeredQps, double* wallSeconds);
    int SetThresholdModel(std::shared_ptr<ThresholdModel> model, float margin);
    uint32_t Slots() const { return static_cast<uint32_t>(m_slots.size()); }

   private:
    struct Request {
        uint64_t id = 0;
        std::vector<float> vec;
        FilterExpr expr;
        uint32_t topK = 0;
        std::chrono::steady_clock::time_point arrival, done;
        std::vector<float> scores;
        std::vector<int64_t> ids;
        uint32_t count = 0;
        int32_t status = 0;
        bool finished = false;
    };
    struct Slot {
        std::unique_ptr<FullRecallSearcher> searcher;
        cudaStream_t stream = nullptr;
        float* hQ = nullptr;  // pinned [maxBatch][dim]
        float* dQ = nullptr;
        float *hSc = nullptr, *dSc = nullptr;  // [maxBatch][kMaxTopK]
        int64_t *hId = nullptr, *dId = nullptr;
        uint32_t *hCnt = nullptr, *dCnt = nullptr;
        uint64_t modelGen = 0;
        uint64_t captures = 0, replays = 0;  // the searcher's graph counters after its last batch
        double captureMs = 0;
        std::thread worker;
    };
    void Worker(Slot* slot);
    void RunBatch(Slot* slot, std::vector<std::shared_ptr<Request>>& batch);

    std::shared_ptr<DataTable> m_table;
    ServingConfig m_cfg;
    bool m_ok = false;
    std::string m_err;
    uint32_t m_dim = 0;
    std::vector<std::unique_ptr<Slot>> m_slots;
    mutable std::mutex m_mu;
    std::condition_variable m_cvQueue, m_cvDone;
    std::deque<std::shared_ptr<Request>> m_queue;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> m_live;
    uint64_t m_nextId = 1;
    bool m_stop = false;
    // threshold model: each slot picks up a new one before its next batch
    std::shared_ptr<ThresholdModel> m_model;
    float m_margin = 0.0f;
    uint64_t m_modelGen = 0;
    // stats
    std::vector<double> m_lat;
    uint64_t m_batches = 0, m_batched = 0;
};

}  // namespace hss
