// searcher.cpp -- FullRecallSearcher: one batch of filtered full-recall queries on the GPU.
//
// Per batch (replacing FullRecallSearcher::BatchSearch, full_recall_searcher.cpp:107-231, with its
// per-query filter launches, host count round trips and host sort):
//   1. filter      all queries' postfix programs over all segments -> per-query doc bitmaps
//   2. eps         per-query error bounds of the approximate scoring passes
//   3. sample      approximate scores of an evenly spaced doc sample; K-th best -> threshold
//   4. candidates  approximate scores of every doc; filter bit && score >= threshold -> candidates
//   5. select      exact FP32 rescoring of the candidates that can still reach the top K, then the
//                  deterministic top K (score desc, doc id asc) with global doc ids
// A query whose candidate list overflowed gets a higher (still safe) threshold from step 5 and is
// re-run through steps 4-5 alone.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "../hss_device.cuh"
#include "../hss_kernels.h"
#include "hss_host.h"

namespace hss {

namespace {
// Error bound of an FP32 FFMA dot product of length d (any summation order) plus the one of the
// ground truth's own sequential sum, relative to sum |q_i v_i|: 2 * gamma_d, gamma_d = d u/(1 - d u),
// u = 2^-24, doubled for slack.
double SimtRelBound(uint32_t d) {
    const double u = std::ldexp(1.0, -24);
    const double g = d * u / (1.0 - d * u);
    return 4.0 * g;
}

size_t AlignUp(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Accumulation error of one tensor-core dot product, relative to |q~||v~| (the quantised vectors'
// norms), for d terms in the pass's format.
//
// Model: every MMA instruction adds its k products (k = 32 bytes of K: 8 TF32, 16 BF16, 32 E4M3
// terms) to the FP32 accumulator as one fused sum. The products are exact; the k + 1 addends are
// aligned to the largest of them and cut to p bits (truncation, no rounding), and the sum is
// normalised to p bits by truncation again. That is the behaviour Fasi, Higham, Mikaitis and Pranesh
// measured on the V100, T4 and A100 tensor cores ("Numerical behavior of NVIDIA tensor cores", PeerJ
// Computer Science 7:e330, 2021), where the FP32-accumulating modes kept no fewer bits than the FP32
// significand. For FP8, the DeepSeek-V3 technical report (arXiv:2412.19437, section 3.3.2) measured
// Hopper's FP8 MMA keeping only about 14 bits of the accumulation.
//
// Each addend loses less than one unit in the p-th bit of the largest addend, and the normalisation
// less than one of the sum, so one instruction's error is below (k + 2) 2^(1-p) M, where M bounds
// every partial sum and product: M <= sum_i |q~_i v~_i| <= |q~||v~| (Cauchy-Schwarz). Over ceil(d/k)
// instructions: (d + 2 ceil(d/k)) 2^(1-p) |q~||v~|, with p one bit below what was measured (23 for
// TF32 and BF16, 13 for E4M3) and a factor (1 + 2^-10) for the second-order growth of M. The 2^-21
// covers the E4M3 dequantising multiplies (acc * q scale * doc scale, two roundings). The GPU test
// test_accumulation_bound_under_cancellation drives the passes with high-cancellation,
// wide-dynamic-range rows and reports the measured fraction of this bound.
double TcAccumulationBound(int format, uint32_t d) {
    const uint32_t k = format == kTcTF32 ? 8u : (format == kTcBF16 ? 16u : 32u);
    const int p = format == kTcE4M3 ? 13 : 23;
    const double steps = static_cast<double>((d + k - 1) / k);
    return (static_cast<double>(d) + 2.0 * steps) * std::ldexp(1.0, 1 - p) * (1.0 + std::ldexp(1.0, -10)) +
           std::ldexp(1.0, -21);
}

// Offsets of the packed per-batch staging buffer.
struct StageLayout {
    size_t progOff, opndOff, topk, epsMain, epsSamp, negInf, theta, thetaPr, qlist, errWord, counters, passCount,
        candCount, sampCount, status, theta1, prog, opnd, total;
};

StageLayout MakeLayout(uint32_t B) {
    StageLayout L{};
    size_t at = 0;
    auto take = [&](size_t bytes) {
        const size_t r = at;
        at = AlignUp(at + bytes, 256);
        return r;
    };
    L.progOff = take((B + 1) * 4ull);
    L.opndOff = take((B + 1) * 4ull);
    L.topk = take(B * 4ull);
    L.epsMain = take(B * 4ull);
    L.epsSamp = take(B * 4ull);
    L.negInf = take(B * 4ull);
    L.theta = take(B * 4ull);
    L.thetaPr = take(B * 4ull);  // proven thresholds beside predicted ones (learned threshold)
    L.qlist = take(B * 4ull);
    L.errWord = take(4);  // host copy of the tensor-core pass's error bits
    L.counters = at;  // zeroed per batch: passCount, status and theta1
    L.passCount = take(B * 4ull);
    L.status = take(B * 4ull);
    L.theta1 = take(B * 4ull);  // the doc sample's proven thresholds, copied out with the statuses
    // the programs, then their operand rows (one host-to-device copy of [0, prog + words))
    L.prog = take(static_cast<size_t>(B) * (kMaxProgram + kMaxOperands) * 4ull);
    L.opnd = take(static_cast<size_t>(B) * kMaxOperands * 4ull);  // host only: operands while programs are laid out
    // per-segment candidate counts: every producing CTA writes its own, no clearing
    L.candCount = take(static_cast<size_t>(B) * kMaxCandSegs * 4ull);
    L.sampCount = take(static_cast<size_t>(B) * kMaxCandSegs * 4ull);
    L.total = at;
    return L;
}
}  // namespace

namespace {
// The clamps every searcher applies to its configuration.
SearcherConfig Normalised(SearcherConfig c) {
    if (c.candidateCap < static_cast<uint32_t>(kMaxTopK)) c.candidateCap = kMaxTopK;
    if (c.maxBatch == 0) c.maxBatch = 1;
    // the tensor-core pass stages at most 2 x 128 query rows per launch
    if (c.method != ScoreMethod::SIMT_FP32 && c.maxBatch > 256) c.maxBatch = 256;
    if (c.maxBatch > kMaxSimtBatch) c.maxBatch = kMaxSimtBatch;
    return c;
}

// Entries of the doc-sample buffer per query: room for the sample a K of up to 1024 asks for (see
// SearchDevice) plus the rounding of its tiles to segments; a larger K's sample overflows it, which
// only weakens its threshold (the stored part is still a subset).
uint32_t SampleCap(const DataTable& T, const SearcherConfig& c) {
    const uint64_t forK = (4ull * 1024 * T.GetDocNum() + c.candidateCap - 1) / c.candidateCap;
    return static_cast<uint32_t>(
        std::min<uint64_t>(std::max<uint64_t>({forK, c.sampleDocs, static_cast<uint64_t>(kMaxTopK)}), 1u << 19) +
        128ull * kMaxCandSegs);
}
}  // namespace

// Byte offsets of every device buffer of a searcher inside its arena (256-byte aligned).
FullRecallSearcher::ArenaLayout FullRecallSearcher::Layout(const DataTable& T, const SearcherConfig& cfgIn) {
    const SearcherConfig c = Normalised(cfgIn);
    ArenaLayout A{};
    size_t at = 0;
    auto take = [&](size_t bytes) {
        const size_t r = at;
        at = AlignUp(at + bytes, 256);
        return r;
    };
    const uint64_t B = c.maxBatch, C = c.candidateCap, dim = T.GetDimension();
    A.sampCap = SampleCap(T, c);
    A.bits = take(B * T.GetBitmapWords() * 8);
    A.candScore = take(B * C * 4);
    A.candLoc = take(B * C * 4);
    A.work = take(B * C * 8);
    A.sampScore = take(B * A.sampCap * 4ull);
    A.sampLoc = take(B * A.sampCap * 4ull);
    A.stageBytes = MakeLayout(c.maxBatch).total;
    A.stage = take(A.stageBytes);
    A.queries = take(B * dim * 4);
    A.outScore = take(B * kMaxTopK * 4ull);
    A.outId = take(B * kMaxTopK * 8ull);
    A.outCount = take(B * 4);
    A.stats = take(B * static_cast<uint64_t>(kSampleStats) * sizeof(float));
    A.features = take(B * (dim + T.PostingRows() + kFeatureTail) * sizeof(float));
    A.predictions = take(B * sizeof(float));
    if (c.method != ScoreMethod::SIMT_FP32) {
        A.staged = take(256ull * dim * 4);
        A.qScale = take(256 * sizeof(float));
        A.error = take(sizeof(int32_t));
    }
    A.total = at;
    return A;
}

size_t FullRecallSearcher::WorkspaceBytes(const DataTable& T, const SearcherConfig& cfg) {
    return Layout(T, cfg).total;
}

FullRecallSearcher::FullRecallSearcher(int32_t deviceId, std::shared_ptr<DataTable> dataTable,
                                       const SearcherConfig& cfg, void* dArena, size_t arenaBytes)
    : m_deviceId(deviceId), m_table(std::move(dataTable)), m_cfg(Normalised(cfg)) {
    if (!m_table) {
        m_err = "null DataTable";
        return;
    }
    m_ok = Allocate(dArena, arenaBytes);
}

FullRecallSearcher::~FullRecallSearcher() {
    cudaSetDevice(m_deviceId);
    if (m_arenaOwned && m_dArena) cudaFree(m_dArena);
    void* hptrs[] = {m_hStage, m_hOutScore, m_hOutId, m_hOutCount, m_hThetaA};
    for (void* p : hptrs)
        if (p) cudaFreeHost(p);
    for (auto& e : m_ev)
        if (e) cudaEventDestroy(e);
    if (m_evStatus) cudaEventDestroy(m_evStatus);
    DropGraphs();
}

bool FullRecallSearcher::Allocate(void* dArena, size_t arenaBytes) {
    auto ck = [&](cudaError_t e, const char* what) {
        if (e == cudaSuccess) return true;
        m_err = std::string(what) + ": " + cudaGetErrorString(e);
        return false;
    };
    if (!ck(cudaSetDevice(m_deviceId), "cudaSetDevice")) return false;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m_deviceId) == cudaSuccess && sms > 0)
        m_numSms = sms;
    // Index-side residency first (it belongs to the table and is shared by its searchers): the
    // dense posting matrix and the copy of the rows the tensor-core pass reads.
    if (m_cfg.densePostings) {
        // every posting decoded once into a dense bitmap when that takes at most 40% of free memory
        size_t freeB = 0, totalB = 0;
        if (!ck(cudaMemGetInfo(&freeB, &totalB), "cudaMemGetInfo")) return false;
        if (!m_table->EnableDensePostings(static_cast<uint64_t>(freeB) / 5 * 2, &m_err)) return false;
    }
    if (m_cfg.method != ScoreMethod::SIMT_FP32) {
        m_tcFormat = static_cast<int>(m_cfg.method) - 1;
        if (!m_table->EnableFormat(m_tcFormat, &m_err)) return false;
        const uint32_t elem = m_tcFormat == kTcTF32 ? 4 : (m_tcFormat == kTcBF16 ? 2 : 1);
        m_tcKblocks = m_table->GetDimension() * elem / 128;
    }
    // The searcher's own device buffers: one arena, the caller's or allocated here.
    const ArenaLayout A = Layout(*m_table, m_cfg);
    if (dArena) {
        cudaPointerAttributes at{};
        if (arenaBytes < A.total || (reinterpret_cast<uintptr_t>(dArena) & 255u)) {
            m_err = "workspace smaller than hss_searcher_workspace_bytes() or not 256-byte aligned";
            return false;
        }
        if (cudaPointerGetAttributes(&at, dArena) != cudaSuccess || at.type != cudaMemoryTypeDevice ||
            at.device != m_deviceId) {
            cudaGetLastError();
            m_err = "workspace is not device memory of the table's device";
            return false;
        }
        m_dArena = static_cast<uint8_t*>(dArena);
        m_arenaOwned = false;
    } else {
        void* p = nullptr;
        if (!ck(cudaMalloc(&p, A.total), "cudaMalloc searcher workspace")) return false;
        m_dArena = static_cast<uint8_t*>(p);
        m_arenaOwned = true;
    }
    uint8_t* W = m_dArena;
    m_sampCap = A.sampCap;
    m_stageBytes = A.stageBytes;
    m_dBits = reinterpret_cast<uint64_t*>(W + A.bits);
    m_dCandScore = reinterpret_cast<float*>(W + A.candScore);
    m_dCandLoc = reinterpret_cast<uint32_t*>(W + A.candLoc);
    m_dWork = reinterpret_cast<unsigned long long*>(W + A.work);
    m_dSampScore = reinterpret_cast<float*>(W + A.sampScore);
    m_dSampLoc = reinterpret_cast<uint32_t*>(W + A.sampLoc);
    m_dStage = W + A.stage;
    m_dQueries = reinterpret_cast<float*>(W + A.queries);
    m_dOutScore = reinterpret_cast<float*>(W + A.outScore);
    m_dOutId = reinterpret_cast<int64_t*>(W + A.outId);
    m_dOutCount = reinterpret_cast<uint32_t*>(W + A.outCount);
    m_dStats = reinterpret_cast<float*>(W + A.stats);
    m_dX = reinterpret_cast<float*>(W + A.features);
    m_dYp = reinterpret_cast<float*>(W + A.predictions);

    const uint64_t B = m_cfg.maxBatch;
    if (!ck(cudaMallocHost(&m_hStage, m_stageBytes), "cudaMallocHost staging")) return false;
    std::memset(m_hStage, 0, m_stageBytes);
    const StageLayout L = MakeLayout(static_cast<uint32_t>(B));
    float* negInf = reinterpret_cast<float*>(m_hStage + L.negInf);
    for (uint64_t i = 0; i < B; ++i) negInf[i] = -INFINITY;
    if (!ck(cudaMallocHost(&m_hOutScore, B * kMaxTopK * 4ull), "cudaMallocHost results")) return false;
    if (!ck(cudaMallocHost(&m_hOutId, B * kMaxTopK * 8ull), "cudaMallocHost results")) return false;
    if (!ck(cudaMallocHost(&m_hOutCount, B * 4ull), "cudaMallocHost results")) return false;
    if (!ck(cudaMallocHost(&m_hThetaA, B * sizeof(float)), "cudaMallocHost thresholds")) return false;
    for (auto& e : m_ev)
        if (!ck(cudaEventCreate(&e), "cudaEventCreate")) return false;
    if (m_tcFormat >= 0) {
        const uint32_t dim = m_table->GetDimension();
        m_dStaged = W + A.staged;
        m_dQScale = reinterpret_cast<float*>(W + A.qScale);
        m_dError = reinterpret_cast<int32_t*>(W + A.error);
        if (!ck(cudaMemset(m_dError, 0, sizeof(int32_t)), "cudaMemset error word")) return false;
        if (!make_tc_map(&m_docMap, m_tcFormat, m_table->DeviceRows(m_tcFormat), m_table->GetTileNum() * 128, dim) ||
            !make_tc_map(&m_qryMap, m_tcFormat, m_dStaged, 256, dim)) {
            m_err = "cuTensorMapEncodeTiled failed";
            return false;
        }
    }
    return true;
}

void FullRecallSearcher::AddQuery(QueryNode* queryTree, const std::vector<float>& queryVector, uint32_t topK) {
    m_queries.push_back(queryTree);
    m_queryVectors.insert(m_queryVectors.end(), queryVector.begin(), queryVector.end());
    m_topKs.push_back(topK);
}

void FullRecallSearcher::ClearQueries() {
    m_queries.clear();
    m_queryVectors.clear();
    m_topKs.clear();
}

FullRecallSearcher::BatchInputs FullRecallSearcher::PrepareInputs(uint32_t nq, uint32_t rows,
                                                                  const FilterExpr* const* exprs,
                                                                  const uint32_t* topks, uint32_t padK) {
    const StageLayout SL = MakeLayout(m_cfg.maxBatch);
    uint8_t* H = m_hStage;
    auto* progOff = reinterpret_cast<uint32_t*>(H + SL.progOff);
    auto* opndOff = reinterpret_cast<uint32_t*>(H + SL.opndOff);
    auto* topk = reinterpret_cast<uint32_t*>(H + SL.topk);
    auto* prog = reinterpret_cast<uint32_t*>(H + SL.prog);
    auto* opnd = reinterpret_cast<uint32_t*>(H + SL.opnd);
    BatchInputs in;
    uint32_t np = 0, no = 0;
    // match-nothing: [AND, 1, 0] over the all-zero posting row
    auto matchNothing = [&] {
        prog[np++] = AND;
        prog[np++] = 1;
        prog[np++] = 0;
        opnd[no++] = m_table->PostingRows() - 1;
        in.maxOpnd = std::max(in.maxOpnd, 1u);
    };
    for (uint32_t q = 0; q < rows; ++q) {
        progOff[q] = np;
        opndOff[q] = no;
        if (q >= nq) {
            topk[q] = padK;
            in.maxK = std::max(in.maxK, padK);
            matchNothing();
            continue;
        }
        topk[q] = topks ? topks[q] : 0u;
        in.maxK = std::max(in.maxK, topk[q]);
        const FilterExpr* e = exprs[q];
        if (e == nullptr || e->emptyTree) continue;  // empty program: match all
        const uint32_t pl = static_cast<uint32_t>(e->postExpr.size());
        const uint32_t ol = static_cast<uint32_t>(e->postingRows.size());
        if (pl > static_cast<uint32_t>(kMaxProgram) || ol > static_cast<uint32_t>(kMaxOperands) || pl == 0) {
            // Over the kernel's limits: reported in the status and run as match-nothing.
            m_lastStatus[q] |= kStatusBadProgram;
            matchNothing();
            continue;
        }
        std::memcpy(prog + np, e->postExpr.data(), pl * 4ull);
        std::memcpy(opnd + no, e->postingRows.data(), ol * 4ull);
        np += pl;
        no += ol;
        in.maxOpnd = std::max(in.maxOpnd, ol);
    }
    progOff[rows] = np;
    opndOff[rows] = no;
    for (uint32_t q = 0; q < nq; ++q)
        if (topk[q] > static_cast<uint32_t>(kMaxTopK)) m_lastStatus[q] |= kStatusTopKTooLarge;
    // the operand rows follow the programs (offsets from the program array's start), and the
    // counters go over zeroed, so that one copy brings every input
    std::memcpy(prog + np, opnd, no * 4ull);
    for (uint32_t q = 0; q <= rows; ++q) opndOff[q] += np;
    std::memset(H + SL.counters, 0, SL.prog - SL.counters);
    in.np = np;
    in.no = no;
    return in;
}

size_t FullRecallSearcher::InputBytes(const BatchInputs& in) const {
    return MakeLayout(m_cfg.maxBatch).prog + std::max(in.np + in.no, 1u) * 4ull;
}

int FullRecallSearcher::EnqueueFilter(uint32_t rows, const BatchInputs& in, uint64_t* dBits, uint64_t bitsStride,
                                      cudaStream_t stream) {
    const StageLayout SL = MakeLayout(m_cfg.maxBatch);
    uint8_t* H = m_hStage;
    uint8_t* D = m_dStage;
    const DataTable& T = *m_table;
    cudaError_t ce = cudaSuccess;
    auto ck = [&](cudaError_t e) {
        if (ce == cudaSuccess && e != cudaSuccess) ce = e;
    };
    // the per-batch inputs in one copy: offsets and K, the zeroed counters, the programs and their
    // operands (at least one word, so that a replayed graph can resize the copy)
    ck(cudaMemcpyAsync(D, H, InputBytes(in), cudaMemcpyHostToDevice, stream));

    if (m_cfg.densePostings && T.DeviceDensePostings()) {
        DenseFilterLaunch F{};
        F.prog = reinterpret_cast<const uint32_t*>(D + SL.prog);
        F.prog_off = reinterpret_cast<const uint32_t*>(D + SL.progOff);
        F.opnd_row = reinterpret_cast<const uint32_t*>(D + SL.prog);
        F.opnd_off = reinterpret_cast<const uint32_t*>(D + SL.opndOff);
        F.dense = T.DeviceDensePostings();
        F.rows = T.PostingRows();
        F.seg_words = T.GetDocNumPerSegment() / 64;
        F.out = dBits;
        F.out_stride = bitsStride;
        F.pass_count = reinterpret_cast<uint32_t*>(D + SL.passCount);
        F.status = reinterpret_cast<int32_t*>(D + SL.status);
        F.nq = rows;
        F.seg_num = T.GetSegmentNum();
        F.doc_num = T.GetDocNum();
        F.max_opnd = in.maxOpnd;
        F.sm_count = m_numSms;
        ck(launch_filter_dense(F, stream));
        return ce == cudaSuccess ? 0 : static_cast<int>(ce);
    }
    FilterLaunch F{};
    F.prog = reinterpret_cast<const uint32_t*>(D + SL.prog);
    F.prog_off = reinterpret_cast<const uint32_t*>(D + SL.progOff);
    F.opnd_row = reinterpret_cast<const uint32_t*>(D + SL.prog);
    F.opnd_off = reinterpret_cast<const uint32_t*>(D + SL.opndOff);
    F.table = T.DevicePostingTable();
    F.row_stride = T.GetSegmentNum();
    F.seg_stride = 1;
    F.out = dBits;
    F.out_stride = bitsStride;
    F.pass_count = reinterpret_cast<uint32_t*>(D + SL.passCount);
    F.status = reinterpret_cast<int32_t*>(D + SL.status);
    F.nq = rows;
    F.seg_num = T.GetSegmentNum();
    F.docs_per_seg = T.GetDocNumPerSegment();
    F.doc_num = T.GetDocNum();
    F.max_opnd = in.maxOpnd;
    ck(launch_filter_batch(F, stream));
    return ce == cudaSuccess ? 0 : static_cast<int>(ce);
}

int FullRecallSearcher::FilterDevice(uint32_t nq, const FilterExpr* const* exprs, uint64_t* dOutBits,
                                     uint64_t outStrideWords, uint32_t* dPassCounts, cudaStream_t stream) {
    if (!m_ok) return -1;
    m_lastStatus.assign(nq, 0);
    if (nq == 0) return 0;
    if (nq > m_cfg.maxBatch || outStrideWords < m_table->GetBitmapWords()) {
        m_err = "batch larger than maxBatch or bitmap row too short";
        return -1;
    }
    if (cudaSetDevice(m_deviceId) != cudaSuccess) return -2;
    const BatchInputs in = PrepareInputs(nq, nq, exprs, nullptr, 0);
    if (EnqueueFilter(nq, in, dOutBits, outStrideWords, stream) != 0) return -2;
    const StageLayout SL = MakeLayout(m_cfg.maxBatch);
    auto* hStatus = reinterpret_cast<int32_t*>(m_hStage + SL.status);
    cudaError_t e = cudaSuccess;
    if (dPassCounts)
        e = cudaMemcpyAsync(dPassCounts, m_dStage + SL.passCount, nq * 4ull, cudaMemcpyDeviceToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hStatus, m_dStage + SL.status, nq * 4ull, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        m_err = cudaGetErrorString(e);
        return -2;
    }
    int bad = 0;
    for (uint32_t q = 0; q < nq; ++q) {
        m_lastStatus[q] |= hStatus[q];
        bad += m_lastStatus[q] != 0;
    }
    return bad;
}

uint32_t FullRecallSearcher::FeatureDim() const {
    return m_table ? m_table->GetDimension() + m_table->PostingRows() + kFeatureTail : 0;
}

int FullRecallSearcher::SetThresholdModel(std::shared_ptr<ThresholdModel> model, float margin) {
    if (!m_ok) return -1;
    if (model && (!model->Ok() || model->Din() != FeatureDim() || model->DeviceId() != m_deviceId)) {
        m_err = "threshold model does not fit this searcher (feature width or device)";
        return -1;
    }
    m_model = std::move(model);
    m_margin = margin;
    DropGraphs();  // the captured launches hold the model's parameters and the margin
    return 0;
}

// Features of the staged batch (the filter stage and the doc sample have run: pass counts, operands
// and sample statistics are on the device).
static cudaError_t LaunchFeatures(const DataTable& T, const uint8_t* D, size_t opndOff, size_t opnd, size_t passCount,
                                  size_t topk, const float* stats, const float* dQueries, uint32_t nq, uint32_t din,
                                  float* dX, cudaStream_t stream) {
    FeatureLaunch F{};
    F.qry = dQueries;
    F.stats = stats;
    F.opnd_row = reinterpret_cast<const uint32_t*>(D + opnd);
    F.opnd_off = reinterpret_cast<const uint32_t*>(D + opndOff);
    F.pass_count = reinterpret_cast<const uint32_t*>(D + passCount);
    F.topk = reinterpret_cast<const uint32_t*>(D + topk);
    F.row_density = T.DeviceRowDensity();
    F.x = dX;
    F.nq = nq;
    F.dim = T.GetDimension();
    F.rows = T.PostingRows();
    F.din = din;
    F.doc_num = T.GetDocNum();
    return launch_features(F, stream);
}

int FullRecallSearcher::LastCandidateCounts(uint32_t n, uint32_t* counts) {
    if (!m_ok || n > m_cfg.maxBatch) return -1;
    std::fill(counts, counts + n, 0u);
    if (n == 0 || m_lastSegs.empty()) return 0;
    if (cudaSetDevice(m_deviceId) != cudaSuccess) return -2;
    const StageLayout SL = MakeLayout(m_cfg.maxBatch);
    std::vector<uint32_t> c(static_cast<size_t>(n) * kMaxCandSegs);
    if (cudaMemcpy(c.data(), m_dStage + SL.candCount, c.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
    const uint32_t m = std::min<uint32_t>(n, static_cast<uint32_t>(m_lastSegs.size()));
    for (uint32_t q = 0; q < m; ++q)
        for (uint32_t g = 0; g < m_lastSegs[q].first; ++g) counts[q] += c[static_cast<size_t>(q) * kMaxCandSegs + g];
    return 0;
}

int FullRecallSearcher::Features(const float* dQueries, uint32_t nq, const FilterExpr* const* exprs,
                                 const uint32_t* topks, float* dX, cudaStream_t stream) {
    // the batch's own filter, staging and doc sample, stopping at the features
    m_featuresOut = dX;
    const int rc = SearchDevice(dQueries, nq, exprs, topks, nullptr, nullptr, nullptr, kMaxTopK, stream);
    m_featuresOut = nullptr;
    return rc;
}

uint32_t FullRecallSearcher::UnitOf(uint32_t rows, bool simt) const {
    return UseSimt(simt) ? 128u : tc_tile_docs(rows, m_tcKblocks);
}

uint64_t FullRecallSearcher::TilesOf(uint32_t unit) const { return (m_table->GetDocNum() + unit - 1) / unit; }

uint32_t FullRecallSearcher::CtasOf(uint32_t rows, uint64_t countTiles, uint32_t cap, bool simt) const {
    return UseSimt(simt) ? cand_simt_segments(countTiles, m_numSms, cap)
                         : tc_cand_ctas(rows, m_tcKblocks, countTiles, m_numSms, cap);
}

uint32_t FullRecallSearcher::SegsOf(uint32_t rows, uint64_t countTiles, uint32_t cap, bool simt) const {
    const uint32_t g = CtasOf(rows, countTiles, cap, simt);
    return UseSimt(simt) ? g : 2 * g;  // a tensor-core CTA fills two segments
}

// Entries per segment: the docs one segment can see at most, within the list's share.
uint32_t FullRecallSearcher::SegCapOf(uint32_t rows, uint64_t countTiles, uint32_t cap, uint32_t segs,
                                      bool simt) const {
    const uint32_t g = CtasOf(rows, countTiles, cap, simt);
    // SIMT: a CTA's tiles; single SM: half of a CTA's tiles' docs; pair: a quarter of a pair's
    const uint64_t groups = UseSimt(simt) ? g : (UnitOf(rows, simt) == 256 ? g / 2 : g);
    const uint64_t perTile = UseSimt(simt) ? 128ull : 64ull;
    const uint64_t perSeg = (countTiles + groups - 1) / groups * perTile;
    return static_cast<uint32_t>(std::min<uint64_t>(perSeg, cap / segs));
}

// Error bounds (and, for the tensor-core pass, the staged queries in its format) of queries dList
// (or 0..rows-1).
void FullRecallSearcher::Stage(const uint32_t* dList, uint32_t rows) {
    const DataTable& T = *m_table;
    const StageLayout SL = MakeLayout(m_cfg.maxBatch);
    auto* dEpsMain = reinterpret_cast<float*>(m_dStage + SL.epsMain);
    auto* dEpsSamp = reinterpret_cast<float*>(m_dStage + SL.epsSamp);
    const uint32_t dim = T.GetDimension();
    if (m_tcFormat < 0) {
        const double rel = SimtRelBound(dim);
        Ck(launch_query_eps(m_b.dQueries, dList, rows, dim, T.GetMaxNorm(), rel, rel, dEpsMain, dEpsSamp, m_b.stream));
        return;
    }
    StageQueriesLaunch Q{};
    Q.qry = m_b.dQueries;
    Q.qlist = dList;
    Q.nq_rows = rows;
    Q.rows_alloc = 256;
    Q.dim = dim;
    Q.format = m_tcFormat;
    Q.staged = m_dStaged;
    Q.q_scale = m_dQScale;
    Q.eps_main = dEpsMain;
    Q.eps_sample = dEpsSamp;
    Q.doc_norm_max = T.NormMax(m_tcFormat);
    Q.doc_err_max = T.ErrMax(m_tcFormat);
    Q.acc_rel = TcAccumulationBound(m_tcFormat, dim);
    Ck(launch_stage_queries(Q, m_b.stream));
}

// A candidate pass: tiles begin + i * step (or, with skip >= 2, all tiles that are not multiples of
// skip), i < countTiles, for `rows` queries (dList or 0..rows-1), writing the list segments
// [segBase, segBase + its segments) of segCap entries each. Tiles hold UnitOf() docs: 128 for the
// SIMT pass and the single-SM tensor-core pass, 256 for the SM-pair pass.
void FullRecallSearcher::Cand(const float* theta, float* score, uint32_t* loc, uint32_t* count, uint32_t cap,
                              uint32_t segBase, uint32_t segCap, uint64_t begin, uint64_t step, uint32_t skip,
                              uint64_t countTiles, const uint32_t* dList, uint32_t rows, bool simt) {
    const DataTable& T = *m_table;
    const uint32_t g = CtasOf(rows, countTiles, cap, simt);
    if (UseSimt(simt)) {
        CandLaunch C{};
        C.vec = T.DeviceVectors();
        C.qry = m_b.dQueries;
        C.bits = m_dBits;
        C.bits_stride = T.GetBitmapWords();
        C.theta = theta;
        C.qlist = dList;
        C.nq_list = rows;
        C.cand_score = score;
        C.cand_loc = loc;
        C.cand_count = count;
        C.cap = cap;
        C.segs = g;
        C.seg_cap = segCap;
        C.seg_base = segBase;
        C.dim = T.GetDimension();
        C.tile_begin = begin;
        C.tile_step = step;
        C.tile_count = countTiles;
        C.tile_skip = skip;
        Ck(launch_cand_simt(C, m_numSms, m_b.stream));
        return;
    }
    TcCandLaunch C{};
    C.format = m_tcFormat;
    C.kblocks = m_tcKblocks;
    C.doc_scale = T.DeviceDocScale();
    C.tile_scale = T.DeviceTileScale();
    C.q_scale = m_dQScale;
    C.bits = m_dBits;
    C.bits_stride = T.GetBitmapWords();
    C.theta = theta;
    C.qlist = dList;
    C.nq_rows = rows;
    C.cand_score = score;
    C.cand_loc = loc;
    C.cand_count = count;
    C.cap = cap;
    C.ctas = g;
    C.seg_cap = segCap;
    C.seg_base = segBase;
    C.tile_begin = begin;
    C.tile_step = step;
    C.tile_count = countTiles;
    C.tile_skip = skip;
    C.tiles128 = T.GetTileNum();
    C.error = m_dError;
    C.emit_all = theta == reinterpret_cast<const float*>(m_dStage + MakeLayout(m_cfg.maxBatch).negInf) ? 1 : 0;
    if (m_testHold && tc_tile_docs(rows, m_tcKblocks) == 128u) {  // the single-SM kernel only
        C.hold_load = m_testHold;
        C.wait_budget = m_testBudget;
        m_testHold = 0;
    }
    Ck(launch_tc_cand(C, m_docMap, m_qryMap, m_numSms, m_b.stream));
}

// The doc sample: evenly spaced tiles, every filtered doc kept; its K-th best bounds the threshold.
// Returns the sample's tile count.
// Tiles (and their step) of a doc sample of `want` docs for `rows` queries.
void FullRecallSearcher::SampleTiles(uint64_t want, uint32_t rows, bool simt, uint64_t* count, uint64_t* step) const {
    const uint32_t unit = UnitOf(rows, simt);
    const uint64_t tilesU = TilesOf(unit);
    const uint64_t sampTiles = std::min<uint64_t>(tilesU, std::max<uint64_t>(1, (want + unit - 1) / unit));
    *step = std::max<uint64_t>(1, tilesU / sampTiles);
    *count = std::min<uint64_t>(sampTiles, (tilesU + *step - 1) / *step);
}

uint64_t FullRecallSearcher::Sample(const uint32_t* dList, uint32_t rows, bool simt, bool raiseOnly, float* stats,
                                    float* thetaCopy, const float* emitTheta) {
    const StageLayout SL = MakeLayout(m_cfg.maxBatch);
    uint8_t* D = m_dStage;
    uint64_t count = 0, step = 1;
    SampleTiles(m_b.want, rows, simt, &count, &step);
    const uint32_t segs = SegsOf(rows, count, m_sampCap, simt);
    const uint32_t segCap = SegCapOf(rows, count, m_sampCap, segs, simt);
    auto* dSampCount = reinterpret_cast<uint32_t*>(D + SL.sampCount);
    Cand(emitTheta ? emitTheta : reinterpret_cast<const float*>(D + SL.negInf), m_dSampScore, m_dSampLoc, dSampCount,
         m_sampCap, 0, segCap, 0, step, 0, count, dList, rows, simt);
    SampleThresholdLaunch ST{};
    ST.score = m_dSampScore;
    ST.count = dSampCount;
    ST.cap = m_sampCap;
    ST.segs = segs;
    ST.seg_cap = segCap;
    ST.raise_only = raiseOnly ? 1 : 0;
    ST.topk = reinterpret_cast<const uint32_t*>(D + SL.topk);
    ST.eps_sample = reinterpret_cast<const float*>(D + SL.epsSamp);
    ST.eps_main = reinterpret_cast<const float*>(D + SL.epsMain);
    ST.theta = reinterpret_cast<float*>(D + SL.theta);
    ST.qlist = dList;
    ST.nq_list = rows;
    ST.stats = stats;
    ST.theta_also = thetaCopy;  // a copy of theta, or (raise_only) raised with it
    Ck(launch_sample_threshold(ST, m_b.stream));
    return count;
}

int FullRecallSearcher::SearchDevice(const float* dQueries, uint32_t nq, const FilterExpr* const* exprs,
                                     const uint32_t* topks, float* dOutScores, int64_t* dOutIds,
                                     uint32_t* dOutCounts, uint32_t outStride, cudaStream_t stream) {
    const int rc = SearchEnqueue(dQueries, nq, exprs, topks, dOutScores, dOutIds, dOutCounts, outStride, stream);
    if (rc != 0 || !m_b.pending) return rc;
    return SearchFinish();
}

int FullRecallSearcher::SearchEnqueue(const float* dQueries, uint32_t nq, const FilterExpr* const* exprs,
                                      const uint32_t* topks, float* dOutScores, int64_t* dOutIds,
                                      uint32_t* dOutCounts, uint32_t outStride, cudaStream_t stream) {
    if (!m_ok) return -1;
    if (m_b.pending) {
        m_err = "the searcher's previous batch was not finished";
        return -1;
    }
    m_times = StageTimes{};
    m_lastStatus.assign(nq, 0);
    m_lastMiss.assign(nq, 0);
    if (nq == 0) return 0;
    if (nq > m_cfg.maxBatch) {
        m_err = "batch larger than the searcher's maxBatch";
        return -1;
    }
    for (uint32_t q = 0; q < nq; ++q) {
        // the result rows hold outStride entries; a K the kernel accepts must fit in them
        if (std::min(topks[q], static_cast<uint32_t>(kMaxTopK)) > outStride) {
            m_err = "topK larger than the output row stride";
            return -1;
        }
    }
    if (cudaSetDevice(m_deviceId) != cudaSuccess) return -2;
    m_b = Batch{};
    m_b.dQueries = dQueries;
    m_b.nq = nq;
    m_b.stream = stream;
    if (!m_evStatus && cudaEventCreateWithFlags(&m_evStatus, cudaEventDisableTiming) != cudaSuccess) return -2;
    const bool graph = m_graphs && !m_timing && m_featuresOut == nullptr && m_testHold == 0;
    const uint32_t rows = graph ? GraphRows(nq, m_cfg.maxBatch) : nq;
    BatchInputs in = PrepareInputs(nq, rows, exprs, topks, std::min(1u, outStride));
    int rc;
    if (graph) {
        in.maxK = PlanTopK(in.maxK);
        in.maxOpnd = GraphOperands(in.maxOpnd);
        GraphKey key;
        key.rows = rows;
        key.maxK = in.maxK;
        key.maxOpnd = in.maxOpnd;
        key.outStride = outStride;
        key.model = m_model.get();
        key.scale = m_model ? m_model->scale : 0.0f;
        key.shift = m_model ? m_model->shift : 0.0f;
        key.dQueries = dQueries;
        key.dOutScores = dOutScores;
        key.dOutIds = dOutIds;
        key.dOutCounts = dOutCounts;
        rc = EnqueueGraph(key, rows, in, dOutScores, dOutIds, dOutCounts, outStride);
    } else {
        rc = EnqueueAttempt(rows, in, dOutScores, dOutIds, dOutCounts, outStride);
        if (rc == 1) {  // Features: done, nothing pending
            if (m_b.ce == cudaSuccess) return 0;
            m_err = cudaGetErrorString(m_b.ce);
            return -2;
        }
        rc = 0;
    }
    if (rc == 0) Ck(cudaEventRecord(m_evStatus, stream));
    m_lastSegs.assign(nq, {m_b.se.segs, m_b.se.seg_cap});
    if (rc != 0 || m_b.ce != cudaSuccess) {
        if (m_err.empty() || m_b.ce != cudaSuccess) m_err = cudaGetErrorString(m_b.ce);
        return -2;
    }
    m_b.pending = true;
    return 0;
}

uint32_t FullRecallSearcher::GraphRows(uint32_t nq, uint32_t maxBatch) {
    uint32_t r = 1;
    if (nq <= 16) {
        while (r < nq) r <<= 1;
    } else {
        r = (nq + 15) / 16 * 16;
    }
    return std::max(nq, std::min(r, maxBatch));
}

uint32_t FullRecallSearcher::GraphTopK(uint32_t maxK) {
    uint32_t k = 1;
    while (k < maxK && k < static_cast<uint32_t>(kMaxTopK)) k <<= 1;
    return maxK == 0 ? 0u : std::max(maxK, std::min(k, static_cast<uint32_t>(kMaxTopK)));
}

uint64_t FullRecallSearcher::SampleWant(uint32_t maxK) const {
    // the doc sample whose threshold keeps the full pass within the list capacity
    return std::max<uint64_t>(m_cfg.sampleDocs, (4ull * std::max<uint32_t>(maxK, 1u) * m_table->GetDocNum() +
                                                 m_cfg.candidateCap - 1) / m_cfg.candidateCap);
}

uint32_t FullRecallSearcher::PlanTopK(uint32_t maxK) const {
    // A batch's K enters its launch plan through the doc sample's size (without a model: the sample;
    // with one: pass A's share) and the select variant (K > 256): every K up to `flat` plans as
    // K = 1 does.
    uint32_t flat = 1;
    while (flat < 256 && SampleWant(flat * 2) == SampleWant(1)) flat <<= 1;
    return maxK == 0 ? 0u : std::max(GraphTopK(maxK), flat);
}

uint32_t FullRecallSearcher::GraphOperands(uint32_t maxOpnd) {
    // powers of two: the filter kernel takes any bound at least the batch's largest operand count,
    // and up to 8 (its shared-memory form) a power of two stays within 8
    uint32_t o = 1;
    while (o < maxOpnd) o <<= 1;
    return maxOpnd == 0 ? 0u : o;
}

void FullRecallSearcher::SetGraphs(bool on) {
    if (!on) DropGraphs();
    m_graphs = on;
}

void FullRecallSearcher::DropGraphs() {
    for (GraphEntry& g : m_graphCache) {
        // an exec still running is released when it completes
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
    }
    m_graphCache.clear();
}

int FullRecallSearcher::EnqueueGraph(const GraphKey& key, uint32_t rows, const BatchInputs& in, float* dOutScores,
                                     int64_t* dOutIds, uint32_t* dOutCounts, uint32_t outStride) {
    cudaStream_t stream = m_b.stream;
    GraphEntry* g = nullptr;
    for (GraphEntry& e : m_graphCache)
        if (e.key == key) g = &e;
    if (g == nullptr) {
        // capture this shape's launches (nothing runs while the stream captures)
        GraphEntry e;
        e.key = key;
        const auto t0 = std::chrono::steady_clock::now();
        cudaError_t ce = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
        if (ce == cudaSuccess) {
            (void)EnqueueAttempt(rows, in, dOutScores, dOutIds, dOutCounts, outStride);
            ce = cudaStreamEndCapture(stream, &e.graph);
        }
        if (ce == cudaSuccess && m_b.ce == cudaSuccess)
            ce = cudaGraphInstantiate(&e.exec, e.graph, 0);
        // the input copy, whose size follows the batch's programs
        size_t n = 0;
        if (ce == cudaSuccess && m_b.ce == cudaSuccess) ce = cudaGraphGetNodes(e.graph, nullptr, &n);
        std::vector<cudaGraphNode_t> nodes(n);
        if (ce == cudaSuccess && m_b.ce == cudaSuccess && n) ce = cudaGraphGetNodes(e.graph, nodes.data(), &n);
        for (size_t i = 0; ce == cudaSuccess && i < n; ++i) {
            cudaGraphNodeType t;
            if (cudaGraphNodeGetType(nodes[i], &t) != cudaSuccess || t != cudaGraphNodeTypeMemcpy) continue;
            cudaMemcpy3DParms p{};
            if (cudaGraphMemcpyNodeGetParams(nodes[i], &p) != cudaSuccess) continue;
            if (p.dstPtr.ptr == m_dStage) e.inputCopy = nodes[i];
        }
        if (ce == cudaSuccess && m_b.ce == cudaSuccess && !e.inputCopy) ce = cudaErrorUnknown;
        if (ce != cudaSuccess || m_b.ce != cudaSuccess) {
            // nothing of the batch ran: graphs off for this searcher, the batch launched directly
            if (e.exec) cudaGraphExecDestroy(e.exec);
            if (e.graph) cudaGraphDestroy(e.graph);
            m_graphFailure = cudaGetErrorString(ce != cudaSuccess ? ce : m_b.ce);
            cudaGetLastError();
            m_graphs = false;
            const uint32_t nq = m_b.nq;
            const float* dq = m_b.dQueries;
            m_b = Batch{};
            m_b.dQueries = dq;
            m_b.nq = nq;
            m_b.stream = stream;
            return EnqueueAttempt(rows, in, dOutScores, dOutIds, dOutCounts, outStride) == 0 && m_b.ce == cudaSuccess
                       ? 0
                       : -2;
        }
        e.batch = m_b;
        if (m_graphCache.size() >= kGraphCacheSize) {
            auto lru = std::min_element(m_graphCache.begin(), m_graphCache.end(),
                                        [](const GraphEntry& x, const GraphEntry& y) { return x.used < y.used; });
            cudaGraphExecDestroy(lru->exec);
            cudaGraphDestroy(lru->graph);
            m_graphCache.erase(lru);
        }
        m_graphCache.push_back(e);
        g = &m_graphCache.back();
        ++m_graphCaptures;
        m_graphCaptureMs += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    } else {
        // the launch plan is the shape's: restore it around this batch's own rows and stream
        const uint32_t nq = m_b.nq;
        m_b = g->batch;
        m_b.nq = nq;
        m_b.stream = stream;
        m_b.ce = cudaSuccess;
        m_b.pending = false;
        ++m_graphReplays;
    }
    g->used = ++m_graphClock;
    uint8_t* H = m_hStage;
    uint8_t* D = m_dStage;
    Ck(cudaGraphExecMemcpyNodeSetParams1D(g->exec, g->inputCopy, D, H, InputBytes(in), cudaMemcpyHostToDevice));
    Ck(cudaGraphLaunch(g->exec, stream));
    return m_b.ce == cudaSuccess ? 0 : -2;
}

int FullRecallSearcher::EnqueueAttempt(uint32_t nq, const BatchInputs& in, float* dOutScores, int64_t* dOutIds,
                                       uint32_t* dOutCounts, uint32_t outStride) {
    const StageLayout SL = MakeLayout(m_cfg.maxBatch);
    uint8_t* H = m_hStage;
    uint8_t* D = m_dStage;
    const float* dQueries = m_b.dQueries;
    cudaStream_t stream = m_b.stream;
    auto* dTopk = reinterpret_cast<uint32_t*>(D + SL.topk);
    auto* dEpsMain = reinterpret_cast<float*>(D + SL.epsMain);
    auto* dTheta = reinterpret_cast<float*>(D + SL.theta);
    auto* dCandCount = reinterpret_cast<uint32_t*>(D + SL.candCount);
    auto* dStatus = reinterpret_cast<int32_t*>(D + SL.status);

    const DataTable& T = *m_table;
    const uint64_t words = T.GetBitmapWords();
    if (m_timing) Ck(cudaEventRecord(m_ev[0], stream));
    const uint32_t maxK = in.maxK;
    if (EnqueueFilter(nq, in, m_dBits, words, stream) != 0) Ck(cudaErrorUnknown);
    ++m_b.launches;
    Stage(nullptr, nq);
    ++m_b.launches;
    if (m_timing) Ck(cudaEventRecord(m_ev[1], stream));

    // 1. doc sample: evenly spaced tiles, every filtered doc kept; its K-th best bounds the threshold.
    // Without a model it grows with K so that its threshold keeps the full pass within the list
    // capacity; with one, the prediction sets the threshold and the sample only feeds the features
    // (which are made from the same sample size, with or without a model set).
    const bool learned = static_cast<bool>(m_model);
    m_b.wantRerun = SampleWant(maxK);
    m_b.want = learned || m_featuresOut != nullptr ? m_cfg.sampleDocs : m_b.wantRerun;
    m_b.learned = learned;
    const bool wantStats = learned || m_featuresOut != nullptr;
    // the sample's proven thresholds (theta_1) are also kept in theta1, copied to the host with the
    // statuses (a copy here would stall the stream between the sample and the passes)
    auto* dTheta1 = reinterpret_cast<float*>(D + SL.theta1);
    uint64_t sampCount;
    if (m_b.want > m_cfg.sampleDocs) {
        // A sample grown with K in two steps: the sample_docs sample's proven threshold first, then the
        // grown sample keeps only the docs above it. Its K-th best is the same whenever it has K docs
        // above that threshold (and raises theta_1 then); otherwise theta_1 stays. Every doc of the
        // grown sample is otherwise stored and walked (K = 1000 at 10M: about 76k per query).
        const uint64_t grown = m_b.want;
        m_b.want = m_cfg.sampleDocs;
        (void)Sample(nullptr, nq, false, false, nullptr, dTheta1);
        m_b.want = grown;
        sampCount = Sample(nullptr, nq, false, true, nullptr, dTheta1, dTheta);
        m_b.launches += 4;
    } else {
        sampCount = Sample(nullptr, nq, false, false, wantStats ? m_dStats : nullptr, dTheta1);
        m_b.launches += 2;
    }
    if (m_featuresOut) {
        Ck(LaunchFeatures(T, D, SL.opndOff, SL.prog, SL.passCount, SL.topk, m_dStats, dQueries, nq, FeatureDim(),
                          m_featuresOut, stream));
        Ck(cudaStreamSynchronize(stream));
        return 1;
    }
    auto* dThetaPr = reinterpret_cast<float*>(D + SL.thetaPr);
    if (learned) {
        // the model's predicted K-th score minus the margin and the error bound, never below theta_1;
        // theta_1 stays in dThetaPr for the select step's check
        Ck(LaunchFeatures(T, D, SL.opndOff, SL.prog, SL.passCount, SL.topk, m_dStats, dQueries, nq, FeatureDim(),
                          m_dX, stream));
        if (m_model->Forward(m_dX, nq, m_dYp, stream) != 0) Ck(cudaErrorUnknown);
        Ck(launch_predict_theta(m_dYp, dEpsMain, reinterpret_cast<const uint32_t*>(D + SL.passCount), dTopk,
                                m_dStats, nq, m_model->scale, m_model->shift, m_margin, dTheta, dThetaPr, m_dYp,
                                stream));
        m_b.launches += 5;
    }
    if (m_timing) Ck(cudaEventRecord(m_ev[2], stream));

    // 2. the full pass, progressively: first every split-th tile (about sqrt(sample / corpus) of it)
    // with the sample's threshold; the K-th best of that part then raises each query's threshold
    // (every doc of the top K scores at least K-th best - 2 eps) for the remaining tiles. Both parts'
    // candidates form one segmented list.
    const uint32_t C = m_cfg.candidateCap;
    const uint64_t tilesM = TilesOf(UnitOf(nq, false));
    // Pass A's share as the sample that bounds the full pass would set it: with a model the sample
    // stays small, but pass A's proven K-th best still raises the threshold of pass B as far as
    // without one (a pass A of 1/8 of the corpus at K = 1000 and 10M docs rather than 1/17)
    uint64_t splitSample = sampCount;
    if (learned) {
        uint64_t step = 1;
        SampleTiles(m_b.wantRerun, nq, false, &splitSample, &step);
    }
    uint32_t split = static_cast<uint32_t>(std::sqrt(static_cast<double>(tilesM) / static_cast<double>(splitSample)));
    split = std::min<uint32_t>(split, 64);
    SelectLaunch& SE = m_b.se;
    SE.vec = T.DeviceVectors();
    SE.qry = dQueries;
    SE.dim = T.GetDimension();
    SE.cand_score = m_dCandScore;
    SE.cand_loc = m_dCandLoc;
    SE.cand_count = dCandCount;
    SE.cap = C;
    SE.work = m_dWork;
    SE.topk = dTopk;
    SE.eps_main = dEpsMain;
    SE.theta = dTheta;
    SE.gdocid = T.DeviceGDocIds();
    SE.out_score = dOutScores;
    SE.out_id = dOutIds;
    SE.out_count = dOutCounts;
    SE.out_stride = outStride;
    SE.status = dStatus;
    SE.qlist = nullptr;
    SE.nq_list = nq;
    // a batch with a large K keeps long candidate lists (K = 1000: about 13k per query at 10M, past
    // the default shared-memory buffer): select K from {10, 100, 1000} 0.302 -> 0.199 ms
    SE.fast_large = maxK > 256 ? 1 : 0;
    // With a model, theta is the prediction: the passes below run at it (raised like a proven one
    // when pass A's K-th best allows), and the select step checks every query whose theta stayed
    // above its proven threshold; a query that fails is re-run at a proven threshold.
    SE.theta_proven = learned ? dThetaPr : nullptr;
    if (split >= 2) {
        const uint64_t countA = (tilesM + split - 1) / split, countB = tilesM - countA;
        const uint32_t segsA = SegsOf(nq, countA, C, false), segsB = SegsOf(nq, countB, C, false);
        const uint32_t segCap = std::min(SegCapOf(nq, countA, C, segsA + segsB, false),
                                         SegCapOf(nq, countB, C, segsA + segsB, false));
        Cand(dTheta, m_dCandScore, m_dCandLoc, dCandCount, C, 0, segCap, 0, split, 0, countA, nullptr, nq, false);
        SampleThresholdLaunch RT{};
        RT.score = m_dCandScore;
        RT.count = dCandCount;
        RT.cap = C;
        RT.segs = segsA;
        RT.seg_cap = segCap;
        RT.raise_only = 1;
        RT.topk = dTopk;
        RT.eps_sample = dEpsMain;  // t - 2 eps_main
        RT.eps_main = dEpsMain;
        RT.theta = dTheta;
        RT.theta_also = learned ? dThetaPr : nullptr;
        RT.qlist = nullptr;
        RT.nq_list = nq;
        Ck(launch_sample_threshold(RT, stream));
        Cand(dTheta, m_dCandScore, m_dCandLoc, dCandCount, C, segsA, segCap, 0, 1, split, countB, nullptr, nq, false);
        m_b.launches += 3;
        SE.segs = segsA + segsB;
        SE.seg_cap = segCap;
    } else {
        const uint32_t segs = SegsOf(nq, tilesM, C, false);
        SE.segs = segs;
        SE.seg_cap = SegCapOf(nq, tilesM, C, segs, false);
        Cand(dTheta, m_dCandScore, m_dCandLoc, dCandCount, C, 0, SE.seg_cap, 0, 1, 0, tilesM, nullptr, nq, false);
        ++m_b.launches;
    }
    if (m_timing) Ck(cudaEventRecord(m_ev[3], stream));

    // 3. exact rescoring and the top K
    Ck(launch_select_topk(SE, stream));
    ++m_b.launches;
    if (m_timing) Ck(cudaEventRecord(m_ev[4], stream));
    // the statuses that decide re-runs (and the tensor-core pass's error bits), on the host when
    // m_evStatus (recorded by the caller) completes
    // one copy for the statuses and theta_1 (theta1 follows status in the staging layout)
    Ck(cudaMemcpyAsync(H + SL.status, dStatus, (SL.theta1 - SL.status) + nq * 4ull, cudaMemcpyDeviceToHost, stream));
    if (m_tcFormat >= 0) Ck(cudaMemcpyAsync(H + SL.errWord, m_dError, 4, cudaMemcpyDeviceToHost, stream));
    // the model's thresholds (m_dYp is not written after the prediction)
    if (learned) Ck(cudaMemcpyAsync(m_hThetaA, m_dYp, nq * 4ull, cudaMemcpyDeviceToHost, stream));
    return 0;
}

int FullRecallSearcher::SearchFinish() {
    if (!m_b.pending) return 0;
    m_b.pending = false;
    if (cudaSetDevice(m_deviceId) != cudaSuccess) return -2;
    const StageLayout SL = MakeLayout(m_cfg.maxBatch);
    uint8_t* H = m_hStage;
    uint8_t* D = m_dStage;
    const uint32_t nq = m_b.nq;
    cudaStream_t stream = m_b.stream;
    auto* dQlist = reinterpret_cast<uint32_t*>(D + SL.qlist);
    auto* dStatus = reinterpret_cast<int32_t*>(D + SL.status);
    auto* dTheta = reinterpret_cast<float*>(D + SL.theta);
    auto* dCandCount = reinterpret_cast<uint32_t*>(D + SL.candCount);
    auto* hStatus = reinterpret_cast<int32_t*>(H + SL.status);
    auto* hQlist = reinterpret_cast<uint32_t*>(H + SL.qlist);
    const bool tc = m_tcFormat >= 0;
    const uint32_t C = m_cfg.candidateCap;
    SelectLaunch& SE = m_b.se;
    uint32_t retries = 0;
    bool firstSync = true;
    for (;;) {
        if (firstSync) {
            Ck(cudaEventSynchronize(m_evStatus));
        } else {
            Ck(cudaMemcpyAsync(hStatus, dStatus, nq * 4ull, cudaMemcpyDeviceToHost, stream));
            Ck(cudaStreamSynchronize(stream));
        }
        if (firstSync && m_b.ce == cudaSuccess) {
            const float* h1 = reinterpret_cast<const float*>(H + SL.theta1);
            m_lastTheta1.assign(h1, h1 + nq);
            if (m_b.learned)
                m_lastThetaA.assign(m_hThetaA, m_hThetaA + nq);
            else
                m_lastThetaA.assign(nq, -INFINITY);
        }
        firstSync = false;
        if (m_b.ce != cudaSuccess) break;
        uint32_t nre = 0;
        for (uint32_t q = 0; q < nq; ++q) {
            m_lastStatus[q] |= hStatus[q] & ~(kStatusOverflow | kStatusThresholdMiss);
            if (hStatus[q] & kStatusThresholdMiss) m_lastMiss[q] = 1;
            if (hStatus[q] & kStatusOverflow) hQlist[nre++] = q;
        }
        if (nre == 0) break;
        if (retries >= m_cfg.maxRetries) {
            for (uint32_t i = 0; i < nre; ++i) m_lastStatus[hQlist[i]] |= kStatusOverflow;
            break;
        }
        ++retries;
        Ck(cudaMemcpyAsync(dQlist, hQlist, nre * 4ull, cudaMemcpyHostToDevice, stream));
        Ck(cudaMemsetAsync(dStatus, 0, nq * 4ull, stream));
        // A tensor-core re-run helps when the first threshold was loose. When the docs inside the
        // 2 eps band around the K-th score alone overflow the list, only a tighter bound helps: from the
        // second re-run on, the queries go through the FP32 SIMT pass (bound ~2 gamma_d |q||v|). Their
        // thresholds stay valid (every bound derived so far was at least the SIMT one).
        const bool simt = tc && retries >= 2;
        if (simt) {
            // the plain path for these queries: SIMT bounds (for the re-run queries only, so every other
            // query keeps the bound its own pass used), a SIMT doc sample for a fresh threshold
            const DataTable& T = *m_table;
            const double rel = SimtRelBound(T.GetDimension());
            Ck(launch_query_eps(m_b.dQueries, dQlist, nre, T.GetDimension(), T.GetMaxNorm(), rel, rel,
                                reinterpret_cast<float*>(D + SL.epsMain), reinterpret_cast<float*>(D + SL.epsSamp),
                                stream));
            m_b.want = m_b.wantRerun;
            (void)Sample(dQlist, nre, true);
            m_b.launches += 3;
        } else if (tc) {
            Stage(dQlist, nre);  // the staged rows become the re-run queries (their bounds unchanged)
            ++m_b.launches;
        }
        // one pass over every tile with the raised threshold; on the tensor-core path in two parts, as
        // in the first attempt: every kRerunSplit-th tile first, whose K-th best raises the threshold
        // for the rest (a query re-run because its predicted threshold kept fewer than K docs comes
        // back with only its doc sample's threshold, which may be far too low for one full pass)
        const uint64_t tilesR = TilesOf(UnitOf(nre, simt));
        uint32_t segs, segCap;
        if (!simt && tilesR >= 2ull * kRerunSplit) {
            const uint64_t countA = (tilesR + kRerunSplit - 1) / kRerunSplit, countB = tilesR - countA;
            const uint32_t segsA = SegsOf(nre, countA, C, false), segsB = SegsOf(nre, countB, C, false);
            segCap = std::min(SegCapOf(nre, countA, C, segsA + segsB, false),
                              SegCapOf(nre, countB, C, segsA + segsB, false));
            segs = segsA + segsB;
            Cand(dTheta, m_dCandScore, m_dCandLoc, dCandCount, C, 0, segCap, 0, kRerunSplit, 0, countA, dQlist, nre,
                 false);
            SampleThresholdLaunch RT{};
            RT.score = m_dCandScore;
            RT.count = dCandCount;
            RT.cap = C;
            RT.segs = segsA;
            RT.seg_cap = segCap;
            RT.raise_only = 1;
            RT.topk = reinterpret_cast<const uint32_t*>(D + SL.topk);
            RT.eps_sample = reinterpret_cast<const float*>(D + SL.epsMain);  // t - 2 eps_main
            RT.eps_main = reinterpret_cast<const float*>(D + SL.epsMain);
            RT.theta = dTheta;
            RT.theta_also = SE.theta_proven;
            RT.qlist = dQlist;
            RT.nq_list = nre;
            Ck(launch_sample_threshold(RT, stream));
            Cand(dTheta, m_dCandScore, m_dCandLoc, dCandCount, C, segsA, segCap, 0, 1, kRerunSplit, countB, dQlist,
                 nre, false);
            m_b.launches += 2;
        } else {
            segs = SegsOf(nre, tilesR, C, simt);
            segCap = SegCapOf(nre, tilesR, C, segs, simt);
            Cand(dTheta, m_dCandScore, m_dCandLoc, dCandCount, C, 0, segCap, 0, 1, 0, tilesR, dQlist, nre, simt);
        }
        for (uint32_t i = 0; i < nre; ++i) m_lastSegs[hQlist[i]] = {segs, segCap};
        SE.segs = segs;
        SE.seg_cap = segCap;
        SE.qlist = dQlist;
        SE.nq_list = nre;
        Ck(launch_select_topk(SE, stream));
        m_b.launches += 2;
    }
    if (tc && m_b.ce == cudaSuccess) {
        // the copy made with the statuses covers the first attempt; re-runs need a fresh one (stream
        // ordered: no device-wide synchronisation, so another searcher's batch queued behind this one
        // keeps running)
        auto* hErr = reinterpret_cast<int32_t*>(H + SL.errWord);
        if (retries > 0) {
            Ck(cudaMemcpyAsync(hErr, m_dError, 4, cudaMemcpyDeviceToHost, stream));
            Ck(cudaStreamSynchronize(stream));
        }
        const int32_t herr = *hErr;
        if (m_b.ce == cudaSuccess && herr != 0) {
            m_err = "tensor-core candidate pass timed out waiting on its pipeline (error bits " +
                    std::to_string(herr) + ")";
            cudaMemsetAsync(m_dError, 0, sizeof(int32_t), stream);
            cudaStreamSynchronize(stream);
            return -2;
        }
    }
    if (m_timing && m_b.ce == cudaSuccess) {
        cudaEventSynchronize(m_ev[4]);
        cudaEventElapsedTime(&m_times.filter, m_ev[0], m_ev[1]);
        cudaEventElapsedTime(&m_times.sample, m_ev[1], m_ev[2]);
        cudaEventElapsedTime(&m_times.candidates, m_ev[2], m_ev[3]);
        cudaEventElapsedTime(&m_times.select, m_ev[3], m_ev[4]);
        cudaEventElapsedTime(&m_times.total, m_ev[0], m_ev[4]);
    }
    m_times.retries = retries;
    m_times.launches = m_b.launches;
    if (m_b.ce != cudaSuccess) {
        m_err = cudaGetErrorString(m_b.ce);
        return -2;
    }
    int bad = 0;
    for (uint32_t q = 0; q < nq; ++q) bad += m_lastStatus[q] != 0;
    return bad;
}

int FullRecallSearcher::LastCandidates(uint32_t q, float* scores, uint32_t* locs, uint32_t cap, uint32_t* count,
                                       float* theta, float* eps) {
    if (!m_ok || q >= m_cfg.maxBatch) return -1;
    if (cudaSetDevice(m_deviceId) != cudaSuccess) return -2;
    if (q >= m_lastSegs.size()) return -1;
    const StageLayout SL = MakeLayout(m_cfg.maxBatch);
    const auto sg = m_lastSegs[q];
    std::vector<uint32_t> cnt(kMaxCandSegs);
    cudaError_t e = cudaMemcpy(cnt.data(), m_dStage + SL.candCount + 4ull * kMaxCandSegs * q, 4ull * kMaxCandSegs,
                               cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(theta, m_dStage + SL.theta + 4ull * q, 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(eps, m_dStage + SL.epsMain + 4ull * q, 4, cudaMemcpyDeviceToHost);
    // the stored entries of every segment, in segment order
    uint32_t total = 0, got = 0;
    const uint64_t row = static_cast<uint64_t>(q) * m_cfg.candidateCap;
    for (uint32_t g = 0; g < sg.first && e == cudaSuccess; ++g) {
        total += cnt[g];
        const uint32_t k = std::min({cnt[g], sg.second, cap - got});
        if (k == 0) continue;
        const uint64_t at = row + static_cast<uint64_t>(g) * sg.second;
        e = cudaMemcpy(scores + got, m_dCandScore + at, 4ull * k, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(locs + got, m_dCandLoc + at, 4ull * k, cudaMemcpyDeviceToHost);
        got += k;
    }
    *count = total;
    return e == cudaSuccess ? 0 : -2;
}

bool FullRecallSearcher::BatchSearch(std::vector<std::shared_ptr<FullRecallResult>>& results,
                                     const std::string& vectorFieldName, bool isMultiShard) {
    const uint32_t nq = static_cast<uint32_t>(m_queries.size());
    const uint32_t dim = m_table ? m_table->GetDimension() : 0;
    auto finish = [&](bool ok) {
        ClearQueries();
        return ok;
    };
    if (!m_ok) return finish(false);
    if (vectorFieldName != m_table->GetConfig().vectorField) {
        m_err = "unknown vector field " + vectorFieldName;
        return finish(false);
    }
    if (m_queryVectors.size() != static_cast<size_t>(nq) * dim) {
        m_err = "query vector dimension mismatch";
        return finish(false);
    }
    results.clear();
    for (uint32_t b0 = 0; b0 < nq; b0 += m_cfg.maxBatch) {
        const uint32_t nb = std::min(m_cfg.maxBatch, nq - b0);
        std::vector<FilterExpr> exprs(nb);
        std::vector<const FilterExpr*> ptrs(nb);
        for (uint32_t i = 0; i < nb; ++i) {
            if (!PrepareExpr(m_queries[b0 + i], *m_table, exprs[i], &m_err)) return finish(false);
            ptrs[i] = &exprs[i];
        }
        cudaStream_t stream = nullptr;
        if (cudaSetDevice(m_deviceId) != cudaSuccess) return finish(false);
        if (cudaMemcpyAsync(m_dQueries, m_queryVectors.data() + static_cast<size_t>(b0) * dim, nb * dim * 4ull,
                            cudaMemcpyHostToDevice, stream) != cudaSuccess)
            return finish(false);
        const int rc = SearchDevice(m_dQueries, nb, ptrs.data(), m_topKs.data() + b0, m_dOutScore, m_dOutId,
                                    m_dOutCount, kMaxTopK, stream);
        if (rc < 0) return finish(false);
        cudaMemcpyAsync(m_hOutCount, m_dOutCount, nb * 4ull, cudaMemcpyDeviceToHost, stream);
        cudaMemcpyAsync(m_hOutScore, m_dOutScore, nb * kMaxTopK * 4ull, cudaMemcpyDeviceToHost, stream);
        cudaMemcpyAsync(m_hOutId, m_dOutId, nb * kMaxTopK * 8ull, cudaMemcpyDeviceToHost, stream);
        if (cudaStreamSynchronize(stream) != cudaSuccess) return finish(false);
        for (uint32_t i = 0; i < nb; ++i) {
            auto r = std::make_shared<FullRecallResult>();
            r->isMultiShard = isMultiShard;
            const uint32_t c = m_lastStatus[i] ? 0u : m_hOutCount[i];
            const float* sc = m_hOutScore + static_cast<size_t>(i) * kMaxTopK;
            const int64_t* id = m_hOutId + static_cast<size_t>(i) * kMaxTopK;
            for (uint32_t j = 0; j < c; ++j) {
                if (isMultiShard) {
                    ScoreWithIndex s(sc[j], static_cast<uint32_t>(id[j] - static_cast<int64_t>(m_table->GetConfig().docOffset)));
                    s.id = static_cast<uint64_t>(id[j]);
                    r->scoreWithIndexes.push_back(s);
                } else {
                    r->scores.push_back(sc[j]);
                    r->docIds.push_back(id[j]);
                }
            }
            results.push_back(r);
        }
        if (rc > 0) {
            m_err = "some queries failed (see per-query status)";
        }
    }
    return finish(true);
}

}  // namespace hss
