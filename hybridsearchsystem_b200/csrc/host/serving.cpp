// serving.cpp -- ServingLoop: continuous batching of single filtered top-K queries over a resident
// table (the request loop around FullRecallSearcher; the reference's counterpart is its
// RunContext/schedule_* request drivers, run_context.cpp:121-274, whose batches are formed before
// they are run).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>

#include "../hss_device.cuh"
#include "hss_host.h"

namespace hss {

namespace {
bool CudaOkS(cudaError_t e, std::string* err, const char* what) {
    if (e == cudaSuccess) return true;
    *err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}
}  // namespace

ServingLoop::ServingLoop(std::shared_ptr<DataTable> table, const ServingConfig& cfg)
    : m_table(std::move(table)), m_cfg(cfg) {
    if (!m_table || m_table->DeviceVectors() == nullptr) {
        m_err = "table has no device residency";
        return;
    }
    if (m_cfg.slots == 0) m_cfg.slots = 1;
    if (m_cfg.maxBatch == 0) m_cfg.maxBatch = 1;
    m_dim = m_table->GetDimension();
    const int dev = m_table->GetDeviceId();
    if (!CudaOkS(cudaSetDevice(dev), &m_err, "cudaSetDevice")) return;
    SearcherConfig sc = m_cfg.searcher;
    sc.maxBatch = m_cfg.maxBatch;
    size_t free0 = 0, total = 0;
    if (!CudaOkS(cudaMemGetInfo(&free0, &total), &m_err, "cudaMemGetInfo")) return;
    const uint64_t budget = m_cfg.memoryBudget ? m_cfg.memoryBudget : free0 / 2;
    uint64_t perSlot = 0;
    for (uint32_t i = 0; i < m_cfg.slots; ++i) {
        // admission by device memory: a slot is added only while the arenas fit the budget
        size_t before = 0, after = 0;
        cudaMemGetInfo(&before, &total);
        if (i > 0 && perSlot * (i + 1) > budget) break;
        auto slot = std::make_unique<Slot>();
        slot->searcher = std::make_unique<FullRecallSearcher>(dev, m_table, sc);
        if (!slot->searcher->Ok()) {
            m_err = slot->searcher->Error();
            return;
        }
        const size_t B = sc.maxBatch;
        const size_t K = kMaxTopK;
        if (!CudaOkS(cudaStreamCreateWithFlags(&slot->stream, cudaStreamNonBlocking), &m_err, "cudaStreamCreate") ||
            !CudaOkS(cudaMallocHost(&slot->hQ, B * m_dim * 4), &m_err, "cudaMallocHost") ||
            !CudaOkS(cudaMalloc(&slot->dQ, B * m_dim * 4), &m_err, "cudaMalloc") ||
            !CudaOkS(cudaMallocHost(&slot->hSc, B * K * 4), &m_err, "cudaMallocHost") ||
            !CudaOkS(cudaMalloc(&slot->dSc, B * K * 4), &m_err, "cudaMalloc") ||
            !CudaOkS(cudaMallocHost(&slot->hId, B * K * 8), &m_err, "cudaMallocHost") ||
            !CudaOkS(cudaMalloc(&slot->dId, B * K * 8), &m_err, "cudaMalloc") ||
            !CudaOkS(cudaMallocHost(&slot->hCnt, B * 4), &m_err, "cudaMallocHost") ||
            !CudaOkS(cudaMalloc(&slot->dCnt, B * 4), &m_err, "cudaMalloc")) {
            m_slots.push_back(std::move(slot));
            return;
        }
        // rows past a batch's own (graph replay pads a batch to its shape) read finite queries
        if (!CudaOkS(cudaMemset(slot->dQ, 0, B * m_dim * 4), &m_err, "cudaMemset")) {
            m_slots.push_back(std::move(slot));
            return;
        }
        slot->searcher->SetGraphs(m_cfg.graphs);
        cudaMemGetInfo(&after, &total);
        if (i == 0) perSlot = before > after ? before - after : 1;
        m_slots.push_back(std::move(slot));
    }
    for (auto& s : m_slots) s->worker = std::thread(&ServingLoop::Worker, this, s.get());
    m_ok = true;
}

ServingLoop::~ServingLoop() {
    {
        std::lock_guard<std::mutex> lk(m_mu);
        m_stop = true;
    }
    m_cvQueue.notify_all();
    for (auto& s : m_slots)
        if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(m_table ? m_table->GetDeviceId() : 0);
    for (auto& s : m_slots) {
        void* d[] = {s->dQ, s->dSc, s->dId, s->dCnt};
        for (void* p : d)
            if (p) cudaFree(p);
        void* h[] = {s->hQ, s->hSc, s->hId, s->hCnt};
        for (void* p : h)
            if (p) cudaFreeHost(p);
        if (s->stream) cudaStreamDestroy(s->stream);
        s->searcher.reset();
    }
}

int ServingLoop::Submit(const float* vec, uint32_t dim, const char* filter, uint32_t topK, uint64_t* id) {
    if (!m_ok || !vec || !id || dim != m_dim) return -1;
    auto r = std::make_shared<Request>();
    bool ok = true;
    auto ast = ParseFilter(filter ? filter : "", ok);
    if (!ok) return -3;
    auto tree = BuildQueryNode(ast.get(), m_table->GetConfig().postingField);
    std::string err;
    if (!PrepareExpr(tree.get(), *m_table, r->expr, &err)) return -4;
    r->vec.assign(vec, vec + dim);
    r->topK = topK;
    r->arrival = std::chrono::steady_clock::now();
    {
        std::lock_guard<std::mutex> lk(m_mu);
        r->id = m_nextId++;
        m_live[r->id] = r;
        m_queue.push_back(r);
    }
    m_cvQueue.notify_one();
    *id = r->id;
    return 0;
}

void ServingLoop::Worker(Slot* slot) {
    cudaSetDevice(m_table->GetDeviceId());
    const auto maxWait = std::chrono::microseconds(m_cfg.maxWaitUs);
    std::vector<std::shared_ptr<Request>> batch;
    for (;;) {
        std::shared_ptr<ThresholdModel> model;
        float margin = 0.0f;
        bool newModel = false, more = false;
        {
            std::unique_lock<std::mutex> lk(m_mu);
            m_cvQueue.wait(lk, [&] { return m_stop || !m_queue.empty(); });
            if (m_queue.empty()) return;  // stopping
            // fewer than a full batch queued: wait a little for more, measured from the oldest request
            const auto deadline = m_queue.front()->arrival + maxWait;
            while (!m_stop && m_queue.size() < m_cfg.maxBatch && std::chrono::steady_clock::now() < deadline)
                m_cvQueue.wait_until(lk, deadline);
            batch.clear();
            while (!m_queue.empty() && batch.size() < m_cfg.maxBatch) {
                batch.push_back(m_queue.front());
                m_queue.pop_front();
            }
            if (slot->modelGen != m_modelGen) {
                model = m_model;
                margin = m_margin;
                newModel = true;
                slot->modelGen = m_modelGen;
            }
            more = !m_queue.empty();
        }
        if (more) m_cvQueue.notify_one();  // more work for another slot
        if (newModel) slot->searcher->SetThresholdModel(model, margin);
        RunBatch(slot, batch);
    }
}

void ServingLoop::RunBatch(Slot* slot, std::vector<std::shared_ptr<Request>>& batch) {
    const uint32_t n = static_cast<uint32_t>(batch.size());
    std::vector<const FilterExpr*> exprs(n);
    std::vector<uint32_t> topks(n);
    uint32_t stride = 1;
    for (uint32_t i = 0; i < n; ++i) {
        std::memcpy(slot->hQ + static_cast<size_t>(i) * m_dim, batch[i]->vec.data(), m_dim * 4ull);
        exprs[i] = &batch[i]->expr;
        topks[i] = batch[i]->topK;
        stride = std::max(stride, std::min<uint32_t>(batch[i]->topK, kMaxTopK));
    }
    // graph replay: device rows of kMaxTopK entries whatever the batch's K (one stride for every
    // batch shape); the host takes the first `stride` entries of each row
    const uint32_t dStride = m_cfg.graphs ? static_cast<uint32_t>(kMaxTopK) : stride;
    cudaError_t e = cudaMemcpyAsync(slot->dQ, slot->hQ, static_cast<size_t>(n) * m_dim * 4, cudaMemcpyHostToDevice,
                                    slot->stream);
    int rc = e == cudaSuccess ? slot->searcher->SearchDevice(slot->dQ, n, exprs.data(), topks.data(), slot->dSc,
                                                             slot->dId, slot->dCnt, dStride, slot->stream)
                              : -2;
    if (rc >= 0) {
        e = cudaMemcpyAsync(slot->hCnt, slot->dCnt, n * 4ull, cudaMemcpyDeviceToHost, slot->stream);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(slot->hSc, stride * 4ull, slot->dSc, dStride * 4ull, stride * 4ull, n,
                                  cudaMemcpyDeviceToHost, slot->stream);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(slot->hId, stride * 8ull, slot->dId, dStride * 8ull, stride * 8ull, n,
                                  cudaMemcpyDeviceToHost, slot->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(slot->stream);
        if (e != cudaSuccess) rc = -2;
    }
    const auto now = std::chrono::steady_clock::now();
    const std::vector<int32_t>& st = slot->searcher->LastStatus();
    {
        std::lock_guard<std::mutex> lk(m_mu);
        for (uint32_t i = 0; i < n; ++i) {
            Request& r = *batch[i];
            r.done = now;
            if (rc < 0) {
                r.status = -2;
            } else {
                r.status = i < st.size() ? st[i] : 0;
                const uint32_t c = r.status ? 0u : std::min(slot->hCnt[i], stride);
                r.count = c;
                r.scores.assign(slot->hSc + static_cast<size_t>(i) * stride, slot->hSc + static_cast<size_t>(i) * stride + c);
                r.ids.assign(slot->hId + static_cast<size_t>(i) * stride, slot->hId + static_cast<size_t>(i) * stride + c);
            }
            r.finished = true;
            m_lat.push_back(std::chrono::duration<double, std::milli>(r.done - r.arrival).count());
        }
        ++m_batches;
        m_batched += n;
        slot->captures = slot->searcher->GraphCaptures();
        slot->replays = slot->searcher->GraphReplays();
        slot->captureMs = slot->searcher->GraphCaptureMs();
    }
    m_cvDone.notify_all();
}

int ServingLoop::Wait(uint64_t id, float* scores, int64_t* ids, uint32_t cap, uint32_t* count, double* latencyMs,
                      int32_t* status, int timeoutMs) {
    std::unique_lock<std::mutex> lk(m_mu);
    auto it = m_live.find(id);
    if (it == m_live.end()) return -1;
    std::shared_ptr<Request> r = it->second;
    auto pred = [&] { return r->finished; };
    if (timeoutMs < 0)
        m_cvDone.wait(lk, pred);
    else if (!m_cvDone.wait_for(lk, std::chrono::milliseconds(timeoutMs), pred))
        return 1;
    const uint32_t c = std::min(r->count, cap);
    if (scores) std::copy(r->scores.begin(), r->scores.begin() + c, scores);
    if (ids) std::copy(r->ids.begin(), r->ids.begin() + c, ids);
    if (count) *count = r->count;
    if (latencyMs) *latencyMs = std::chrono::duration<double, std::milli>(r->done - r->arrival).count();
    if (status) *status = r->status;
    m_live.erase(id);
    return 0;
}

ServingStats ServingLoop::Stats() const {
    std::lock_guard<std::mutex> lk(m_mu);
    ServingStats s;
    s.completed = m_lat.size();
    s.batches = m_batches;
    s.slots = static_cast<uint32_t>(m_slots.size());
    s.meanBatch = m_batches ? static_cast<double>(m_batched) / m_batches : 0.0;
    if (!m_lat.empty()) {
        std::vector<double> v = m_lat;
        std::sort(v.begin(), v.end());
        // percentile p = sorted[floor(p * n)] (report.cpp:67-70 of the reference's harness)
        auto pct = [&](double p) { return v[std::min(v.size() - 1, static_cast<size_t>(p * v.size()))]; };
        s.p50Ms = pct(0.50);
        s.p99Ms = pct(0.99);
        s.maxMs = v.back();
    }
    for (const auto& slot : m_slots) {
        s.graphCaptures += slot->captures;
        s.graphReplays += slot->replays;
        s.graphCaptureMs += slot->captureMs;
    }
    return s;
}

void ServingLoop::ResetStats() {
    std::lock_guard<std::mutex> lk(m_mu);
    m_lat.clear();
    m_batches = m_batched = 0;
}

int ServingLoop::RunPoisson(const float* queries, uint32_t n, const char* const* filters, const uint32_t* topks,
                            double rateQps, uint64_t seed, double* latencyMs, double* offeredQps, double* wallSeconds) {
    if (!m_ok || n == 0 || !queries || !filters || !topks || rateQps <= 0) return -1;
    std::vector<uint64_t> ids(n, 0);
    std::vector<int> rcs(n, 0);
    std::mt19937_64 rng(seed);
    std::exponential_distribution<double> gap(rateQps);
    std::vector<double> at(n);
    double t = 0;
    for (uint32_t i = 0; i < n; ++i) at[i] = (t += gap(rng));
    std::atomic<uint32_t> submitted{0};
    const auto t0 = std::chrono::steady_clock::now();
    std::chrono::steady_clock::time_point tEnd;
    // open-loop arrivals: each request is submitted at its Poisson arrival time, whatever the
    // completions do (a submitter that falls behind schedule is reported as a lower offered rate)
    std::thread submitter([&] {
        for (uint32_t i = 0; i < n; ++i) {
            const auto due = t0 + std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                                      std::chrono::duration<double>(at[i]));
            while (std::chrono::steady_clock::now() < due) {
            }
            rcs[i] = Submit(queries + static_cast<size_t>(i) * m_dim, m_dim, filters[i], topks[i], &ids[i]);
            submitted.store(i + 1, std::memory_order_release);
        }
        tEnd = std::chrono::steady_clock::now();
    });
    int bad = 0;
    for (uint32_t i = 0; i < n; ++i) {
        while (submitted.load(std::memory_order_acquire) <= i) std::this_thread::yield();
        double lat = -1;
        int32_t st = 0;
        if (rcs[i] != 0 || Wait(ids[i], nullptr, nullptr, 0, nullptr, &lat, &st, -1) != 0 || st != 0) ++bad;
        if (latencyMs) latencyMs[i] = lat;
    }
    submitter.join();
    const double subSeconds = std::chrono::duration<double>(tEnd - t0).count();
    if (offeredQps) *offeredQps = subSeconds > 0 ? n / subSeconds : 0;
    if (wallSeconds) *wallSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return bad;
}

int ServingLoop::SetThresholdModel(std::shared_ptr<ThresholdModel> model, float margin) {
    if (!m_ok) return -1;
    if (model && (!model->Ok() || model->Din() != m_slots[0]->searcher->FeatureDim())) return -1;
    std::lock_guard<std::mutex> lk(m_mu);
    m_model = std::move(model);
    m_margin = margin;
    ++m_modelGen;
    return 0;
}

}  // namespace hss
