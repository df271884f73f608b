// data_table.cpp -- index build, persistence and HBM residency (the reference's DataTable /
// PostingFieldData / VectorFieldData / DocIdMapping, src/engine/index/).
//
// Index directory written by Save() and read by LoadData():
//   hss_meta.json                                  doc count, dim, segment geometry, codec options
//   vectors.f32                                    [docNum][dim] float32, row-major
//   gdocid.i64                                     [docNum] int64 global doc ids
//   <field>/poissonengine_<ver>_<seg>_<field>.posting   one file per segment in the reference's
//        posting-file format (inverted_builder.cpp:178-250, file_writer.cpp:4-26): 9-byte file head
//        [version:1][reserved:5][extLen:2 = 1][type: '0' matrix / '1' bitmap], u32 tokenNum, the
//        token dict tokenNum x {u64 Hash64(token), u32 postingOffset, u32 tokenOffset} (offsets from
//        the file start), the postings (each padded to 4 bytes), then the token literals {u32 len, bytes}.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <sys/stat.h>
#include <thread>

#include "../hss_kernels.h"
#include "hss_host.h"

namespace hss {

namespace {
constexpr uint32_t kIndexVersion = 1;

unsigned HostThreads() {
    const unsigned n = std::thread::hardware_concurrency();
    return n == 0 ? 1 : std::min(n, 32u);
}

template <class F>
void ParallelFor(uint64_t n, F f) {
    const unsigned t = static_cast<unsigned>(std::min<uint64_t>(HostThreads(), n == 0 ? 1 : n));
    std::vector<std::thread> pool;
    for (unsigned i = 0; i < t; ++i)
        pool.emplace_back([&, i]() {
            for (uint64_t j = i; j < n; j += t) f(j);
        });
    for (auto& th : pool) th.join();
}

size_t Align16(size_t x) { return (x + 15) & ~static_cast<size_t>(15); }

bool Fail(std::string* err, const std::string& m) {
    if (err) *err = m;
    return false;
}

bool CudaOk(cudaError_t e, std::string* err, const char* what) {
    if (e == cudaSuccess) return true;
    return Fail(err, std::string(what) + ": " + cudaGetErrorString(e));
}

// Smallest float >= x.
float RoundUp(double x) {
    float f = static_cast<float>(x);
    if (static_cast<double>(f) < x) f = std::nextafter(f, INFINITY);
    return f;
}

std::string PostingFileName(uint32_t seg, const std::string& field) {
    return "poissonengine_" + std::to_string(kIndexVersion) + "_" + std::to_string(seg) + "_" + field + ".posting";
}

// Minimal flat JSON object writer/reader for the meta file (string and number values only).
std::string JsonGet(const std::string& s, const std::string& key) {
    const std::string k = "\"" + key + "\"";
    size_t p = s.find(k);
    if (p == std::string::npos) return "";
    p = s.find(':', p + k.size());
    if (p == std::string::npos) return "";
    ++p;
    while (p < s.size() && (s[p] == ' ' || s[p] == '\n' || s[p] == '\t')) ++p;
    if (p < s.size() && s[p] == '"') {
        const size_t e = s.find('"', p + 1);
        return s.substr(p + 1, e - p - 1);
    }
    size_t e = p;
    while (e < s.size() && s[e] != ',' && s[e] != '}' && s[e] != '\n') ++e;
    return s.substr(p, e - p);
}
}  // namespace

DataTable::~DataTable() { Release(); }

bool DataTable::EnableFormat(int format, std::string* err) {
    if (format < 0 || format > 2) return Fail(err, "unknown tensor-core format");
    if (m_fmtReady[format]) return true;
    if (m_dVectors == nullptr) return Fail(err, "table has no device residency");
    if (!CudaOk(cudaSetDevice(m_deviceId), err, "cudaSetDevice")) return false;
    const uint64_t rows = GetTileNum() * 128;
    const uint32_t elem = format == kTcBF16 ? 2 : (format == kTcE4M3 ? 1 : 4);
    if ((static_cast<uint64_t>(m_dim) * elem) % 128 != 0)
        return Fail(err, "dim * element size must be a multiple of 128 bytes for the tensor-core formats");
    void* out = nullptr;
    if (format != kTcTF32 && !CudaOk(cudaMalloc(&out, rows * m_dim * elem), err, "cudaMalloc quantised rows"))
        return false;
    float *scale = nullptr, *norm = nullptr, *errn = nullptr;
    bool ok = CudaOk(cudaMalloc(&norm, rows * sizeof(float)), err, "cudaMalloc norms") &&
              CudaOk(cudaMalloc(&errn, rows * sizeof(float)), err, "cudaMalloc norms");
    if (ok && format == kTcE4M3) ok = CudaOk(cudaMalloc(&scale, rows * sizeof(float)), err, "cudaMalloc scales");
    if (ok)
        ok = CudaOk(launch_quantize_docs(m_dVectors, rows, m_docNum, m_dim, format, out, scale, norm, errn, nullptr), err,
                    "quantise");
    std::vector<float> hn(rows), he(rows);
    if (ok) ok = CudaOk(cudaMemcpy(hn.data(), norm, rows * 4, cudaMemcpyDeviceToHost), err, "download norms");
    if (ok) ok = CudaOk(cudaMemcpy(he.data(), errn, rows * 4, cudaMemcpyDeviceToHost), err, "download norms");
    if (ok && format == kTcE4M3) {
        ok = CudaOk(cudaMalloc(&m_dTileScale, GetTileNum() * sizeof(float2)), err, "cudaMalloc tile scales") &&
             CudaOk(launch_tile_scale_minmax(scale, GetTileNum(), m_dTileScale, nullptr), err, "tile scales");
        m_dDocScale = scale;
        scale = nullptr;
    }
    cudaFree(norm);
    cudaFree(errn);
    if (scale) cudaFree(scale);
    if (!ok || !CudaOk(cudaDeviceSynchronize(), err, "quantise")) {
        if (out) cudaFree(out);
        return false;
    }
    double nm = 0, em = 0;
    for (uint64_t i = 0; i < rows; ++i) {
        nm = std::max(nm, static_cast<double>(hn[i]));
        em = std::max(em, static_cast<double>(he[i]));
    }
    m_dQuant[format] = out;
    m_fmtNormMax[format] = nm;
    m_fmtErrMax[format] = em;
    m_fmtReady[format] = true;
    return true;
}

bool DataTable::EnableDensePostings(uint64_t budgetBytes, std::string* err) {
    if (m_dDense) return true;
    if (m_dPostingTable == nullptr) return Fail(err, "table has no device residency");
    const uint64_t segBytes = GetSegmentByteSize();
    const uint64_t n = static_cast<uint64_t>(m_rows) * m_segmentNum;
    if (n * segBytes > budgetBytes) return true;  // over budget: batches keep decoding postings in place
    if (!CudaOk(cudaSetDevice(m_deviceId), err, "cudaSetDevice")) return false;
    uint64_t* dense = nullptr;
    uint64_t* ptrs = nullptr;  // [2][n]: source posting addresses, destination bitmap addresses
    int32_t* status = nullptr;
    bool ok = CudaOk(cudaMalloc(&dense, n * segBytes), err, "cudaMalloc dense postings") &&
              CudaOk(cudaMalloc(&ptrs, 2 * n * sizeof(uint64_t)), err, "cudaMalloc dense postings") &&
              CudaOk(cudaMalloc(&status, sizeof(int32_t)), err, "cudaMalloc dense postings") &&
              CudaOk(cudaMemset(status, 0, sizeof(int32_t)), err, "cudaMemset");
    // ordered full segments first, then the last (possibly partial) segment, which decodes with its
    // own doc count
    std::vector<uint64_t> table(n), hp(2 * n);
    if (ok) ok = CudaOk(cudaMemcpy(table.data(), m_dPostingTable, n * 8, cudaMemcpyDeviceToHost), err, "download");
    const uint32_t S = m_segmentNum;
    uint64_t at = 0;
    for (int pass = 0; pass < 2 && ok; ++pass)
        for (uint32_t r = 0; r < m_rows; ++r)
            for (uint32_t s = 0; s < S; ++s) {
                if ((s + 1 == S) != (pass == 1)) continue;
                hp[at] = table[static_cast<uint64_t>(r) * S + s];
                hp[n + at] = reinterpret_cast<uint64_t>(dense) + (static_cast<uint64_t>(r) * S + s) * segBytes;
                ++at;
            }
    if (ok) ok = CudaOk(cudaMemcpy(ptrs, hp.data(), 2 * n * 8, cudaMemcpyHostToDevice), err, "upload");
    const uint64_t full = static_cast<uint64_t>(m_rows) * (S - 1);
    const uint32_t lastDocs = static_cast<uint32_t>(m_docNum - static_cast<uint64_t>(S - 1) * m_cfg.docNumPerSegment);
    if (ok && full)
        ok = CudaOk(launch_posting_expand(ptrs, ptrs + n, static_cast<uint32_t>(full), static_cast<uint32_t>(segBytes),
                                          m_cfg.docNumPerSegment, status, nullptr),
                    err, "expand postings");
    if (ok)
        ok = CudaOk(launch_posting_expand(ptrs + full, ptrs + n + full, m_rows, static_cast<uint32_t>(segBytes),
                                          lastDocs, status, nullptr),
                    err, "expand postings");
    int32_t hs = 0;
    if (ok) ok = CudaOk(cudaMemcpy(&hs, status, 4, cudaMemcpyDeviceToHost), err, "expand postings");
    cudaFree(ptrs);
    cudaFree(status);
    if (!ok || hs != 0) {
        // a malformed posting: leave the in-place path, which reports it per query
        if (dense) cudaFree(dense);
        return ok;
    }
    m_dDense = dense;
    return true;
}

void DataTable::Release() {
    for (int f = 0; f < 3; ++f) m_fmtReady[f] = false;
    if (m_dDense) {
        if (m_deviceId >= 0) cudaSetDevice(m_deviceId);
        cudaFree(m_dDense);
        m_dDense = nullptr;
    }
    if (m_dVectors == nullptr && m_dArena == nullptr && m_dPostingTable == nullptr && m_dGDocIds == nullptr) return;
    if (m_deviceId >= 0) cudaSetDevice(m_deviceId);
    for (int f = 1; f < 3; ++f) {
        if (m_dQuant[f]) cudaFree(m_dQuant[f]);
        m_dQuant[f] = nullptr;
    }
    if (m_dDocScale) cudaFree(m_dDocScale);
    if (m_dTileScale) cudaFree(m_dTileScale);
    m_dDocScale = nullptr;
    m_dTileScale = nullptr;
    if (m_dVectors) cudaFree(m_dVectors);
    if (m_dArena) cudaFree(m_dArena);
    if (m_dPostingTable) cudaFree(m_dPostingTable);
    if (m_dGDocIds) cudaFree(m_dGDocIds);
    if (m_dRowDensity) cudaFree(m_dRowDensity);
    m_dRowDensity = nullptr;
    m_dVectors = nullptr;
    m_dArena = nullptr;
    m_dPostingTable = nullptr;
    m_dGDocIds = nullptr;
}

uint32_t DataTable::TokenRow(uint64_t token, bool& tokenExist) const {
    auto it = m_tokenRow.find(token);
    tokenExist = it != m_tokenRow.end();
    return tokenExist ? it->second : m_rows - 1;
}

const uint8_t* DataTable::HostPosting(uint32_t row, uint32_t seg, uint32_t* len) const {
    if (row + 1 >= m_rows || seg >= m_segmentNum) return nullptr;
    const int64_t off = m_rowSegOffset[row][seg];
    if (off < 0) return nullptr;
    if (len) *len = m_rowSegLen[row][seg];
    return reinterpret_cast<const uint8_t*>(m_segPostings[seg].data()) + off;
}

std::vector<uint8_t> DataTable::PostingTypes(uint32_t row) const {
    std::vector<uint8_t> t(m_segmentNum, 0);
    for (uint32_t s = 0; s < m_segmentNum; ++s) {
        const uint8_t* p = HostPosting(row, s, nullptr);
        if (p) t[s] = p[3] >> 4;
    }
    return t;
}

bool DataTable::Build(int32_t deviceId, const float* vectors, const uint64_t* tagBits, uint64_t docNum, uint32_t dim,
                      uint32_t tagNum, const IndexConfig& cfg, std::string* err) {
    return BuildImpl(deviceId, vectors, false, tagBits, docNum, dim, tagNum, cfg, err);
}

bool DataTable::BuildFromDevice(int32_t deviceId, const float* dVectors, const uint64_t* tagBits, uint64_t docNum,
                                uint32_t dim, uint32_t tagNum, const IndexConfig& cfg, std::string* err) {
    if (deviceId < 0) return Fail(err, "a build from device vectors needs a device");
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, dVectors) != cudaSuccess || at.type != cudaMemoryTypeDevice ||
        at.device != deviceId) {
        cudaGetLastError();
        return Fail(err, "vectors are not device memory of the table's device");
    }
    return BuildImpl(deviceId, dVectors, true, tagBits, docNum, dim, tagNum, cfg, err);
}

bool DataTable::BuildImpl(int32_t deviceId, const float* vectors, bool onDevice, const uint64_t* tagBits,
                          uint64_t docNum, uint32_t dim, uint32_t tagNum, const IndexConfig& cfg, std::string* err) {
    Release();
    if (docNum == 0 || docNum >= 0xffffffffull) return Fail(err, "docNum must be in [1, 2^32-1)");
    if (dim == 0 || dim % 4 != 0 || dim > 4096) return Fail(err, "dim must be a multiple of 4 in [4, 4096]");
    if (cfg.docNumPerSegment == 0 || cfg.docNumPerSegment % 128 != 0)
        return Fail(err, "doc_num_per_segment must be a positive multiple of 128");
    if (cfg.sparsePacked && cfg.docNumPerSegment > 16u * 65536u)
        return Fail(err, "SPARSE_PACKED needs doc_num_per_segment <= 1048576");
    m_deviceId = deviceId;
    m_cfg = cfg;
    m_docNum = docNum;
    m_dim = dim;
    const uint32_t P = cfg.docNumPerSegment;
    m_segmentNum = static_cast<uint32_t>((docNum + P - 1) / P);
    m_postingFields = {cfg.postingField};
    const uint32_t words = (tagNum + 63) / 64;

    // gdocids and the corpus norm bound (device vectors: after the upload, on the device)
    m_gdocids.resize(docNum);
    for (uint64_t i = 0; i < docNum; ++i) m_gdocids[i] = static_cast<int64_t>(cfg.docOffset + i);
    if (!onDevice) {
        const unsigned t = HostThreads();
        std::vector<double> mx(t, 0.0);
        const uint64_t per = (docNum + t - 1) / t;
        std::vector<std::thread> pool;
        for (unsigned i = 0; i < t; ++i)
            pool.emplace_back([&, i]() {
                const uint64_t a = std::min<uint64_t>(docNum, i * per), b = std::min<uint64_t>(docNum, a + per);
                double m = 0;
                for (uint64_t r = a; r < b; ++r) {
                    const float* v = vectors + r * dim;
                    double s = 0;
                    for (uint32_t d = 0; d < dim; ++d) s += static_cast<double>(v[d]) * v[d];
                    m = std::max(m, s);
                }
                mx[i] = m;
            });
        for (auto& th : pool) th.join();
        double m = 0;
        for (double x : mx) m = std::max(m, x);
        m_maxNorm = RoundUp(std::sqrt(m) * (1.0 + 1e-12));
    }

    // Postings: per segment, per tag, the sorted local ids (fr_converter + InvertedBuilder).
    std::vector<std::vector<std::vector<uint32_t>>> ids(m_segmentNum);
    ParallelFor(m_segmentNum, [&](uint64_t s) {
        auto& per = ids[s];
        per.assign(tagNum, {});
        const uint64_t d0 = s * P, d1 = std::min<uint64_t>(docNum, d0 + P);
        for (uint64_t doc = d0; doc < d1; ++doc) {
            const uint64_t* bm = tagBits + doc * words;
            for (uint32_t w = 0; w < words; ++w) {
                uint64_t x = bm[w];
                while (x) {
                    const uint32_t b = static_cast<uint32_t>(__builtin_ctzll(x));
                    const uint32_t tag = w * 64 + b;
                    if (tag < tagNum) per[tag].push_back(static_cast<uint32_t>(doc - d0));
                    x &= x - 1;
                }
            }
        }
    });
    std::vector<uint32_t> tagRow(tagNum, 0xffffffffu);
    m_tokens.clear();
    m_tokenText.clear();
    m_tokenRow.clear();
    for (uint32_t tag = 0; tag < tagNum; ++tag) {
        bool any = false;
        for (uint32_t s = 0; s < m_segmentNum && !any; ++s) any = !ids[s][tag].empty();
        if (!any) continue;
        tagRow[tag] = static_cast<uint32_t>(m_tokens.size());
        const std::string text = std::to_string(tag);
        m_tokenText.push_back(text);
        m_tokens.push_back(Hash64(text));
        m_tokenRow[m_tokens.back()] = tagRow[tag];
    }
    m_rows = static_cast<uint32_t>(m_tokens.size()) + 1;
    m_segPostings.assign(m_segmentNum, {});
    m_rowSegOffset.assign(m_rows - 1, std::vector<int64_t>(m_segmentNum, -1));
    m_rowSegLen.assign(m_rows - 1, std::vector<uint32_t>(m_segmentNum, 0));
    bool ok = true;
    ParallelFor(m_segmentNum, [&](uint64_t s) {
        const uint32_t segDocs = static_cast<uint32_t>(std::min<uint64_t>(P, docNum - s * P));
        std::string& buf = m_segPostings[s];
        for (uint32_t tag = 0; tag < tagNum; ++tag) {
            if (ids[s][tag].empty()) continue;
            const size_t at = buf.size();
            if (!PostingSerializer::Serialize(ids[s][tag], segDocs, cfg.matrixPosting, cfg.densityThreshold,
                                              cfg.sparsePacked, buf)) {
                ok = false;
                return;
            }
            m_rowSegLen[tagRow[tag]][s] = static_cast<uint32_t>(buf.size() - at);
            buf.resize((buf.size() + 3) & ~static_cast<size_t>(3), '\0');  // 4-byte padding
            m_rowSegOffset[tagRow[tag]][s] = static_cast<int64_t>(at);
        }
        std::vector<std::vector<uint32_t>>().swap(ids[s]);
    });
    if (!ok) return Fail(err, "posting serialisation failed");
    if (deviceId < 0) {  // host-only table: index build, filter compilation and Save without a GPU
        m_vectors.assign(vectors, vectors + docNum * dim);
        return true;
    }

    if (!CudaOk(cudaSetDevice(deviceId), err, "cudaSetDevice")) return false;
    const uint64_t rowsAlloc = GetTileNum() * 128;
    if (!CudaOk(cudaMalloc(&m_dVectors, rowsAlloc * dim * sizeof(float)), err, "cudaMalloc vectors")) return false;
    if (!CudaOk(cudaMemcpy(m_dVectors, vectors, docNum * dim * sizeof(float),
                           onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice),
                err, "upload vectors"))
        return false;
    if (rowsAlloc > docNum &&
        !CudaOk(cudaMemset(m_dVectors + docNum * dim, 0, (rowsAlloc - docNum) * dim * sizeof(float)), err,
                "memset vectors"))
        return false;
    if (onDevice) {
        // per-row norms (FP64 sums, rounded up) by the quantiser's FP32 mode, maximum on the host
        float* norm = nullptr;
        bool ok = CudaOk(cudaMalloc(&norm, rowsAlloc * sizeof(float)), err, "cudaMalloc norms") &&
                  CudaOk(launch_quantize_docs(m_dVectors, rowsAlloc, docNum, dim, kTcTF32, nullptr, nullptr, norm,
                                              nullptr, nullptr),
                         err, "row norms");
        std::vector<float> hn(rowsAlloc, 0.0f);
        if (ok) ok = CudaOk(cudaMemcpy(hn.data(), norm, rowsAlloc * sizeof(float), cudaMemcpyDeviceToHost), err,
                            "download norms");
        if (norm) cudaFree(norm);
        if (!ok) return false;
        float m = 0.0f;
        for (float x : hn) m = std::max(m, x);
        m_maxNorm = m;
    }
    return Upload(err);
}

// Postings, posting table and doc ids to the device. Vectors are uploaded by the caller.
bool DataTable::Upload(std::string* err) {
    const uint32_t P = m_cfg.docNumPerSegment;
    // The all-zero posting (PostingFieldData::BuildZeroPosting: an empty id set serialised dense).
    std::string zero;
    PostingSerializer::Serialize({}, P, m_cfg.matrixPosting, -1.0f, false, zero);
    std::vector<std::vector<size_t>> slot(m_rows - 1, std::vector<size_t>(m_segmentNum, 0));
    size_t cur = Align16(zero.size());
    for (uint32_t r = 0; r + 1 < m_rows; ++r)
        for (uint32_t s = 0; s < m_segmentNum; ++s)
            if (m_rowSegOffset[r][s] >= 0) {
                slot[r][s] = cur;
                cur += Align16(m_rowSegLen[r][s] + 8);
            }
    // Slack past the last posting: 8-byte reads may run past a posting's last byte, and an operand
    // given in the reference's dense-bitset convention is read for a whole segment bitset (P/8 bytes)
    // even when its (last-segment) payload is shorter.
    const size_t arenaBytes = cur + std::max<size_t>(128, P / 8 + 16);
    std::vector<uint8_t> arena(arenaBytes, 0);
    std::memcpy(arena.data(), zero.data(), zero.size());
    for (uint32_t r = 0; r + 1 < m_rows; ++r)
        for (uint32_t s = 0; s < m_segmentNum; ++s)
            if (m_rowSegOffset[r][s] >= 0)
                std::memcpy(arena.data() + slot[r][s], m_segPostings[s].data() + m_rowSegOffset[r][s],
                            m_rowSegLen[r][s]);
    if (!CudaOk(cudaSetDevice(m_deviceId), err, "cudaSetDevice")) return false;
    if (!CudaOk(cudaMalloc(&m_dArena, arenaBytes), err, "cudaMalloc postings")) return false;
    if (!CudaOk(cudaMemcpy(m_dArena, arena.data(), arenaBytes, cudaMemcpyHostToDevice), err, "upload postings"))
        return false;
    const uint64_t base = reinterpret_cast<uint64_t>(m_dArena);
    std::vector<uint64_t> table(static_cast<size_t>(m_rows) * m_segmentNum, base);  // default: zero posting
    for (uint32_t r = 0; r + 1 < m_rows; ++r)
        for (uint32_t s = 0; s < m_segmentNum; ++s)
            if (m_rowSegOffset[r][s] >= 0) table[static_cast<size_t>(r) * m_segmentNum + s] = base + slot[r][s];
    if (!CudaOk(cudaMalloc(&m_dPostingTable, table.size() * sizeof(uint64_t)), err, "cudaMalloc posting table"))
        return false;
    if (!CudaOk(cudaMemcpy(m_dPostingTable, table.data(), table.size() * sizeof(uint64_t), cudaMemcpyHostToDevice),
                err, "upload posting table"))
        return false;
    if (!CudaOk(cudaMalloc(&m_dGDocIds, m_docNum * sizeof(int64_t)), err, "cudaMalloc gdocids")) return false;
    if (!CudaOk(cudaMemcpy(m_dGDocIds, m_gdocids.data(), m_docNum * sizeof(int64_t), cudaMemcpyHostToDevice), err,
                "upload gdocids"))
        return false;
    // fraction of docs holding each row's token: the hit counts of the posting heads ([layout:4|hits:28])
    std::vector<float> density(m_rows, 0.0f);
    for (uint32_t r = 0; r + 1 < m_rows; ++r) {
        uint64_t hits = 0;
        for (uint32_t s = 0; s < m_segmentNum; ++s)
            if (m_rowSegOffset[r][s] >= 0 && m_rowSegLen[r][s] >= 4) {
                uint32_t head = 0;
                std::memcpy(&head, m_segPostings[s].data() + m_rowSegOffset[r][s], 4);
                hits += head & 0x0fffffffu;
            }
        density[r] = m_docNum ? static_cast<float>(static_cast<double>(hits) / static_cast<double>(m_docNum)) : 0.0f;
    }
    if (!CudaOk(cudaMalloc(&m_dRowDensity, m_rows * sizeof(float)), err, "cudaMalloc row density")) return false;
    if (!CudaOk(cudaMemcpy(m_dRowDensity, density.data(), m_rows * sizeof(float), cudaMemcpyHostToDevice), err,
                "upload row density"))
        return false;
    return true;
}

bool DataTable::Save(const std::string& dir, std::string* err) const {
    if (m_dVectors == nullptr && m_vectors.size() != m_docNum * m_dim) return Fail(err, "table not loaded");
    ::mkdir(dir.c_str(), 0755);
    const std::string pdir = dir + "/" + m_cfg.postingField;
    ::mkdir(pdir.c_str(), 0755);
    {
        std::ofstream m(dir + "/hss_meta.json");
        m << "{\n  \"version\": " << kIndexVersion << ",\n  \"doc_num\": " << m_docNum << ",\n  \"dim\": " << m_dim
          << ",\n  \"doc_num_per_segment\": " << m_cfg.docNumPerSegment << ",\n  \"segment_num\": " << m_segmentNum
          << ",\n  \"doc_offset\": " << m_cfg.docOffset << ",\n  \"density_threshold\": "
          << m_cfg.densityThreshold << ",\n  \"matrix_posting\": " << (m_cfg.matrixPosting ? 1 : 0)
          << ",\n  \"sparse_packed\": " << (m_cfg.sparsePacked ? 1 : 0) << ",\n  \"posting_field\": \""
          << m_cfg.postingField << "\",\n  \"vector_field\": \"" << m_cfg.vectorField << "\"\n}\n";
        if (!m) return Fail(err, "write meta");
    }
    {
        std::vector<float> v(m_docNum * m_dim);
        if (m_dVectors) {
            if (!CudaOk(cudaSetDevice(m_deviceId), err, "cudaSetDevice")) return false;
            if (!CudaOk(cudaMemcpy(v.data(), m_dVectors, v.size() * sizeof(float), cudaMemcpyDeviceToHost), err,
                        "download vectors"))
                return false;
        } else {
            v = m_vectors;
        }
        std::ofstream f(dir + "/vectors.f32", std::ios::binary);
        f.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(float)));
        std::ofstream g(dir + "/gdocid.i64", std::ios::binary);
        g.write(reinterpret_cast<const char*>(m_gdocids.data()),
                static_cast<std::streamsize>(m_gdocids.size() * sizeof(int64_t)));
        if (!f || !g) return Fail(err, "write vectors / gdocids");
    }
    for (uint32_t s = 0; s < m_segmentNum; ++s) {
        std::vector<uint32_t> rows;
        for (uint32_t r = 0; r + 1 < m_rows; ++r)
            if (m_rowSegOffset[r][s] >= 0) rows.push_back(r);
        std::string head;
        const uint8_t ver = static_cast<uint8_t>(kIndexVersion);
        head.push_back(static_cast<char>(ver));
        head.append(5, '\0');
        const uint16_t extLen = 1;
        head.append(reinterpret_cast<const char*>(&extLen), 2);
        head.push_back(m_cfg.matrixPosting ? '0' : '1');
        const uint32_t tokenNum = static_cast<uint32_t>(rows.size());
        const uint64_t prefix = head.size() + 4 + 16ull * tokenNum;
        std::string postings, literals, dict;
        std::vector<uint32_t> pOff, tOff;
        for (uint32_t r : rows) {
            pOff.push_back(static_cast<uint32_t>(prefix + postings.size()));
            postings.append(m_segPostings[s].data() + m_rowSegOffset[r][s], m_rowSegLen[r][s]);
            postings.resize((postings.size() + 3) & ~static_cast<size_t>(3), '\0');
            tOff.push_back(static_cast<uint32_t>(literals.size()));
            const uint32_t tl = static_cast<uint32_t>(m_tokenText[r].size());
            literals.append(reinterpret_cast<const char*>(&tl), 4);
            literals.append(m_tokenText[r]);
        }
        if (prefix + postings.size() + literals.size() > 0xffffffffull) return Fail(err, "posting file over 4 GiB");
        const uint32_t postingEnd = static_cast<uint32_t>(prefix + postings.size());
        for (size_t i = 0; i < rows.size(); ++i) {
            const uint64_t h = m_tokens[rows[i]];
            const uint32_t to = tOff[i] + postingEnd;
            dict.append(reinterpret_cast<const char*>(&h), 8);
            dict.append(reinterpret_cast<const char*>(&pOff[i]), 4);
            dict.append(reinterpret_cast<const char*>(&to), 4);
        }
        std::ofstream f(pdir + "/" + PostingFileName(s, m_cfg.postingField), std::ios::binary);
        f.write(head.data(), static_cast<std::streamsize>(head.size()));
        f.write(reinterpret_cast<const char*>(&tokenNum), 4);
        f.write(dict.data(), static_cast<std::streamsize>(dict.size()));
        f.write(postings.data(), static_cast<std::streamsize>(postings.size()));
        f.write(literals.data(), static_cast<std::streamsize>(literals.size()));
        if (!f) return Fail(err, "write posting file");
    }
    return true;
}

bool DataTable::LoadData(int32_t deviceId, const std::string& dir, std::string* err) {
    Release();
    std::ifstream mf(dir + "/hss_meta.json");
    if (!mf) return Fail(err, "meta file not found in " + dir);
    std::stringstream ss;
    ss << mf.rdbuf();
    const std::string meta = ss.str();
    IndexConfig cfg;
    try {
        m_docNum = std::stoull(JsonGet(meta, "doc_num"));
        m_dim = static_cast<uint32_t>(std::stoul(JsonGet(meta, "dim")));
        cfg.docNumPerSegment = static_cast<uint32_t>(std::stoul(JsonGet(meta, "doc_num_per_segment")));
        m_segmentNum = static_cast<uint32_t>(std::stoul(JsonGet(meta, "segment_num")));
        cfg.docOffset = std::stoull(JsonGet(meta, "doc_offset"));
        cfg.densityThreshold = std::stof(JsonGet(meta, "density_threshold"));
        cfg.matrixPosting = std::stoi(JsonGet(meta, "matrix_posting")) != 0;
        cfg.sparsePacked = std::stoi(JsonGet(meta, "sparse_packed")) != 0;
        cfg.postingField = JsonGet(meta, "posting_field");
        cfg.vectorField = JsonGet(meta, "vector_field");
    } catch (...) {
        return Fail(err, "malformed meta file");
    }
    if (m_docNum == 0 || m_dim == 0 || m_dim % 4 || cfg.docNumPerSegment == 0 || cfg.docNumPerSegment % 128 ||
        m_segmentNum != (m_docNum + cfg.docNumPerSegment - 1) / cfg.docNumPerSegment)
        return Fail(err, "inconsistent meta file");
    m_cfg = cfg;
    m_deviceId = deviceId;
    m_postingFields = {cfg.postingField};
    const uint32_t P = cfg.docNumPerSegment;

    // postings (PostingFieldData::AddSegment / ParseTokenDict / FinishAdd)
    m_tokens.clear();
    m_tokenText.clear();
    m_tokenRow.clear();
    m_segPostings.assign(m_segmentNum, {});
    std::vector<std::vector<std::pair<uint32_t, std::pair<int64_t, uint32_t>>>> segEntries(m_segmentNum);
    for (uint32_t s = 0; s < m_segmentNum; ++s) {
        std::ifstream f(dir + "/" + cfg.postingField + "/" + PostingFileName(s, cfg.postingField), std::ios::binary);
        if (!f) return Fail(err, "posting file missing for segment " + std::to_string(s));
        std::string file((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
        if (file.size() < 13) return Fail(err, "posting file too short");
        uint16_t extLen;
        std::memcpy(&extLen, file.data() + 6, 2);
        const size_t dictAt = 8 + extLen;
        if (file.size() < dictAt + 4) return Fail(err, "posting file header");
        uint32_t tokenNum;
        std::memcpy(&tokenNum, file.data() + dictAt, 4);
        const size_t regionAt = dictAt + 4 + 16ull * tokenNum;
        if (file.size() < regionAt) return Fail(err, "posting dict truncated");
        const uint32_t segDocs = static_cast<uint32_t>(std::min<uint64_t>(P, m_docNum - static_cast<uint64_t>(s) * P));
        m_segPostings[s] = file.substr(regionAt);
        for (uint32_t i = 0; i < tokenNum; ++i) {
            uint64_t h;
            uint32_t po, to;
            const char* e = file.data() + dictAt + 4 + 16ull * i;
            std::memcpy(&h, e, 8);
            std::memcpy(&po, e + 8, 4);
            std::memcpy(&to, e + 12, 4);
            if (po < regionAt || po >= to || to > file.size()) return Fail(err, "posting dict offsets");
            const uint8_t* p = reinterpret_cast<const uint8_t*>(file.data()) + po;
            std::string why;
            if (!ValidatePosting(p, to - po, segDocs, &why)) return Fail(err, "corrupt posting: " + why);
            uint32_t plen;
            std::memcpy(&plen, p + 4, 4);
            auto it = m_tokenRow.find(h);
            uint32_t row;
            if (it == m_tokenRow.end()) {
                row = static_cast<uint32_t>(m_tokens.size());
                m_tokenRow[h] = row;
                m_tokens.push_back(h);
                uint32_t tl = 0;
                std::string text;
                if (to + 4ull <= file.size()) {
                    std::memcpy(&tl, file.data() + to, 4);
                    if (to + 4ull + tl <= file.size()) text.assign(file.data() + to + 4, tl);
                }
                m_tokenText.push_back(text);
            } else {
                row = it->second;
            }
            segEntries[s].push_back({row, {static_cast<int64_t>(po - regionAt), 8 + plen}});
        }
    }
    // Canonical row order: by token literal, shorter first (numeric order for decimal tag tokens), the
    // order Build() assigns, so a saved and reloaded index is the same table.
    std::vector<uint32_t> order(m_tokens.size());
    for (uint32_t i = 0; i < order.size(); ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        const std::string &x = m_tokenText[a], &y = m_tokenText[b];
        if (x.size() != y.size()) return x.size() < y.size();
        if (x != y) return x < y;
        return m_tokens[a] < m_tokens[b];
    });
    std::vector<uint32_t> rowOf(order.size());
    std::vector<uint64_t> tokens(order.size());
    std::vector<std::string> texts(order.size());
    for (uint32_t r = 0; r < order.size(); ++r) {
        rowOf[order[r]] = r;
        tokens[r] = m_tokens[order[r]];
        texts[r] = m_tokenText[order[r]];
        m_tokenRow[tokens[r]] = r;
    }
    m_tokens.swap(tokens);
    m_tokenText.swap(texts);
    m_rows = static_cast<uint32_t>(m_tokens.size()) + 1;
    m_rowSegOffset.assign(m_rows - 1, std::vector<int64_t>(m_segmentNum, -1));
    m_rowSegLen.assign(m_rows - 1, std::vector<uint32_t>(m_segmentNum, 0));
    for (uint32_t s = 0; s < m_segmentNum; ++s)
        for (auto& e : segEntries[s]) {
            m_rowSegOffset[rowOf[e.first]][s] = e.second.first;
            m_rowSegLen[rowOf[e.first]][s] = e.second.second;
        }

    // vectors, doc ids, norm bound
    std::vector<float> v(m_docNum * m_dim);
    {
        std::ifstream f(dir + "/vectors.f32", std::ios::binary);
        f.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(float)));
        if (!f) return Fail(err, "vectors.f32 missing or short");
        m_gdocids.resize(m_docNum);
        std::ifstream g(dir + "/gdocid.i64", std::ios::binary);
        g.read(reinterpret_cast<char*>(m_gdocids.data()), static_cast<std::streamsize>(m_docNum * sizeof(int64_t)));
        if (!g) return Fail(err, "gdocid.i64 missing or short");
    }
    double mx = 0;
    for (uint64_t r = 0; r < m_docNum; ++r) {
        double s = 0;
        for (uint32_t d = 0; d < m_dim; ++d) s += static_cast<double>(v[r * m_dim + d]) * v[r * m_dim + d];
        mx = std::max(mx, s);
    }
    m_maxNorm = RoundUp(std::sqrt(mx) * (1.0 + 1e-12));
    if (deviceId < 0) {
        m_vectors = std::move(v);
        return true;
    }
    if (!CudaOk(cudaSetDevice(deviceId), err, "cudaSetDevice")) return false;
    const uint64_t rowsAlloc = GetTileNum() * 128;
    if (!CudaOk(cudaMalloc(&m_dVectors, rowsAlloc * m_dim * sizeof(float)), err, "cudaMalloc vectors")) return false;
    if (!CudaOk(cudaMemset(m_dVectors, 0, rowsAlloc * m_dim * sizeof(float)), err, "memset vectors")) return false;
    if (!CudaOk(cudaMemcpy(m_dVectors, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice), err,
                "upload vectors"))
        return false;
    return Upload(err);
}

}  // namespace hss
