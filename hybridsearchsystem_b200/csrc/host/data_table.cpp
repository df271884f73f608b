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
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <dirent.h>
#include <fstream>
#include <sstream>
#include <chrono>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <thread>
#include <unistd.h>

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

std::string PostingFileName(uint32_t seg, const std::string& field, uint32_t ver = kIndexVersion) {
    return "poissonengine_" + std::to_string(ver) + "_" + std::to_string(seg) + "_" + field + ".posting";
}

using Clock = std::chrono::steady_clock;
double MsSince(Clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

// A read-only mapping of a whole file.
struct MappedFile {
    const uint8_t* data = nullptr;
    size_t size = 0;
    bool Open(const std::string& path) {
        const int fd = ::open(path.c_str(), O_RDONLY);
        if (fd < 0) return false;
        struct stat st {};
        if (::fstat(fd, &st) != 0) {
            ::close(fd);
            return false;
        }
        size = static_cast<size_t>(st.st_size);
        void* p = size ? ::mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0) : nullptr;
        ::close(fd);
        if (size && p == MAP_FAILED) return false;
        data = static_cast<const uint8_t*>(p);
        return true;
    }
    ~MappedFile() {
        if (data) ::munmap(const_cast<uint8_t*>(data), size);
    }
};

// The reference's file head (file_writer.cpp:4-26, file_header.cpp:20-38):
// [version:1][reserved:5][extendedLen:2][extended:extendedLen].
std::string FileHead(uint8_t ver, const std::string& ext) {
    std::string h(1, static_cast<char>(ver));
    h.append(5, '\0');
    const uint16_t n = static_cast<uint16_t>(ext.size());
    h.append(reinterpret_cast<const char*>(&n), 2);
    h.append(ext);
    return h;
}
bool ParseHead(const uint8_t* p, size_t size, uint8_t* ver, std::string* ext, size_t* bodyAt) {
    if (size < 8) return false;
    uint16_t n;
    std::memcpy(&n, p + 6, 2);
    if (size < 8ull + n) return false;
    *ver = p[0];
    ext->assign(reinterpret_cast<const char*>(p) + 8, n);
    *bodyAt = 8ull + n;
    return true;
}

// IEEE binary16 <-> binary32 as the reference's Float32ToFloat16 / Float16ToFloat32 convert
// (trans_number.cpp:38-105): round to nearest even; inputs and results below the normal range of
// binary16 become signed zero; overflow becomes infinity; NaN stays NaN.
uint16_t HalfFromFloat(float f) {
    uint32_t b;
    std::memcpy(&b, &f, 4);
    const uint32_t sign = (b >> 16) & 0x8000u, e = (b >> 23) & 0xffu, m = b & 0x7fffffu;
    if (e == 0) return static_cast<uint16_t>(sign);
    // (an infinity, whose payload is zero, becomes the NaN 0x7c01 as well, as the reference's does)
    if (e == 0xff) return static_cast<uint16_t>(sign | 0x7c00u | std::max<uint32_t>(1u, (m >> 13) & 0x3ffu));
    int32_t he = static_cast<int32_t>(e) - 112;  // rebias 127 -> 15
    if (he >= 31) return static_cast<uint16_t>(sign | 0x7c00u);
    if (he <= 0) return static_cast<uint16_t>(sign);
    uint32_t hm = m >> 13;
    const uint32_t rest = m & 0x1fffu;  // the 13 dropped bits: half-way is 0x1000
    if (rest > 0x1000u || (rest == 0x1000u && (hm & 1u))) {
        if (++hm == 0x400u) {
            hm = 0;
            if (++he >= 31) return static_cast<uint16_t>(sign | 0x7c00u);
        }
    }
    return static_cast<uint16_t>(sign | (static_cast<uint32_t>(he) << 10) | hm);
}
float FloatFromHalf(uint16_t h) {
    const uint32_t sign = (h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
    uint32_t b;
    if (e == 0)
        b = sign;  // subnormal halves read as signed zero
    else if (e == 31)
        b = sign | 0x7f800000u | (m << 13);
    else
        b = sign | ((e + 112) << 23) | (m << 13);
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

// A small JSON reader for the reference's meta file (protobuf's JSON form of IndexMeta: objects,
// arrays, strings and numbers).
struct Json {
    enum Kind { kNull, kNum, kStr, kArr, kObj } kind = kNull;
    double num = 0;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;
    const Json* Get(const std::string& a, const std::string& b = "") const {
        for (const auto& kv : obj)
            if (kv.first == a || (!b.empty() && kv.first == b)) return &kv.second;
        return nullptr;
    }
};
bool ParseJson(const std::string& s, size_t& i, Json& out, int depth = 0) {
    auto ws = [&]() {
        while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
    };
    auto str = [&](std::string& o) {
        if (i >= s.size() || s[i] != '"') return false;
        for (++i; i < s.size() && s[i] != '"'; ++i) {
            if (s[i] == '\\' && i + 1 < s.size()) ++i;
            o.push_back(s[i]);
        }
        if (i >= s.size()) return false;
        ++i;
        return true;
    };
    if (depth > 16) return false;
    ws();
    if (i >= s.size()) return false;
    if (s[i] == '{') {
        out.kind = Json::kObj;
        ++i;
        ws();
        if (i < s.size() && s[i] == '}') return ++i, true;
        for (;;) {
            ws();
            std::string k;
            if (!str(k)) return false;
            ws();
            if (i >= s.size() || s[i] != ':') return false;
            ++i;
            Json v;
            if (!ParseJson(s, i, v, depth + 1)) return false;
            out.obj.emplace_back(std::move(k), std::move(v));
            ws();
            if (i < s.size() && s[i] == ',') {
                ++i;
                continue;
            }
            if (i < s.size() && s[i] == '}') return ++i, true;
            return false;
        }
    }
    if (s[i] == '[') {
        out.kind = Json::kArr;
        ++i;
        ws();
        if (i < s.size() && s[i] == ']') return ++i, true;
        for (;;) {
            Json v;
            if (!ParseJson(s, i, v, depth + 1)) return false;
            out.arr.push_back(std::move(v));
            ws();
            if (i < s.size() && s[i] == ',') {
                ++i;
                continue;
            }
            if (i < s.size() && s[i] == ']') return ++i, true;
            return false;
        }
    }
    if (s[i] == '"') {
        out.kind = Json::kStr;
        return str(out.str);
    }
    size_t e = i;
    while (e < s.size() && (std::isalnum(static_cast<unsigned char>(s[e])) || s[e] == '-' || s[e] == '+' || s[e] == '.'))
        ++e;
    const std::string tok = s.substr(i, e - i);
    i = e;
    if (tok == "null" || tok == "true" || tok == "false") return true;
    try {
        out.num = std::stod(tok);
    } catch (...) {
        return false;
    }
    out.kind = Json::kNum;
    return true;
}
// A uint32 field of IndexMeta's JSON form: the number, or its decimal string (protobuf's printer
// writes 64-bit integers as strings), 0 when absent (proto3 JSON omits zero values).
uint64_t JsonUint(const Json* v) {
    if (!v) return 0;
    if (v->kind == Json::kNum) return v->num < 0 ? 0 : static_cast<uint64_t>(v->num);
    if (v->kind == Json::kStr) {
        try {
            return std::stoull(v->str);
        } catch (...) {
        }
    }
    return 0;
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
    return WritePostingFiles(dir, err);
}

// The posting files of the table's posting field (inverted_builder.cpp:178-250, file_writer.cpp:4-26).
bool DataTable::WritePostingFiles(const std::string& dir, std::string* err) const {
    const std::string pdir = dir + "/" + m_cfg.postingField;
    ::mkdir(pdir.c_str(), 0755);
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
    m_loadTimes = LoadTimes{};
    const auto t0 = Clock::now();
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
    m_loadTimes.meta = MsSince(t0);
    if (!ReadPostingFiles(dir, cfg.postingField, kIndexVersion, err)) return false;
    m_gdocids.resize(m_docNum);
    {
        std::ifstream g(dir + "/gdocid.i64", std::ios::binary);
        g.read(reinterpret_cast<char*>(m_gdocids.data()), static_cast<std::streamsize>(m_docNum * sizeof(int64_t)));
        if (!g) return Fail(err, "gdocid.i64 missing or short");
    }
    MappedFile vf;
    if (!vf.Open(dir + "/vectors.f32") || vf.size < m_docNum * m_dim * sizeof(float))
        return Fail(err, "vectors.f32 missing or short");
    const uint32_t dim = m_dim;
    const bool ok = FinishRows(
        deviceId,
        [&](uint64_t r0, uint64_t r1, float* dst) {
            std::memcpy(dst, vf.data + r0 * dim * sizeof(float), (r1 - r0) * dim * sizeof(float));
        },
        err);
    m_loadTimes.total = MsSince(t0);
    return ok;
}

bool DataTable::ReadPostingFiles(const std::string& dir, const std::string& field, uint32_t ver, std::string* err) {
    // PostingFieldData::AddSegment / ParseTokenDict / FinishAdd
    const auto t0 = Clock::now();
    const uint32_t P = m_cfg.docNumPerSegment;
    m_tokens.clear();
    m_tokenText.clear();
    m_tokenRow.clear();
    m_segPostings.assign(m_segmentNum, {});
    std::vector<std::vector<std::pair<uint32_t, std::pair<int64_t, uint32_t>>>> segEntries(m_segmentNum);
    uint64_t bytes = 0;
    for (uint32_t s = 0; s < m_segmentNum; ++s) {
        std::ifstream f(dir + "/" + field + "/" + PostingFileName(s, field, ver), std::ios::binary);
        if (!f) return Fail(err, "posting file missing for segment " + std::to_string(s));
        std::string file((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
        bytes += file.size();
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
    m_loadTimes.postingsRead = MsSince(t0);
    m_loadTimes.postingBytes = bytes;
    return true;
}

bool DataTable::FinishRows(int32_t deviceId, const std::function<void(uint64_t, uint64_t, float*)>& fill,
                           std::string* err) {
    const auto t0 = Clock::now();
    const uint32_t dim = m_dim;
    const unsigned T = HostThreads();
    m_loadTimes.threads = T;
    m_loadTimes.vectorBytes = m_docNum * dim * sizeof(float);
    // rows [r0, r1) into dst on T threads
    auto parallelFill = [&](uint64_t r0, uint64_t r1, float* dst) {
        const uint64_t n = r1 - r0, per = (n + T - 1) / T;
        std::vector<std::thread> pool;
        for (unsigned i = 0; i < T; ++i) {
            const uint64_t a = std::min(n, i * per), b = std::min(n, a + per);
            if (a < b) pool.emplace_back([&, a, b]() { fill(r0 + a, r0 + b, dst + a * dim); });
        }
        for (auto& th : pool) th.join();
    };
    if (deviceId < 0) {  // host-only table
        m_vectors.assign(m_docNum * dim, 0.0f);
        parallelFill(0, m_docNum, m_vectors.data());
        double mx = 0;
        for (uint64_t r = 0; r < m_docNum; ++r) {
            double s2 = 0;
            for (uint32_t d = 0; d < dim; ++d) s2 += static_cast<double>(m_vectors[r * dim + d]) * m_vectors[r * dim + d];
            mx = std::max(mx, s2);
        }
        m_maxNorm = RoundUp(std::sqrt(mx) * (1.0 + 1e-12));
        m_loadTimes.vectorsRead = MsSince(t0);
        return true;
    }
    if (!CudaOk(cudaSetDevice(deviceId), err, "cudaSetDevice")) return false;
    const uint64_t rowsAlloc = GetTileNum() * 128;
    if (!CudaOk(cudaMalloc(&m_dVectors, rowsAlloc * dim * sizeof(float)), err, "cudaMalloc vectors")) return false;
    if (rowsAlloc > m_docNum &&
        !CudaOk(cudaMemset(m_dVectors + m_docNum * dim, 0, (rowsAlloc - m_docNum) * dim * sizeof(float)), err,
                "memset vectors"))
        return false;
    // two pinned staging chunks of ~64 MB: host threads fill one while the other is copied
    const uint64_t chunkRows = std::max<uint64_t>(1, (64ull << 20) / (dim * sizeof(float)));
    float* pin[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaStream_t st = nullptr;
    bool ok = CudaOk(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), err, "cudaStreamCreate");
    for (int b = 0; b < 2 && ok; ++b)
        ok = CudaOk(cudaMallocHost(&pin[b], chunkRows * dim * sizeof(float)), err, "cudaMallocHost staging") &&
             CudaOk(cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming), err, "cudaEventCreate");
    double fillMs = 0;
    for (uint64_t r0 = 0, c = 0; ok && r0 < m_docNum; r0 += chunkRows, ++c) {
        const uint64_t r1 = std::min(m_docNum, r0 + chunkRows);
        const int b = static_cast<int>(c & 1);
        if (c >= 2) ok = CudaOk(cudaEventSynchronize(ev[b]), err, "staging copy");
        if (!ok) break;
        const auto f0 = Clock::now();
        parallelFill(r0, r1, pin[b]);
        fillMs += MsSince(f0);
        ok = CudaOk(cudaMemcpyAsync(m_dVectors + r0 * dim, pin[b], (r1 - r0) * dim * sizeof(float),
                                    cudaMemcpyHostToDevice, st),
                    err, "upload vectors") &&
             CudaOk(cudaEventRecord(ev[b], st), err, "cudaEventRecord");
    }
    if (ok) ok = CudaOk(cudaStreamSynchronize(st), err, "upload vectors");
    for (int b = 0; b < 2; ++b) {
        if (pin[b]) cudaFreeHost(pin[b]);
        if (ev[b]) cudaEventDestroy(ev[b]);
    }
    if (st) cudaStreamDestroy(st);
    if (!ok) return false;
    m_loadTimes.vectorsRead = fillMs;
    m_loadTimes.vectorsH2D = MsSince(t0);
    // the corpus norm bound: per-row FP64 norms rounded up (the quantiser's FP32 mode), maximum here
    {
        float* norm = nullptr;
        bool nok = CudaOk(cudaMalloc(&norm, rowsAlloc * sizeof(float)), err, "cudaMalloc norms") &&
                   CudaOk(launch_quantize_docs(m_dVectors, rowsAlloc, m_docNum, dim, kTcTF32, nullptr, nullptr, norm,
                                               nullptr, nullptr),
                          err, "row norms");
        std::vector<float> hn(rowsAlloc, 0.0f);
        if (nok) nok = CudaOk(cudaMemcpy(hn.data(), norm, rowsAlloc * sizeof(float), cudaMemcpyDeviceToHost), err,
                              "download norms");
        if (norm) cudaFree(norm);
        if (!nok) return false;
        float m = 0.0f;
        for (float x : hn) m = std::max(m, x);
        m_maxNorm = m;
    }
    const auto u0 = Clock::now();
    const bool up = Upload(err);
    m_loadTimes.postingsH2D = MsSince(u0);
    return up;
}

bool DataTable::LoadReferenceIndex(int32_t deviceId, const std::string& dir, std::string* err) {
    Release();
    m_loadTimes = LoadTimes{};
    const auto t0 = Clock::now();
    // the meta file: the first *.meta of the directory (by name); its version is the name's 2nd field
    std::string metaName;
    {
        struct stat st {};
        if (::stat(dir.c_str(), &st) != 0 || !S_ISDIR(st.st_mode)) return Fail(err, "index directory not found: " + dir);
        std::vector<std::string> names;
        if (DIR* d = ::opendir(dir.c_str())) {
            while (dirent* e = ::readdir(d)) {
                const std::string n = e->d_name;
                if (n.size() > 5 && n.compare(n.size() - 5, 5, ".meta") == 0) names.push_back(n);
            }
            ::closedir(d);
        }
        if (names.empty()) return Fail(err, "meta file not exist in " + dir);
        std::sort(names.begin(), names.end());
        metaName = names[0];
    }
    uint32_t ver = 0;
    {
        const std::string stem = metaName.substr(0, metaName.size() - 5);
        const size_t a = stem.find('_');
        const size_t b = a == std::string::npos ? a : stem.find('_', a + 1);
        try {
            if (a == std::string::npos) throw 0;
            ver = static_cast<uint32_t>(std::stoul(stem.substr(a + 1, b == std::string::npos ? b : b - a - 1)));
        } catch (...) {
            return Fail(err, "meta filename invalid: " + metaName);
        }
        if (ver > 255) return Fail(err, "meta filename invalid: " + metaName);
    }
    Json meta;
    {
        std::ifstream mf(dir + "/" + metaName);
        std::stringstream ss;
        ss << mf.rdbuf();
        size_t i = 0;
        if (!mf || !ParseJson(ss.str(), i, meta) || meta.kind != Json::kObj) return Fail(err, "malformed meta file");
    }
    const Json* config = meta.Get("config");
    const Json* schema = meta.Get("schema");
    const Json* stats = meta.Get("statistics");
    if (!config || !schema || !stats) return Fail(err, "meta file lacks config / schema / statistics");
    const uint64_t P = JsonUint(config->Get("docNumPerSegment", "doc_num_per_segment"));
    const uint64_t zn = JsonUint(config->Get("splitDocNumZn", "split_doc_num_zn"));
    m_docNum = JsonUint(stats->Get("docNum", "doc_num"));
    m_segmentNum = static_cast<uint32_t>(JsonUint(stats->Get("segmentNum", "segment_num")));
    const Json* pf = schema->Get("posting");
    const Json* vfs = schema->Get("vector");
    if (!pf || pf->kind != Json::kArr || pf->arr.empty() || pf->arr[0].kind != Json::kStr || !vfs ||
        vfs->kind != Json::kArr || vfs->arr.empty() || vfs->arr[0].kind != Json::kStr)
        return Fail(err, "meta schema needs a posting and a vector field");
    if (m_docNum == 0 || m_docNum >= 0xffffffffull || P == 0 || zn == 0 ||
        m_segmentNum != (m_docNum + P - 1) / P)
        return Fail(err, "inconsistent meta file");
    if (P % 128 != 0)
        return Fail(err, "doc_num_per_segment " + std::to_string(P) +
                             " is not a multiple of 128 (this library's segment geometry; the reference needs 8)");
    IndexConfig cfg;
    cfg.docNumPerSegment = static_cast<uint32_t>(P);
    cfg.postingField = pf->arr[0].str;
    cfg.vectorField = vfs->arr[0].str;
    m_cfg = cfg;
    m_deviceId = deviceId;
    m_postingFields = {cfg.postingField};
    m_loadTimes.meta = MsSince(t0);
    if (!ReadPostingFiles(dir, cfg.postingField, ver, err)) return false;

    // doc ids (DocIdMapping::Load, doc_id_mapping.cpp:38-114): the global-id form only
    m_gdocids.clear();
    m_gdocids.reserve(m_docNum);
    for (uint32_t s = 0; s < m_segmentNum; ++s) {
        const uint64_t segDocs = std::min<uint64_t>(P, m_docNum - s * P);
        MappedFile f;
        const std::string path = dir + "/id/poissonengine_" + std::to_string(ver) + "_" + std::to_string(s) + ".idm";
        uint8_t fv;
        std::string ext;
        size_t at;
        if (!f.Open(path) || !ParseHead(f.data, f.size, &fv, &ext, &at)) return Fail(err, "id mapping file: " + path);
        if (fv != ver) return Fail(err, "id mapping version differs from the meta file's: " + path);
        if (ext == "1")
            return Fail(err, "string doc ids (sdocid) are not supported: results carry 64-bit global ids");
        if (f.size - at < segDocs * 8) return Fail(err, "id mapping file short: " + path);
        for (uint64_t l = 0; l < segDocs; ++l) {
            uint64_t g;
            std::memcpy(&g, f.data + at + 8 * l, 8);
            m_gdocids.push_back(static_cast<int64_t>(g));
        }
    }
    // vectors (VectorFieldData::AddSegment, vector_field_data.cpp:10-47): FP16, per segment in blocks of
    // Zn docs; inside a block, for each group of 16 dims, the block's docs' 16 halves in doc order
    std::vector<MappedFile> vf(m_segmentNum);
    std::vector<size_t> bodyAt(m_segmentNum);
    uint32_t dim = 0;
    for (uint32_t s = 0; s < m_segmentNum; ++s) {
        const std::string path = dir + "/" + cfg.vectorField + "/poissonengine_" + std::to_string(ver) + "_" +
                                 std::to_string(s) + "_" + cfg.vectorField + ".vector";
        uint8_t fv;
        std::string ext;
        if (!vf[s].Open(path) || !ParseHead(vf[s].data, vf[s].size, &fv, &ext, &bodyAt[s]) || ext.size() != 2)
            return Fail(err, "vector file: " + path);
        uint16_t d;
        std::memcpy(&d, ext.data(), 2);
        if (d == 0 || (dim && d != dim)) return Fail(err, "vector dimension invalid or differs between segments");
        dim = d;
        const uint64_t segDocs = std::min<uint64_t>(P, m_docNum - s * P);
        const uint64_t groups = (dim + 15) / 16;
        // the last doc's last 16-dim group must lie inside the body
        const uint64_t l = segDocs - 1;
        const uint64_t end = ((l / zn) * zn * groups + (zn * (groups - 1) + l % zn)) * 32 + 32;
        if (vf[s].size - bodyAt[s] < end) return Fail(err, "vector file short: " + path);
    }
    if (dim % 4 != 0 || dim > 4096) return Fail(err, "vector dimension must be a multiple of 4 up to 4096");
    m_dim = dim;
    const uint64_t groups = (dim + 15) / 16;
    const bool ok = FinishRows(
        deviceId,
        [&](uint64_t r0, uint64_t r1, float* dst) {
            for (uint64_t g = r0; g < r1; ++g, dst += dim) {
                const uint64_t s = g / P, l = g % P;
                const uint8_t* body = vf[s].data + bodyAt[s];
                const uint64_t blockAt = (l / zn) * zn * groups * 16, slot = l % zn;
                for (uint64_t j = 0; j < groups; ++j) {
                    const uint8_t* h = body + (blockAt + (zn * j + slot) * 16) * 2;
                    for (uint32_t k = 0; k < 16 && j * 16 + k < dim; ++k) {
                        uint16_t v;
                        std::memcpy(&v, h + 2 * k, 2);
                        dst[j * 16 + k] = FloatFromHalf(v);
                    }
                }
            }
        },
        err);
    m_loadTimes.total = MsSince(t0);
    return ok;
}

bool DataTable::SaveReferenceIndex(const std::string& dir, uint32_t zn, std::string* err) const {
    if (m_dVectors == nullptr && m_vectors.size() != m_docNum * m_dim) return Fail(err, "table not loaded");
    if (zn == 0) return Fail(err, "splitDocNumZn must be positive");
    if (m_dim > 0xffff) return Fail(err, "dimension does not fit the vector file's 16-bit field");
    const uint32_t P = m_cfg.docNumPerSegment;
    const uint8_t ver = static_cast<uint8_t>(kIndexVersion);
    const std::string& vfield = m_cfg.vectorField;
    const std::string& pfield = m_cfg.postingField;
    ::mkdir(dir.c_str(), 0755);
    ::mkdir((dir + "/id").c_str(), 0755);
    ::mkdir((dir + "/" + vfield).c_str(), 0755);
    // meta: IndexMeta in protobuf's JSON form (MetaBuilder::WriteMeta, meta_builder.cpp:8-27)
    {
        std::ofstream m(dir + "/poissonengine_" + std::to_string(kIndexVersion) + ".meta");
        m << "{\"config\":{\"docNumPerSegment\":" << P << ",\"splitDocNumZn\":" << zn << "},\"schema\":{\"posting\":[\""
          << pfield << "\"],\"vector\":[\"" << vfield << "\"]},\"statistics\":{\"docNum\":" << m_docNum
          << ",\"segmentNum\":" << m_segmentNum << "}}";
        if (!m) return Fail(err, "write meta");
    }
    std::vector<float> v;
    const float* rows = m_vectors.data();
    if (m_dVectors) {
        v.resize(m_docNum * m_dim);
        if (!CudaOk(cudaSetDevice(m_deviceId), err, "cudaSetDevice") ||
            !CudaOk(cudaMemcpy(v.data(), m_dVectors, v.size() * sizeof(float), cudaMemcpyDeviceToHost), err,
                    "download vectors"))
            return false;
        rows = v.data();
    }
    const uint32_t groups = (m_dim + 15) / 16;
    for (uint32_t s = 0; s < m_segmentNum; ++s) {
        const uint64_t d0 = static_cast<uint64_t>(s) * P;
        const uint64_t segDocs = std::min<uint64_t>(P, m_docNum - d0);
        // id mapping (IDMappingBuilder, idmapping_builder.cpp:11-70): head extension '0' (global ids)
        {
            std::ofstream f(dir + "/id/poissonengine_" + std::to_string(kIndexVersion) + "_" + std::to_string(s) + ".idm",
                            std::ios::binary);
            const std::string h = FileHead(ver, "0");
            f.write(h.data(), static_cast<std::streamsize>(h.size()));
            for (uint64_t l = 0; l < segDocs; ++l) {
                const uint64_t g = static_cast<uint64_t>(m_gdocids[d0 + l]);
                f.write(reinterpret_cast<const char*>(&g), 8);
            }
            if (!f) return Fail(err, "write id mapping");
        }
        // vectors (VectorBuilder::WriteDocVectorBlocks, vector_builder.cpp:34-72): FP16, blocks of zn
        // docs, 16-dim groups, the tail group zero-padded; the last segment padded to whole blocks
        {
            const uint64_t padded = (segDocs + zn - 1) / zn * zn;
            std::vector<uint16_t> body(padded * groups * 16, 0);
            for (uint64_t l = 0; l < segDocs; ++l) {
                const float* x = rows + (d0 + l) * m_dim;
                const uint64_t blockAt = (l / zn) * zn * groups * 16, slot = l % zn;
                for (uint32_t j = 0; j < groups; ++j)
                    for (uint32_t k = 0; k < 16 && j * 16 + k < m_dim; ++k)
                        body[blockAt + (zn * j + slot) * 16 + k] = HalfFromFloat(x[j * 16 + k]);
            }
            std::string ext(2, '\0');
            const uint16_t d = static_cast<uint16_t>(m_dim);
            std::memcpy(&ext[0], &d, 2);
            std::ofstream f(dir + "/" + vfield + "/poissonengine_" + std::to_string(kIndexVersion) + "_" +
                                std::to_string(s) + "_" + vfield + ".vector",
                            std::ios::binary);
            const std::string h = FileHead(ver, ext);
            f.write(h.data(), static_cast<std::streamsize>(h.size()));
            f.write(reinterpret_cast<const char*>(body.data()), static_cast<std::streamsize>(body.size() * 2));
            if (!f) return Fail(err, "write vector file");
        }
    }
    return WritePostingFiles(dir, err);
}

}  // namespace hss
