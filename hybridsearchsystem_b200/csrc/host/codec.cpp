// codec.cpp -- token hash, filter grammar and posting codec of the host library.
#include <algorithm>
#include <cstring>

#include "hss_host.h"

namespace hss {

// ---------------------------------------------------------------------------------------------
// Hash64 (hash.cpp:10-16): the 128-bit x64 variant of Austin Appleby's public-domain MurmurHash3,
// seed 0x20160713, folded to 64 bits as h1 ^ h2. Written from the published algorithm.
namespace {
inline uint64_t Rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
inline uint64_t Fmix(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}
}  // namespace

uint64_t Hash64(const char* data, uint32_t len) {
    const auto* d = reinterpret_cast<const uint8_t*>(data);
    constexpr uint64_t c1 = 0x87c37b91114253d5ull, c2 = 0x4cf5ad432745937full;
    uint64_t h1 = 0x20160713u, h2 = 0x20160713u;
    const uint32_t blocks = len / 16;
    for (uint32_t i = 0; i < blocks; ++i) {
        uint64_t k1, k2;
        std::memcpy(&k1, d + 16 * i, 8);
        std::memcpy(&k2, d + 16 * i + 8, 8);
        k1 = Rotl(k1 * c1, 31) * c2;
        h1 ^= k1;
        h1 = (Rotl(h1, 27) + h2) * 5 + 0x52dce729;
        k2 = Rotl(k2 * c2, 33) * c1;
        h2 ^= k2;
        h2 = (Rotl(h2, 31) + h1) * 5 + 0x38495ab5;
    }
    const uint8_t* tail = d + 16 * blocks;
    const uint32_t rem = len & 15u;
    uint64_t k1 = 0, k2 = 0;
    for (uint32_t i = 8; i < rem; ++i) k2 |= static_cast<uint64_t>(tail[i]) << (8 * (i - 8));
    for (uint32_t i = 0; i < rem && i < 8; ++i) k1 |= static_cast<uint64_t>(tail[i]) << (8 * i);
    if (rem > 8) h2 ^= Rotl(k2 * c2, 33) * c1;
    if (rem > 0) h1 ^= Rotl(k1 * c1, 31) * c2;
    h1 ^= len;
    h2 ^= len;
    h1 += h2;
    h2 += h1;
    h1 = Fmix(h1);
    h2 = Fmix(h2);
    h1 += h2;
    h2 += h1;
    return h1 ^ h2;
}

// ---------------------------------------------------------------------------------------------
// Filter grammar (filter_expr.h:1-177). A token is "(", ")", a digit run (a tag id, wrapping modulo
// 2^64), or a run of ASCII letters that must spell AND / OR / NOT exactly.
namespace {
class Parser {
   public:
    explicit Parser(const std::string& s) : m_s(s) {}

    bool AtEnd() {
        SkipWs();
        return m_i >= m_s.size();
    }

    std::unique_ptr<FilterNode> ParseOr(bool& ok) {
        auto first = ParseAnd(ok);
        if (!ok) return nullptr;
        std::vector<std::unique_ptr<FilterNode>> parts;
        parts.push_back(std::move(first));
        while (PeekWord("OR")) {
            m_i += 2;
            auto next = ParseAnd(ok);
            if (!ok) return nullptr;
            parts.push_back(std::move(next));
        }
        return Join(FilterOp::Or, std::move(parts));
    }

   private:
    void SkipWs() {
        while (m_i < m_s.size() && (m_s[m_i] == ' ' || m_s[m_i] == '\t' || m_s[m_i] == '\r' || m_s[m_i] == '\n')) ++m_i;
    }
    static bool IsLetter(char c) { return (c >= 'A' && c <= 'Z') || (c >= 'a' && c <= 'z'); }
    static bool IsDigit(char c) { return c >= '0' && c <= '9'; }

    // True when the next token is the letter run `kw` exactly.
    bool PeekWord(const char* kw) {
        SkipWs();
        size_t j = m_i;
        while (j < m_s.size() && IsLetter(m_s[j])) ++j;
        const size_t n = std::strlen(kw);
        return j - m_i == n && m_s.compare(m_i, n, kw) == 0;
    }

    static std::unique_ptr<FilterNode> Join(FilterOp op, std::vector<std::unique_ptr<FilterNode>> parts) {
        if (parts.size() == 1) return std::move(parts[0]);
        auto n = std::make_unique<FilterNode>();
        n->op = op;
        n->children = std::move(parts);
        return n;
    }

    std::unique_ptr<FilterNode> ParseAnd(bool& ok) {
        auto first = ParseNot(ok);
        if (!ok) return nullptr;
        std::vector<std::unique_ptr<FilterNode>> parts;
        parts.push_back(std::move(first));
        while (PeekWord("AND")) {
            m_i += 3;
            auto next = ParseNot(ok);
            if (!ok) return nullptr;
            parts.push_back(std::move(next));
        }
        return Join(FilterOp::And, std::move(parts));
    }

    std::unique_ptr<FilterNode> ParseNot(bool& ok) {
        if (PeekWord("NOT")) {
            m_i += 3;
            auto child = ParseNot(ok);
            if (!ok) return nullptr;
            auto n = std::make_unique<FilterNode>();
            n->op = FilterOp::Not;
            n->children.push_back(std::move(child));
            return n;
        }
        return ParseAtom(ok);
    }

    std::unique_ptr<FilterNode> ParseAtom(bool& ok) {
        SkipWs();
        if (m_i < m_s.size() && m_s[m_i] == '(') {
            ++m_i;
            auto inner = ParseOr(ok);
            if (!ok) return nullptr;
            SkipWs();
            if (m_i >= m_s.size() || m_s[m_i] != ')') {
                ok = false;
                return nullptr;
            }
            ++m_i;
            return inner;
        }
        if (m_i < m_s.size() && IsDigit(m_s[m_i])) {
            uint64_t v = 0;
            while (m_i < m_s.size() && IsDigit(m_s[m_i])) v = v * 10u + static_cast<uint64_t>(m_s[m_i++] - '0');
            auto n = std::make_unique<FilterNode>();
            n->op = FilterOp::Term;
            n->tag = v;
            return n;
        }
        ok = false;
        return nullptr;
    }

    const std::string& m_s;
    size_t m_i = 0;
};
}  // namespace

std::unique_ptr<FilterNode> ParseFilter(const std::string& expr, bool& ok) {
    ok = true;
    Parser p(expr);
    if (p.AtEnd()) return nullptr;  // empty -> match all
    auto n = p.ParseOr(ok);
    if (!ok) return nullptr;
    if (!p.AtEnd()) {  // trailing garbage
        ok = false;
        return nullptr;
    }
    return n;
}

// ---------------------------------------------------------------------------------------------
// Posting codec. Head word [layout:4][hitCount:28], then the payload byte length; the layout is
// sparse iff hits / docNum (as float) < threshold (posting_serializer.cpp:15-79).
namespace {
void Put32(std::string& b, uint32_t v) { b.append(reinterpret_cast<const char*>(&v), 4); }
void Put16(std::string& b, uint16_t v) { b.append(reinterpret_cast<const char*>(&v), 2); }
uint32_t Get32(const uint8_t* p) {
    uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}
}  // namespace

PostingLayout PostingSerializer::SelectLayout(bool isMatrixType, uint32_t targetDocNum, uint32_t docNum,
                                              float densityThreshold, bool sparsePacked) {
    if (docNum == 0) return PostingLayout::DENSE_BITMAP;
    const float density = static_cast<float>(targetDocNum * 1.0 / docNum);
    if (density < densityThreshold) {
        if (isMatrixType) return PostingLayout::SPARSE_IDLIST;
        return sparsePacked ? PostingLayout::SPARSE_PACKED : PostingLayout::SPARSE_BITMAP;
    }
    return isMatrixType ? PostingLayout::DENSE_BYTEMAP : PostingLayout::DENSE_BITMAP;
}

bool PostingSerializer::Serialize(const std::vector<uint32_t>& docIds, uint32_t docNum, bool isMatrixType,
                                  float densityThreshold, bool sparsePacked, std::string& buffer) {
    const uint32_t hits = static_cast<uint32_t>(docIds.size());
    if (hits > 0x0fffffffu) return false;
    const PostingLayout layout = SelectLayout(isMatrixType, hits, docNum, densityThreshold, sparsePacked);
    const uint32_t units = (docNum + 15) / 16;
    const uint32_t head = (static_cast<uint32_t>(layout) << 28) | hits;
    if (layout == PostingLayout::DENSE_BYTEMAP) {
        Put32(buffer, head);
        Put32(buffer, docNum);
        const size_t at = buffer.size();
        buffer.append(docNum, '\0');
        for (uint32_t id : docIds)
            if (id < docNum) buffer[at + id] = 1;
        return true;
    }
    if (layout == PostingLayout::SPARSE_IDLIST) {
        Put32(buffer, head);
        Put32(buffer, hits * 4u);
        for (uint32_t id : docIds) Put32(buffer, id);
        return true;
    }
    std::vector<uint16_t> masks(units, 0);
    for (uint32_t id : docIds)
        if (id < units * 16u) masks[id / 16] |= static_cast<uint16_t>(1u << (id % 16));
    if (layout == PostingLayout::DENSE_BITMAP) {
        Put32(buffer, head);
        Put32(buffer, units * 2u);
        for (uint16_t m : masks) Put16(buffer, m);
        return true;
    }
    uint32_t nz = 0;
    for (uint16_t m : masks) nz += m != 0;
    if (layout == PostingLayout::SPARSE_PACKED) {
        if (units > 0x10000u) return false;
        Put32(buffer, head);
        Put32(buffer, nz * 4u);
        for (uint32_t u = 0; u < units; ++u)
            if (masks[u]) Put32(buffer, (u << 16) | masks[u]);
        return true;
    }
    Put32(buffer, head);
    Put32(buffer, nz * 6u);
    for (uint32_t u = 0; u < units; ++u)
        if (masks[u]) Put32(buffer, u * 2u);
    for (uint32_t u = 0; u < units; ++u)
        if (masks[u]) Put16(buffer, masks[u]);
    return true;
}

bool ValidatePosting(const uint8_t* p, size_t len, uint32_t segDocs, std::string* err) {
    auto fail = [&](const char* m) {
        if (err) *err = m;
        return false;
    };
    if (len < 8) return fail("posting shorter than its 8-byte head");
    const uint32_t head = Get32(p), plen = Get32(p + 4);
    const uint32_t layout = head >> 28, hits = head & 0x0fffffffu;
    if (8ull + plen > len) return fail("posting payload runs past its buffer");
    const uint32_t units = (segDocs + 15) / 16;
    switch (layout) {
        case 0:
            if (plen > units * 2u || (plen & 1u)) return fail("dense bitmap payload length");
            return true;
        case 2:
            if (plen > segDocs) return fail("dense bytemap payload length");
            return true;
        case 3: {
            if (plen % 4 || plen / 4 != hits) return fail("id list length != hit count");
            for (uint32_t i = 0; i < plen / 4; ++i)
                if (Get32(p + 8 + 4 * i) >= segDocs) return fail("id list entry out of range");
            return true;
        }
        case 1:
        case 4: {
            const uint32_t per = layout == 1 ? 6 : 4;
            if (plen % per) return fail("sparse payload length");
            const uint32_t k = plen / per;
            uint32_t prev = 0;
            for (uint32_t i = 0; i < k; ++i) {
                const uint32_t w = Get32(p + 8 + 4 * i);
                if (layout == 1 && (w & 1u)) return fail("sparse byte offset not unit aligned");
                const uint32_t u = layout == 1 ? w / 2 : w >> 16;
                if (u >= units) return fail("sparse unit out of range");
                if (i > 0 && u <= prev) return fail("sparse units not strictly increasing");
                prev = u;
            }
            return true;
        }
        default:
            return fail("unknown posting layout");
    }
}

}  // namespace hss
