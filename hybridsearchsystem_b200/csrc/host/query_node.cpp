// query_node.cpp -- the filter-expression AST lowered to the reference's postfix filter program.
//
// Program words (query_node_imp.cpp:8-47,65-96,120-160,295-342):
//   AND / OR:     [op, postingNum, stackNum]; the non-term children are emitted first (each leaves
//                 one entry on the stack), then the direct term children as postings.
//   NOT:          [NOT, 1, 0] over a posting or [NOT, 0, 1] over the stack top.
//   CONJUNCTION:  [0, parts, n_1 .. n_parts]: AND over parts of the OR of each part's postings.
// Postings are consumed in the order they are appended, so operand i of the program is
// FilterExpr::postingRows[i].
#include "hss_host.h"

namespace hss {

void QueryNode::AddChild(std::unique_ptr<QueryNode>& child) {
    if (child) m_children.emplace_back(std::move(child));
}

namespace {
bool EmitAndOr(const std::vector<std::unique_ptr<QueryNode>>& children, FilterOpType op, const DataTable& table,
               FilterExpr& out) {
    uint32_t postingNum = 0, stackNum = 0;
    for (const auto& c : children) {
        if (!c || c->GetNodeType() == QueryNodeType::TermNode) continue;
        if (c->GetPostOrderExpression(table, out)) ++stackNum;
    }
    for (const auto& c : children) {
        if (!c || c->GetNodeType() != QueryNodeType::TermNode) continue;
        if (c->GetPostOrderExpression(table, out)) ++postingNum;
    }
    out.postExpr.push_back(static_cast<uint32_t>(op));
    out.postExpr.push_back(postingNum);
    out.postExpr.push_back(stackNum);
    out.opNum += 1;
    return true;
}
}  // namespace

bool AndNode::GetPostOrderExpression(const DataTable& table, FilterExpr& out) const {
    return EmitAndOr(m_children, FilterOpType::AND, table, out);
}

bool OrNode::GetPostOrderExpression(const DataTable& table, FilterExpr& out) const {
    return EmitAndOr(m_children, FilterOpType::OR, table, out);
}

bool NotNode::GetPostOrderExpression(const DataTable& table, FilterExpr& out) const {
    if (m_children.size() != 1 || !m_children[0]) return false;
    const QueryNode& child = *m_children[0];
    if (!child.GetPostOrderExpression(table, out)) return false;
    const bool term = child.GetNodeType() == QueryNodeType::TermNode;
    out.postExpr.push_back(static_cast<uint32_t>(FilterOpType::NOT));
    out.postExpr.push_back(term ? 1u : 0u);
    out.postExpr.push_back(term ? 0u : 1u);
    out.opNum += 1;
    return true;
}

// An absent token reads the all-zero posting (TermNode::AppendPostings, query_node_imp.cpp:124-160).
bool TermNode::AppendPostings(const DataTable& table, FilterExpr& out) const {
    if (table.GetPostingFields().count(m_fieldName) == 0) return false;
    bool exist = true;
    out.postingRows.push_back(table.TokenRow(m_token, exist));
    return true;
}

bool TermNode::GetPostOrderExpression(const DataTable& table, FilterExpr& out) const {
    return AppendPostings(table, out);
}

// Absent tokens add the all-zero posting once at most (TermsNode::AppendPostings, :195-232).
bool TermsNode::AppendPostings(const DataTable& table, FilterExpr& out) const {
    if (table.GetPostingFields().count(m_fieldName) == 0) return false;
    bool added = false;
    for (uint64_t tok : m_tokens) {
        bool exist = true;
        const uint32_t row = table.TokenRow(tok, exist);
        if (!exist && added) continue;
        out.postingRows.push_back(row);
        added = true;
    }
    return true;
}

bool TermsNode::GetPostOrderExpression(const DataTable& table, FilterExpr& out) const {
    const size_t base = out.postingRows.size();
    if (!AppendPostings(table, out)) return false;
    const uint32_t n = static_cast<uint32_t>(out.postingRows.size() - base);
    if (n == 0) return false;
    out.postExpr.push_back(static_cast<uint32_t>(FilterOpType::OR));
    out.postExpr.push_back(n);
    out.postExpr.push_back(0);
    out.opNum += 1;
    return true;
}

bool OrTermsNode::AppendPostings(const DataTable& table, FilterExpr& out) const {
    for (const auto& c : m_children) {
        const auto* leaf = dynamic_cast<const QueryLeafNode*>(c.get());
        if (!leaf) continue;
        const QueryNodeType t = leaf->GetNodeType();
        if (t != QueryNodeType::TermNode && t != QueryNodeType::TermsNode) continue;
        leaf->AppendPostings(table, out);
    }
    return true;
}

bool OrTermsNode::GetPostOrderExpression(const DataTable& table, FilterExpr& out) const {
    const size_t base = out.postingRows.size();
    AppendPostings(table, out);
    const uint32_t n = static_cast<uint32_t>(out.postingRows.size() - base);
    if (n == 0) return false;
    out.postExpr.push_back(static_cast<uint32_t>(FilterOpType::OR));
    out.postExpr.push_back(n);
    out.postExpr.push_back(0);
    out.opNum += 1;
    return true;
}

bool ConjunctionNode::GetPostOrderExpression(const DataTable& table, FilterExpr& out) const {
    std::vector<uint32_t> groups;
    for (const auto& c : m_children) {
        const auto* leaf = dynamic_cast<const QueryLeafNode*>(c.get());
        if (!leaf) continue;
        const QueryNodeType t = leaf->GetNodeType();
        if (t != QueryNodeType::TermNode && t != QueryNodeType::TermsNode && t != QueryNodeType::OrTermsNode) continue;
        const size_t base = out.postingRows.size();
        if (!leaf->AppendPostings(table, out)) continue;
        const uint32_t n = static_cast<uint32_t>(out.postingRows.size() - base);
        if (n > 0) groups.push_back(n);
    }
    if (groups.empty()) return false;
    out.postExpr.push_back(static_cast<uint32_t>(FilterOpType::CONJUNCTION));
    out.postExpr.push_back(static_cast<uint32_t>(groups.size()));
    for (uint32_t g : groups) out.postExpr.push_back(g);
    out.opNum += 1;
    return true;
}

std::unique_ptr<QueryNode> BuildQueryNode(const FilterNode* n, const std::string& field) {
    if (n == nullptr) return std::make_unique<AndNode>();
    switch (n->op) {
        case FilterOp::Term:
            return std::make_unique<TermNode>(field, Hash64(std::to_string(n->tag)));
        case FilterOp::And:
        case FilterOp::Or: {
            std::unique_ptr<QueryNode> node;
            if (n->op == FilterOp::And)
                node = std::make_unique<AndNode>();
            else
                node = std::make_unique<OrNode>();
            for (const auto& c : n->children) {
                auto child = BuildQueryNode(c.get(), field);
                node->AddChild(child);
            }
            return node;
        }
        case FilterOp::Not: {
            auto node = std::make_unique<NotNode>();
            auto child = BuildQueryNode(n->children[0].get(), field);
            node->AddChild(child);
            return node;
        }
    }
    return std::make_unique<AndNode>();
}

// CheckPostExpr (text_filter.cpp:1233-1352): every operator finds its operands, exactly one value is
// left on the stack and every posting is consumed.
bool CheckPostExpr(const std::vector<uint32_t>& e, uint32_t postingNums) {
    uint32_t inStack = 0, remained = postingNums;
    for (size_t i = 0; i < e.size(); ++i) {
        const uint32_t op = e[i];
        if (op == AND || op == OR || op == NOT) {
            if (e.size() <= i + 2) return false;
            const uint32_t pn = e[i + 1], sn = e[i + 2];
            if (op == NOT ? (pn + sn != 1) : (pn + sn == 0)) return false;
            if (remained < pn || inStack < sn) return false;
            remained -= pn;
            inStack = inStack - sn + 1;
            i += 2;
        } else if (op == CONJUNCTION) {
            if (e.size() <= i + 1) return false;
            const uint32_t parts = e[i + 1];
            if (parts == 0 || e.size() <= i + 1 + parts) return false;
            uint32_t total = 0;
            for (uint32_t p = 0; p < parts; ++p) {
                if (e[i + 2 + p] == 0) return false;
                total += e[i + 2 + p];
            }
            if (remained < total) return false;
            remained -= total;
            inStack += 1;
            i += 1 + parts;
        } else {
            return false;
        }
    }
    return remained == 0 && inStack == 1;
}

bool PrepareExpr(const QueryNode* tree, const DataTable& table, FilterExpr& out, std::string* err) {
    out = FilterExpr{};
    if (tree == nullptr) {
        if (err) *err = "null query tree";
        return false;
    }
    const QueryNodeType rootType = tree->GetNodeType();
    if (tree->GetChildrenNum() == 0 && rootType != QueryNodeType::TermNode && rootType != QueryNodeType::TermsNode) {
        out.emptyTree = true;  // empty tree: match all (text_filter.cpp:443-447)
        return true;
    }
    if (rootType == QueryNodeType::TermNode) {
        // A bare term at the root (filter "t"). The reference's PrepareExpr takes any childless root for
        // an empty tree and matches everything, which contradicts its own ground truth
        // (EvalFilterBitmap); the ground truth is what results are checked against, so the term is
        // evaluated: one posting under a single-operand OR.
        if (!static_cast<const TermNode*>(tree)->AppendPostings(table, out)) {
            if (err) *err = "term field is not indexed";
            return false;
        }
        out.postExpr = {static_cast<uint32_t>(FilterOpType::OR), 1u, 0u};
        out.opNum = 1;
        return true;
    }
    if (!tree->GetPostOrderExpression(table, out)) {
        if (err) *err = "query tree produced no filter program";
        return false;
    }
    if (!CheckPostExpr(out.postExpr, static_cast<uint32_t>(out.postingRows.size()))) {
        if (err) *err = "invalid postfix filter program";
        return false;
    }
    return true;
}

}  // namespace hss
