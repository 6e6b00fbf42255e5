#include "query_ir.h"

#include <cmath>
#include <map>
#include <stdexcept>

#include "plan_builder.h"

namespace gpudb {
namespace ir {

// ---- factories (reference: Expr::col / lit / binary, Predicate::cmp ...,
// query_plan.h:60-160) ----------------------------------------------------
ExprPtr Expr::col(const std::string& table, const std::string& column) {
    auto e = std::make_shared<Expr>();
    e->node = ColRef{table, column};
    return e;
}
ExprPtr Expr::lit(long long v) {
    auto e = std::make_shared<Expr>();
    e->node = Literal{v};
    return e;
}
ExprPtr Expr::litf(double v) {
    auto e = std::make_shared<Expr>();
    e->node = Literal{v};
    return e;
}
ExprPtr Expr::lits(const std::string& v) {
    auto e = std::make_shared<Expr>();
    e->node = Literal{v};
    return e;
}
ExprPtr Expr::binary(ExprOp op, ExprPtr l, ExprPtr r) {
    auto e = std::make_shared<Expr>();
    e->node = BinaryExpr{op, std::move(l), std::move(r)};
    return e;
}
PredPtr Predicate::cmp(CmpOp op, ExprPtr l, ExprPtr r) {
    auto p = std::make_shared<Predicate>();
    p->node = Comparison{op, std::move(l), std::move(r)};
    return p;
}
PredPtr Predicate::between(ExprPtr e, ExprPtr lo, ExprPtr hi) {
    auto p = std::make_shared<Predicate>();
    p->node = Between{std::move(e), std::move(lo), std::move(hi)};
    return p;
}
PredPtr Predicate::inList(ExprPtr e, std::vector<ExprPtr> vals) {
    auto p = std::make_shared<Predicate>();
    p->node = InList{std::move(e), std::move(vals)};
    return p;
}
PredPtr Predicate::logAnd(std::vector<PredPtr> ch) {
    auto p = std::make_shared<Predicate>();
    p->node = LogicalAnd{std::move(ch)};
    return p;
}
PredPtr Predicate::logOr(std::vector<PredPtr> ch) {
    auto p = std::make_shared<Predicate>();
    p->node = LogicalOr{std::move(ch)};
    return p;
}
PredPtr Predicate::logNot(PredPtr ch) {
    auto p = std::make_shared<Predicate>();
    p->node = LogicalNot{std::move(ch)};
    return p;
}

bool AnalyzedQuery::hasAggregation() const {
    for (const auto& t : targets)
        if (t.isAgg) return true;
    return false;
}

// ---- catalog resolution ---------------------------------------------------
namespace {

// TPC-H lineitem names of the fact table's columns (the reference's Q1 / Q6
// analyses name lineitem; the fact table stands in for it).
const std::map<std::string, std::string>& lineitemNames() {
    static const std::map<std::string, std::string> m = {
        {"l_shipdate", "f_ship_day"},     {"l_quantity", "f_quantity"}, {"l_extendedprice", "f_price"},
        {"l_discount", "f_discount"},     {"l_tax", "f_tax"},           {"l_returnflag", "f_flag_a"},
        {"l_linestatus", "f_flag_b"}};
    return m;
}

constexpr int kMaxScale = 12;

long long pow10(int s) {
    long long v = 1;
    for (int i = 0; i < s; i++) v *= 10;
    return v;
}

std::string L(long long v) { return std::to_string(v) + "ll"; }

// A literal at a given scale: exact integer or nothing. Decimal literals
// may carry single-precision noise (a float 0.05 is 0.0500000007...): a
// value within one part in 10^6 of itself from an integer at that scale
// counts as that integer (so 1e-20 is never taken for 0).
std::optional<long long> literalAt(const Literal& lit, int scale) {
    if (scale > kMaxScale) return std::nullopt;
    if (auto* i = std::get_if<long long>(&lit.value)) {
        const long double v = (long double)*i * (long double)pow10(scale);
        if (std::fabs(v) > 9.0e18L) return std::nullopt;
        return (long long)v;
    }
    if (auto* d = std::get_if<double>(&lit.value)) {
        const long double v = (long double)*d * (long double)pow10(scale);
        const long double r = std::nearbyint(v);
        if (std::fabs(r) > 9.0e18L) return std::nullopt;
        if (std::fabs(v - r) <= 1e-6L * std::fabs(v)) return (long long)r;
        return std::nullopt;
    }
    return std::nullopt;
}

// Smallest scale at which a numeric literal is exact.
int literalScale(const Literal& lit) {
    for (int s = 0; s <= kMaxScale; s++)
        if (literalAt(lit, s)) return s;
    throw std::runtime_error("IR: decimal literal " + std::to_string(std::get<double>(lit.value)) +
                             " has no exact fixed-point form within " + std::to_string(kMaxScale) + " digits");
}

// Lowering result that remembers a bare literal, so that aligning scales
// rescales the literal itself instead of multiplying at run time.
struct Low {
    Lowered v;
    std::optional<Literal> lit;
};

Low lower(const ExprPtr& e, const std::string& idx);

Lowered atScale(const Low& x, int scale) {
    if (x.v.isText) throw std::runtime_error("IR: character value in arithmetic");
    if (x.v.scale == scale) return x.v;
    if (x.v.scale > scale) throw std::runtime_error("IR: internal scale alignment error");
    if (scale > kMaxScale) throw std::runtime_error("IR: expression needs more than " + std::to_string(kMaxScale) +
                                                    " decimal digits");
    if (x.lit) {
        auto v = literalAt(*x.lit, scale);
        if (!v) throw std::runtime_error("IR: literal out of range at scale " + std::to_string(scale));
        return {L(*v), scale, false};
    }
    return {"(" + x.v.code + " * " + L(pow10(scale - x.v.scale)) + ")", scale, false};
}

Low lower(const ExprPtr& e, const std::string& idx) {
    if (!e) throw std::runtime_error("IR: missing expression");
    return std::visit(
        [&](auto&& n) -> Low {
            using T = std::decay_t<decltype(n)>;
            if constexpr (std::is_same_v<T, ColRef>) {
                const ResolvedColumn c = resolveColumn(n.table, n.column);
                Low r;
                r.v.code = c.column + "[" + idx + "]";
                r.v.scale = c.scale;
                r.v.isText = c.cudaType == "unsigned char" && !catalogTable(c.table).col(c.column).domain.empty();
                if (c.cudaType == "unsigned char" && !r.v.isText) r.v.code = "(long long)" + r.v.code;
                return r;
            } else if constexpr (std::is_same_v<T, Literal>) {
                Low r;
                if (auto* s = std::get_if<std::string>(&n.value)) {
                    if (s->size() != 1) throw std::runtime_error("IR: only one-character string literals ('A')");
                    const unsigned char ch = (unsigned char)(*s)[0];
                    if (ch < 32 || ch > 126 || ch == '\'' || ch == '\\')
                        throw std::runtime_error("IR: unsupported character literal");
                    r.v = {std::string("'") + (char)ch + "'", 0, true};
                    return r;
                }
                const int s = literalScale(n);
                r.v = {L(*literalAt(n, s)), s, false};
                r.lit = n;
                return r;
            } else {
                const Low a = lower(n.left, idx), b = lower(n.right, idx);
                Low r;
                switch (n.op) {
                    case ExprOp::ADD:
                    case ExprOp::SUB: {
                        const int s = std::max(a.v.scale, b.v.scale);
                        const Lowered x = atScale(a, s), y = atScale(b, s);
                        r.v = {"(" + x.code + (n.op == ExprOp::ADD ? " + " : " - ") + y.code + ")", s, false};
                        return r;
                    }
                    case ExprOp::MUL: {
                        if (a.v.isText || b.v.isText) throw std::runtime_error("IR: character value in arithmetic");
                        const int s = a.v.scale + b.v.scale;
                        if (s > kMaxScale) throw std::runtime_error("IR: product needs too many decimal digits");
                        r.v = {"(" + a.v.code + " * " + b.v.code + ")", s, false};
                        return r;
                    }
                    case ExprOp::DIV:
                    default:
                        throw std::runtime_error(
                            "IR: division has no exact fixed-point result on the device (ratios are derived on the "
                            "host from exact sums)");
                }
            }
        },
        e->node);
}

const char* cmpText(CmpOp op) {
    switch (op) {
        case CmpOp::EQ: return " == ";
        case CmpOp::NE: return " != ";
        case CmpOp::LT: return " < ";
        case CmpOp::LE: return " <= ";
        case CmpOp::GT: return " > ";
        case CmpOp::GE: return " >= ";
    }
    return " == ";
}

std::string compare(const Low& a, const Low& b, const char* op) {
    if (a.v.isText || b.v.isText) {
        if (!(a.v.isText && b.v.isText)) throw std::runtime_error("IR: character compared with a number");
        return a.v.code + op + b.v.code;
    }
    const int s = std::max(a.v.scale, b.v.scale);
    return atScale(a, s).code + op + atScale(b, s).code;
}

}  // namespace

std::string resolveTable(const std::string& table) {
    if (table == "lineitem") return "fact";
    return table;
}

ResolvedColumn resolveColumn(const std::string& table, const std::string& column) {
    std::string col = column;
    auto it = lineitemNames().find(column);
    if (it != lineitemNames().end()) col = it->second;
    std::string tab = table.empty() ? "" : resolveTable(table);
    if (tab.empty()) {
        for (const auto& t : catalogTables())
            for (const auto& c : catalogTable(t).columns)
                if (c.name == col) tab = t;
        if (tab.empty()) throw std::runtime_error("IR: unknown column '" + column + "'");
    }
    const ColumnDef& cd = catalogTable(tab).col(col);
    return {tab, cd.name, cd.cudaType, cd.scale};
}

Lowered exprToCuda(const ExprPtr& e, const std::string& idx) { return lower(e, idx).v; }

std::string predToCuda(const PredPtr& p, const std::string& idx) {
    if (!p) return "true";
    return std::visit(
        [&](auto&& n) -> std::string {
            using T = std::decay_t<decltype(n)>;
            if constexpr (std::is_same_v<T, Comparison>) {
                return compare(lower(n.left, idx), lower(n.right, idx), cmpText(n.op));
            } else if constexpr (std::is_same_v<T, Between>) {
                const Low e = lower(n.expr, idx), lo = lower(n.low, idx), hi = lower(n.high, idx);
                return "(" + compare(e, lo, " >= ") + " && " + compare(e, hi, " <= ") + ")";
            } else if constexpr (std::is_same_v<T, InList>) {
                if (n.values.empty()) return "false";
                const Low e = lower(n.expr, idx);
                std::string c;
                for (size_t i = 0; i < n.values.size(); i++)
                    c += (i ? " || " : "") + compare(e, lower(n.values[i], idx), " == ");
                return "(" + c + ")";
            } else if constexpr (std::is_same_v<T, LogicalAnd>) {
                if (n.children.empty()) return "true";
                std::string c;
                for (size_t i = 0; i < n.children.size(); i++)
                    c += (i ? " && " : "") + std::string("(") + predToCuda(n.children[i], idx) + ")";
                return "(" + c + ")";
            } else if constexpr (std::is_same_v<T, LogicalOr>) {
                if (n.children.empty()) return "false";
                std::string c;
                for (size_t i = 0; i < n.children.size(); i++)
                    c += (i ? " || " : "") + std::string("(") + predToCuda(n.children[i], idx) + ")";
                return "(" + c + ")";
            } else {
                return "!(" + predToCuda(n.child, idx) + ")";
            }
        },
        p->node);
}

std::string combineFilters(const std::vector<PredPtr>& filters, const std::string& idx) {
    if (filters.empty()) return "";
    if (filters.size() == 1) return predToCuda(filters[0], idx);
    std::string c;
    for (size_t i = 0; i < filters.size(); i++) c += (i ? " && " : "") + std::string("(") + predToCuda(filters[i], idx) + ")";
    return c;
}

void collectColumns(const ExprPtr& e, std::vector<ResolvedColumn>& out) {
    if (!e) return;
    std::visit(
        [&](auto&& n) {
            using T = std::decay_t<decltype(n)>;
            if constexpr (std::is_same_v<T, ColRef>) {
                if (n.table.empty() && !lineitemNames().count(n.column)) {
                    // an alias reference resolves only if it is a column
                    bool known = false;
                    for (const auto& t : catalogTables())
                        for (const auto& c : catalogTable(t).columns) known |= c.name == n.column;
                    if (!known) return;
                }
                const ResolvedColumn c = resolveColumn(n.table, n.column);
                for (const auto& x : out)
                    if (x.table == c.table && x.column == c.column) return;
                out.push_back(c);
            } else if constexpr (std::is_same_v<T, BinaryExpr>) {
                collectColumns(n.left, out);
                collectColumns(n.right, out);
            }
        },
        e->node);
}

void collectColumns(const PredPtr& p, std::vector<ResolvedColumn>& out) {
    if (!p) return;
    std::visit(
        [&](auto&& n) {
            using T = std::decay_t<decltype(n)>;
            if constexpr (std::is_same_v<T, Comparison>) {
                collectColumns(n.left, out);
                collectColumns(n.right, out);
            } else if constexpr (std::is_same_v<T, Between>) {
                collectColumns(n.expr, out);
                collectColumns(n.low, out);
                collectColumns(n.high, out);
            } else if constexpr (std::is_same_v<T, InList>) {
                collectColumns(n.expr, out);
                for (const auto& v : n.values) collectColumns(v, out);
            } else if constexpr (std::is_same_v<T, LogicalNot>) {
                collectColumns(n.child, out);
            } else {
                for (const auto& c : n.children) collectColumns(c, out);
            }
        },
        p->node);
}

}  // namespace ir
}  // namespace gpudb
