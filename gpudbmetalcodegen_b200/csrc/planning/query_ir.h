#pragma once
// ===================================================================
// Analyzed-query IR: the planning layer's input, restated.
//
// The reference plans from an AnalyzedQuery that its SQL analyser fills
// (codegen/planning/query_plan.h:14-183 — expressions, predicates,
// aggregate specs; codegen/planning/query_analyzer.h:14-81 — join
// clauses, select targets, GROUP BY / ORDER BY / LIMIT) and lowers it with
// buildMetalPlan(aq, name) (metal_plan_builder.cpp:2035-2109), turning
// expressions into kernel source with exprToMetal / predToMetal
// (:64-228). The same shapes are kept here so a caller that builds an
// AnalyzedQuery for the reference can build it for this engine; the
// lowering emits CUDA over the engine's exact columns:
//   * decimal columns are scaled int64 (price in cents, discount / tax in
//     hundredths), so every expression carries a decimal scale: literals
//     are converted to fixed point exactly, ADD / SUB / comparisons align
//     the operands' scales, MUL adds them; a value that is not exact at
//     the needed scale is refused rather than rounded;
//   * columns are named by the engine's catalog, or by the TPC-H names of
//     lineitem (l_shipdate, l_quantity, l_extendedprice, l_discount,
//     l_tax, l_returnflag, l_linestatus), which resolve to the fact table.
// ===================================================================
#include <memory>
#include <optional>
#include <string>
#include <variant>
#include <vector>

namespace gpudb {
namespace ir {

enum class ExprOp { ADD, SUB, MUL, DIV };
enum class AggFunc { SUM, COUNT, AVG, MIN, MAX, COUNT_DISTINCT };
enum class CmpOp { EQ, NE, LT, LE, GT, GE };

struct ColRef {
    std::string table;   // "" = a select target's alias (ORDER BY revenue)
    std::string column;
};
struct Literal {
    std::variant<long long, double, std::string> value;  // integer, decimal, character / string
};

struct Expr;
using ExprPtr = std::shared_ptr<Expr>;
struct BinaryExpr {
    ExprOp op;
    ExprPtr left, right;
};
struct Expr {
    std::variant<ColRef, Literal, BinaryExpr> node;
    static ExprPtr col(const std::string& table, const std::string& column);
    static ExprPtr lit(long long v);
    static ExprPtr litf(double v);
    static ExprPtr lits(const std::string& v);
    static ExprPtr binary(ExprOp op, ExprPtr l, ExprPtr r);
};

struct Predicate;
using PredPtr = std::shared_ptr<Predicate>;
struct Comparison {
    CmpOp op;
    ExprPtr left, right;
};
struct Between {
    ExprPtr expr, low, high;
};
struct InList {
    ExprPtr expr;
    std::vector<ExprPtr> values;
};
struct LogicalAnd {
    std::vector<PredPtr> children;
};
struct LogicalOr {
    std::vector<PredPtr> children;
};
struct LogicalNot {
    PredPtr child;
};
struct Predicate {
    std::variant<Comparison, Between, InList, LogicalAnd, LogicalOr, LogicalNot> node;
    static PredPtr cmp(CmpOp op, ExprPtr l, ExprPtr r);
    static PredPtr between(ExprPtr e, ExprPtr lo, ExprPtr hi);
    static PredPtr inList(ExprPtr e, std::vector<ExprPtr> vals);
    static PredPtr logAnd(std::vector<PredPtr> ch);
    static PredPtr logOr(std::vector<PredPtr> ch);
    static PredPtr logNot(PredPtr ch);
};

struct JoinClause {
    std::string leftTable, rightTable, leftCol, rightCol;
};
struct AggTarget {
    AggFunc func;
    ExprPtr innerExpr;  // null for COUNT(*)
    std::string alias;
    bool isStar = false;
};
struct SelectTarget {
    ExprPtr expr;
    std::string alias;
    bool isAgg = false;
    std::optional<AggTarget> agg;
};
struct OrderByItem {
    ExprPtr expr;
    bool descending = false;
};

struct AnalyzedQuery {
    std::vector<std::string> tables;
    std::vector<JoinClause> joins;
    std::vector<PredPtr> filters;
    std::vector<SelectTarget> targets;
    std::vector<ExprPtr> groupBy;
    std::vector<OrderByItem> orderBy;
    int limit = -1;
    bool isSingleTable() const { return tables.size() == 1 && joins.empty(); }
    bool hasAggregation() const;
    bool hasGroupBy() const { return !groupBy.empty(); }
};

// ---- lowering of expressions to CUDA over the engine's columns ---------
// A column resolved against the catalog (TPC-H lineitem names included).
struct ResolvedColumn {
    std::string table, column, cudaType;
    int scale = 0;  // decimal digits of the stored integer
};
ResolvedColumn resolveColumn(const std::string& table, const std::string& column);
// Engine table a (possibly TPC-H) table name stands for.
std::string resolveTable(const std::string& table);

struct Lowered {
    std::string code;  // CUDA expression (long long arithmetic)
    int scale = 0;     // decimal digits of its value
    bool isText = false;
};
// Reference: exprToMetal (metal_plan_builder.cpp:64-117). Throws
// std::runtime_error on what cannot be computed exactly (division, a
// literal not exact at the needed scale, an unknown column).
Lowered exprToCuda(const ExprPtr& e, const std::string& idx);
// Reference: predToMetal (:119-185) and combineFilters (:188-198).
std::string predToCuda(const PredPtr& p, const std::string& idx);
std::string combineFilters(const std::vector<PredPtr>& filters, const std::string& idx);
// Columns (engine names) an expression / predicate reads, per table.
void collectColumns(const ExprPtr& e, std::vector<ResolvedColumn>& out);
void collectColumns(const PredPtr& p, std::vector<ResolvedColumn>& out);

}  // namespace ir
}  // namespace gpudb
