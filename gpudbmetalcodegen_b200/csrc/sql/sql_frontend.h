#pragma once
// ===================================================================
// SQL front end for the engine's pipeline templates.
//
// The reference parses SQL with libpg_query and maps the analysed query
// to a plan builder (query_analyzer.cpp:640-727, then buildMetalPlan by
// query shape). libpg_query is not available here, so this is a small
// recursive-descent parser for the SELECT subset the templates cover:
//   SELECT items FROM tables [WHERE p AND p ...] [GROUP BY cols]
//   [ORDER BY expr [ASC|DESC], ...] [LIMIT n]
// with comparisons (= <> < <= > >=), BETWEEN, + - * / and the aggregates
// sum / avg / count(*). Column and table names are the engine catalog's;
// constants are integers in the columns' own units (scaled decimals, day
// numbers). The analyser matches the statement to a template (Q1 and Q6
// shapes over `fact`, the semi-join of `dim` and `probe` as a grouped
// top-k or as materialised rows, the group-by over `zprobe`, the hash join
// of `zbuild` and `zprobe`, and the mixed-workload shapes over `mix`:
// filtered count + sum, the same through the `mixdim` semi-join, grouped by
// a key modulo a cardinality, and its top-k) and returns that template's
// spec string.
// ===================================================================

#include <string>

namespace gpudb {

// Spec string ("template=...;key=value;...") of the statement; throws
// std::runtime_error naming what it cannot map.
std::string sqlToSpec(const std::string& sql);

}  // namespace gpudb
