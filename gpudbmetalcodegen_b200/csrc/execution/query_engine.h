#pragma once
// ===================================================================
// Query driver: the per-query flow of the reference's runCodegenQuery
// (codegen/codegen_main.cpp:271-1776) restricted to the hot path —
// plan -> generate -> compile -> size -> execute -> collect.
// ===================================================================
#include <map>
#include <memory>
#include <string>

#include "../planning/plan_builder.h"
#include "executor.h"

namespace gpudb {

struct PreparedQuery {
    CudaQueryPlan plan;
    CudaCodegen cg;
    TuneConfig tune;
    std::string source;
    std::string describe;
    std::string compileLog;
    std::vector<std::string> kernelNames;
    std::shared_ptr<RuntimeCompiler::CompiledQuery> compiled;
    double planMs = 0, codegenMs = 0, compileMs = 0;
    // columns whose max-key symbol a size expression references (found
    // once, on the first run)
    std::vector<std::string> maxKeyColumns;
    bool maxKeyColumnsFound = false;
};

// Everything that lives as long as a gpudb_ctx.
struct QueryContext {
    explicit QueryContext(int device) : ex(device) {}
    CudaGenericExecutor ex;
    struct MaxKeyEntry {
        uint64_t generation;
        long long max;
    };
    std::map<std::string, MaxKeyEntry> maxKeys;
    std::map<std::string, std::shared_ptr<PreparedQuery>> helperQueries;  // colmax plans
};

// Plan + generate (+ compile, + load when `load`). Throws std::runtime_error.
std::shared_ptr<PreparedQuery> prepareQuery(const std::string& spec, const std::string& tune, bool compile, bool load);

// The same from a plan already built (e.g. from an analyzed query).
std::shared_ptr<PreparedQuery> prepareFromPlan(CudaQueryPlan plan, const TuneConfig& tune, double planMs, bool compile,
                                               bool load);

// Load a prepared-but-unloaded query into the current context.
void loadQuery(PreparedQuery& q);

// Exact max of a registered column -> symbol "max_<column>" (GPU pass, cached).
long long registerMaxKey(QueryContext& qc, const std::string& column);

// Execute all phases, splitting at sizing steps; returns 0 or a negative
// status with `err` set; GPUDB_E_DEVICE-style status -7 on device errors.
int runQuery(QueryContext& qc, PreparedQuery& q, int warmup, int measured, bool collect, ExecutionResult& out,
             std::string& err);

std::string describePlan(const PreparedQuery& q);

}  // namespace gpudb
