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

// Device chunk buffers, copy stream and events of chunked streaming runs
// (created on first use, reused by later runs).
struct StreamRing {
    static constexpr int kSlots = 3;  // chunks in flight: copying, waiting, being scanned
    cudaStream_t copy = nullptr;
    cudaEvent_t ready[kSlots] = {}, consumed[kSlots] = {};
    std::map<std::string, std::pair<void*, size_t>> buf[kSlots];  // column -> (device buffer, bytes)
    ~StreamRing();
};

// Everything that lives as long as a gpudb_ctx.
struct QueryContext {
    explicit QueryContext(int device) : ex(device) {}
    CudaGenericExecutor ex;
    std::unique_ptr<StreamRing> ring;  // destroyed before the executor
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

// One column of a table streamed from host memory.
struct StreamColumn {
    std::string column;
    const void* host = nullptr;  // its row 0, in pinned host memory
    size_t elemBytes = 0;
    bool inPlace = false;        // read in place over the host link (mapped), not copied per chunk
};

// Chunked streaming run (the reference's chunked path, codegen_main.cpp:
// 686-808): the phases before the first phase that scans `table` run
// once (with their sizing steps), the phases that scan it run once per
// chunk of `chunkRows` rows, accumulating (zero fills on the first chunk
// only), and the remaining phases run once after the last chunk. Copied
// columns move host -> device on a copy stream into a ring of device
// chunk buffers while the previous chunks are scanned. Size expressions
// see the whole table (`rows`); no phase outside the streamed ones may
// read the table. Returns like runQuery.
int runStreamed(QueryContext& qc, PreparedQuery& q, const std::string& table, const std::vector<StreamColumn>& cols,
                uint64_t rows, uint64_t chunkRows, bool collect, ExecutionResult& out, std::string& err);

std::string describePlan(const PreparedQuery& q);

}  // namespace gpudb
