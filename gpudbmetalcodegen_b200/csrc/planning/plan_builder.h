#pragma once
// ===================================================================
// Query plans and plan builders.
//
// CudaQueryPlan mirrors the reference's MetalQueryPlan
// (codegen/planning/metal_plan_builder.h:22-68): an ordered list of phases,
// each one operator tree = one kernel, plus helpers, the chunkable flag and
// the CPU post-sort descriptor. B200 additions:
//   * `sizing`: symbols a later phase's buffers depend on, produced by an
//     earlier phase (exact count pass) or supplied by the caller (learned
//     sizer); the driver splits execution at `afterPhase`.
//   * `decorate`: post-generation edits of the result schema (group-key
//     labels, FP64 derived columns).
//
// The reference builds plans from an AnalyzedQuery produced by its SQL
// front end (buildMetalPlan, metal_plan_builder.cpp:2035). Here plans are
// built from such an analysis (buildCudaPlan(const ir::AnalyzedQuery&),
// query_ir.h) or from a `key=value;...` spec naming a pipeline template
// and its constants (buildCudaPlan(spec)), which also covers the reference
// chains that no analysis shape reaches (anti-join, histogram, ...).
// ===================================================================

#include <functional>
#include <map>
#include <memory>
#include <optional>
#include <string>
#include <vector>

#include "../operators/cuda_operators.h"

namespace gpudb {

// ------------------------------------------------------------------
// Synthetic schema catalog (the role of tpch_schema.h for the workloads
// this backend is measured on). Decimals are scaled int64 fixed point.
// ------------------------------------------------------------------
struct ColumnDef {
    std::string name;
    std::string cudaType;  // "int", "long long", "unsigned char"
    int scale = 0;         // decimal digits of a fixed-point decimal (2: cents / hundredths)
    std::string domain;    // CHAR1 columns with a known value set, in bucket order ("ANR")
};
struct TableDef {
    std::string name;
    std::vector<ColumnDef> columns;
    const ColumnDef& col(const std::string& n) const;
};
const TableDef& catalogTable(const std::string& table);
std::vector<std::string> catalogTables();

struct CudaQueryPlan {
    std::string name;
    struct Phase {
        std::string name;
        std::unique_ptr<CudaOperator> root;
        int threadgroupSize = 256;
        int minBlocksPerSM = 1;
        int smemCarveout = -1;
        bool singleThread = false;
        std::vector<std::pair<std::string, std::string>> bitmapReads;   // (name, sizeExpr)
        std::vector<std::pair<std::string, std::string>> scalarParams;  // (name, type)
        // scalars whose value is a size expression over registered symbols
        // (name, type, expression): constants bound at launch, not compiled in
        struct SizeScalar {
            std::string name, type, expr;
        };
        std::vector<SizeScalar> sizeScalars;
        std::vector<std::string> prologue;  // lines before the root operator's code
        struct ExtraBuffer {
            std::string name, type;
            bool readOnly = true;
            bool zeroInit = false;
        };
        std::vector<ExtraBuffer> extraBuffers;
    };
    std::vector<Phase> phases;
    std::vector<std::string> helpers;
    bool chunkable = false;

    struct CpuSort {
        struct SortKey {
            std::string column;
            bool descending;
        };
        std::vector<SortKey> keys;
        int limit = -1;
    };
    std::optional<CpuSort> cpuSort;

    struct SizingStep {
        std::string symbol;       // symbol registered before phase `afterPhase`
        int afterPhase = 0;       // phases [0, afterPhase) produce it
        std::string counterBuffer;// u64 buffer holding the exact value
        std::string minCounterBuffer;  // optional second bound: the smaller of the two
        std::string fallbackExpr; // when no counter: a size expression
    };
    std::vector<SizingStep> sizing;

    std::vector<std::function<void(CudaResultSchema&)>> decorate;

    // Tables the plan scans (for registration checks and algorithmic bytes).
    std::vector<std::string> tables;
    std::string spec;  // canonical spec string the plan was built from
};

// Tunables the autotuner sweeps. Every field changes the generated source
// (hence the compile-cache key) but never an answer.
struct TuneConfig {
    int blockSize = 512;
    ScanConfig scan;
    HashLayout hashLayout = HashLayout::Linear;
    int smemPreAggLog2 = 10;    // hash group-by shared-memory table (0 = off)
    int smemProbe = 0;          // slots tried in that table per row (0 = the operator's default)
    int minBlocksPerSM = 1;     // __launch_bounds__ occupancy hint (caps registers)
    bool warpAggregate = true;  // match_any pre-aggregation in hash / atomic aggregation
    int keyedStrategy = 0;      // CudaKeyedAgg::Strategy (0 = auto)
    int maxProbe = 128;
    // Hash-table slots requested per expected group, in percent (200: the
    // table is requested for twice the groups, then rounded up to a power of
    // two). Lower fills keep a large table inside L2.
    int hashFill = 200;
    // Warm tier of a group-by table (log2 of its slots, 0 = none) and its
    // probe count: an L2-resident table between the shared-memory one and
    // the main table.
    int warmLog2 = 0;
    int warmProbe = 4;
    // CTAs of the join's top-k phase (each keeps its own list; the last to
    // finish merges them all)
    int topkBlocks = 296;
    bool lateMaterialize = true;  // columns read only by surviving rows are not staged
    // join_topk: the probe lists matched rows and later phases aggregate
    // them, sized on the device (split=0: probe and group-by in one kernel,
    // sized by a host read of the build's distinct count)
    bool splitJoin = true;
    // Preferred shared-memory carveout (percent of the SM's maximum) of
    // phases that use dynamic shared memory; -1 leaves it to the driver,
    // which may then fit fewer staged-ring blocks per SM.
    int smemCarveout = -1;
    // Block size and vector rows of a join's build phase when they should
    // differ from the probe's (0 = same as the plan's).
    int buildBlockSize = 0;
    int buildVectorRows = 0;
    TuneConfig forBuild() const;
    std::string toString() const;
    static TuneConfig parse(const std::string& s);  // "bs=512;scan=tma;tile=1024;stages=4;..."
};

using SpecMap = std::map<std::string, std::string>;
SpecMap parseSpec(const std::string& spec);
std::string canonicalSpec(const SpecMap& m);

// Build a plan for `spec` (template=...; constants). Throws
// std::runtime_error on an unknown template / bad constant.
CudaQueryPlan buildCudaPlan(const std::string& spec, const TuneConfig& tune = {});

namespace ir {
struct AnalyzedQuery;
}
// Plan an analyzed query (reference: buildMetalPlan(const AnalyzedQuery&,
// name), metal_plan_builder.cpp:2035-2109): the analysis' shape selects the
// operator chain and its expressions are lowered with ir::exprToCuda /
// predToCuda:
//   * one table, aggregates, no GROUP BY      -> Scan -> Selection -> TGReduce
//     (the Q6 shape, buildQ6Plan :253-303);
//   * one table, GROUP BY character columns with known value sets (at most
//     64 groups)                              -> Scan -> Selection -> KeyedAgg
//     (the Q1 shape, buildQ1Plan :309-354); AVG becomes SUM / COUNT derived
//     on the host;
//   * one table, GROUP BY one integer column  -> hash group-by (the Q18
//     shape, :1529-1545, with an open-addressing table for any key range);
//   * dim JOIN probe ON b_key = p_fk, GROUP BY the key, one SUM over probe
//     columns, optionally ORDER BY it DESC (then the key ASC) LIMIT k <= 32
//                                             -> the semi-join group-by and
//     GPU top-k (the Q3 shape, :1170-1239).
// Throws std::runtime_error naming what it cannot plan (the reference
// returns nullopt).
CudaQueryPlan buildCudaPlan(const ir::AnalyzedQuery& aq, const std::string& queryName, const TuneConfig& tune = {});

// Generate CUDA source metadata from a plan. Reference:
// generateFromPlan (metal_plan_builder.cpp:2115-2154).
CudaCodegen generateFromPlan(const CudaQueryPlan& plan);

// Algorithmic bytes of one execution of the plan (each referenced column
// read once, at its declared width), given registered row counts.
long long planAlgorithmicBytes(const CudaQueryPlan& plan, const std::map<std::string, long long>& rows);

// Template names understood by buildCudaPlan.
std::vector<std::string> planTemplates();

}  // namespace gpudb
