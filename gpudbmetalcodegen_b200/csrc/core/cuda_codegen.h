#pragma once
// ===================================================================
// CudaCodegen — composable CUDA C++ kernel generation.
//
// Same emission / phase / binding / result-schema surface as the
// reference's MetalCodegen (codegen/core/metal_codegen_base.h:34-147), so
// operators are written the same way: produce() emits lines into the
// current phase, registers its parameters, and a terminal operator
// registers the result schema. print() returns one NVRTC translation unit:
// the hand-written device template library (gpudb_device.cuh) + helpers +
// one `extern "C" __global__` kernel per phase.
//
// B200 specifics carried as phase metadata (all consumed by the executor):
//   * blockSize / minBlocksPerSM  -> __launch_bounds__ and occupancy;
//   * dynamicSmemBytes            -> TMA-bulk staging ring (cp.async.bulk);
//   * tileRows                    -> grid = min(tiles, SMs x occupancy),
//                                    a persistent one-wave grid;
//   * rowsPerThread               -> grid for plain grid-stride phases.
// ===================================================================

#include <functional>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "param_binding.h"

namespace gpudb {

using ConsumerFn = std::function<void()>;

class CudaCodegen {
public:
    // ---- code emission -------------------------------------------------
    void addLine(const std::string& line);
    void addBlock(const std::string& header, const std::function<void()>& body,
                  const std::string& trailing = "");
    void addIf(const std::string& condition, const std::function<void()>& body);
    void addComment(const std::string& comment);
    void increaseIndent();
    void decreaseIndent();
    void addRawCode(const std::string& code);

    // Device helpers emitted once, before all kernels.
    void addHelper(const std::string& code);

    // Unique identifier for temporaries (e.g. "_t3").
    std::string fresh(const std::string& stem);

    // ---- scan hints ------------------------------------------------------
    // An operator pushes a hint before it calls its child's produce() and
    // pops it afterwards, so the scan at the bottom of the chain sees, top
    // down, what the operators above it will do with each row: a selection's
    // guard, a bitmap probe's word it may load ahead (BitmapPrefetch), or a
    // barrier (an operator that defines names the scan cannot evaluate).
    struct ScanHint {
        enum Kind { Guard, BitmapPrefetch, Barrier } kind;
        std::string expr;    // guard predicate / probe key expression
        std::string bitmap;  // BitmapPrefetch: bitmap buffer name
    };
    int pushScanHint(const ScanHint& h);
    void popScanHint();
    const std::vector<ScanHint>& scanHints() const { return scanHints_; }
    // Set by the scan while it emits a row body whose bitmap word for hint
    // `id` is already in a register; empty when not prefetched.
    void setPrefetchVar(int id, const std::string& var);
    std::string prefetchVar(int id) const;

    // ---- phases: one phase = one kernel --------------------------------
    void beginPhase(const std::string& phaseName);
    void endPhase();
    int phaseCount() const { return (int)phases_.size(); }

    void setPhaseScannedTable(const std::string& tableName);
    void setPhaseThreadgroupSize(int size);
    void setPhaseSingleThread(bool single);
    void setPhaseMaxThreadgroups(int max);
    void setPhaseDynamicSmem(int bytes);
    void setPhaseTileRows(int rows);
    void setPhaseRowsPerThread(int rows);
    void setPhaseMinBlocksPerSM(int n);
    void setPhaseSmemCarveout(int percent);
    int currentThreadgroupSize() const;

    // ---- parameters ----------------------------------------------------
    void addColumnParam(const std::string& paramName, const std::string& elemType,
                        const std::string& tableName, bool late = false);
    void addTableSizeParam(const std::string& table);
    void addBufferParam(const std::string& name, const std::string& elemType,
                        const std::string& sizeExpr, bool zeroInit = true, int fillByte = 0);
    void addReadBufferParam(const std::string& name, const std::string& elemType);
    void addAtomicBufferParam(const std::string& name, const std::string& elemType,
                              const std::string& sizeExpr);
    void addScalarParam(const std::string& name, const std::string& type);
    // Scalar whose value is a size expression resolved by the executor.
    void addSizeScalarParam(const std::string& name, const std::string& type, const std::string& sizeExpr);
    // `long long <name>` = element count of buffer `bufferName` at launch.
    void addBufferLengthParam(const std::string& name, const std::string& bufferName);
    // Carve `bytes` (128-byte aligned) out of the phase's dynamic shared
    // memory; returns the byte offset from `gpudb_smem`.
    int allocDynamicSmem(int bytes);
    int dynamicSmemBytes() const { return current_ < 0 ? 0 : phases_[current_].dynamicSmemBytes; }
    void addConstantDataParam(const std::string& name, const std::string& type, size_t bytes);
    void addBitmapReadParam(const std::string& name, const std::string& sizeExpr);
    void addBitmapWriteParam(const std::string& name, const std::string& sizeExpr);
    // Open-addressing hash table: keys (0xFF-filled = empty) + per-slot values.
    void addHashMapParam(const std::string& keysName, const std::string& keyType,
                         const std::string& capacityExpr);
    void addHashMapReadParam(const std::string& keysName, const std::string& keyType);

    void setBufferSize(const std::string& name, const std::string& sizeExpr);
    const std::unordered_map<std::string, std::string>& getGlobalBufferSizes() const {
        return globalBufferSizes_;
    }

    // ---- result schema ---------------------------------------------------
    void registerScalarAggColumn(const std::string& displayName, const std::string& buffer,
                                 bool isWide, int scaleDown = 0);
    void registerMaterializeOutput(const std::string& counterBuffer);
    void registerOutputColumn(const std::string& displayName, const std::string& bufferName,
                              const std::string& elementType);
    void registerKeyedAggOutput(const std::string& bufferName, int numBuckets,
                                int valuesPerBucket,
                                const std::vector<CudaResultSchema::KeyedAggSlot>& slots);
    CudaResultSchema& resultSchema() { return resultSchema_; }
    const CudaResultSchema& getResultSchema() const { return resultSchema_; }

    // ---- output ----------------------------------------------------------
    std::string print();

    struct PhaseInfo {
        std::string name;
        std::string code;
        std::string scannedTable;
        int threadgroupSize = 256;
        int maxThreadgroups = 0;
        bool isSingleThread = false;
        int dynamicSmemBytes = 0;
        int tileRows = 0;
        int rowsPerThread = 1;
        int minBlocksPerSM = 1;
        int smemCarveout = -1;  // preferred carveout percent, -1 = driver default
        std::vector<CudaParamBinding> bindings;
    };
    const std::vector<PhaseInfo>& getPhases() const { return phases_; }
    std::vector<PhaseInfo>& getPhasesMutable() { return phases_; }
    std::vector<CudaParamBinding> getAllBindings() const;

    static const char* deviceHeader();

private:
    std::vector<PhaseInfo> phases_;
    int current_ = -1;
    std::string helperCode_;
    std::unordered_map<std::string, std::string> globalBufferSizes_;
    CudaResultSchema resultSchema_;
    unsigned indentLevel_ = 1;
    int freshCounter_ = 0;
    std::vector<ScanHint> scanHints_;
    std::unordered_map<int, std::string> prefetchVars_;

    PhaseInfo& cur(const char* op);
    std::string indent() const { return std::string(indentLevel_ * 4, ' '); }
    void pushBinding(const char* op, CudaParamBinding b, bool dedup);
    void assignArgIndices(PhaseInfo& phase);
    std::string generateSignature(const PhaseInfo& phase) const;
};

class IndentGuard {
public:
    explicit IndentGuard(CudaCodegen& cg) : cg_(cg) { cg_.increaseIndent(); }
    ~IndentGuard() { cg_.decreaseIndent(); }
    IndentGuard(const IndentGuard&) = delete;
    IndentGuard& operator=(const IndentGuard&) = delete;

private:
    CudaCodegen& cg_;
};

}  // namespace gpudb
