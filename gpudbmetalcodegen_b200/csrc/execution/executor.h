#pragma once
// ===================================================================
// CudaGenericExecutor — data-driven launch of generated phases.
//
// Replaces the reference's MetalGenericExecutor
// (codegen/execution/metal_generic_executor.h:46-164) with the same
// responsibilities and lifetimes: register non-owned columns / row counts /
// buffers / symbols / scalars, allocate phase buffers from symbolic sizes,
// zero/0xFF-fill them every iteration (unless skip-zero-init), launch the
// phases in order, time them, and hand buffers to the collector.
// B200 design:
//   * one CUDA stream per executor; all fills and launches are
//     stream-ordered, the host synchronises once per execute();
//   * per-phase CUDA events (the reference's GPU timestamps);
//   * launch = min(work, SMs x occupancy) persistent CTAs, with the
//     dynamic shared memory each phase declares (TMA ring, smem tables);
//   * the device error word is cleared before and read after each run;
//   * optional CUDA-graph replay of a whole iteration (fills + kernels).
// ===================================================================
#include <cuda_runtime.h>

#include <deque>
#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../core/cuda_codegen.h"
#include "result_collector.h"
#include "runtime_compiler.h"

namespace gpudb {

struct ExecutionResult {
    GenericResult result;
    double totalKernelTimeMs = 0.0;        // device time of one iteration (fills + kernels), mean over measured
    std::vector<double> phaseTimesMs;      // per phase, mean over measured iterations
    std::vector<std::string> phaseNames;
    std::vector<int> phaseGrid, phaseBlock, phaseSmem;
    unsigned deviceError = 0;              // OR of GPUDB_ERR_* bits seen
    long long launches = 0;                // kernels launched per iteration
    double bufferAllocTimeMs = 0.0;
    // filled by the query driver
    double planTimeMs = 0.0, codegenTimeMs = 0.0, compileTimeMs = 0.0, collectTimeMs = 0.0;
};

class CudaGenericExecutor {
public:
    explicit CudaGenericExecutor(int device);
    ~CudaGenericExecutor();
    CudaGenericExecutor(const CudaGenericExecutor&) = delete;
    CudaGenericExecutor& operator=(const CudaGenericExecutor&) = delete;

    // --- registration (non-owning) ---------------------------------------
    void registerTableBuffer(const std::string& column, const void* dptr, size_t rows, size_t elemBytes);
    void registerTableRowCount(const std::string& table, size_t rows);
    void registerAllocatedBuffer(const std::string& name, void* dptr, size_t bytes, size_t elemBytes = 1);
    void registerSymbol(const std::string& name, uint64_t value);
    bool tryGetSymbol(const std::string& name, uint64_t& out) const;
    void registerScalarInt(const std::string& name, long long value);
    void registerScalarFloat(const std::string& name, double value);
    CudaSizeResolver& sizeResolver() { return resolver_; }

    // Owned column: copy `rows*elemBytes` host bytes into an executor-owned
    // device buffer (reused across calls when large enough) on the stream.
    void uploadColumn(const std::string& column, const std::string& table, const void* host, size_t rows,
                      size_t elemBytes);
    // Column left in pinned, mapped host memory and read in place by the
    // kernels (over the host link, at access time). Only a late-materialised
    // binding may use it: rows that fail earlier selections never touch it.
    void registerHostColumn(const std::string& column, const std::string& table, const void* host, size_t rows,
                            size_t elemBytes);

    // Chunked streaming (the reference's chunk loop, codegen_main.cpp:686-808):
    // `dptr` holds one chunk of `rows` rows of a streamed column (device
    // memory, or the mapped device address of pinned host memory when
    // `host`, then read in place by late-materialised bindings only).
    // Neither call touches the table's row-count symbol, so size
    // expressions keep seeing the whole table while setScanRows() sets the
    // extent the scanning phases walk.
    void registerStreamChunk(const std::string& column, const void* dptr, size_t rows, size_t elemBytes, bool host);
    void setScanRows(const std::string& table, size_t rows) { tableRows_[table] = rows; }
    // Drop a column registration (a streamed chunk must not outlive its run).
    void forgetColumn(const std::string& column) { columns_.erase(column); }

    // --- execution -----------------------------------------------------------
    // Run phases [first, last) (last < 0 = all) `warmup` + `measured` times.
    // Returns 0, or a negative status with `error` filled.
    int execute(const RuntimeCompiler::CompiledQuery& cq, const std::vector<CudaCodegen::PhaseInfo>& phases,
                int warmup, int measured, int first, int last, ExecutionResult& out, std::string& error);

    void setSkipZeroInit(bool skip) { skipZeroInit_ = skip; }
    void setUseGraphs(bool on) { useGraphs_ = on; }
    // Deferred completion: an untimed execute() returns once its work is enqueued,
    // without waiting or reading the device error word; the bits of such
    // runs accumulate until syncErrors() (or a waiting execute) reads them.
    void setDeferSync(bool on) { deferSync_ = on; }
    // Waits for the stream and returns (and clears) the accumulated device
    // error bits; false if the stream itself failed.
    bool syncErrors(unsigned& bits, std::string& error);

    // --- buffers -------------------------------------------------------------
    bool readBuffer(const std::string& name, void* host, size_t bytes);
    void* bufferPtr(const std::string& name, size_t* bytes = nullptr) const;
    void releaseAllocatedBuffers();
    GenericResult collectResult(const CudaResultSchema& schema);

    cudaStream_t stream() const { return stream_; }
    int device() const { return device_; }
    int numSMs() const { return numSMs_; }
    size_t tableRows(const std::string& table) const;
    const void* columnPtr(const std::string& column, size_t* rows = nullptr) const;
    // Bumped on every (re)registration or upload of the column; caches of
    // column-derived values (max-key symbols) compare it.
    uint64_t columnGeneration(const std::string& column) const;

private:
    struct Buffer {
        void* ptr = nullptr;
        size_t bytes = 0;     // logical size of the current run (length params, fills, reads)
        size_t elemBytes = 1;
        bool owned = false;
        size_t capacity = 0;  // bytes allocated; reused while a run's size fits
    };
    struct Column {
        const void* ptr = nullptr;
        size_t rows = 0;
        size_t elemBytes = 0;
        uint64_t generation = 0;
        bool host = false;  // pinned host memory read in place
    };
    uint64_t generationCounter_ = 0;
    struct Launch {
        CUfunction fn;
        unsigned grid, block, smem;
        std::vector<uint64_t> slots;
        std::string name;
    };
    struct Fill {
        void* ptr;
        size_t bytes;
        int value;
    };

    int device_ = 0;
    int numSMs_ = 148;
    cudaStream_t stream_ = nullptr;
    unsigned* errWord_ = nullptr;
    unsigned* errHost_ = nullptr;
    static constexpr size_t kMaxGraphs = 512;  // captured graphs kept per context
    bool skipZeroInit_ = false;
    bool useGraphs_ = false;
    bool deferSync_ = false;
    bool pendingErr_ = false;  // deferred runs whose error bits are unread
    CudaSizeResolver resolver_;
    std::unordered_map<std::string, Column> columns_;
    std::unordered_map<std::string, size_t> tableRows_;
    std::unordered_map<std::string, Buffer> buffers_;
    std::unordered_map<std::string, Buffer> ownedColumns_;
    std::unordered_map<std::string, long long> scalarInts_;
    std::unordered_map<std::string, double> scalarFloats_;
    // keyed by (load id, function): handles of an unloaded module recur
    std::map<std::pair<uint64_t, CUfunction>, int> smemConfigured_;
    std::map<std::pair<uint64_t, CUfunction>, int> carveoutSet_;
    std::vector<cudaEvent_t> events_;
    struct GraphEntry {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
    };
    std::map<std::string, GraphEntry> graphs_;
    std::deque<std::string> graphOrder_;          // graph keys in capture order, oldest first
    std::unordered_set<std::string> seenOnce_;    // keys run once, eagerly, not captured yet
    static constexpr size_t kMaxSeen = 4096;

    void ensureEvents(size_t n);
    bool allocateBuffers(const CudaCodegen::PhaseInfo& phase, std::string& error);
    bool buildLaunch(const RuntimeCompiler::CompiledQuery& cq, const CudaCodegen::PhaseInfo& phase, Launch& l,
                     std::string& error);
    void clearGraphs();
    void evictOldestGraph();
};

}  // namespace gpudb
