#include "executor.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <stdexcept>

#include "cuda_api.h"

namespace gpudb {

namespace {

std::string cudaErr(const char* what, cudaError_t e) { return std::string(what) + ": " + cudaGetErrorString(e); }

#define GPUDB_CUDA_OR_THROW(call)                                              \
    do {                                                                       \
        const cudaError_t _e = (call);                                         \
        if (_e != cudaSuccess) throw std::runtime_error(cudaErr(#call, _e));   \
    } while (0)

uint64_t encodeScalar(const std::string& type, long long iv, double dv, bool isFloat) {
    uint64_t slot = 0;
    if (type == "double") {
        const double d = isFloat ? dv : (double)iv;
        std::memcpy(&slot, &d, 8);
    } else if (type == "float") {
        const float f = (float)(isFloat ? dv : (double)iv);
        std::memcpy(&slot, &f, 4);
    } else if (type == "int" || type == "unsigned" || type == "unsigned int") {
        const int32_t v = (int32_t)(isFloat ? (long long)dv : iv);
        std::memcpy(&slot, &v, 4);
    } else {
        const int64_t v = isFloat ? (int64_t)dv : (int64_t)iv;
        std::memcpy(&slot, &v, 8);
    }
    return slot;
}

}  // namespace

CudaGenericExecutor::CudaGenericExecutor(int device) : device_(device) {
    GPUDB_CUDA_OR_THROW(cudaSetDevice(device));
    GPUDB_CUDA_OR_THROW(cudaDeviceGetAttribute(&numSMs_, cudaDevAttrMultiProcessorCount, device));
    GPUDB_CUDA_OR_THROW(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    GPUDB_CUDA_OR_THROW(cudaMalloc((void**)&errWord_, sizeof(unsigned)));
    GPUDB_CUDA_OR_THROW(cudaMemset(errWord_, 0, sizeof(unsigned)));
    GPUDB_CUDA_OR_THROW(cudaHostAlloc((void**)&errHost_, sizeof(unsigned), cudaHostAllocDefault));
    const DriverApi& api = driverApi();
    if (!api.loaded) throw std::runtime_error("CUDA driver API unavailable: " + api.error);
}

CudaGenericExecutor::~CudaGenericExecutor() {
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(stream_);
    clearGraphs();
    releaseAllocatedBuffers();
    for (auto& [_, b] : ownedColumns_)
        if (b.ptr) cudaFree(b.ptr);
    ownedColumns_.clear();
    for (auto e : events_) cudaEventDestroy(e);
    if (errWord_) cudaFree(errWord_);
    if (errHost_) cudaFreeHost(errHost_);
    if (stream_) cudaStreamDestroy(stream_);
}

void CudaGenericExecutor::clearGraphs() {
    // deferred replays may still be running on the stream
    if (pendingErr_ && stream_ && !graphs_.empty()) cudaStreamSynchronize(stream_);
    for (auto& [_, g] : graphs_) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
    }
    graphs_.clear();
    graphOrder_.clear();
    seenOnce_.clear();
}

void CudaGenericExecutor::evictOldestGraph() {
    while (!graphOrder_.empty()) {
        auto g = graphs_.find(graphOrder_.front());
        graphOrder_.pop_front();
        if (g == graphs_.end()) continue;
        // a deferred replay of it may still be running on the stream
        if (pendingErr_ && stream_) cudaStreamSynchronize(stream_);
        if (g->second.exec) cudaGraphExecDestroy(g->second.exec);
        if (g->second.graph) cudaGraphDestroy(g->second.graph);
        graphs_.erase(g);
        return;
    }
}

// ---------------------------------------------------------------------------
// registration
// ---------------------------------------------------------------------------
void CudaGenericExecutor::registerTableRowCount(const std::string& table, size_t rows) {
    tableRows_[table] = rows;
    resolver_.registerSymbol(tableSizeName(table), rows);
    resolver_.registerSymbol("num" + table, rows);
}

// Registering a column frees nothing, so the captured graphs stay: a graph
// is looked up by every launch argument (column pointers and sizes among
// them), so one captured over other pointers is simply never matched.
void CudaGenericExecutor::registerTableBuffer(const std::string& column, const void* dptr, size_t rows,
                                              size_t elemBytes) {
    columns_[column] = {dptr, rows, elemBytes, ++generationCounter_};
}

void CudaGenericExecutor::registerAllocatedBuffer(const std::string& name, void* dptr, size_t bytes, size_t elemBytes) {
    auto it = buffers_.find(name);
    if (it != buffers_.end() && it->second.owned && it->second.ptr) cudaFree(it->second.ptr);
    buffers_[name] = {dptr, bytes, elemBytes ? elemBytes : 1, false, bytes};
    clearGraphs();
}

void CudaGenericExecutor::registerSymbol(const std::string& name, uint64_t value) { resolver_.registerSymbol(name, value); }

bool CudaGenericExecutor::tryGetSymbol(const std::string& name, uint64_t& out) const {
    if (!resolver_.hasSymbol(name)) return false;
    out = resolver_.getSymbol(name);
    return true;
}

void CudaGenericExecutor::registerScalarInt(const std::string& name, long long v) {
    scalarInts_[name] = v;
    scalarFloats_.erase(name);
}

void CudaGenericExecutor::registerScalarFloat(const std::string& name, double v) {
    scalarFloats_[name] = v;
    scalarInts_.erase(name);
}

void CudaGenericExecutor::uploadColumn(const std::string& column, const std::string& table, const void* host,
                                       size_t rows, size_t elemBytes) {
    const size_t bytes = rows * elemBytes;
    Buffer& b = ownedColumns_[column];
    if (b.bytes < bytes || !b.ptr) {
        if (b.ptr) {
            cudaStreamSynchronize(stream_);
            cudaFree(b.ptr);
        }
        b.ptr = nullptr;
        GPUDB_CUDA_OR_THROW(cudaMalloc(&b.ptr, bytes ? bytes : 16));
        b.bytes = bytes;
        clearGraphs();
    }
    b.elemBytes = elemBytes;
    b.owned = true;
    if (bytes) GPUDB_CUDA_OR_THROW(cudaMemcpyAsync(b.ptr, host, bytes, cudaMemcpyHostToDevice, stream_));
    columns_[column] = {b.ptr, rows, elemBytes, ++generationCounter_};
    registerTableRowCount(table, rows);
}

void CudaGenericExecutor::registerHostColumn(const std::string& column, const std::string& table, const void* host,
                                             size_t rows, size_t elemBytes) {
    void* dptr = nullptr;
    if (rows) {
        const cudaError_t e = cudaHostGetDevicePointer(&dptr, const_cast<void*>(host), 0);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw std::runtime_error("host column '" + column + "': not pinned, mapped host memory (" +
                                     cudaGetErrorString(e) + ")");
        }
    }
    columns_[column] = {dptr, rows, elemBytes, ++generationCounter_, true};
    registerTableRowCount(table, rows);
}

void CudaGenericExecutor::registerStreamChunk(const std::string& column, const void* dptr, size_t rows,
                                              size_t elemBytes, bool host) {
    columns_[column] = {dptr, rows, elemBytes, ++generationCounter_, host};
}

size_t CudaGenericExecutor::tableRows(const std::string& table) const {
    auto it = tableRows_.find(table);
    if (it != tableRows_.end()) return it->second;
    const std::string sym = tableSizeName(table);
    return resolver_.hasSymbol(sym) ? resolver_.getSymbol(sym) : 0;
}

uint64_t CudaGenericExecutor::columnGeneration(const std::string& column) const {
    auto it = columns_.find(column);
    return it == columns_.end() ? 0 : it->second.generation;
}

const void* CudaGenericExecutor::columnPtr(const std::string& column, size_t* rows) const {
    auto it = columns_.find(column);
    if (it == columns_.end()) return nullptr;
    if (rows) *rows = it->second.rows;
    return it->second.ptr;
}

// ---------------------------------------------------------------------------
// buffers
// ---------------------------------------------------------------------------
bool CudaGenericExecutor::allocateBuffers(const CudaCodegen::PhaseInfo& phase, std::string& error) {
    for (const auto& b : phase.bindings) {
        if (b.kind != CudaParamKind::DeviceBuffer || b.readOnly || b.sizeExpr.empty()) continue;
        uint64_t count = 0;
        try {
            count = resolver_.resolve(b.sizeExpr);
        } catch (const std::exception& e) {
            error = "buffer '" + b.name + "': " + e.what();
            return false;
        }
        const size_t elem = b.elemSizeBytes();
        const size_t bytes = (size_t)(count ? count : 1) * elem;
        auto it = buffers_.find(b.name);
        if (it != buffers_.end() && !it->second.owned) continue;  // caller-provided buffer
        if (it != buffers_.end() && it->second.ptr && it->second.capacity >= bytes && it->second.elemBytes == elem) {
            // reuse the allocation (its capacity stays); remember the
            // logical size for length params / fills
            it->second.bytes = bytes;
            continue;
        }
        // a buffer that has to grow again gets a quarter of headroom, so
        // sizes that creep upward do not free and allocate on every run
        size_t cap = bytes;
        if (it != buffers_.end() && it->second.ptr) {
            if (it->second.elemBytes == elem) cap = std::max(bytes, it->second.capacity + it->second.capacity / 4);
            cudaStreamSynchronize(stream_);
            cudaFree(it->second.ptr);
            it->second.ptr = nullptr;
        }
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, cap);
        if (e != cudaSuccess && cap > bytes) {
            cudaGetLastError();  // the headroom did not fit: the exact size may
            cap = bytes;
            e = cudaMalloc(&p, cap);
        }
        if (e != cudaSuccess) {
            buffers_.erase(b.name);
            error = "cudaMalloc(" + std::to_string(bytes) + " B) for '" + b.name + "': " + cudaGetErrorString(e);
            return false;
        }
        buffers_[b.name] = {p, bytes, elem, true, cap};
        clearGraphs();
    }
    return true;
}

bool CudaGenericExecutor::readBuffer(const std::string& name, void* host, size_t bytes) {
    auto it = buffers_.find(name);
    if (it == buffers_.end() || !it->second.ptr) return false;
    if (bytes > it->second.bytes) return false;
    if (cudaMemcpyAsync(host, it->second.ptr, bytes, cudaMemcpyDeviceToHost, stream_) != cudaSuccess) return false;
    return cudaStreamSynchronize(stream_) == cudaSuccess;
}

void* CudaGenericExecutor::bufferPtr(const std::string& name, size_t* bytes) const {
    auto it = buffers_.find(name);
    if (it == buffers_.end()) return nullptr;
    if (bytes) *bytes = it->second.bytes;
    return it->second.ptr;
}

void CudaGenericExecutor::releaseAllocatedBuffers() {
    if (stream_) cudaStreamSynchronize(stream_);
    clearGraphs();
    for (auto& [_, b] : buffers_)
        if (b.owned && b.ptr) cudaFree(b.ptr);
    buffers_.clear();
}

GenericResult CudaGenericExecutor::collectResult(const CudaResultSchema& schema) {
    return CudaResultCollector::collect(
        schema, [this](const std::string& n, void* dst, size_t bytes) { return readBuffer(n, dst, bytes); },
        [this](const std::string& e) { return resolver_.resolve(e); });
}

// ---------------------------------------------------------------------------
// launch preparation
// ---------------------------------------------------------------------------
void CudaGenericExecutor::ensureEvents(size_t n) {
    while (events_.size() < n) {
        cudaEvent_t e;
        GPUDB_CUDA_OR_THROW(cudaEventCreate(&e));
        events_.push_back(e);
    }
}

bool CudaGenericExecutor::buildLaunch(const RuntimeCompiler::CompiledQuery& cq, const CudaCodegen::PhaseInfo& ph,
                                      Launch& l, std::string& error) {
    const DriverApi& api = driverApi();
    int fi = -1;
    for (size_t i = 0; i < cq.kernelNames.size(); i++)
        if (cq.kernelNames[i] == ph.name) fi = (int)i;
    if (fi < 0) {
        error = "kernel for phase '" + ph.name + "' not found in module";
        return false;
    }
    l.fn = cq.functions[fi];
    l.name = ph.name;
    l.block = ph.isSingleThread ? 1u : (unsigned)ph.threadgroupSize;
    l.smem = (unsigned)ph.dynamicSmemBytes;
    const std::pair<uint64_t, CUfunction> fkey{cq.loadId, l.fn};
    auto sc = smemConfigured_.find(fkey);
    // any dynamic shared memory gets the opt-in: 48 KB of it plus the
    // kernel's static shared memory already exceeds the default limit
    if (l.smem > 0 && (sc == smemConfigured_.end() || sc->second < (int)l.smem)) {
        const CUresult r = api.cuFuncSetAttribute(l.fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)l.smem);
        if (r != CUDA_SUCCESS) {
            error = "phase '" + ph.name + "': cannot reserve " + std::to_string(l.smem) + " B shared memory (" +
                    cuErrorString(r) + ")";
            return false;
        }
        smemConfigured_[fkey] = (int)l.smem;
    }
    if (ph.smemCarveout >= 0 && l.smem > 0) {
        auto cv = carveoutSet_.find(fkey);
        if (cv == carveoutSet_.end() || cv->second != ph.smemCarveout) {
            const CUresult r = api.cuFuncSetAttribute(l.fn, CU_FUNC_ATTRIBUTE_PREFERRED_SHARED_MEMORY_CARVEOUT,
                                                      ph.smemCarveout);
            if (r != CUDA_SUCCESS) {
                error = "phase '" + ph.name + "': cannot set the shared-memory carveout (" + cuErrorString(r) + ")";
                return false;
            }
            carveoutSet_[fkey] = ph.smemCarveout;
        }
    }
    int occ = 0;
    const CUresult r = api.cuOccupancyMaxActiveBlocksPerMultiprocessor(&occ, l.fn, (int)l.block, l.smem);
    if (r != CUDA_SUCCESS || occ <= 0) {
        error = "phase '" + ph.name + "' cannot be resident (block " + std::to_string(l.block) + ", smem " +
                std::to_string(l.smem) + "): " + (r != CUDA_SUCCESS ? cuErrorString(r) : std::string("occupancy 0"));
        return false;
    }
    const long long maxRes = (long long)occ * numSMs_;
    long long grid = maxRes;
    if (ph.isSingleThread) grid = 1;
    else if (!ph.scannedTable.empty()) {
        const long long rows = (long long)tableRows(ph.scannedTable);
        long long work;
        if (ph.tileRows > 0 && rows >= ph.tileRows) work = rows / ph.tileRows;
        else work = (rows + (long long)l.block * ph.rowsPerThread - 1) / ((long long)l.block * ph.rowsPerThread);
        grid = std::min(maxRes, std::max(1ll, work));
    }
    if (ph.maxThreadgroups > 0) grid = std::min<long long>(grid, ph.maxThreadgroups);
    l.grid = (unsigned)std::max(1ll, grid);

    l.slots.assign(ph.bindings.size(), 0);
    for (const auto& b : ph.bindings) {
        uint64_t& s = l.slots[b.argIndex];
        switch (b.kind) {
            case CudaParamKind::TableData: {
                auto it = columns_.find(b.name);
                if (it == columns_.end()) {
                    error = "required column '" + b.name + "' (table '" + b.tableName + "') is not registered";
                    return false;
                }
                if (it->second.host && !b.late) {
                    error = "phase '" + ph.name + "': column '" + b.name +
                            "' is in host memory but every row reads it; only late-materialised columns may stay "
                            "on the host (upload it instead)";
                    return false;
                }
                s = (uint64_t)(uintptr_t)it->second.ptr;
                break;
            }
            case CudaParamKind::TableSize: {
                const uint64_t rows = tableRows(b.tableName);
                std::memcpy(&s, &rows, 8);
                break;
            }
            case CudaParamKind::DeviceBuffer:
            case CudaParamKind::ConstantData: {
                auto it = buffers_.find(b.name);
                if (it == buffers_.end() || !it->second.ptr) {
                    error = "phase '" + ph.name + "': buffer '" + b.name +
                            "' was neither produced by an earlier phase nor registered";
                    return false;
                }
                s = (uint64_t)(uintptr_t)it->second.ptr;
                break;
            }
            case CudaParamKind::ConstantScalar: {
                if (!b.sizeExpr.empty()) {
                    try {
                        s = encodeScalar(b.elementType, (long long)resolver_.resolve(b.sizeExpr), 0, false);
                    } catch (const std::exception& e) {
                        error = "scalar '" + b.name + "': " + e.what();
                        return false;
                    }
                } else if (scalarInts_.count(b.name)) {
                    s = encodeScalar(b.elementType, scalarInts_[b.name], 0, false);
                } else if (scalarFloats_.count(b.name)) {
                    s = encodeScalar(b.elementType, 0, scalarFloats_[b.name], true);
                } else {
                    error = "scalar '" + b.name + "' is not registered";
                    return false;
                }
                break;
            }
            case CudaParamKind::ErrorWord: s = (uint64_t)(uintptr_t)errWord_; break;
            case CudaParamKind::BufferLength: {
                auto it = buffers_.find(b.tableName);
                if (it == buffers_.end()) {
                    error = "length of unknown buffer '" + b.tableName + "'";
                    return false;
                }
                const uint64_t n = it->second.bytes / (it->second.elemBytes ? it->second.elemBytes : 1);
                std::memcpy(&s, &n, 8);
                break;
            }
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// execute
// ---------------------------------------------------------------------------
int CudaGenericExecutor::execute(const RuntimeCompiler::CompiledQuery& cq,
                                 const std::vector<CudaCodegen::PhaseInfo>& phases, int warmup, int measured,
                                 int first, int last, ExecutionResult& out, std::string& error) {
    if (phases.empty()) {
        error = "no phases to execute";
        return -2;
    }
    if (last < 0) last = (int)phases.size();
    if (first < 0 || first >= last || last > (int)phases.size()) {
        error = "bad phase range";
        return -2;
    }
    // a deferred run is one untimed pass; timed runs (the max-key pass's
    // among them) always complete here
    const bool defer = deferSync_ && measured <= 0;
    if (warmup < 0) warmup = 0;
    if (defer) {
        measured = 0;
        warmup = std::max(warmup, 1);
    } else if (measured < 1) {
        measured = 1;
    }
    cudaSetDevice(device_);
    const DriverApi& api = driverApi();

    const auto a0 = std::chrono::steady_clock::now();
    for (int p = first; p < last; p++)
        if (!allocateBuffers(phases[p], error)) return -3;
    out.bufferAllocTimeMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a0).count();

    std::vector<Launch> launches(last - first);
    for (int p = first; p < last; p++)
        if (!buildLaunch(cq, phases[p], launches[p - first], error)) return -4;

    std::vector<Fill> fills;
    if (!skipZeroInit_) {
        std::map<void*, bool> seen;
        for (int p = first; p < last; p++)
            for (const auto& b : phases[p].bindings) {
                if (b.kind != CudaParamKind::DeviceBuffer || !b.zeroInit || b.readOnly) continue;
                auto it = buffers_.find(b.name);
                if (it == buffers_.end() || !it->second.ptr || seen[it->second.ptr]) continue;
                seen[it->second.ptr] = true;
                fills.push_back({it->second.ptr, it->second.bytes, b.fillByte});
            }
    }

    const size_t nl = launches.size();
    ensureEvents(2 * nl + 2);
    out.phaseNames.clear();
    out.phaseTimesMs.assign(nl, 0.0);
    out.phaseGrid.clear();
    out.phaseBlock.clear();
    out.phaseSmem.clear();
    for (const auto& l : launches) {
        out.phaseNames.push_back(l.name);
        out.phaseGrid.push_back((int)l.grid);
        out.phaseBlock.push_back((int)l.block);
        out.phaseSmem.push_back((int)l.smem);
    }
    out.launches = (long long)nl;
    out.totalKernelTimeMs = 0.0;

    auto launchAll = [&](bool timed) -> bool {
        for (const auto& f : fills)
            if (cudaMemsetAsync(f.ptr, f.value, f.bytes, stream_) != cudaSuccess) {
                error = "cudaMemsetAsync failed";
                return false;
            }
        if (timed) cudaEventRecord(events_[2 * nl], stream_);
        for (size_t i = 0; i < nl; i++) {
            Launch& l = launches[i];
            std::vector<void*> args(l.slots.size());
            for (size_t k = 0; k < l.slots.size(); k++) args[k] = &l.slots[k];
            if (timed) cudaEventRecord(events_[2 * i], stream_);
            const CUresult r =
                api.cuLaunchKernel(l.fn, l.grid, 1, 1, l.block, 1, 1, l.smem, (CUstream)stream_, args.data(), nullptr);
            if (r != CUDA_SUCCESS) {
                error = "launch of '" + l.name + "' failed: " + cuErrorString(r);
                return false;
            }
            if (timed) cudaEventRecord(events_[2 * i + 1], stream_);
        }
        if (timed) cudaEventRecord(events_[2 * nl + 1], stream_);
        return true;
    };

    // the word still holds the bits of deferred runs until they are read
    if (!pendingErr_ && cudaMemsetAsync(errWord_, 0, sizeof(unsigned), stream_) != cudaSuccess) {
        error = "cannot clear the device error word";
        return -5;
    }
    const int total = warmup + measured;
    std::map<std::string, GraphEntry>::iterator it = graphs_.end();
    if (useGraphs_) {
        // the load id: a graph captured from a module that was unloaded and
        // loaded again (same source key) must never be replayed
        std::string key = cq.key + "#" + std::to_string(cq.loadId) + ":" + std::to_string(first) + ":" +
                          std::to_string(last);
        for (const auto& l : launches) {
            key += ":" + std::to_string(l.grid);
            for (auto s : l.slots) key += "," + std::to_string(s);
        }
        for (const auto& f : fills) key += ";" + std::to_string((uintptr_t)f.ptr) + "/" + std::to_string(f.bytes);
        it = graphs_.find(key);
        // A launch sequence met for the first time runs eagerly, unless this
        // call repeats it: a query run once (its constants are launch
        // arguments) never pays for a capture or holds a cache entry.
        if (it == graphs_.end() && total == 1 && seenOnce_.count(key) == 0) {
            if (seenOnce_.size() >= kMaxSeen) seenOnce_.clear();
            seenOnce_.insert(key);
        } else if (it == graphs_.end()) {
            seenOnce_.erase(key);
            // the oldest graph makes room: argument sets that no longer
            // occur (columns registered elsewhere since) age out
            if (graphs_.size() >= kMaxGraphs) evictOldestGraph();
            GraphEntry g;
            if (cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                error = "cudaStreamBeginCapture failed";
                return -6;
            }
            const bool ok = launchAll(false);
            const cudaError_t ce = cudaStreamEndCapture(stream_, &g.graph);
            if (!ok || ce != cudaSuccess) {
                if (g.graph) cudaGraphDestroy(g.graph);
                if (error.empty()) error = cudaErr("cudaStreamEndCapture", ce);
                return -6;
            }
            if (cudaGraphInstantiate(&g.exec, g.graph, 0) != cudaSuccess) {
                cudaGraphDestroy(g.graph);
                error = "cudaGraphInstantiate failed";
                return -6;
            }
            it = graphs_.emplace(key, g).first;
            graphOrder_.push_back(key);
        }
    }
    if (it != graphs_.end()) {
        for (int iter = 0; iter < total; iter++) {
            const bool timed = iter >= warmup;
            if (timed) cudaEventRecord(events_[2 * nl], stream_);
            if (cudaGraphLaunch(it->second.exec, stream_) != cudaSuccess) {
                error = "cudaGraphLaunch failed";
                return -6;
            }
            if (timed) {
                cudaEventRecord(events_[2 * nl + 1], stream_);
                if (cudaEventSynchronize(events_[2 * nl + 1]) != cudaSuccess) {
                    error = cudaErr("graph replay", cudaGetLastError());
                    return -7;
                }
                float ms = 0;
                cudaEventElapsedTime(&ms, events_[2 * nl], events_[2 * nl + 1]);
                out.totalKernelTimeMs += ms / measured;
            }
        }
    } else {
        for (int iter = 0; iter < total; iter++) {
            const bool timed = iter >= warmup;
            if (!launchAll(timed)) return -6;
            if (timed) {
                const cudaError_t e = cudaEventSynchronize(events_[2 * nl + 1]);
                if (e != cudaSuccess) {
                    error = cudaErr("kernel execution", e);
                    return -7;
                }
                for (size_t i = 0; i < nl; i++) {
                    float ms = 0;
                    cudaEventElapsedTime(&ms, events_[2 * i], events_[2 * i + 1]);
                    out.phaseTimesMs[i] += ms / measured;
                }
                float ms = 0;
                cudaEventElapsedTime(&ms, events_[2 * nl], events_[2 * nl + 1]);
                out.totalKernelTimeMs += ms / measured;
            }
        }
    }
    if (defer) {
        pendingErr_ = true;
        return 0;
    }
    unsigned bits = 0;
    if (!syncErrors(bits, error)) return -7;
    out.deviceError |= bits;
    return 0;
}

bool CudaGenericExecutor::syncErrors(unsigned& bits, std::string& error) {
    cudaError_t e = cudaMemcpyAsync(errHost_, errWord_, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) {
        error = cudaErr("kernel execution", e);
        return false;
    }
    bits = *errHost_;
    if (pendingErr_) {
        // read: the next run starts from a clear word
        pendingErr_ = false;
        if (cudaMemsetAsync(errWord_, 0, sizeof(unsigned), stream_) != cudaSuccess) {
            error = "cannot clear the device error word";
            return false;
        }
    }
    return true;
}

}  // namespace gpudb
