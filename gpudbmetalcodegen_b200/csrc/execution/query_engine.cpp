#include "query_engine.h"

#include <algorithm>

#include <chrono>
#include <regex>
#include <set>
#include <sstream>
#include <stdexcept>

namespace gpudb {

namespace {
double msSince(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Table that owns a catalog column.
std::string tableOf(const std::string& column) {
    for (const auto& t : catalogTables())
        for (const auto& c : catalogTable(t).columns)
            if (c.name == column) return t;
    return "";
}
}  // namespace

std::string describePlan(const PreparedQuery& q) {
    std::ostringstream o;
    o << "plan " << q.plan.name << "  spec={" << q.plan.spec << "}  tune={" << q.tune.toString() << "}\n";
    const auto& phases = q.cg.getPhases();
    for (size_t i = 0; i < q.plan.phases.size() && i < phases.size(); i++) {
        const auto& pp = q.plan.phases[i];
        const auto& ph = phases[i];
        o << "  phase " << i << " " << ph.name << ": " << (pp.root ? pp.root->describe() : "<empty>") << "\n";
        o << "    block=" << ph.threadgroupSize << " tileRows=" << ph.tileRows << " dynSmem=" << ph.dynamicSmemBytes
          << " maxBlocks=" << ph.maxThreadgroups << " scanned=" << ph.scannedTable << "\n";
        for (const auto& b : ph.bindings)
            o << "    arg" << b.argIndex << " " << paramKindName(b.kind) << " " << b.cudaTypeDecl << " " << b.name
              << (b.sizeExpr.empty() ? "" : "  [" + b.sizeExpr + "]") << (b.zeroInit ? "  fill=" + std::to_string(b.fillByte) : "")
              << "\n";
    }
    for (const auto& s : q.plan.sizing)
        o << "  sizing " << s.symbol << " after phase " << s.afterPhase << " from "
          << (s.counterBuffer.empty() ? "'" + s.fallbackExpr + "'" : "counter " + s.counterBuffer)
          << (s.minCounterBuffer.empty() ? "" : " (min with " + s.minCounterBuffer + ")") << "\n";
    return o.str();
}

std::shared_ptr<PreparedQuery> prepareQuery(const std::string& spec, const std::string& tuneStr, bool compile,
                                            bool load) {
    auto t0 = std::chrono::steady_clock::now();
    const TuneConfig tune = TuneConfig::parse(tuneStr);
    CudaQueryPlan plan = buildCudaPlan(spec, tune);
    return prepareFromPlan(std::move(plan), tune, msSince(t0), compile, load);
}

std::shared_ptr<PreparedQuery> prepareFromPlan(CudaQueryPlan plan, const TuneConfig& tune, double planMs, bool compile,
                                               bool load) {
    auto q = std::make_shared<PreparedQuery>();
    q->tune = tune;
    q->plan = std::move(plan);
    q->planMs = planMs;
    auto t0 = std::chrono::steady_clock::now();
    q->cg = generateFromPlan(q->plan);
    q->source = q->cg.print();
    for (const auto& ph : q->cg.getPhases()) q->kernelNames.push_back(ph.name);
    q->codegenMs = msSince(t0);
    q->describe = describePlan(*q);
    if (compile && !load) {
        CubinArtifact art;
        std::string err;
        if (!RuntimeCompiler::compileToCubin(q->source, art, err)) throw std::runtime_error(err);
        q->compileLog = art.log;
        q->compileMs = art.compileMs;
    }
    if (load) loadQuery(*q);
    return q;
}

void loadQuery(PreparedQuery& q) {
    if (q.compiled) return;
    std::string err;
    auto t0 = std::chrono::steady_clock::now();
    q.compiled = RuntimeCompiler::compileAndLoad(q.source, q.kernelNames, err);
    if (!q.compiled) throw std::runtime_error(err);
    q.compileMs = msSince(t0);
    q.compileLog = q.compiled->log;
}

long long registerMaxKey(QueryContext& qc, const std::string& column) {
    size_t rows = 0;
    const void* ptr = qc.ex.columnPtr(column, &rows);
    if (!ptr) throw std::runtime_error("max-key pass: column '" + column + "' is not registered");
    auto it = qc.maxKeys.find(column);
    const uint64_t gen = qc.ex.columnGeneration(column);
    if (it != qc.maxKeys.end() && it->second.generation == gen) {
        qc.ex.registerSymbol("max_" + column, (uint64_t)std::max(0ll, it->second.max));
        return it->second.max;
    }
    const std::string table = tableOf(column);
    if (table.empty()) throw std::runtime_error("max-key pass: '" + column + "' is not a catalog column");
    const std::string spec = "template=colmax;table=" + table + ";col=" + column;
    auto& hq = qc.helperQueries[spec];
    if (!hq) hq = prepareQuery(spec, "bs=512;scan=direct", true, true);
    ExecutionResult r;
    std::string err;
    const bool skip = false;
    qc.ex.setSkipZeroInit(skip);
    if (qc.ex.execute(*hq->compiled, hq->cg.getPhases(), 0, 1, 0, -1, r, err) != 0)
        throw std::runtime_error("max-key pass: " + err);
    uint64_t biased = 0;
    if (!qc.ex.readBuffer("d_colmax_max_biased", &biased, 8)) throw std::runtime_error("max-key pass: no output");
    const long long mx = rows ? (long long)(biased ^ 0x8000000000000000ull) : 0;
    qc.maxKeys[column] = {gen, mx};
    qc.ex.registerSymbol("max_" + column, (uint64_t)std::max(0ll, mx));
    return mx;
}

namespace {

// Load the module and register the max-key symbols its size expressions use.
int prepareRun(QueryContext& qc, PreparedQuery& q, std::string& err) {
    try {
        loadQuery(q);
        // max-key sizing symbols referenced by any size expression
        if (!q.maxKeyColumnsFound) {
            static const std::regex re("max_([A-Za-z][A-Za-z0-9_]*)");
            std::set<std::string> cols;
            for (const auto& ph : q.cg.getPhases())
                for (const auto& b : ph.bindings) {
                    for (std::sregex_iterator it(b.sizeExpr.begin(), b.sizeExpr.end(), re), end; it != end; ++it)
                        cols.insert((*it)[1]);
                }
            q.maxKeyColumns.assign(cols.begin(), cols.end());
            q.maxKeyColumnsFound = true;
        }
        for (const auto& c : q.maxKeyColumns) registerMaxKey(qc, c);
    } catch (const std::exception& e) {
        err = e.what();
        return -2;
    }
    return 0;
}

// Register supplied sizes up front; return the phases after which a
// counter-driven sizing step needs a host round trip.
int sizingCuts(QueryContext& qc, PreparedQuery& q, std::vector<int>& cuts, std::string& err) {
    for (const auto& s : q.plan.sizing) {
        if (!s.counterBuffer.empty()) {
            cuts.push_back(s.afterPhase);
            continue;
        }
        try {
            qc.ex.registerSymbol(s.symbol, qc.ex.sizeResolver().resolve(s.fallbackExpr));
        } catch (const std::exception& e) {
            err = std::string("sizing: ") + e.what();
            return -2;
        }
    }
    return 0;
}

// Register the counter-driven sizing symbols whose producing phases (those
// before `first`) have run; `si` walks the plan's sizing steps.
int registerCounters(QueryContext& qc, PreparedQuery& q, int first, size_t& si, std::string& err) {
    while (si < q.plan.sizing.size() && q.plan.sizing[si].afterPhase <= first) {
        const auto& st = q.plan.sizing[si++];
        if (st.counterBuffer.empty()) continue;
        uint64_t v = 0;
        if (!qc.ex.readBuffer(st.counterBuffer, &v, 8)) {
            err = "sizing: counter '" + st.counterBuffer + "' unavailable";
            return -2;
        }
        if (!st.minCounterBuffer.empty()) {
            uint64_t w = 0;
            if (!qc.ex.readBuffer(st.minCounterBuffer, &w, 8)) {
                err = "sizing: counter '" + st.minCounterBuffer + "' unavailable";
                return -2;
            }
            v = std::min(v, w);
        }
        qc.ex.registerSymbol(st.symbol, v);
    }
    return 0;
}

void appendSegment(ExecutionResult& out, const ExecutionResult& seg) {
    out.totalKernelTimeMs += seg.totalKernelTimeMs;
    out.bufferAllocTimeMs += seg.bufferAllocTimeMs;
    out.deviceError |= seg.deviceError;
    out.launches += seg.launches;
    for (size_t i = 0; i < seg.phaseNames.size(); i++) {
        out.phaseNames.push_back(seg.phaseNames[i]);
        out.phaseTimesMs.push_back(seg.phaseTimesMs[i]);
        out.phaseGrid.push_back(seg.phaseGrid[i]);
        out.phaseBlock.push_back(seg.phaseBlock[i]);
        out.phaseSmem.push_back(seg.phaseSmem[i]);
    }
}

// Phases [from, to) split at the counter-driven sizing steps.
int runPhases(QueryContext& qc, PreparedQuery& q, const std::vector<int>& cuts, int from, int to, int warmup,
              int measured, size_t& si, ExecutionResult& out, std::string& err) {
    const auto& phases = q.cg.getPhases();
    int first = from;
    std::vector<int> ends;
    for (int c : cuts)
        if (c > from && c < to) ends.push_back(c);
    ends.push_back(to);
    std::sort(ends.begin(), ends.end());
    for (int cut : ends) {
        if (int rc = registerCounters(qc, q, first, si, err)) return rc;
        if (cut <= first) continue;
        ExecutionResult seg;
        const int rc = qc.ex.execute(*q.compiled, phases, warmup, measured, first, cut, seg, err);
        if (rc != 0) return rc;
        appendSegment(out, seg);
        first = cut;
    }
    return 0;
}

int finish(QueryContext& qc, PreparedQuery& q, bool collect, ExecutionResult& out, std::string& err) {
    if (out.deviceError) {
        char b[16];
        snprintf(b, sizeof b, "%x", out.deviceError);
        err = std::string("device error word 0x") + b;
        return -7;
    }
    if (collect) {
        const auto t0 = std::chrono::steady_clock::now();
        try {
            out.result = qc.ex.collectResult(q.cg.getResultSchema());
        } catch (const std::exception& e) {
            err = e.what();
            return -2;
        }
        out.collectTimeMs = msSince(t0);
    }
    return 0;
}

}  // namespace

int runQuery(QueryContext& qc, PreparedQuery& q, int warmup, int measured, bool collect, ExecutionResult& out,
             std::string& err) {
    if (int rc = prepareRun(qc, q, err)) return rc;
    const auto& phases = q.cg.getPhases();
    // Only counter-driven sizing needs a host round trip; supplied sizes
    // (learned predictions, explicit constants) are registered up front so
    // the whole plan runs as one stream-ordered sequence.
    std::vector<int> cuts;
    if (int rc = sizingCuts(qc, q, cuts, err)) return rc;
    out = ExecutionResult{};
    out.planTimeMs = q.planMs;
    out.codegenTimeMs = q.codegenMs;
    out.compileTimeMs = q.compileMs;
    size_t si = 0;
    if (int rc = runPhases(qc, q, cuts, 0, (int)phases.size(), warmup, measured, si, out, err)) return rc;
    return finish(qc, q, collect, out, err);
}

StreamRing::~StreamRing() {
    if (copy) cudaStreamSynchronize(copy);
    for (int s = 0; s < kSlots; s++) {
        for (auto& [_, b] : buf[s])
            if (b.first) cudaFree(b.first);
        if (ready[s]) cudaEventDestroy(ready[s]);
        if (consumed[s]) cudaEventDestroy(consumed[s]);
    }
    if (copy) cudaStreamDestroy(copy);
}

int runStreamed(QueryContext& qc, PreparedQuery& q, const std::string& table, const std::vector<StreamColumn>& cols,
                uint64_t rows, uint64_t chunkRows, bool collect, ExecutionResult& out, std::string& err) {
    if (chunkRows == 0) {
        err = "streamed run: chunk rows must be positive";
        return -2;
    }
    if (int rc = prepareRun(qc, q, err)) return rc;
    const auto& phases = q.cg.getPhases();
    const int np = (int)phases.size();
    int firstS = -1, lastS = -1;
    for (int p = 0; p < np; p++)
        if (phases[p].scannedTable == table) {
            if (firstS < 0) firstS = p;
            lastS = p + 1;
        }
    if (firstS < 0) {
        err = "streamed run: no phase of the plan scans table '" + table + "'";
        return -2;
    }
    std::set<std::string> given;
    for (const auto& c : cols) {
        if (c.column.empty() || (!c.host && rows) || c.elemBytes == 0) {
            err = "streamed run: a column needs a name, host memory and an element size";
            return -2;
        }
        given.insert(c.column);
    }
    for (int p = 0; p < np; p++) {
        const bool streamed = p >= firstS && p < lastS;
        if (streamed && phases[p].scannedTable != table) {
            err = "streamed run: the phases that scan '" + table + "' are not consecutive";
            return -2;
        }
        for (const auto& b : phases[p].bindings) {
            const bool ofTable = (b.kind == CudaParamKind::TableData || b.kind == CudaParamKind::TableSize) &&
                                 b.tableName == table;
            if (ofTable && !streamed) {
                err = "streamed run: phase '" + phases[p].name + "' reads table '" + table +
                      "' outside the streamed phases (stream a plan whose later phases do not read it)";
                return -2;
            }
            if (ofTable && b.kind == CudaParamKind::TableData && !given.count(b.name)) {
                err = "streamed run: column '" + b.name + "' of '" + table + "' is not supplied";
                return -2;
            }
        }
    }
    for (const auto& s : q.plan.sizing)
        if (!s.counterBuffer.empty() && s.afterPhase > firstS) {
            err = "streamed run: sizing step '" + s.symbol + "' reads a counter of the streamed phases";
            return -2;
        }
    std::vector<int> cuts;
    if (int rc = sizingCuts(qc, q, cuts, err)) return rc;
    out = ExecutionResult{};
    out.planTimeMs = q.planMs;
    out.codegenTimeMs = q.codegenMs;
    out.compileTimeMs = q.compileMs;
    CudaGenericExecutor& ex = qc.ex;
    ex.registerTableRowCount(table, rows);  // size expressions see the whole table

    // the ring: copy stream, events, device chunk buffers of the copied columns
    if (!qc.ring) {
        auto r = std::make_unique<StreamRing>();
        if (cudaStreamCreateWithFlags(&r->copy, cudaStreamNonBlocking) != cudaSuccess) {
            err = "streamed run: cannot create the copy stream";
            return -3;
        }
        for (int s = 0; s < StreamRing::kSlots; s++)
            if (cudaEventCreateWithFlags(&r->ready[s], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&r->consumed[s], cudaEventDisableTiming) != cudaSuccess) {
                err = "streamed run: cannot create events";
                return -3;
            }
        qc.ring = std::move(r);
    }
    StreamRing& R = *qc.ring;
    cudaStreamSynchronize(R.copy);  // a failed earlier run may have left copies in flight
    std::vector<const char*> mapped(cols.size(), nullptr);
    for (size_t k = 0; k < cols.size(); k++) {
        const auto& c = cols[k];
        if (c.inPlace) {
            void* d = nullptr;
            if (rows && cudaHostGetDevicePointer(&d, const_cast<void*>(c.host), 0) != cudaSuccess) {
                cudaGetLastError();
                err = "streamed run: column '" + c.column + "' is read in place but is not pinned, mapped host memory";
                return -2;
            }
            mapped[k] = static_cast<const char*>(d);
            continue;
        }
        const size_t need = std::max<size_t>(16, (size_t)std::min(rows, chunkRows) * c.elemBytes);
        for (int s = 0; s < StreamRing::kSlots; s++) {
            auto& b = R.buf[s][c.column];
            if (b.second >= need) continue;
            if (b.first) cudaFree(b.first);
            b = {nullptr, 0};
            if (cudaMalloc(&b.first, need) != cudaSuccess) {
                cudaGetLastError();
                err = "streamed run: cannot allocate " + std::to_string(need) + " B for a chunk of '" + c.column + "'";
                return -3;
            }
            b.second = need;
        }
    }

    const uint64_t nChunks = rows ? (rows + chunkRows - 1) / chunkRows : 1;
    const int S = StreamRing::kSlots;
    cudaStream_t cs = ex.stream();
    auto enqueueCopy = [&](uint64_t c) -> bool {
        const int slot = (int)(c % S);
        const uint64_t r0 = c * chunkRows, n = std::min(chunkRows, rows - r0);
        // the slot's previous chunk must have been scanned
        if (c >= (uint64_t)S && cudaStreamWaitEvent(R.copy, R.consumed[slot], 0) != cudaSuccess) return false;
        for (const auto& col : cols) {
            if (col.inPlace || n == 0) continue;
            if (cudaMemcpyAsync(R.buf[slot][col.column].first, static_cast<const char*>(col.host) + r0 * col.elemBytes,
                                n * col.elemBytes, cudaMemcpyHostToDevice, R.copy) != cudaSuccess)
                return false;
        }
        return cudaEventRecord(R.ready[slot], R.copy) == cudaSuccess;
    };
    // the first chunks start copying now, under the pre-stream phases
    int rc = 0;
    for (uint64_t c = 0; c < std::min<uint64_t>(S, nChunks) && rc == 0; c++)
        if (!enqueueCopy(c)) {
            err = "streamed run: chunk copy failed";
            rc = -6;
        }
    // pre-stream phases, with their sizing steps
    size_t si = 0;
    if (rc == 0) rc = runPhases(qc, q, cuts, 0, firstS, 0, 1, si, out, err);
    if (rc == 0) rc = registerCounters(qc, q, firstS, si, err);
    if (rc != 0) {
        cudaStreamSynchronize(R.copy);  // the host columns stay untouched once the call returns
        return rc;
    }
    {
        struct Deferred {
            CudaGenericExecutor& ex;
            explicit Deferred(CudaGenericExecutor& e) : ex(e) { ex.setDeferSync(true); }
            ~Deferred() {
                ex.setDeferSync(false);
                ex.setSkipZeroInit(false);
            }
        } deferred(ex);
        for (uint64_t c = 0; c < nChunks && rc == 0; c++) {
            const int slot = (int)(c % S);
            const uint64_t r0 = c * chunkRows, n = rows ? std::min(chunkRows, rows - r0) : 0;
            if (cudaStreamWaitEvent(cs, R.ready[slot], 0) != cudaSuccess) {
                err = "streamed run: cannot order a chunk after its copy";
                rc = -6;
                break;
            }
            for (size_t k = 0; k < cols.size(); k++) {
                const auto& col = cols[k];
                const void* p = col.inPlace ? static_cast<const void*>(mapped[k] ? mapped[k] + r0 * col.elemBytes : nullptr)
                                            : R.buf[slot][col.column].first;
                ex.registerStreamChunk(col.column, p, n, col.elemBytes, col.inPlace);
            }
            ex.setScanRows(table, n);
            ex.setSkipZeroInit(c > 0);  // chunks accumulate into the first chunk's zeroed buffers
            ExecutionResult seg;
            rc = ex.execute(*q.compiled, phases, 0, 0, firstS, lastS, seg, err);
            if (rc != 0) break;
            if (c == 0) appendSegment(out, seg);
            else out.launches += seg.launches;
            if (cudaEventRecord(R.consumed[slot], cs) != cudaSuccess ||
                (c + S < nChunks && !enqueueCopy(c + S))) {
                err = "streamed run: chunk copy failed";
                rc = -6;
            }
        }
    }
    // no chunk buffer stays registered past the run
    for (const auto& col : cols) ex.forgetColumn(col.column);
    ex.setScanRows(table, rows);
    if (rc != 0) {
        cudaStreamSynchronize(R.copy);
        unsigned bits = 0;
        std::string ignored;
        ex.syncErrors(bits, ignored);
        return rc;
    }
    if (lastS < np) {
        if (int r = runPhases(qc, q, cuts, lastS, np, 0, 1, si, out, err)) return r;
    } else {
        unsigned bits = 0;
        if (!ex.syncErrors(bits, err)) return -7;
        out.deviceError |= bits;
    }
    return finish(qc, q, collect, out, err);
}

}  // namespace gpudb
