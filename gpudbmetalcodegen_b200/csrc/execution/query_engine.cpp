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

int runQuery(QueryContext& qc, PreparedQuery& q, int warmup, int measured, bool collect, ExecutionResult& out,
             std::string& err) {
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
    const auto& phases = q.cg.getPhases();
    // Only counter-driven sizing needs a host round trip; supplied sizes
    // (learned predictions, explicit constants) are registered up front so
    // the whole plan runs as one stream-ordered sequence.
    std::vector<int> cuts;
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
    cuts.push_back((int)phases.size());
    out = ExecutionResult{};
    out.planTimeMs = q.planMs;
    out.codegenTimeMs = q.codegenMs;
    out.compileTimeMs = q.compileMs;
    int first = 0;
    size_t si = 0;
    for (int cut : cuts) {
        // register sizing symbols whose producing phases have run
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
        if (cut <= first) continue;
        ExecutionResult seg;
        const int rc = qc.ex.execute(*q.compiled, phases, warmup, measured, first, cut, seg, err);
        if (rc != 0) return rc;
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
        first = cut;
    }
    if (out.deviceError) {
        err = "device error word 0x" + [&] {
            char b[16];
            snprintf(b, sizeof b, "%x", out.deviceError);
            return std::string(b);
        }();
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

}  // namespace gpudb
