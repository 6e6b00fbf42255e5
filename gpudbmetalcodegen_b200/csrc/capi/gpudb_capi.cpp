// C-ABI of libgpudb.so: include/gpudb_rt.h and include/gpudb_engine.h.
// Every entry point catches C++ exceptions and turns them into a status +
// context error text; nothing C++ crosses the boundary.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>
#include <memory>
#include <string>

#include "../../../include/gpudb_engine.h"
#include "../../../include/gpudb_rt.h"
#include "../execution/query_engine.h"
#include "../io/colbin.h"
#include "../sql/sql_frontend.h"
#include "../planning/plan_builder.h"
#include "../planning/query_ir.h"

struct gpudb_ctx {
    std::unique_ptr<gpudb::QueryContext> qc;
    std::string lastError;
};
struct gpudb_module {
    std::shared_ptr<gpudb::RuntimeCompiler::CompiledQuery> cq;
};
struct gpudb_query {
    std::shared_ptr<gpudb::PreparedQuery> q;
};
struct gpudb_result {
    gpudb::GenericResult r;
};
// An analyzed query under construction: its nodes are owned here and handed
// out as opaque pointers (checked against this pool before use).
struct gpudb_expr {
    gpudb::ir::ExprPtr e;
};
struct gpudb_pred {
    gpudb::ir::PredPtr p;
};
struct gpudb_aq {
    gpudb::ir::AnalyzedQuery q;
    std::vector<std::unique_ptr<gpudb_expr>> exprs;
    std::vector<std::unique_ptr<gpudb_pred>> preds;
    bool owns(const gpudb_expr* e) const {
        for (const auto& x : exprs)
            if (x.get() == e) return true;
        return false;
    }
    bool owns(const gpudb_pred* p) const {
        for (const auto& x : preds)
            if (x.get() == p) return true;
        return false;
    }
    gpudb_expr* add(gpudb::ir::ExprPtr e) {
        exprs.push_back(std::make_unique<gpudb_expr>(gpudb_expr{std::move(e)}));
        return exprs.back().get();
    }
    gpudb_pred* add(gpudb::ir::PredPtr p) {
        preds.push_back(std::make_unique<gpudb_pred>(gpudb_pred{std::move(p)}));
        return preds.back().get();
    }
};

namespace {

thread_local std::string tlCreateError;

size_t copyOut(const std::string& s, char* buf, size_t cap) {
    if (buf && cap) {
        const size_t n = s.size() < cap - 1 ? s.size() : cap - 1;
        std::memcpy(buf, s.data(), n);
        buf[n] = '\0';
    }
    return s.size();
}

int fail(gpudb_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->lastError = msg;
    else tlCreateError = msg;
    return code;
}

int mapStatus(int rc) {
    switch (rc) {
        case 0: return GPUDB_OK;
        case -2: return GPUDB_E_PLAN;
        case -3: return GPUDB_E_ALLOC;
        case -4: return GPUDB_E_LAUNCH;
        case -5: return GPUDB_E_CUDA;
        case -6: return GPUDB_E_LAUNCH;
        case -7: return GPUDB_E_DEVICE;
        default: return GPUDB_E_CUDA;
    }
}

void fillTiming(const gpudb::ExecutionResult& r, gpudb_timing* t) {
    if (!t) return;
    std::memset(t, 0, sizeof *t);
    t->total_ms = r.totalKernelTimeMs;
    t->nphases = (int)std::min<size_t>(r.phaseNames.size(), GPUDB_MAX_PHASES);
    for (int i = 0; i < t->nphases; i++) {
        t->phase_ms[i] = r.phaseTimesMs[i];
        t->phase_grid[i] = r.phaseGrid[i];
        t->phase_block[i] = r.phaseBlock[i];
    }
    t->device_error = r.deviceError;
    t->launches = r.launches;
    t->alloc_ms = r.bufferAllocTimeMs;
    t->plan_ms = r.planTimeMs;
    t->codegen_ms = r.codegenTimeMs;
    t->compile_ms = r.compileTimeMs;
    t->collect_ms = r.collectTimeMs;
}

#define GPUDB_GUARD(ctx, ...)                                    \
    try {                                                        \
        __VA_ARGS__                                              \
    } catch (const std::exception& e) {                          \
        return fail(ctx, GPUDB_E_INVALID, e.what());             \
    } catch (...) {                                              \
        return fail(ctx, GPUDB_E_INVALID, "unknown C++ exception"); \
    }

}  // namespace

namespace gpudb {
// Error text of context-free entry points, read back by gpudb_last_error(NULL).
void setThreadError(const std::string& message) { tlCreateError = message; }
}  // namespace gpudb

extern "C" {

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
int gpudb_create(int device, gpudb_ctx** out) {
    if (!out) return fail(nullptr, GPUDB_E_INVALID, "out is NULL");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(nullptr, GPUDB_E_NOGPU, "no CUDA device available");
    }
    if (device < 0 || device >= n) return fail(nullptr, GPUDB_E_INVALID, "device index out of range");
    try {
        auto c = std::make_unique<gpudb_ctx>();
        c->qc = std::make_unique<gpudb::QueryContext>(device);
        *out = c.release();
        return GPUDB_OK;
    } catch (const std::exception& e) {
        return fail(nullptr, GPUDB_E_CUDA, e.what());
    }
}

void gpudb_destroy(gpudb_ctx* ctx) { delete ctx; }

size_t gpudb_last_error(gpudb_ctx* ctx, char* buf, size_t cap) {
    return copyOut(ctx ? ctx->lastError : tlCreateError, buf, cap);
}

void* gpudb_stream(gpudb_ctx* ctx) { return ctx ? (void*)ctx->qc->ex.stream() : nullptr; }

int gpudb_device_info(gpudb_ctx* ctx, int* num_sms, int* cc_major, int* cc_minor) {
    if (!ctx) return GPUDB_E_INVALID;
    const int d = ctx->qc->ex.device();
    if (num_sms) *num_sms = ctx->qc->ex.numSMs();
    if (cc_major) cudaDeviceGetAttribute(cc_major, cudaDevAttrComputeCapabilityMajor, d);
    if (cc_minor) cudaDeviceGetAttribute(cc_minor, cudaDevAttrComputeCapabilityMinor, d);
    return GPUDB_OK;
}

int gpudb_synchronize(gpudb_ctx* ctx) {
    if (!ctx) return GPUDB_E_INVALID;
    const cudaError_t e = cudaStreamSynchronize(ctx->qc->ex.stream());
    return e == cudaSuccess ? GPUDB_OK : fail(ctx, GPUDB_E_CUDA, cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// compile
// ---------------------------------------------------------------------------
int gpudb_compile(gpudb_ctx* ctx, const char* src, const char* const* kernels, int nkernels, gpudb_module** out) {
    if (!ctx || !src || !out || (nkernels > 0 && !kernels)) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    GPUDB_GUARD(ctx, {
        std::vector<std::string> names;
        for (int i = 0; i < nkernels; i++) names.push_back(kernels[i]);
        std::string err;
        cudaSetDevice(ctx->qc->ex.device());
        auto cq = gpudb::RuntimeCompiler::compileAndLoad(src, names, err);
        if (!cq) return fail(ctx, GPUDB_E_COMPILE, err);
        *out = new gpudb_module{cq};
        return GPUDB_OK;
    })
}

void gpudb_module_free(gpudb_module* m) { delete m; }

int gpudb_compile_check(const char* src, char* log, size_t cap, double* compile_ms) {
    if (!src) return GPUDB_E_INVALID;
    try {
        gpudb::CubinArtifact art;
        std::string err;
        const bool ok = gpudb::RuntimeCompiler::compileToCubin(src, art, err);
        copyOut(ok ? art.log : err, log, cap);
        if (compile_ms) *compile_ms = art.compileMs;
        return ok ? GPUDB_OK : GPUDB_E_COMPILE;
    } catch (const std::exception& e) {
        copyOut(e.what(), log, cap);
        return GPUDB_E_COMPILE;
    }
}

void gpudb_set_fast_math(int on) { gpudb::RuntimeCompiler::setFastMathEnabled(on != 0); }
void gpudb_set_kernel_cache_dir(const char* dir) { gpudb::RuntimeCompiler::setCacheDir(dir ? dir : ""); }

// ---------------------------------------------------------------------------
// registration
// ---------------------------------------------------------------------------
int gpudb_register_column(gpudb_ctx* ctx, const char* table, const char* column, const void* dptr, uint64_t rows,
                          int elem_bytes) {
    if (!ctx || !table || !column || (!dptr && rows) || elem_bytes <= 0) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    GPUDB_GUARD(ctx, {
        ctx->qc->ex.registerTableBuffer(column, dptr, rows, (size_t)elem_bytes);
        ctx->qc->ex.registerTableRowCount(table, rows);
        return GPUDB_OK;
    })
}

int gpudb_upload_column(gpudb_ctx* ctx, const char* table, const char* column, const void* host, uint64_t rows,
                        int elem_bytes) {
    if (!ctx || !table || !column || (!host && rows) || elem_bytes <= 0) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    try {
        ctx->qc->ex.uploadColumn(column, table, host, rows, (size_t)elem_bytes);
        return GPUDB_OK;
    } catch (const std::exception& e) {
        return fail(ctx, GPUDB_E_ALLOC, e.what());
    }
}

int gpudb_register_host_column(gpudb_ctx* ctx, const char* table, const char* column, const void* host,
                               uint64_t rows, int elem_bytes) {
    if (!ctx || !table || !column || (!host && rows) || elem_bytes <= 0) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    try {
        ctx->qc->ex.registerHostColumn(column, table, host, rows, (size_t)elem_bytes);
        return GPUDB_OK;
    } catch (const std::exception& e) {
        return fail(ctx, GPUDB_E_INVALID, e.what());
    }
}

int gpudb_sql_to_spec(const char* sql, char* spec, size_t cap) {
    if (!sql || (!spec && cap)) return fail(nullptr, GPUDB_E_INVALID, "bad argument");
    try {
        const std::string s = gpudb::sqlToSpec(sql);
        if (s.size() + 1 > cap) return fail(nullptr, GPUDB_E_INVALID, "spec buffer too small");
        std::memcpy(spec, s.c_str(), s.size() + 1);
        return GPUDB_OK;
    } catch (const std::exception& e) {
        return fail(nullptr, GPUDB_E_PLAN, e.what());
    }
}

int gpudb_colbin_inspect(const char* path, uint64_t* rows, uint32_t* ncols, gpudb_colbin_column* cols, uint32_t cap) {
    if (!path) return fail(nullptr, GPUDB_E_INVALID, "bad argument");
    try {
        gpudb::ColbinFile f(path);
        if (rows) *rows = f.rows();
        if (ncols) *ncols = (uint32_t)f.columns().size();
        for (uint32_t i = 0; cols && i < cap && i < (uint32_t)f.columns().size(); i++) {
            const auto& d = f.columns()[i];
            cols[i] = {d.columnIndex, d.dtype, d.fixedWidth, d.offset, d.sizeBytes};
        }
        return GPUDB_OK;
    } catch (const std::exception& e) {
        return fail(nullptr, GPUDB_E_INVALID, e.what());
    }
}

int gpudb_colbin_load(gpudb_ctx* ctx, const char* path, const char* table, const gpudb_colbin_load_spec* specs,
                      int n) {
    if (!ctx || !path || !table || (!specs && n) || n < 0) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    try {
        cudaSetDevice(ctx->qc->ex.device());
        gpudb::ColbinFile f(path);
        const gpudb::TableDef td = gpudb::catalogTable(table);  // a copy: no reference tied to the name temporary
        const uint64_t rows = f.rows();
        for (int k = 0; k < n; k++) {
            const auto& s = specs[k];
            if (!s.column) return fail(ctx, GPUDB_E_INVALID, "colbin: a load spec names no column");
            const gpudb::ColbinDesc& d = f.find(s.column_index);
            const size_t want = gpudb::cudaTypeBytes(td.col(s.column).cudaType);
            const std::string what = std::string("colbin: column ") + std::to_string(s.column_index) + " -> " +
                                     table + "." + s.column;
            const unsigned char* src = f.payload(d);
            std::vector<unsigned char> conv;
            size_t width = gpudb::ColbinFile::width(d);
            switch (s.transform) {
                case GPUDB_COLBIN_AS_IS:
                    if (d.dtype == 1 || d.dtype == 4 || width != want)
                        return fail(ctx, GPUDB_E_INVALID, what + ": stored type does not match the column as is");
                    break;
                case GPUDB_COLBIN_WIDEN: {
                    if ((d.dtype != 0 && d.dtype != 2) || want != 8)
                        return fail(ctx, GPUDB_E_INVALID, what + ": widening needs an int32 source and an int64 column");
                    conv.resize(rows * 8);
                    for (uint64_t i = 0; i < rows; i++) {
                        int32_t v;
                        std::memcpy(&v, src + i * 4, 4);
                        const int64_t w = v;
                        std::memcpy(conv.data() + i * 8, &w, 8);
                    }
                    width = 8;
                    break;
                }
                case GPUDB_COLBIN_DECIMAL: {
                    if (d.dtype != 1 || want != 8 || s.scale <= 0)
                        return fail(ctx, GPUDB_E_INVALID,
                                    what + ": decimals need a float32 source, an int64 column and a positive scale");
                    conv.resize(rows * 8);
                    for (uint64_t i = 0; i < rows; i++) {
                        float v;
                        std::memcpy(&v, src + i * 4, 4);
                        const int64_t w = std::llround((double)v * (double)s.scale);
                        std::memcpy(conv.data() + i * 8, &w, 8);
                    }
                    width = 8;
                    break;
                }
                case GPUDB_COLBIN_DAYS: {
                    if (d.dtype != 2 || want != 4)
                        return fail(ctx, GPUDB_E_INVALID, what + ": day numbers need a date source and an int32 column");
                    conv.resize(rows * 4);
                    for (uint64_t i = 0; i < rows; i++) {
                        int32_t v;
                        std::memcpy(&v, src + i * 4, 4);
                        const int32_t w = gpudb::colbinDayNumber(v);
                        std::memcpy(conv.data() + i * 4, &w, 4);
                    }
                    break;
                }
                default: return fail(ctx, GPUDB_E_INVALID, what + ": unknown transform");
            }
            ctx->qc->ex.uploadColumn(s.column, table, conv.empty() ? (const void*)src : conv.data(), rows, width);
            // the source (mapped file or converted copy) must outlive the copy
            const cudaError_t e = cudaStreamSynchronize(ctx->qc->ex.stream());
            if (e != cudaSuccess) return fail(ctx, GPUDB_E_CUDA, cudaGetErrorString(e));
        }
        return GPUDB_OK;
    } catch (const std::exception& e) {
        return fail(ctx, GPUDB_E_INVALID, e.what());
    }
}

int gpudb_register_rows(gpudb_ctx* ctx, const char* table, uint64_t rows) {
    if (!ctx || !table) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    ctx->qc->ex.registerTableRowCount(table, rows);
    return GPUDB_OK;
}

int gpudb_register_buffer(gpudb_ctx* ctx, const char* name, void* dptr, uint64_t bytes, int elem_bytes) {
    if (!ctx || !name || !dptr) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    ctx->qc->ex.registerAllocatedBuffer(name, dptr, bytes, elem_bytes > 0 ? (size_t)elem_bytes : 1);
    return GPUDB_OK;
}

int gpudb_register_symbol(gpudb_ctx* ctx, const char* name, uint64_t value) {
    if (!ctx || !name) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    ctx->qc->ex.registerSymbol(name, value);
    return GPUDB_OK;
}

int gpudb_get_symbol(gpudb_ctx* ctx, const char* name, uint64_t* value) {
    if (!ctx || !name || !value) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    return ctx->qc->ex.tryGetSymbol(name, *value) ? GPUDB_OK
                                                  : fail(ctx, GPUDB_E_INVALID, std::string("unknown symbol ") + name);
}

int gpudb_register_scalar_i64(gpudb_ctx* ctx, const char* name, long long value) {
    if (!ctx || !name) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    ctx->qc->ex.registerScalarInt(name, value);
    return GPUDB_OK;
}

int gpudb_register_scalar_f64(gpudb_ctx* ctx, const char* name, double value) {
    if (!ctx || !name) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    ctx->qc->ex.registerScalarFloat(name, value);
    return GPUDB_OK;
}

// ---------------------------------------------------------------------------
// execute
// ---------------------------------------------------------------------------
int gpudb_execute(gpudb_ctx* ctx, gpudb_module* m, const gpudb_phase_desc* phases, int nphases, int first, int last,
                  int warmup, int measured, gpudb_timing* timing) {
    if (!ctx || !m || !phases || nphases <= 0) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    GPUDB_GUARD(ctx, {
        std::vector<gpudb::CudaCodegen::PhaseInfo> ph(nphases);
        for (int i = 0; i < nphases; i++) {
            const auto& d = phases[i];
            auto& p = ph[i];
            if (!d.name) return fail(ctx, GPUDB_E_INVALID, "phase without a name");
            p.name = d.name;
            p.scannedTable = d.scanned_table ? d.scanned_table : "";
            p.threadgroupSize = d.block_size > 0 ? d.block_size : 256;
            p.maxThreadgroups = d.max_blocks;
            p.isSingleThread = d.single_thread != 0;
            p.dynamicSmemBytes = d.dynamic_smem_bytes;
            p.tileRows = d.tile_rows;
            p.rowsPerThread = d.rows_per_thread > 0 ? d.rows_per_thread : 1;
            for (int k = 0; k < d.nbindings; k++) {
                const auto& bd = d.bindings[k];
                if (!bd.name || bd.kind < 0 || bd.kind > GPUDB_PARAM_BUFFER_LENGTH)
                    return fail(ctx, GPUDB_E_INVALID, "bad binding in phase " + p.name);
                gpudb::CudaParamBinding b;
                b.name = bd.name;
                b.kind = (gpudb::CudaParamKind)bd.kind;
                b.elementType = bd.elem_type ? bd.elem_type : "unsigned";
                b.tableName = bd.table ? bd.table : "";
                b.sizeExpr = bd.size_expr ? bd.size_expr : "";
                b.zeroInit = bd.zero_init != 0;
                b.fillByte = bd.fill_byte;
                b.readOnly = bd.read_only != 0;
                b.argIndex = k;
                p.bindings.push_back(b);
            }
        }
        gpudb::ExecutionResult r;
        std::string err;
        const int rc = ctx->qc->ex.execute(*m->cq, ph, warmup, measured, first, last, r, err);
        fillTiming(r, timing);
        if (rc != 0) return fail(ctx, mapStatus(rc), err);
        if (r.deviceError) return fail(ctx, GPUDB_E_DEVICE, "device error word set");
        return GPUDB_OK;
    })
}

int gpudb_set_skip_zero_init(gpudb_ctx* ctx, int skip) {
    if (!ctx) return GPUDB_E_INVALID;
    ctx->qc->ex.setSkipZeroInit(skip != 0);
    return GPUDB_OK;
}

int gpudb_set_use_graphs(gpudb_ctx* ctx, int on) {
    if (!ctx) return GPUDB_E_INVALID;
    ctx->qc->ex.setUseGraphs(on != 0);
    return GPUDB_OK;
}

int gpudb_read_buffer(gpudb_ctx* ctx, const char* name, void* host, uint64_t bytes) {
    if (!ctx || !name || (!host && bytes)) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    return ctx->qc->ex.readBuffer(name, host, bytes) ? GPUDB_OK
                                                     : fail(ctx, GPUDB_E_INVALID, std::string("cannot read buffer ") + name);
}

int gpudb_buffer_ptr(gpudb_ctx* ctx, const char* name, void** dptr, uint64_t* bytes) {
    if (!ctx || !name || !dptr) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    size_t b = 0;
    *dptr = ctx->qc->ex.bufferPtr(name, &b);
    if (bytes) *bytes = b;
    return *dptr ? GPUDB_OK : fail(ctx, GPUDB_E_INVALID, std::string("unknown buffer ") + name);
}

int gpudb_release_buffers(gpudb_ctx* ctx) {
    if (!ctx) return GPUDB_E_INVALID;
    ctx->qc->ex.releaseAllocatedBuffers();
    return GPUDB_OK;
}

void* gpudb_host_alloc(uint64_t bytes) {
    void* p = nullptr;
    if (cudaHostAlloc(&p, bytes ? bytes : 1, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void gpudb_host_free(void* p) {
    if (p) cudaFreeHost(p);
}

// ---------------------------------------------------------------------------
// queries
// ---------------------------------------------------------------------------
int gpudb_query_prepare(gpudb_ctx* ctx, const char* spec, const char* tune, gpudb_query** out) {
    if (!spec || !out) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    *out = nullptr;
    try {
        if (ctx) cudaSetDevice(ctx->qc->ex.device());
        auto q = gpudb::prepareQuery(spec, tune ? tune : "", true, ctx != nullptr);
        *out = new gpudb_query{q};
        return GPUDB_OK;
    } catch (const std::exception& e) {
        const std::string m = e.what();
        const bool compile = m.find("NVRTC") != std::string::npos || m.find("cuModule") != std::string::npos;
        return fail(ctx, compile ? GPUDB_E_COMPILE : GPUDB_E_PLAN, m);
    }
}

void gpudb_query_free(gpudb_query* q) { delete q; }

size_t gpudb_query_source(gpudb_query* q, char* buf, size_t cap) { return q ? copyOut(q->q->source, buf, cap) : 0; }
size_t gpudb_query_describe(gpudb_query* q, char* buf, size_t cap) { return q ? copyOut(q->q->describe, buf, cap) : 0; }
size_t gpudb_query_compile_log(gpudb_query* q, char* buf, size_t cap) {
    return q ? copyOut(q->q->compileLog, buf, cap) : 0;
}

int gpudb_query_algorithmic_bytes(gpudb_ctx* ctx, gpudb_query* q, long long* bytes) {
    if (!ctx || !q || !bytes) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    GPUDB_GUARD(ctx, {
        std::map<std::string, long long> rows;
        for (const auto& t : q->q->plan.tables) rows[t] = (long long)ctx->qc->ex.tableRows(t);
        *bytes = gpudb::planAlgorithmicBytes(q->q->plan, rows);
        return GPUDB_OK;
    })
}

int gpudb_query_run(gpudb_ctx* ctx, gpudb_query* q, int warmup, int measured, gpudb_result** result,
                    gpudb_timing* timing) {
    if (!ctx || !q) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    if (result) *result = nullptr;
    GPUDB_GUARD(ctx, {
        cudaSetDevice(ctx->qc->ex.device());
        gpudb::ExecutionResult r;
        std::string err;
        ctx->qc->ex.setSkipZeroInit(false);
        const int rc = gpudb::runQuery(*ctx->qc, *q->q, warmup, measured, result != nullptr, r, err);
        fillTiming(r, timing);
        if (rc != 0) return fail(ctx, mapStatus(rc), err);
        if (result) *result = new gpudb_result{std::move(r.result)};
        return GPUDB_OK;
    })
}

int gpudb_query_run_streamed(gpudb_ctx* ctx, gpudb_query* q, const char* table, const gpudb_stream_column* cols,
                             int ncols, uint64_t rows, uint64_t chunk_rows, gpudb_result** result,
                             gpudb_timing* timing) {
    if (!ctx || !q || !table || ncols < 0 || (ncols && !cols) || chunk_rows == 0)
        return fail(ctx, GPUDB_E_INVALID, "bad argument");
    if (result) *result = nullptr;
    std::vector<gpudb::StreamColumn> sc;
    for (int i = 0; i < ncols; i++) {
        if (!cols[i].column || (!cols[i].host && rows) || cols[i].elem_bytes <= 0)
            return fail(ctx, GPUDB_E_INVALID, "bad stream column");
        sc.push_back({cols[i].column, cols[i].host, (size_t)cols[i].elem_bytes, cols[i].in_place != 0});
    }
    GPUDB_GUARD(ctx, {
        cudaSetDevice(ctx->qc->ex.device());
        gpudb::ExecutionResult r;
        std::string err;
        ctx->qc->ex.setSkipZeroInit(false);
        const int rc = gpudb::runStreamed(*ctx->qc, *q->q, table, sc, rows, chunk_rows, result != nullptr, r, err);
        fillTiming(r, timing);
        if (rc != 0) return fail(ctx, mapStatus(rc), err);
        if (result) *result = new gpudb_result{std::move(r.result)};
        return GPUDB_OK;
    })
}

int gpudb_query_collect(gpudb_ctx* ctx, gpudb_query* q, gpudb_result** result) {
    if (!ctx || !q || !result) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    *result = nullptr;
    GPUDB_GUARD(ctx, {
        cudaSetDevice(ctx->qc->ex.device());
        if (!q->q->compiled) return fail(ctx, GPUDB_E_INVALID, "the query has not run in this context");
        if (cudaStreamSynchronize(static_cast<cudaStream_t>(ctx->qc->ex.stream())) != cudaSuccess)
            return fail(ctx, GPUDB_E_CUDA, "stream synchronize failed");
        *result = new gpudb_result{ctx->qc->ex.collectResult(q->q->cg.getResultSchema())};
        return GPUDB_OK;
    })
}

int gpudb_query_enqueue(gpudb_ctx* ctx, gpudb_query* q) {
    if (!ctx || !q) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    GPUDB_GUARD(ctx, {
        cudaSetDevice(ctx->qc->ex.device());
        gpudb::ExecutionResult r;
        std::string err;
        ctx->qc->ex.setSkipZeroInit(false);
        struct Deferred {
            gpudb::CudaGenericExecutor& ex;
            explicit Deferred(gpudb::CudaGenericExecutor& e) : ex(e) { ex.setDeferSync(true); }
            ~Deferred() { ex.setDeferSync(false); }
        } deferred(ctx->qc->ex);
        const int rc = gpudb::runQuery(*ctx->qc, *q->q, 1, 0, false, r, err);
        if (rc != 0) return fail(ctx, mapStatus(rc), err);
        return GPUDB_OK;
    })
}

int gpudb_ctx_sync(gpudb_ctx* ctx, unsigned* device_error) {
    if (!ctx) return GPUDB_E_INVALID;
    if (device_error) *device_error = 0;
    GPUDB_GUARD(ctx, {
        cudaSetDevice(ctx->qc->ex.device());
        unsigned bits = 0;
        std::string err;
        if (!ctx->qc->ex.syncErrors(bits, err)) return fail(ctx, GPUDB_E_CUDA, err);
        if (device_error) *device_error = bits;
        if (bits) {
            char b[64];
            snprintf(b, sizeof b, "device error word 0x%x", bits);
            return fail(ctx, GPUDB_E_DEVICE, b);
        }
        return GPUDB_OK;
    })
}

// ---------------------------------------------------------------------------
// results
// ---------------------------------------------------------------------------
int gpudb_result_shape(gpudb_result* r, int* ncols, long long* nrows) {
    if (!r) return GPUDB_E_INVALID;
    if (ncols) *ncols = (int)r->r.columns.size();
    if (nrows) *nrows = (long long)r->r.rows.size();
    return GPUDB_OK;
}

int gpudb_result_column(gpudb_result* r, int col, char* name, size_t cap, int* type) {
    if (!r || col < 0 || col >= (int)r->r.columns.size()) return GPUDB_E_INVALID;
    copyOut(r->r.columns[col].name, name, cap);
    if (type) {
        const auto& t = r->r.columns[col].type;
        *type = t == "int" ? GPUDB_COL_INT : t == "double" ? GPUDB_COL_DOUBLE : GPUDB_COL_STRING;
    }
    return GPUDB_OK;
}

int gpudb_result_get_int(gpudb_result* r, long long row, int col, int64_t* lo, int64_t* hi) {
    if (!r || row < 0 || row >= (long long)r->r.rows.size() || col < 0 || col >= (int)r->r.rows[row].size())
        return GPUDB_E_INVALID;
    const auto* v = std::get_if<gpudb::int128>(&r->r.rows[row][col]);
    if (!v) return GPUDB_E_INVALID;
    if (lo) *lo = (int64_t)(unsigned long long)(*v);
    if (hi) *hi = (int64_t)(*v >> 64);
    return GPUDB_OK;
}

int gpudb_result_get_f64(gpudb_result* r, long long row, int col, double* out) {
    if (!r || row < 0 || row >= (long long)r->r.rows.size() || col < 0 || col >= (int)r->r.rows[row].size())
        return GPUDB_E_INVALID;
    const auto* v = std::get_if<double>(&r->r.rows[row][col]);
    if (!v) return GPUDB_E_INVALID;
    if (out) *out = *v;
    return GPUDB_OK;
}

size_t gpudb_result_get_str(gpudb_result* r, long long row, int col, char* buf, size_t cap) {
    if (!r || row < 0 || row >= (long long)r->r.rows.size() || col < 0 || col >= (int)r->r.rows[row].size()) return 0;
    const auto* v = std::get_if<std::string>(&r->r.rows[row][col]);
    return v ? copyOut(*v, buf, cap) : 0;
}

int gpudb_result_export_i64(gpudb_result* r, int col, int64_t* out, long long n) {
    if (!r || !out || col < 0 || col >= (int)r->r.columns.size() || n < (long long)r->r.rows.size())
        return GPUDB_E_INVALID;
    for (size_t i = 0; i < r->r.rows.size(); i++) {
        const auto* v = std::get_if<gpudb::int128>(&r->r.rows[i][col]);
        if (!v || *v > (gpudb::int128)INT64_MAX || *v < (gpudb::int128)INT64_MIN) return GPUDB_E_INVALID;
        out[i] = (int64_t)*v;
    }
    return GPUDB_OK;
}

size_t gpudb_result_canonical(gpudb_result* r, int exact, char* buf, size_t cap) {
    if (!r) return 0;
    return copyOut(exact ? r->r.toExact() : r->r.toCanonical(), buf, cap);
}

void gpudb_result_free(gpudb_result* r) { delete r; }

int gpudb_compare_canonical(const char* got, const char* expected, double abs_tol, double rel_tol, char* buf,
                            size_t cap) {
    if (!got || !expected) return 0;
    const std::string why = gpudb::compareCanonical(got, expected, abs_tol, rel_tol);
    copyOut(why, buf, cap);
    return why.empty() ? 1 : 0;
}

int gpudb_register_max_key(gpudb_ctx* ctx, const char* column, long long* max_out) {
    if (!ctx || !column) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    GPUDB_GUARD(ctx, {
        const long long m = gpudb::registerMaxKey(*ctx->qc, column);
        if (max_out) *max_out = m;
        return GPUDB_OK;
    })
}

size_t gpudb_list_templates(char* buf, size_t cap) {
    std::string s;
    for (const auto& t : gpudb::planTemplates()) s += (s.empty() ? "" : ",") + t;
    return copyOut(s, buf, cap);
}

const char* gpudb_version(void) { return "gpudb-b200 0.1 (sm_100a, NVRTC)"; }

}  // extern "C"

// ===================================================================
// analyzed queries
// ===================================================================
namespace {
using namespace gpudb::ir;
bool okExpr(const gpudb_aq* aq, const gpudb_expr* e) { return aq && e && aq->owns(e); }
bool okPred(const gpudb_aq* aq, const gpudb_pred* p) { return aq && p && aq->owns(p); }
}  // namespace

extern "C" {

int gpudb_aq_create(gpudb_aq** out) {
    if (!out) return GPUDB_E_INVALID;
    *out = new gpudb_aq();
    return GPUDB_OK;
}

void gpudb_aq_free(gpudb_aq* aq) { delete aq; }

gpudb_expr* gpudb_aq_col(gpudb_aq* aq, const char* table, const char* column) {
    if (!aq || !column) return nullptr;
    return aq->add(Expr::col(table ? table : "", column));
}
gpudb_expr* gpudb_aq_lit_int(gpudb_aq* aq, int64_t v) { return aq ? aq->add(Expr::lit((long long)v)) : nullptr; }
gpudb_expr* gpudb_aq_lit_decimal(gpudb_aq* aq, double v) { return aq ? aq->add(Expr::litf(v)) : nullptr; }
gpudb_expr* gpudb_aq_lit_str(gpudb_aq* aq, const char* v) { return aq && v ? aq->add(Expr::lits(v)) : nullptr; }
gpudb_expr* gpudb_aq_binary(gpudb_aq* aq, int op, gpudb_expr* l, gpudb_expr* r) {
    if (!okExpr(aq, l) || !okExpr(aq, r) || op < GPUDB_EXPR_ADD || op > GPUDB_EXPR_DIV) return nullptr;
    return aq->add(Expr::binary((ExprOp)op, l->e, r->e));
}
gpudb_pred* gpudb_aq_cmp(gpudb_aq* aq, int op, gpudb_expr* l, gpudb_expr* r) {
    if (!okExpr(aq, l) || !okExpr(aq, r) || op < GPUDB_CMP_EQ || op > GPUDB_CMP_GE) return nullptr;
    return aq->add(Predicate::cmp((CmpOp)op, l->e, r->e));
}
gpudb_pred* gpudb_aq_between(gpudb_aq* aq, gpudb_expr* e, gpudb_expr* lo, gpudb_expr* hi) {
    if (!okExpr(aq, e) || !okExpr(aq, lo) || !okExpr(aq, hi)) return nullptr;
    return aq->add(Predicate::between(e->e, lo->e, hi->e));
}
gpudb_pred* gpudb_aq_in_list(gpudb_aq* aq, gpudb_expr* e, gpudb_expr* const* values, int n) {
    if (!okExpr(aq, e) || n < 0 || (n && !values)) return nullptr;
    std::vector<ExprPtr> v;
    for (int i = 0; i < n; i++) {
        if (!okExpr(aq, values[i])) return nullptr;
        v.push_back(values[i]->e);
    }
    return aq->add(Predicate::inList(e->e, std::move(v)));
}
static gpudb_pred* logical(gpudb_aq* aq, gpudb_pred* const* ch, int n, bool isAnd) {
    if (!aq || n < 0 || (n && !ch)) return nullptr;
    std::vector<PredPtr> v;
    for (int i = 0; i < n; i++) {
        if (!okPred(aq, ch[i])) return nullptr;
        v.push_back(ch[i]->p);
    }
    return aq->add(isAnd ? Predicate::logAnd(std::move(v)) : Predicate::logOr(std::move(v)));
}
gpudb_pred* gpudb_aq_and(gpudb_aq* aq, gpudb_pred* const* children, int n) { return logical(aq, children, n, true); }
gpudb_pred* gpudb_aq_or(gpudb_aq* aq, gpudb_pred* const* children, int n) { return logical(aq, children, n, false); }
gpudb_pred* gpudb_aq_not(gpudb_aq* aq, gpudb_pred* child) {
    return okPred(aq, child) ? aq->add(Predicate::logNot(child->p)) : nullptr;
}

int gpudb_aq_add_table(gpudb_aq* aq, const char* table) {
    if (!aq || !table) return GPUDB_E_INVALID;
    aq->q.tables.push_back(table);
    return GPUDB_OK;
}
int gpudb_aq_add_join(gpudb_aq* aq, const char* lt, const char* lc, const char* rt, const char* rc) {
    if (!aq || !lt || !lc || !rt || !rc) return GPUDB_E_INVALID;
    aq->q.joins.push_back({lt, rt, lc, rc});
    return GPUDB_OK;
}
int gpudb_aq_add_filter(gpudb_aq* aq, gpudb_pred* p) {
    if (!okPred(aq, p)) return GPUDB_E_INVALID;
    aq->q.filters.push_back(p->p);
    return GPUDB_OK;
}
int gpudb_aq_add_target(gpudb_aq* aq, gpudb_expr* e, const char* alias) {
    if (!okExpr(aq, e)) return GPUDB_E_INVALID;
    SelectTarget t;
    t.expr = e->e;
    t.alias = alias ? alias : "";
    aq->q.targets.push_back(t);
    return GPUDB_OK;
}
int gpudb_aq_add_agg(gpudb_aq* aq, int func, gpudb_expr* e, const char* alias) {
    if (!aq || func < GPUDB_AGGF_SUM || func > GPUDB_AGGF_MAX || (e && !aq->owns(e))) return GPUDB_E_INVALID;
    if (!e && func != GPUDB_AGGF_COUNT) return GPUDB_E_INVALID;
    SelectTarget t;
    t.isAgg = true;
    t.alias = alias ? alias : "";
    AggTarget a;
    a.func = (AggFunc)func;
    a.innerExpr = e ? e->e : nullptr;
    a.alias = t.alias;
    a.isStar = e == nullptr;
    t.agg = a;
    t.expr = a.innerExpr;
    aq->q.targets.push_back(t);
    return GPUDB_OK;
}
int gpudb_aq_add_group_by(gpudb_aq* aq, gpudb_expr* e) {
    if (!okExpr(aq, e)) return GPUDB_E_INVALID;
    aq->q.groupBy.push_back(e->e);
    return GPUDB_OK;
}
int gpudb_aq_add_order_by(gpudb_aq* aq, gpudb_expr* e, int descending) {
    if (!okExpr(aq, e)) return GPUDB_E_INVALID;
    aq->q.orderBy.push_back({e->e, descending != 0});
    return GPUDB_OK;
}
int gpudb_aq_set_limit(gpudb_aq* aq, int limit) {
    if (!aq || limit < -1) return GPUDB_E_INVALID;
    aq->q.limit = limit;
    return GPUDB_OK;
}

int gpudb_aq_lower_expr(gpudb_expr* e, char* code, size_t cap, int* scale) {
    if (!e) return GPUDB_E_INVALID;
    try {
        const Lowered l = exprToCuda(e->e, "i");
        copyOut(l.code, code, cap);
        if (scale) *scale = l.scale;
        return GPUDB_OK;
    } catch (const std::exception& ex) {
        return fail(nullptr, GPUDB_E_PLAN, ex.what());
    }
}

int gpudb_aq_lower_pred(gpudb_pred* p, char* code, size_t cap) {
    if (!p) return GPUDB_E_INVALID;
    try {
        copyOut(predToCuda(p->p, "i"), code, cap);
        return GPUDB_OK;
    } catch (const std::exception& ex) {
        return fail(nullptr, GPUDB_E_PLAN, ex.what());
    }
}

int gpudb_query_prepare_analyzed(gpudb_ctx* ctx, const gpudb_aq* aq, const char* name, const char* tune,
                                 gpudb_query** out) {
    if (!aq || !out) return fail(ctx, GPUDB_E_INVALID, "bad argument");
    *out = nullptr;
    try {
        if (ctx) cudaSetDevice(ctx->qc->ex.device());
        auto t0 = std::chrono::steady_clock::now();
        const gpudb::TuneConfig tc = gpudb::TuneConfig::parse(tune ? tune : "");
        gpudb::CudaQueryPlan plan = gpudb::buildCudaPlan(aq->q, name ? name : "", tc);
        const double planMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        *out = new gpudb_query{gpudb::prepareFromPlan(std::move(plan), tc, planMs, true, ctx != nullptr)};
        return GPUDB_OK;
    } catch (const std::exception& e) {
        const std::string m = e.what();
        const bool compile = m.find("NVRTC") != std::string::npos || m.find("cuModule") != std::string::npos;
        return fail(ctx, compile ? GPUDB_E_COMPILE : GPUDB_E_PLAN, m);
    }
}

}  // extern "C"
