/*
 * gpudb_engine.h — C-ABI of the query layer above the runtime.
 *
 * What the reference's driver does per query (codegen/codegen_main.cpp:
 * runCodegenQuery :271-1776): plan -> generate source -> compile -> size
 * (max-key pass, exact counts) -> execute -> collect -> post-process. Here
 * the plan comes from an analyzed query (the reference's planning input,
 * built through the gpudb_aq_* functions below), from a `key=value;...`
 * spec naming a pipeline template, or from SQL through the engine's own
 * front end; the generated language is CUDA C++ for sm_100a.
 */
#ifndef GPUDB_ENGINE_H
#define GPUDB_ENGINE_H

#include "gpudb_rt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gpudb_query gpudb_query;
typedef struct gpudb_result gpudb_result;

/* Result column types. */
#define GPUDB_COL_INT 0     /* exact integer (read as int128 lo/hi)   */
#define GPUDB_COL_DOUBLE 1  /* FP64 derived column                    */
#define GPUDB_COL_STRING 2

/* Plan + generate + compile (reference: buildMetalPlan,
 * planning/metal_plan_builder.h:73, .cpp:2035; generateFromPlan :78,
 * .cpp:2115; RuntimeCompiler::compile). `tune` (may be NULL) selects block
 * size, scan mode, hash layout, ... ("bs=512;scan=tma;tile=1024;..."). With
 * ctx == NULL the query is planned and compiled but not loaded (no GPU
 * needed). */
int gpudb_query_prepare(gpudb_ctx* ctx, const char* spec, const char* tune, gpudb_query** out);
void gpudb_query_free(gpudb_query* q);
/* The generated CUDA source (reference --dump-msl, codegen_main.cpp:343-380). */
size_t gpudb_query_source(gpudb_query* q, char* buf, size_t cap);
/* Plan / phase / binding description (reference --print-plan). */
size_t gpudb_query_describe(gpudb_query* q, char* buf, size_t cap);
/* NVRTC log of the compile (ptxas resource usage per kernel). */
size_t gpudb_query_compile_log(gpudb_query* q, char* buf, size_t cap);
/* Algorithmic bytes of one execution given the registered row counts. */
int gpudb_query_algorithmic_bytes(gpudb_ctx* ctx, gpudb_query* q, long long* bytes);

/* Execute (sizing passes included) and collect the result
 * (reference: MetalGenericExecutor::execute + MetalResultCollector::collect).
 * `result` may be NULL to skip collection. Returns GPUDB_E_DEVICE when a
 * kernel raised a device error bit (timing->device_error tells which);
 * the result is not collected then. */
int gpudb_query_run(gpudb_ctx* ctx, gpudb_query* q, int warmup, int measured, gpudb_result** result,
                    gpudb_timing* timing);

/* Chunked streaming execution from host memory (reference: the chunked
 * path of runCodegenQuery, codegen/codegen_main.cpp:686-808, with
 * ChunkedColbinTable::loadChunk, registerTableBuffer,
 * registerTableRowCount and setSkipZeroInit per chunk). The phases before
 * the first one that scans `table` run once; the phases that scan it run
 * once per chunk of `chunk_rows` rows and accumulate (zero fills on the
 * first chunk only); the remaining phases run once after the last chunk.
 * Copied columns move host -> device on a copy stream into a ring of three
 * device chunk buffers while earlier chunks are scanned, so the copies
 * overlap the kernels; in-place columns (pinned, mapped memory) are read
 * over the host link by late-materialised bindings. Size expressions see
 * all `rows` rows. No phase outside the streamed ones may read `table`
 * (stream the unsplit join plan, split=0), and no counter-driven sizing
 * step may depend on the streamed phases (GPUDB_E_PLAN otherwise). The
 * streamed columns are unregistered when the call returns. Timing covers
 * the phases outside the stream. */
typedef struct gpudb_stream_column {
    const char* column; /* a column of `table` read by the streamed phases */
    const void* host;   /* its row 0, in pinned host memory (gpudb_host_alloc) */
    int32_t elem_bytes;
    int32_t in_place;   /* 1: read in place over the host link; 0: copied per chunk */
} gpudb_stream_column;
int gpudb_query_run_streamed(gpudb_ctx* ctx, gpudb_query* q, const char* table, const gpudb_stream_column* cols,
                             int ncols, uint64_t rows, uint64_t chunk_rows, gpudb_result** result,
                             gpudb_timing* timing);

/* Enqueue one execution on the context's stream and return without
 * waiting for it: no timing, no collection. Sizing passes that need a
 * host round trip still wait at their counter reads; a plan without them
 * runs as one stream-ordered launch (a CUDA graph replay when graphs are
 * on), so consecutive enqueues keep the GPU busy back to back. Device
 * errors accumulate until gpudb_ctx_sync (or the next gpudb_query_run)
 * reads them. The reference runs one blocking execution per invocation
 * (MetalGenericExecutor::execute); this is the pipelined form of it. */
int gpudb_query_enqueue(gpudb_ctx* ctx, gpudb_query* q);
/* Collect the result the last execution of `q` left in the context's
 * buffers (after gpudb_ctx_sync for enqueued runs), without executing:
 * e.g. the answer of the last of many back-to-back graph replays
 * (reference: MetalGenericExecutor::collectResult,
 * metal_generic_executor.h:110). The buffers must not have been reused by
 * another query since. */
int gpudb_query_collect(gpudb_ctx* ctx, gpudb_query* q, gpudb_result** result);
/* Wait for everything enqueued on the context's stream; *device_error
 * (may be NULL) receives the accumulated device error bits, which are
 * then cleared. Returns GPUDB_E_DEVICE when any bit was set. */
int gpudb_ctx_sync(gpudb_ctx* ctx, unsigned* device_error);

/* ---- results (reference: GenericResult, metal_result_collector.h:19-38) */
int gpudb_result_shape(gpudb_result* r, int* ncols, long long* nrows);
int gpudb_result_column(gpudb_result* r, int col, char* name, size_t cap, int* type);
/* Integer cell as a two's-complement 128-bit value (lo, hi words). */
int gpudb_result_get_int(gpudb_result* r, long long row, int col, int64_t* lo, int64_t* hi);
int gpudb_result_get_f64(gpudb_result* r, long long row, int col, double* v);
size_t gpudb_result_get_str(gpudb_result* r, long long row, int col, char* buf, size_t cap);
/* Whole integer column as int64 (fails with GPUDB_E_INVALID if a value
 * does not fit). */
int gpudb_result_export_i64(gpudb_result* r, int col, int64_t* out, long long n);
/* GenericResult::toCanonical (%.4f doubles) / full-precision variant. */
size_t gpudb_result_canonical(gpudb_result* r, int exact, char* buf, size_t cap);
void gpudb_result_free(gpudb_result* r);

/* Golden comparison (reference: compareCanonical, codegen_main.cpp:63-188).
 * Returns 1 on match, 0 on mismatch (reason copied to buf). */
int gpudb_compare_canonical(const char* got, const char* expected, double abs_tol, double rel_tol, char* buf,
                            size_t cap);

/* Exact max of a registered integer column (reference: the max-key sizing
 * pass registerMaxKeySymbols, execution/max_key_symbols.cpp:188-235), run
 * on the GPU and registered as symbol "max_<column>". Cached per
 * (column pointer, rows) like the reference's .maxkeys.json cache. */
int gpudb_register_max_key(gpudb_ctx* ctx, const char* column, long long* max_out);

/* SQL front end (reference: query_analyzer.cpp:640-727 over libpg_query,
 * then buildMetalPlan by query shape). Maps a SELECT over the engine's
 * tables to the spec string of the pipeline template that computes it
 * (Q1 / Q6 shapes over fact, the dim-probe semi-join grouped with ORDER BY
 * revenue DESC LIMIT k or as rows, the zprobe group-by, the zbuild-zprobe
 * hash join); constants are integers in the columns' own units. No GPU
 * needed. Copies the NUL-terminated spec into `spec` (up to `cap` bytes)
 * and returns GPUDB_OK, or GPUDB_E_PLAN with the reason in
 * gpudb_last_error(NULL, ...). */
int gpudb_sql_to_spec(const char* sql, char* spec, size_t cap);

/* ---- analyzed queries: the planning layer's input ----------------------
 * The reference plans from an AnalyzedQuery (codegen/planning/query_plan.h:
 * 14-183: Expr / Predicate / AggSpec; query_analyzer.h:14-81: joins, select
 * targets, GROUP BY / ORDER BY / LIMIT) with buildMetalPlan(aq, name)
 * (planning/metal_plan_builder.h:73, .cpp:2035-2109). A caller holding one
 * rebuilds it node for node through these functions and plans it with
 * gpudb_query_prepare_analyzed. Tables and columns are the engine's
 * catalog names, or lineitem's TPC-H names for the fact table. Decimal
 * literals (e.g. 0.05) are converted exactly to the columns' fixed point.
 * Nodes belong to their gpudb_aq and live until gpudb_aq_free; a builder
 * given a NULL or foreign node returns NULL / GPUDB_E_INVALID. */
typedef struct gpudb_aq gpudb_aq;
typedef struct gpudb_expr gpudb_expr;
typedef struct gpudb_pred gpudb_pred;

/* ExprOp (query_plan.h:25) */
#define GPUDB_EXPR_ADD 0
#define GPUDB_EXPR_SUB 1
#define GPUDB_EXPR_MUL 2
#define GPUDB_EXPR_DIV 3
/* CmpOp (query_plan.h:27) */
#define GPUDB_CMP_EQ 0
#define GPUDB_CMP_NE 1
#define GPUDB_CMP_LT 2
#define GPUDB_CMP_LE 3
#define GPUDB_CMP_GT 4
#define GPUDB_CMP_GE 5
/* AggFunc (query_plan.h:26) */
#define GPUDB_AGGF_SUM 0
#define GPUDB_AGGF_COUNT 1
#define GPUDB_AGGF_AVG 2
#define GPUDB_AGGF_MIN 3
#define GPUDB_AGGF_MAX 4

int gpudb_aq_create(gpudb_aq** out);
void gpudb_aq_free(gpudb_aq* aq);
/* Expr::col / lit / litf / lits / binary (query_plan.h:60-90). A column
 * with table "" refers to a select target's alias (ORDER BY revenue). */
gpudb_expr* gpudb_aq_col(gpudb_aq* aq, const char* table, const char* column);
gpudb_expr* gpudb_aq_lit_int(gpudb_aq* aq, int64_t v);
gpudb_expr* gpudb_aq_lit_decimal(gpudb_aq* aq, double v);
gpudb_expr* gpudb_aq_lit_str(gpudb_aq* aq, const char* v);
gpudb_expr* gpudb_aq_binary(gpudb_aq* aq, int op, gpudb_expr* l, gpudb_expr* r);
/* Predicate::cmp / between / inList / logAnd / logOr / logNot (:130-160). */
gpudb_pred* gpudb_aq_cmp(gpudb_aq* aq, int op, gpudb_expr* l, gpudb_expr* r);
gpudb_pred* gpudb_aq_between(gpudb_aq* aq, gpudb_expr* e, gpudb_expr* lo, gpudb_expr* hi);
gpudb_pred* gpudb_aq_in_list(gpudb_aq* aq, gpudb_expr* e, gpudb_expr* const* values, int n);
gpudb_pred* gpudb_aq_and(gpudb_aq* aq, gpudb_pred* const* children, int n);
gpudb_pred* gpudb_aq_or(gpudb_aq* aq, gpudb_pred* const* children, int n);
gpudb_pred* gpudb_aq_not(gpudb_aq* aq, gpudb_pred* child);
/* AnalyzedQuery fields (query_analyzer.h:38-81). */
int gpudb_aq_add_table(gpudb_aq* aq, const char* table);
int gpudb_aq_add_join(gpudb_aq* aq, const char* left_table, const char* left_col, const char* right_table,
                      const char* right_col);
int gpudb_aq_add_filter(gpudb_aq* aq, gpudb_pred* p);
/* A plain select target (a GROUP BY column). */
int gpudb_aq_add_target(gpudb_aq* aq, gpudb_expr* e, const char* alias);
/* An aggregate target (SelectTarget with AggTarget); e = NULL is COUNT(*). */
int gpudb_aq_add_agg(gpudb_aq* aq, int func, gpudb_expr* e, const char* alias);
int gpudb_aq_add_group_by(gpudb_aq* aq, gpudb_expr* e);
int gpudb_aq_add_order_by(gpudb_aq* aq, gpudb_expr* e, int descending);
int gpudb_aq_set_limit(gpudb_aq* aq, int limit);
/* The kernel expressions an expression / predicate lowers to, with the
 * decimal scale of the expression's value (for callers that print or
 * check the lowering; no GPU needed). */
int gpudb_aq_lower_expr(gpudb_expr* e, char* code, size_t cap, int* scale);
int gpudb_aq_lower_pred(gpudb_pred* p, char* code, size_t cap);
/* Plan + generate + compile an analyzed query (reference: buildMetalPlan
 * (aq, name) then generateFromPlan and RuntimeCompiler::compile). `name`
 * (may be NULL) names the plan and its kernels; `tune` as for
 * gpudb_query_prepare; ctx == NULL plans and compiles without loading.
 * GPUDB_E_PLAN with the reason when the analysis has no plan here. */
int gpudb_query_prepare_analyzed(gpudb_ctx* ctx, const gpudb_aq* aq, const char* name, const char* tune,
                                 gpudb_query** out);

/* Template names understood by gpudb_query_prepare, comma separated. */
size_t gpudb_list_templates(char* buf, size_t cap);
/* Library version / build string. */
const char* gpudb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* GPUDB_ENGINE_H */
