/*
 * gpudb_engine.h — C-ABI of the query layer above the runtime.
 *
 * What the reference's driver does per query (codegen/codegen_main.cpp:
 * runCodegenQuery :271-1776): plan -> generate source -> compile -> size
 * (max-key pass, exact counts) -> execute -> collect -> post-process. Here
 * the plan comes from a `key=value;...` spec naming a pipeline template
 * (the SQL front end of the reference is out of scope) and the generated
 * language is CUDA C++ for sm_100a.
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

/* Enqueue one execution on the context's stream and return without
 * waiting for it: no timing, no collection. Sizing passes that need a
 * host round trip still wait at their counter reads; a plan without them
 * runs as one stream-ordered launch (a CUDA graph replay when graphs are
 * on), so consecutive enqueues keep the GPU busy back to back. Device
 * errors accumulate until gpudb_ctx_sync (or the next gpudb_query_run)
 * reads them. The reference runs one blocking execution per invocation
 * (MetalGenericExecutor::execute); this is the pipelined form of it. */
int gpudb_query_enqueue(gpudb_ctx* ctx, gpudb_query* q);
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

/* Template names understood by gpudb_query_prepare, comma separated. */
size_t gpudb_list_templates(char* buf, size_t cap);
/* Library version / build string. */
const char* gpudb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* GPUDB_ENGINE_H */
