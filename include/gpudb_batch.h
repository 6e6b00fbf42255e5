/*
 * gpudb_batch.h — batched mixed-query execution and the learned sizer.
 *
 * No counterpart in the reference (which runs one query per process
 * invocation and sizes every table with an exact max-key / count pass,
 * codegen/execution/max_key_symbols.cpp:188-235). Three layers, none of
 * which changes an answer:
 *   - batch: many queries of the four mixed pipeline shapes (scan-filter-agg,
 *     join-agg, high-cardinality group-by, group-by + top-k) over slices of
 *     resident tables run as one persistent work-queue kernel per shape
 *     (CTAs pull (query, tile) work items from a global counter), optionally
 *     replayed as a CUDA graph;
 *   - sizer: an MLP (16 -> 64 -> 64 -> 64 -> 2, BF16 weights, FP32
 *     accumulate) trained on the GPU by this library's own kernels, predicting
 *     log2 group cardinality and filter selectivity from per-query features,
 *     so hash tables are sized without the exact count pass; any table that
 *     overflows is detected on the device and the query re-runs with exact
 *     sizing;
 *   - exact statistics (the count pass itself, batched) and the 4096-row
 *     feature sample, both on the GPU.
 */
#ifndef GPUDB_BATCH_H
#define GPUDB_BATCH_H

#include "gpudb_rt.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- learned sizer ---------------------------------------------------- */
typedef struct gpudb_sizer gpudb_sizer;
#define GPUDB_SIZER_FEATURES 16
#define GPUDB_SIZER_OUTPUTS 2

int gpudb_sizer_create(int device, uint64_t seed, gpudb_sizer** out);
void gpudb_sizer_free(gpudb_sizer* s);
int gpudb_sizer_param_count(void);
/* FP32 master parameters (gpudb_sizer_param_count floats). */
int gpudb_sizer_get_params(gpudb_sizer* s, float* out);
int gpudb_sizer_set_params(gpudb_sizer* s, const float* in);
/* One forward + backward pass of the mean-squared error over (X, Y) (host
 * arrays, n x 16 and n x 2) with the current BF16 weights; gradients w.r.t.
 * the parameters are copied to grads_out. No update. */
int gpudb_sizer_grads(gpudb_sizer* s, const float* X, const float* Y, int n, float* grads_out, float* loss_out);
/* Adam training on the GPU: `epochs` passes over (X, Y) in shuffled batches,
 * learning rate `lr` decayed to 0 along a half cosine over the call's steps. */
int gpudb_sizer_train(gpudb_sizer* s, const float* X, const float* Y, int n, int epochs, int batch, float lr,
                      uint64_t seed, float* final_loss);
int gpudb_sizer_predict(gpudb_sizer* s, const float* X, int n, float* Y_out);

/* ---- column statistics -------------------------------------------------- */
/* Zone-map min / max of a device column of n int32 (elem_bytes 4) or int64
 * (elem_bytes 8) values, on `stream` (NULL = legacy default); returns after
 * the stream has finished. n = 0 gives (0, 0). These are the sizer's column
 * features (the key / filter domain of a resident table). */
int gpudb_column_minmax(const void* column, uint64_t n, int elem_bytes, int64_t* min_out, int64_t* max_out,
                        void* stream);

/* ---- batched mixed queries --------------------------------------------- */
typedef struct gpudb_batch gpudb_batch;

#define GPUDB_TPL_AGG 0      /* filter -> count + sum(value)                       */
#define GPUDB_TPL_JOIN 1     /* semi-join fk against dim(attr < attr_lt) -> count + sum */
#define GPUDB_TPL_GROUPBY 2  /* filter -> group by key % card: count + sum          */
#define GPUDB_TPL_TOPK 3     /* GROUPBY, then top k groups by (sum desc, key asc)   */

typedef struct {
    int tmpl;             /* GPUDB_TPL_*                                          */
    int32_t thr;          /* filter: filter[i] < thr                              */
    int64_t card;         /* group key = key[i] % card (GROUPBY / TOPK)           */
    int32_t k;            /* TOPK                                                 */
    int32_t attr_lt;      /* JOIN: dim rows with attr < attr_lt                   */
    uint64_t rows;        /* slice length                                         */
    const int32_t* key;   /* device column slices (rows elements)                 */
    const int32_t* filter;
    const int64_t* value;
    const int32_t* fk;
    const int32_t* dim_key;   /* JOIN build side (dim_rows elements)             */
    const int32_t* dim_attr;
    uint64_t dim_rows;
    int64_t dim_max_key;
    uint64_t groups;      /* hash-table sizing: expected groups (exact or predicted) */
    /* column statistics (zone-map min / max of the slice's table), features only */
    int64_t key_min, key_max;
    int32_t filter_min, filter_max;
    int32_t agg_mode;     /* GROUPBY / TOPK aggregation strategy, GPUDB_AGG_*     */
} gpudb_batch_query;

#define GPUDB_AGG_AUTO 0         /* SHARED                                           */
#define GPUDB_AGG_SHARED 1       /* warp + per-CTA shared-memory table, flushed       */
#define GPUDB_AGG_GLOBAL_WARP 2  /* warp aggregation, then the global table          */
#define GPUDB_AGG_GLOBAL 3       /* the global table directly (mostly distinct keys) */
#define GPUDB_AGG_SHARED_DIRECT 4 /* per-CTA shared-memory table indexed by the key   *
                                   * itself, no warp aggregation; card <= 1024 (else  *
                                   * SHARED), flushed like SHARED                     */

int gpudb_batch_create(gpudb_ctx* ctx, gpudb_batch** out);
void gpudb_batch_free(gpudb_batch* b);
/* Describe the batch; allocates / reuses one device arena for every
 * query's outputs and hash tables. */
int gpudb_batch_set_queries(gpudb_batch* b, const gpudb_batch_query* q, int n);
/* Change one query's table sizing / aggregation strategy (before the next
 * execute). */
int gpudb_batch_set_groups(gpudb_batch* b, int q, uint64_t groups);
int gpudb_batch_set_agg_mode(gpudb_batch* b, int q, int agg_mode);
/* Tuning of the persistent kernels: block size, rows per work item, warp
 * aggregation (0 turns GLOBAL_WARP into GLOBAL), hash probe bound. */
int gpudb_batch_set_tuning(gpudb_batch* b, int block, int tile_rows, int warp_aggregate, int max_probe);
/* Named tuning options beyond those: "group_rows" = rows in flight per
 * thread of the group-by kernel: 1 (default; a 32-register cap), 2 (42
 * registers) or 4 (64 registers); blocks of more than 512 threads use 4.
 * "agg_rows" = the same for the agg / join kernel: 2 (default; 32
 * registers, blocks of at most 512) or 4 (64 registers).
 * "shared_warp" = 1 (default): the SHARED strategy aggregates each warp's
 * equal keys before the shared table; 0: every row goes to it directly.
 * GPUDB_E_INVALID for an unknown name or value. */
int gpudb_batch_set_option(gpudb_batch* b, const char* name, long long value);
/* Run every query; per-query device error words go to errors[n] (bit
 * GPUDB_DEVERR_HASH_OVERFLOW = the table was undersized). With use_graph the
 * fills + kernels are captured once and replayed. *ms = device time. */
int gpudb_batch_execute(gpudb_batch* b, int use_graph, double* ms, uint32_t* errors);
/* Exact statistics (the count pass, batched): per query rows passing the
 * filter and distinct group keys among them (GROUPBY / TOPK). */
int gpudb_batch_exact_stats(gpudb_batch* b, uint64_t* passing, uint64_t* distinct, double* ms);
/* Features of each query from a 4096-row sample (GPUDB_SIZER_FEATURES floats
 * per query, see the library's feature definition). */
int gpudb_batch_features(gpudb_batch* b, float* features, double* ms);
/* Results. Scalar: count and 128-bit sum (lo, hi) for AGG / JOIN. Groups:
 * (key, count, sum) of GROUPBY / TOPK tables in slot-list order; ngroups is
 * always set. Top-k: (key, sum) best first. */
int gpudb_batch_result_scalar(gpudb_batch* b, int q, int64_t* count, uint64_t* sum_lo, int64_t* sum_hi);
int gpudb_batch_result_groups(gpudb_batch* b, int q, uint64_t cap, uint64_t* ngroups, int64_t* keys, int64_t* counts,
                              int64_t* sums);
int gpudb_batch_result_topk(gpudb_batch* b, int q, int64_t* keys, int64_t* vals, int* n);
/* Every query's result at once: compacted on the device, then ONE copy to
 * `host` (pinned memory recommended). rows[q] = result rows of query q
 * (1 for AGG / JOIN, groups for GROUPBY, min(k, groups) for TOPK). Each row
 * is three int64: AGG / JOIN (count, sum_lo, sum_hi); GROUPBY (key, count,
 * sum) in table order; TOPK (key, sum, 0) best first. Pass host = NULL to
 * learn *bytes_needed (and rows) without copying. */
int gpudb_batch_collect(gpudb_batch* b, uint64_t* rows, void* host, uint64_t host_bytes, uint64_t* bytes_needed,
                        double* ms);
/* Launches of this library's kernels in the last execute. */
long long gpudb_batch_last_launches(gpudb_batch* b);
/* Device time of each step of the last execute run without a graph:
 * zero fill, join build, agg / join probe, group-by, top-k chunks, top-k merge. */
#define GPUDB_BATCH_STAGES 6
int gpudb_batch_stage_ms(gpudb_batch* b, double* ms);

#ifdef __cplusplus
}
#endif

#endif /* GPUDB_BATCH_H */
