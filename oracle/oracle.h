/*
 * oracle.h — CPU restatement of the reference engine's hot-path operator
 * semantics, used ONLY as test infrastructure: the parity checker of the
 * GPU path (tests/, __graft_entry__.smoke) and the timed CPU baseline leg
 * of bench.py. The product path never calls it.
 *
 * Arithmetic is exact (int64 per row, 128-bit sums; the reference computes
 * in float32 with truncating fixed-point casts, which the benchmark
 * configurations replace by scaled-int64 fixed point). Grouping rules,
 * bucket order, empty-group omission and top-k ordering follow the
 * reference files cited per function.
 *
 * Pinning: the restatement is checked against the reference's own kernels
 * executed on the CPU (oracle/ref_harness, compiled from the reference's
 * plan builder + operator emitters; golden vectors in tests/golden/).
 */
#ifndef GPUDB_ORACLE_H
#define GPUDB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 128-bit two's complement value as (lo, hi) 64-bit words. */
typedef struct {
    uint64_t lo;
    int64_t hi;
} oracle_i128;

/* Scan -> filter(ship_day <= ship_le) -> 6-bucket aggregate.
 * Bucket = (flag_a=='A'?0 : flag_a=='N'?2 : 4) + (flag_b=='F'?0:1)
 * (metal_plan_builder.cpp:335). out[b*6 + j], j = sum_qty, sum_base_price,
 * sum_disc_price = sum price*(100-discount), sum_charge = sum
 * price*(100-discount)*(100+tax), sum_disc, count (metal_plan_builder.cpp:
 * 342-349). Buckets with all-zero slots are empty groups (omitted by the
 * collector, metal_result_collector.cpp:231-235). */
int oracle_q1(uint64_t n, const int32_t* ship_day, const int64_t* quantity, const int64_t* price,
              const int64_t* discount, const int64_t* tax, const uint8_t* flag_a, const uint8_t* flag_b,
              int32_t ship_le, oracle_i128* out /* [36] */, int threads);

/* Scan -> conjunctive filter -> scalar sum of price*discount
 * (metal_plan_builder.cpp:253-303; TGReduce metal_operators.cpp:258-346). */
int oracle_q6(uint64_t n, const int32_t* ship_day, const int64_t* quantity, const int64_t* price,
              const int64_t* discount, int32_t ship_ge, int32_t ship_lt, int64_t disc_lo, int64_t disc_hi,
              int64_t qty_lt, oracle_i128* out, int threads);

/* Build: keys of build rows with segment==seg && order_day<od_lt form a
 * semi-join set (BitmapBuild, metal_operators.cpp:108-116); probe rows with
 * ship_day>ship_gt whose fk is in the set are grouped by fk, summing
 * price*(100-discount) (ArrayLookup + AtomicAgg, metal_plan_builder.cpp:
 * 1189-1236); top k by (sum desc, key asc) (host top-k,
 * codegen_main.cpp:1211-1248, ties broken by key). Returns rows written. */
int oracle_join_topk(uint64_t nb, const int32_t* b_key, const int32_t* b_order_day, const uint8_t* b_segment,
                     uint64_t np, const int32_t* p_fk, const int32_t* p_ship_day, const int64_t* p_price,
                     const int64_t* p_discount, int32_t seg, int32_t od_lt, int32_t ship_gt, int k,
                     int64_t* out_keys, int64_t* out_vals, uint64_t* out_groups, uint64_t* out_build_distinct,
                     int threads);

/* Group by 64-bit key (optionally only rows with filter[i] < thr): count and
 * sum(value). Writes groups sorted by key into out_* (capacity `cap`);
 * returns the group count, or -1 if it exceeds cap. */
int64_t oracle_groupby(uint64_t n, const int64_t* key, const int64_t* value, uint64_t cap, int64_t* out_keys,
                       int64_t* out_count, int64_t* out_sum, int threads);

/* Inner join of probe keys against unique build keys; per build key with
 * at least one match: count of matches and sum of the build payload over
 * matches. Sorted by key; returns groups or -1 if cap is exceeded. */
int64_t oracle_hashjoin(uint64_t nb, const int64_t* b_key, const int32_t* b_payload, uint64_t np,
                        const int64_t* p_key, uint64_t cap, int64_t* out_keys, int64_t* out_count, int64_t* out_sum,
                        int threads);

/* Mixed templates (key = rank % card, filter = filter[i] < thr). */
int oracle_mix_agg(uint64_t n, const int32_t* filter, const int64_t* value, int32_t thr, int64_t* out_count,
                   oracle_i128* out_sum, int threads);
int64_t oracle_mix_groupby(uint64_t n, const int32_t* rank, const int32_t* filter, const int64_t* value, int32_t thr,
                           int64_t card, uint64_t cap, int64_t* out_keys, int64_t* out_count, int64_t* out_sum,
                           int threads);
int oracle_mix_join(uint64_t nd, const int32_t* md_key, const int32_t* md_attr, int32_t attr_lt, uint64_t n,
                    const int32_t* fk, const int32_t* filter, const int64_t* value, int32_t thr, int64_t* out_count,
                    oracle_i128* out_sum, int threads);
/* Top k of (key, sum) rows by (sum desc, key asc). */
int oracle_topk(uint64_t n, const int64_t* keys, const int64_t* vals, int k, int64_t* out_keys, int64_t* out_vals);

/* Exact max of an int32 / int64 column (max_key_symbols.cpp:188-235). */
int64_t oracle_max_i32(uint64_t n, const int32_t* v, int threads);

/* Anti-join (Q22 operator chain): probe rows with ship_day > ship_gt whose
 * key is not a qualifying build key (segment == seg, order_day < od_lt),
 * per discount bin: row count and exact sum of price. 0, or -1 on a bin
 * outside [0, nbins). */
int oracle_anti_join(uint64_t nb, const int32_t* b_key, const int32_t* b_order_day, const uint8_t* b_segment,
                     uint64_t np, const int32_t* p_fk, const int32_t* p_ship_day, const int64_t* p_price,
                     const int64_t* p_discount, int32_t seg, int32_t od_lt, int32_t ship_gt, int nbins,
                     int64_t* out_counts, oracle_i128* out_sums, int threads);

/* Histogram (Q13 operator chain): probe rows with ship_day > ship_gt counted
 * per key, then out_hist[c] = build rows whose key has c of them. 0, or -1
 * on a probe key beyond the largest build key or a count >= nbins. */
int oracle_histogram(uint64_t nb, const int32_t* b_key, uint64_t np, const int32_t* p_fk, const int32_t* p_ship_day,
                     int32_t ship_gt, int nbins, int64_t* out_hist, int threads);

#ifdef __cplusplus
}
#endif

#endif
