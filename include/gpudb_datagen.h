/*
 * gpudb_datagen.h — seeded synthetic tables for the measured workloads.
 *
 * The reference loads dbgen .tbl files into columns (src/infra.h:
 * loadQueryColumns :1045, colbin format :522-910). Neither dbgen nor its
 * data exist here, so the workloads run on seeded synthetic tables with the
 * shapes, sizes and value distributions the benchmark configurations name.
 * Every value is a pure function of (seed, column, row): any row range can
 * be generated independently and reproduces the same values as a full
 * generation (tests use small slices of the full-size tables).
 *
 * All functions fill caller-provided host arrays and return 0, or -1 on a
 * bad argument. `threads` <= 0 means all hardware threads.
 *
 * The generators live in their own library, libgpudb_datagen.so, next to
 * libgpudb.so: a program that only needs the data (a CPU baseline, a test
 * fixture) loads no engine code.
 */
#ifndef GPUDB_DATAGEN_H
#define GPUDB_DATAGEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Fact table (scan-filter-aggregate). ship_day U[0,2526]; quantity
 * U[1,50]; price U[90000,10500000] (cents); discount U[0,10] (hundredths);
 * tax U[0,8]; flag_b = 'O' if ship_day > 1263 else 'F'; flag_a = 'N' if
 * ship_day + U[1,30] > 1263 else uniform {'A','R'}: exactly four populated
 * (flag_a, flag_b) groups. */
int gpudb_gen_fact(uint64_t seed, uint64_t row0, uint64_t n, int32_t* ship_day, int64_t* quantity, int64_t* price,
                   int64_t* discount, int64_t* tax, uint8_t* flag_a, uint8_t* flag_b, int threads);

/* Build side of the join: key = perm(row) + 1 over [1, nrows] (seeded
 * bijection); order_day(key) U[0,2405]; segment U[0,4]. */
int gpudb_gen_dim(uint64_t seed, uint64_t nrows, uint64_t row0, uint64_t n, int32_t* key, int32_t* order_day,
                  uint8_t* segment, int threads);

/* Probe side: fk U[1, dim_rows]; ship_day = order_day(fk) + U[1,121];
 * price / discount as the fact table. */
int gpudb_gen_probe(uint64_t seed, uint64_t dim_rows, uint64_t row0, uint64_t n, int32_t* fk, int32_t* ship_day,
                    int64_t* price, int64_t* discount, int threads);

/* order_day of one build key (what gen_dim stores for that key). */
int32_t gpudb_gen_order_day(uint64_t seed, int64_t key);

/* Skewed keys: key(rank) = seeded 64-bit bijection of rank (never -1).
 * zbuild: one row per rank in [row0, row0+n): key, payload U[0, 2^31-1]. */
int gpudb_gen_zbuild(uint64_t seed, uint64_t row0, uint64_t n, int64_t* key, int32_t* payload, int threads);
/* zprobe: rank ~ Zipf(s) over [0, nkeys); key(rank); value U[90000,10500000]. */
int gpudb_gen_zprobe(uint64_t seed, uint64_t nkeys, double s, uint64_t row0, uint64_t n, int64_t* key, int64_t* value,
                     int threads);
int64_t gpudb_gen_zkey(uint64_t seed, uint64_t rank);

/* Mixed-workload table: rank_u U[0, nranks); rank_z ~ Zipf(s) over
 * [0, nranks); filter U[0,10000); value U[1,1000000]; fk U[1, dim_rows]. */
int gpudb_gen_mix(uint64_t seed, uint64_t nranks, double s, uint64_t dim_rows, uint64_t row0, uint64_t n,
                  int32_t* rank_u, int32_t* rank_z, int32_t* filter, int64_t* value, int32_t* fk, int threads);
/* Mixed-workload dimension: key = row + 1, attr U[0,1000). */
int gpudb_gen_mixdim(uint64_t seed, uint64_t row0, uint64_t n, int32_t* key, int32_t* attr, int threads);
/* Device twins of gpudb_gen_mix / gpudb_gen_mixdim: identical values written
 * straight into device memory on `stream` (NULL = the default stream);
 * return after the stream has finished. */
int gpudb_gen_mix_device(uint64_t seed, uint64_t nranks, double s, uint64_t dim_rows, uint64_t row0, uint64_t n,
                         int32_t* rank_u, int32_t* rank_z, int32_t* filter, int64_t* value, int32_t* fk,
                         void* stream);
int gpudb_gen_mixdim_device(uint64_t seed, uint64_t row0, uint64_t n, int32_t* key, int32_t* attr, void* stream);
/* The snowflake of the multi-join plan (the reference's Q5 shape:
 * region -> nation -> customer / supplier -> orders -> lineitem). nation is
 * 25 rows (key 0..24, region key % 5) built by the caller. cust / supp:
 * key = row + 1, nation U[0,24]. orders: key = row + 1, cust U[1, ncust],
 * day U[0,2405]. lines: order key U[1, norders], supplier U[1, nsupp],
 * price / discount as the fact table. */
int gpudb_gen_snow_cust(uint64_t seed, uint64_t row0, uint64_t n, int32_t* key, int32_t* nation, int threads);
int gpudb_gen_snow_supp(uint64_t seed, uint64_t row0, uint64_t n, int32_t* key, int32_t* nation, int threads);
int gpudb_gen_snow_orders(uint64_t seed, uint64_t ncust, uint64_t row0, uint64_t n, int32_t* key, int32_t* cust,
                          int32_t* day, int threads);
int gpudb_gen_snow_lines(uint64_t seed, uint64_t norders, uint64_t nsupp, uint64_t row0, uint64_t n, int32_t* okey,
                         int32_t* supp, int64_t* price, int64_t* discount, int threads);
/* Text of the last device-generator failure on this thread ("" if none). */
const char* gpudb_datagen_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* GPUDB_DATAGEN_H */
