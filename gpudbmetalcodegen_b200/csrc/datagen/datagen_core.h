// Per-row primitives of the seeded generators, shared by the host
// generators (datagen.cpp) and their device twins (kernels/datagen_device.cu)
// so both produce identical values: integer arithmetic only, plus the exact
// conversion of 53 random bits to a double in [0, 1) and comparisons
// against a host-computed Zipf CDF.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define GPUDB_HD __host__ __device__ __forceinline__
#else
#define GPUDB_HD inline
#endif

namespace gpudb_gen {

// splitmix64 finalizer: a bijection on 64-bit words.
GPUDB_HD uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Independent stream per (seed, column id); value per row.
GPUDB_HD uint64_t rnd(uint64_t seed, uint64_t stream, uint64_t row) {
    return mix64(mix64(seed * 0x9E3779B97F4A7C15ull + stream * 0xD1B54A32D192ED03ull) + row);
}

GPUDB_HD int64_t uni(uint64_t r, int64_t lo, int64_t hi) { return lo + (int64_t)(r % (uint64_t)(hi - lo + 1)); }

GPUDB_HD double unit(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

// Stream ids (one per generated column).
enum : uint64_t {
    S_SHIP = 1, S_QTY, S_PRICE, S_DISC, S_TAX, S_FLAG_A, S_RECV,
    S_PERM, S_ODAY, S_SEG, S_FK, S_SHIPD, S_PPRICE, S_PDISC,
    S_ZKEY, S_ZPAY, S_ZRANK, S_ZVAL,
    S_MRU, S_MRZ, S_MF, S_MV, S_MFK, S_MDA,
    S_CNAT, S_SNAT, S_OCUST, S_ODAY2, S_LOKEY, S_LSUPP, S_LPRICE, S_LDISC
};

// Inverse CDF by binary search: the first rank whose CDF exceeds u.
GPUDB_HD uint64_t zipfRank(const double* cdf, uint64_t n, double u) {
    uint64_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (cdf[mid] > u) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// One row of the mixed-workload table.
struct MixRow {
    int32_t rank_u, rank_z, filter, fk;
    int64_t value;
};

GPUDB_HD MixRow mixRow(uint64_t seed, uint64_t nranks, uint64_t dim_rows, const double* cdf, uint64_t r) {
    MixRow m;
    m.rank_u = (int32_t)uni(rnd(seed, S_MRU, r), 0, (int64_t)nranks - 1);
    m.rank_z = (int32_t)zipfRank(cdf, nranks, unit(rnd(seed, S_MRZ, r)));
    m.filter = (int32_t)uni(rnd(seed, S_MF, r), 0, 9999);
    m.value = uni(rnd(seed, S_MV, r), 1, 1000000);
    m.fk = (int32_t)uni(rnd(seed, S_MFK, r), 1, (int64_t)dim_rows);
    return m;
}

// One row of the mixed-workload dimension table: key r + 1, attr U[0, 999].
GPUDB_HD int32_t mixdimAttr(uint64_t seed, uint64_t r) { return (int32_t)uni(rnd(seed, S_MDA, r), 0, 999); }

}  // namespace gpudb_gen
