// Seeded, row-addressable synthetic table generators (include/gpudb_datagen.h).
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/gpudb_datagen.h"
#include "datagen_core.h"

namespace {

using namespace gpudb_gen;

template <typename F>
void parallelFor(uint64_t n, int threads, F&& f) {
    unsigned t = threads > 0 ? (unsigned)threads : std::max(1u, std::thread::hardware_concurrency());
    if (n < 65536) t = 1;
    if (t > 256) t = 256;
    const uint64_t chunk = (n + t - 1) / t;
    std::vector<std::thread> ts;
    for (unsigned k = 0; k < t; k++) {
        const uint64_t b = k * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        ts.emplace_back([=, &f]() { f(b, e); });
    }
    for (auto& th : ts) th.join();
}

// Seeded bijection on [0, n): 4-round Feistel on the smallest even-width
// bit domain >= n, cycle-walking values that fall outside [0, n).
struct Perm {
    uint64_t n, seed;
    int half;
    uint64_t mask;
    Perm(uint64_t n_, uint64_t seed_) : n(n_), seed(seed_) {
        int bits = 2;
        while ((1ull << bits) < n) bits += 2;
        half = bits / 2;
        mask = (1ull << half) - 1;
    }
    uint64_t once(uint64_t x) const {
        uint64_t l = x >> half, r = x & mask;
        for (uint64_t round = 0; round < 4; round++) {
            const uint64_t f = mix64(r + seed * 0x9E3779B97F4A7C15ull + round * 0xA24BAED4963EE407ull) & mask;
            const uint64_t nl = r;
            r = l ^ f;
            l = nl;
        }
        return (l << half) | r;
    }
    uint64_t operator()(uint64_t x) const {
        uint64_t y = once(x);
        while (y >= n) y = once(y);
        return y;
    }
};

inline int32_t orderDay(uint64_t seed, int64_t key) { return (int32_t)uni(rnd(seed, S_ODAY, (uint64_t)key), 0, 2405); }

// Zipf(s) over [0, n): inverse CDF by binary search on a cached table.
struct ZipfTable {
    std::vector<double> cdf;
};
std::mutex gZipfMu;
std::map<std::pair<uint64_t, uint64_t>, std::shared_ptr<ZipfTable>> gZipf;

std::shared_ptr<ZipfTable> zipf(uint64_t n, double s) {
    uint64_t sbits;
    std::memcpy(&sbits, &s, 8);
    std::lock_guard<std::mutex> g(gZipfMu);
    auto& t = gZipf[{n, sbits}];
    if (!t) {
        t = std::make_shared<ZipfTable>();
        t->cdf.resize(n);
        long double acc = 0;
        for (uint64_t r = 0; r < n; r++) {
            acc += std::pow((long double)(r + 1), -(long double)s);
            t->cdf[r] = (double)acc;
        }
        const double tot = t->cdf[n - 1];
        for (auto& v : t->cdf) v /= tot;
        t->cdf[n - 1] = 1.0;
    }
    return t;
}

inline uint64_t zipfRank(const ZipfTable& t, double u) { return gpudb_gen::zipfRank(t.cdf.data(), t.cdf.size(), u); }

inline int64_t zkey(uint64_t seed, uint64_t rank) {
    uint64_t k = mix64(rank ^ mix64(seed + 0x5851F42D4C957F2Dull));
    if (k == ~0ull) k = 0x7FFFFFFFFFFFFFFFull;  // the empty-slot sentinel is never a key
    return (int64_t)k;
}

}  // namespace

namespace gpudb_gen {
// Zipf(s) CDF over [0, n) (cached for the process), shared with the device
// generators so both search the same table.
const std::vector<double>& zipfCdf(uint64_t n, double s) { return zipf(n, s)->cdf; }

// The last failure of a device generator on this thread (the generators'
// own library keeps its own error text).
thread_local std::string tlError;
void setError(const std::string& message) { tlError = message; }
}  // namespace gpudb_gen

extern "C" {

const char* gpudb_datagen_last_error(void) { return gpudb_gen::tlError.c_str(); }


int gpudb_gen_fact(uint64_t seed, uint64_t row0, uint64_t n, int32_t* ship_day, int64_t* quantity, int64_t* price,
                   int64_t* discount, int64_t* tax, uint8_t* flag_a, uint8_t* flag_b, int threads) {
    if (n && (!ship_day || !quantity || !price || !discount || !tax || !flag_a || !flag_b)) return -1;
    const int32_t cutoff = 1263;
    parallelFor(n, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            const uint64_t r = row0 + i;
            const int32_t sd = (int32_t)uni(rnd(seed, S_SHIP, r), 0, 2526);
            ship_day[i] = sd;
            quantity[i] = uni(rnd(seed, S_QTY, r), 1, 50);
            price[i] = uni(rnd(seed, S_PRICE, r), 90000, 10500000);
            discount[i] = uni(rnd(seed, S_DISC, r), 0, 10);
            tax[i] = uni(rnd(seed, S_TAX, r), 0, 8);
            flag_b[i] = sd > cutoff ? 'O' : 'F';
            const int32_t recv = sd + (int32_t)uni(rnd(seed, S_RECV, r), 1, 30);
            flag_a[i] = recv > cutoff ? 'N' : ((rnd(seed, S_FLAG_A, r) & 1) ? 'R' : 'A');
        }
    });
    return 0;
}

int gpudb_gen_dim(uint64_t seed, uint64_t nrows, uint64_t row0, uint64_t n, int32_t* key, int32_t* order_day,
                  uint8_t* segment, int threads) {
    if ((n && (!key || !order_day || !segment)) || row0 + n > nrows || nrows > 0x7FFFFFFFull) return -1;
    const Perm perm(nrows, seed ^ 0x1234567ull);
    parallelFor(n, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            const uint64_t r = row0 + i;
            const int64_t k = (int64_t)perm(r) + 1;
            key[i] = (int32_t)k;
            order_day[i] = orderDay(seed, k);
            segment[i] = (uint8_t)uni(rnd(seed, S_SEG, r), 0, 4);
        }
    });
    return 0;
}

int32_t gpudb_gen_order_day(uint64_t seed, int64_t key) { return orderDay(seed, key); }

int gpudb_gen_probe(uint64_t seed, uint64_t dim_rows, uint64_t row0, uint64_t n, int32_t* fk, int32_t* ship_day,
                    int64_t* price, int64_t* discount, int threads) {
    if ((n && (!fk || !ship_day || !price || !discount)) || dim_rows == 0 || dim_rows > 0x7FFFFFFFull) return -1;
    parallelFor(n, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            const uint64_t r = row0 + i;
            const int64_t k = uni(rnd(seed, S_FK, r), 1, (int64_t)dim_rows);
            fk[i] = (int32_t)k;
            ship_day[i] = orderDay(seed, k) + (int32_t)uni(rnd(seed, S_SHIPD, r), 1, 121);
            price[i] = uni(rnd(seed, S_PPRICE, r), 90000, 10500000);
            discount[i] = uni(rnd(seed, S_PDISC, r), 0, 10);
        }
    });
    return 0;
}

int64_t gpudb_gen_zkey(uint64_t seed, uint64_t rank) { return zkey(seed, rank); }

int gpudb_gen_zbuild(uint64_t seed, uint64_t row0, uint64_t n, int64_t* key, int32_t* payload, int threads) {
    if (n && (!key || !payload)) return -1;
    parallelFor(n, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            const uint64_t r = row0 + i;
            key[i] = zkey(seed, r);
            payload[i] = (int32_t)uni(rnd(seed, S_ZPAY, r), 0, 0x7FFFFFFF);
        }
    });
    return 0;
}

int gpudb_gen_zprobe(uint64_t seed, uint64_t nkeys, double s, uint64_t row0, uint64_t n, int64_t* key, int64_t* value,
                     int threads) {
    if ((n && (!key || !value)) || nkeys == 0 || !(s > 0.0)) return -1;
    auto t = zipf(nkeys, s);
    parallelFor(n, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            const uint64_t r = row0 + i;
            key[i] = zkey(seed, zipfRank(*t, unit(rnd(seed, S_ZRANK, r))));
            value[i] = uni(rnd(seed, S_ZVAL, r), 90000, 10500000);
        }
    });
    return 0;
}

int gpudb_gen_mix(uint64_t seed, uint64_t nranks, double s, uint64_t dim_rows, uint64_t row0, uint64_t n,
                  int32_t* rank_u, int32_t* rank_z, int32_t* filter, int64_t* value, int32_t* fk, int threads) {
    if ((n && (!rank_u || !rank_z || !filter || !value || !fk)) || nranks == 0 || nranks > 0x7FFFFFFFull ||
        dim_rows == 0 || !(s > 0.0))
        return -1;
    auto t = zipf(nranks, s);
    parallelFor(n, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            const MixRow m = mixRow(seed, nranks, dim_rows, t->cdf.data(), row0 + i);
            rank_u[i] = m.rank_u;
            rank_z[i] = m.rank_z;
            filter[i] = m.filter;
            value[i] = m.value;
            fk[i] = m.fk;
        }
    });
    return 0;
}

int gpudb_gen_mixdim(uint64_t seed, uint64_t row0, uint64_t n, int32_t* key, int32_t* attr, int threads) {
    if (n && (!key || !attr)) return -1;
    parallelFor(n, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            const uint64_t r = row0 + i;
            key[i] = (int32_t)(r + 1);
            attr[i] = mixdimAttr(seed, r);
        }
    });
    return 0;
}


// ---- the snowflake of the multi-join (Q5-shape) plan ----------------------
int gpudb_gen_snow_cust(uint64_t seed, uint64_t row0, uint64_t n, int32_t* key, int32_t* nation, int threads) {
    if (n && (!key || !nation)) return -1;
    parallelFor(n, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            const uint64_t r = row0 + i;
            key[i] = (int32_t)(r + 1);
            nation[i] = (int32_t)uni(rnd(seed, S_CNAT, r), 0, 24);
        }
    });
    return 0;
}

int gpudb_gen_snow_supp(uint64_t seed, uint64_t row0, uint64_t n, int32_t* key, int32_t* nation, int threads) {
    if (n && (!key || !nation)) return -1;
    parallelFor(n, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            const uint64_t r = row0 + i;
            key[i] = (int32_t)(r + 1);
            nation[i] = (int32_t)uni(rnd(seed, S_SNAT, r), 0, 24);
        }
    });
    return 0;
}

int gpudb_gen_snow_orders(uint64_t seed, uint64_t ncust, uint64_t row0, uint64_t n, int32_t* key, int32_t* cust,
                          int32_t* day, int threads) {
    if ((n && (!key || !cust || !day)) || ncust == 0 || ncust > 0x7FFFFFFFull) return -1;
    parallelFor(n, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            const uint64_t r = row0 + i;
            key[i] = (int32_t)(r + 1);
            cust[i] = (int32_t)uni(rnd(seed, S_OCUST, r), 1, (int64_t)ncust);
            day[i] = (int32_t)uni(rnd(seed, S_ODAY2, r), 0, 2405);
        }
    });
    return 0;
}

int gpudb_gen_snow_lines(uint64_t seed, uint64_t norders, uint64_t nsupp, uint64_t row0, uint64_t n, int32_t* okey,
                         int32_t* supp, int64_t* price, int64_t* discount, int threads) {
    if ((n && (!okey || !supp || !price || !discount)) || norders == 0 || nsupp == 0 || norders > 0x7FFFFFFFull ||
        nsupp > 0x7FFFFFFFull)
        return -1;
    parallelFor(n, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            const uint64_t r = row0 + i;
            okey[i] = (int32_t)uni(rnd(seed, S_LOKEY, r), 1, (int64_t)norders);
            supp[i] = (int32_t)uni(rnd(seed, S_LSUPP, r), 1, (int64_t)nsupp);
            price[i] = uni(rnd(seed, S_LPRICE, r), 90000, 10500000);
            discount[i] = uni(rnd(seed, S_LDISC, r), 0, 10);
        }
    });
    return 0;
}

}  // extern "C"
