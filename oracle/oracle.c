/*
 * oracle.c — CPU restatement of the reference's hot-path operator
 * semantics (see oracle.h). TEST INFRASTRUCTURE ONLY: loaded by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the
 * product path. Exact integer arithmetic; OpenMP over host cores.
 */
#include "oracle.h"

#include <omp.h>
#include <stdlib.h>
#include <string.h>

typedef __int128 i128;

static oracle_i128 to_pair(i128 v) {
    oracle_i128 p;
    p.lo = (uint64_t)v;
    p.hi = (int64_t)(v >> 64);
    return p;
}

static int nthreads(int threads) { return threads > 0 ? threads : omp_get_max_threads(); }

/* ---- q1: metal_plan_builder.cpp:309-354, KeyedAgg metal_operators.cpp:375-502 */
int oracle_q1(uint64_t n, const int32_t* ship_day, const int64_t* quantity, const int64_t* price,
              const int64_t* discount, const int64_t* tax, const uint8_t* flag_a, const uint8_t* flag_b,
              int32_t ship_le, oracle_i128* out, int threads) {
    i128 tot[36];
    memset(tot, 0, sizeof tot);
#pragma omp parallel num_threads(nthreads(threads))
    {
        i128 loc[36];
        memset(loc, 0, sizeof loc);
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; i++) {
            if (ship_day[i] > ship_le) continue;
            const int fa = flag_a[i], fb = flag_b[i];
            const int b = (fa == 'A' ? 0 : (fa == 'N' ? 2 : 4)) + (fb == 'F' ? 0 : 1);
            const int64_t p = price[i], d = discount[i];
            const int64_t dp = p * (100 - d);
            i128* r = loc + b * 6;
            r[0] += quantity[i];
            r[1] += p;
            r[2] += dp;
            r[3] += (i128)dp * (100 + tax[i]);
            r[4] += d;
            r[5] += 1;
        }
#pragma omp critical
        for (int j = 0; j < 36; j++) tot[j] += loc[j];
    }
    for (int j = 0; j < 36; j++) out[j] = to_pair(tot[j]);
    return 0;
}

/* ---- q6: metal_plan_builder.cpp:253-303 */
int oracle_q6(uint64_t n, const int32_t* ship_day, const int64_t* quantity, const int64_t* price,
              const int64_t* discount, int32_t ship_ge, int32_t ship_lt, int64_t disc_lo, int64_t disc_hi,
              int64_t qty_lt, oracle_i128* out, int threads) {
    i128 tot = 0;
#pragma omp parallel num_threads(nthreads(threads))
    {
        i128 loc = 0;
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; i++) {
            const int64_t d = discount[i];
            if (ship_day[i] >= ship_ge && ship_day[i] < ship_lt && d >= disc_lo && d <= disc_hi && quantity[i] < qty_lt)
                loc += (i128)price[i] * d;
        }
#pragma omp critical
        tot += loc;
    }
    *out = to_pair(tot);
    return 0;
}

/* ---- top-k helper: (value desc, key asc); codegen_main.cpp:1211-1248 */
static int better(int64_t va, int64_t ka, int64_t vb, int64_t kb) { return va > vb || (va == vb && ka < kb); }

static void topk_push(int k, int* cnt, int64_t* kk, int64_t* vv, int64_t key, int64_t val) {
    int pos = *cnt;
    if (pos == k) {
        if (!better(val, key, vv[k - 1], kk[k - 1])) return;
        pos = k - 1;
    } else {
        (*cnt)++;
    }
    while (pos > 0 && better(val, key, vv[pos - 1], kk[pos - 1])) {
        vv[pos] = vv[pos - 1];
        kk[pos] = kk[pos - 1];
        pos--;
    }
    vv[pos] = val;
    kk[pos] = key;
}

int oracle_topk(uint64_t n, const int64_t* keys, const int64_t* vals, int k, int64_t* out_keys, int64_t* out_vals) {
    int cnt = 0;
    for (uint64_t i = 0; i < n; i++) topk_push(k, &cnt, out_keys, out_vals, keys[i], vals[i]);
    return cnt;
}

/* ---- join + group + top-k: Q3 shape, metal_plan_builder.cpp:1170-1239 */
int oracle_join_topk(uint64_t nb, const int32_t* b_key, const int32_t* b_order_day, const uint8_t* b_segment,
                     uint64_t np, const int32_t* p_fk, const int32_t* p_ship_day, const int64_t* p_price,
                     const int64_t* p_discount, int32_t seg, int32_t od_lt, int32_t ship_gt, int k,
                     int64_t* out_keys, int64_t* out_vals, uint64_t* out_groups, uint64_t* out_build_distinct,
                     int threads) {
    const int T = nthreads(threads);
    int64_t maxk = 0;
    for (uint64_t i = 0; i < nb; i++)
        if (b_key[i] > maxk) maxk = b_key[i];
    const uint64_t words = (uint64_t)maxk / 32 + 1;
    uint32_t* bm = calloc(words, 4);
    int64_t* sum = calloc((size_t)maxk + 1, 8);
    int64_t* cntk = calloc((size_t)maxk + 1, 8);
    if (!bm || !sum || !cntk) {
        free(bm);
        free(sum);
        free(cntk);
        return -1;
    }
#pragma omp parallel for num_threads(T) schedule(static)
    for (int64_t i = 0; i < (int64_t)nb; i++) {
        if (b_segment[i] == seg && b_order_day[i] < od_lt && b_key[i] >= 0)
            __atomic_fetch_or(&bm[b_key[i] >> 5], 1u << (b_key[i] & 31), __ATOMIC_RELAXED);
    }
    uint64_t distinct = 0;
    for (uint64_t w = 0; w < words; w++) distinct += (uint64_t)__builtin_popcount(bm[w]);
#pragma omp parallel for num_threads(T) schedule(static)
    for (int64_t i = 0; i < (int64_t)np; i++) {
        const int32_t f = p_fk[i];
        if (p_ship_day[i] <= ship_gt || f < 0 || f > maxk) continue;
        if (!((bm[f >> 5] >> (f & 31)) & 1u)) continue;
        __atomic_fetch_add(&sum[f], p_price[i] * (100 - p_discount[i]), __ATOMIC_RELAXED);
        __atomic_fetch_add(&cntk[f], 1, __ATOMIC_RELAXED);
    }
    uint64_t groups = 0;
    int total = 0;
    int64_t* tk = malloc(sizeof(int64_t) * (size_t)k * T * 2);
    int* tc = calloc((size_t)T, sizeof(int));
#pragma omp parallel num_threads(T) reduction(+ : groups)
    {
        const int t = omp_get_thread_num();
        int64_t* kk = tk + (size_t)t * k * 2;
        int64_t* vv = kk + k;
#pragma omp for schedule(static)
        for (int64_t key = 0; key <= maxk; key++) {
            if (!cntk[key]) continue;
            groups++;
            topk_push(k, &tc[t], kk, vv, key, sum[key]);
        }
    }
    for (int t = 0; t < T; t++) {
        int64_t* kk = tk + (size_t)t * k * 2;
        for (int j = 0; j < tc[t]; j++) topk_push(k, &total, out_keys, out_vals, kk[j], kk[k + j]);
    }
    free(tk);
    free(tc);
    free(bm);
    free(sum);
    free(cntk);
    if (out_groups) *out_groups = groups;
    if (out_build_distinct) *out_build_distinct = distinct;
    return total;
}

/* ---- hash aggregation helpers (open addressing, empty = all ones) ---- */
typedef struct {
    uint64_t cap, mask;
    uint64_t* keys;
    int64_t* cnt;
    int64_t* sum;
} oht;

static int oht_init(oht* h, uint64_t want) {
    uint64_t c = 16;
    while (c < 2 * want) c <<= 1;
    h->cap = c;
    h->mask = c - 1;
    h->keys = malloc(c * 8);
    h->cnt = calloc(c, 8);
    h->sum = calloc(c, 8);
    if (!h->keys || !h->cnt || !h->sum) return -1;
    memset(h->keys, 0xFF, c * 8);
    return 0;
}

static void oht_free(oht* h) {
    free(h->keys);
    free(h->cnt);
    free(h->sum);
}

static uint64_t oht_hash(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    return k;
}

/* returns slot, or -1 when the table is full */
static int64_t oht_slot(oht* h, uint64_t key) {
    uint64_t s = oht_hash(key) & h->mask;
    for (uint64_t p = 0; p < h->cap; p++) {
        uint64_t cur = __atomic_load_n(&h->keys[s], __ATOMIC_RELAXED);
        if (cur == key) return (int64_t)s;
        if (cur == ~0ull) {
            uint64_t exp = ~0ull;
            if (__atomic_compare_exchange_n(&h->keys[s], &exp, key, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED) ||
                exp == key)
                return (int64_t)s;
        }
        s = (s + 1) & h->mask;
    }
    return -1;
}

typedef struct {
    int64_t key;
    int64_t cnt, sum;
} grp;

static int grp_cmp(const void* a, const void* b) {
    const int64_t x = ((const grp*)a)->key, y = ((const grp*)b)->key;
    return x < y ? -1 : x > y;
}

static int64_t oht_emit(oht* h, uint64_t cap, int64_t* ok, int64_t* oc, int64_t* os) {
    uint64_t g = 0;
    for (uint64_t s = 0; s < h->cap; s++)
        if (h->keys[s] != ~0ull && h->cnt[s]) g++;
    if (g > cap) return -1;
    grp* v = malloc(sizeof(grp) * (g ? g : 1));
    uint64_t j = 0;
    for (uint64_t s = 0; s < h->cap; s++)
        if (h->keys[s] != ~0ull && h->cnt[s]) {
            v[j].key = (int64_t)h->keys[s];
            v[j].cnt = h->cnt[s];
            v[j].sum = h->sum[s];
            j++;
        }
    qsort(v, g, sizeof(grp), grp_cmp);
    for (uint64_t i = 0; i < g; i++) {
        ok[i] = v[i].key;
        oc[i] = v[i].cnt;
        os[i] = v[i].sum;
    }
    free(v);
    return (int64_t)g;
}

/* ---- group-by: Q18 shape (metal_plan_builder.cpp:1529-1545) with 64-bit keys */
int64_t oracle_groupby(uint64_t n, const int64_t* key, const int64_t* value, uint64_t cap, int64_t* out_keys,
                       int64_t* out_count, int64_t* out_sum, int threads) {
    oht h;
    if (oht_init(&h, n < cap ? n : cap) != 0) return -2;
    int full = 0;
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static) reduction(| : full)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        const int64_t s = oht_slot(&h, (uint64_t)key[i]);
        if (s < 0) {
            full = 1;
            continue;
        }
        __atomic_fetch_add(&h.cnt[s], 1, __ATOMIC_RELAXED);
        __atomic_fetch_add(&h.sum[s], value[i], __ATOMIC_RELAXED);
    }
    const int64_t g = full ? -1 : oht_emit(&h, cap, out_keys, out_count, out_sum);
    oht_free(&h);
    return g;
}

/* ---- hash join: host-built HT + probe (query_preprocessing.cpp:443-479,
 *      metal_plan_builder.cpp:1968-1982) */
int64_t oracle_hashjoin(uint64_t nb, const int64_t* b_key, const int32_t* b_payload, uint64_t np,
                        const int64_t* p_key, uint64_t cap, int64_t* out_keys, int64_t* out_count, int64_t* out_sum,
                        int threads) {
    oht h;
    if (oht_init(&h, nb) != 0) return -2;
    int64_t* pay = malloc(h.cap * 8);
    for (uint64_t i = 0; i < nb; i++) {
        const int64_t s = oht_slot(&h, (uint64_t)b_key[i]);
        if (s < 0) {
            free(pay);
            oht_free(&h);
            return -2;
        }
        pay[s] = b_payload[i];
    }
    const uint64_t mask = h.mask;
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (int64_t i = 0; i < (int64_t)np; i++) {
        const uint64_t k = (uint64_t)p_key[i];
        uint64_t s = oht_hash(k) & mask;
        for (;;) {
            const uint64_t cur = h.keys[s];
            if (cur == k) {
                __atomic_fetch_add(&h.cnt[s], 1, __ATOMIC_RELAXED);
                __atomic_fetch_add(&h.sum[s], pay[s], __ATOMIC_RELAXED);
                break;
            }
            if (cur == ~0ull) break;
            s = (s + 1) & mask;
        }
    }
    const int64_t g = oht_emit(&h, cap, out_keys, out_count, out_sum);
    free(pay);
    oht_free(&h);
    return g;
}

/* ---- mixed templates ---------------------------------------------------- */
int oracle_mix_agg(uint64_t n, const int32_t* filter, const int64_t* value, int32_t thr, int64_t* out_count,
                   oracle_i128* out_sum, int threads) {
    int64_t c = 0;
    i128 s = 0;
#pragma omp parallel num_threads(nthreads(threads))
    {
        int64_t lc = 0;
        i128 ls = 0;
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; i++)
            if (filter[i] < thr) {
                lc++;
                ls += value[i];
            }
#pragma omp critical
        {
            c += lc;
            s += ls;
        }
    }
    *out_count = c;
    *out_sum = to_pair(s);
    return 0;
}

int64_t oracle_mix_groupby(uint64_t n, const int32_t* rank, const int32_t* filter, const int64_t* value, int32_t thr,
                           int64_t card, uint64_t cap, int64_t* out_keys, int64_t* out_count, int64_t* out_sum,
                           int threads) {
    oht h;
    const uint64_t want = (uint64_t)card < n ? (uint64_t)card : n;
    if (oht_init(&h, want) != 0) return -2;
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        if (filter[i] >= thr) continue;
        const int64_t s = oht_slot(&h, (uint64_t)((int64_t)rank[i] % card));
        __atomic_fetch_add(&h.cnt[s], 1, __ATOMIC_RELAXED);
        __atomic_fetch_add(&h.sum[s], value[i], __ATOMIC_RELAXED);
    }
    const int64_t g = oht_emit(&h, cap, out_keys, out_count, out_sum);
    oht_free(&h);
    return g;
}

int oracle_mix_join(uint64_t nd, const int32_t* md_key, const int32_t* md_attr, int32_t attr_lt, uint64_t n,
                    const int32_t* fk, const int32_t* filter, const int64_t* value, int32_t thr, int64_t* out_count,
                    oracle_i128* out_sum, int threads) {
    int64_t maxk = 0;
    for (uint64_t i = 0; i < nd; i++)
        if (md_key[i] > maxk) maxk = md_key[i];
    uint8_t* in = calloc((size_t)maxk + 1, 1);
    for (uint64_t i = 0; i < nd; i++)
        if (md_attr[i] < attr_lt && md_key[i] >= 0) in[md_key[i]] = 1;
    int64_t c = 0;
    i128 s = 0;
#pragma omp parallel num_threads(nthreads(threads))
    {
        int64_t lc = 0;
        i128 ls = 0;
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; i++)
            if (filter[i] < thr && fk[i] >= 0 && fk[i] <= maxk && in[fk[i]]) {
                lc++;
                ls += value[i];
            }
#pragma omp critical
        {
            c += lc;
            s += ls;
        }
    }
    free(in);
    *out_count = c;
    *out_sum = to_pair(s);
    return 0;
}

int64_t oracle_max_i32(uint64_t n, const int32_t* v, int threads) {
    int64_t m = INT64_MIN;
#pragma omp parallel for num_threads(nthreads(threads)) reduction(max : m)
    for (int64_t i = 0; i < (int64_t)n; i++)
        if (v[i] > m) m = v[i];
    return m;
}

/* ---- anti_join: Q22 operator chain, metal_plan_builder.cpp:1304-1357 —
 * BitmapBuild over the qualifying build keys, AntiBitmapProbe
 * (metal_operators.cpp:157-165) of the probe rows passing ship_day >
 * ship_gt, bin = discount (ComputeExpr, :86-91), AtomicCount (:550-594)
 * and AtomicAgg of price (:525-533) per bin. A key outside the bitmap is
 * absent, so such a probe row passes the anti-probe. Returns 0, or -1 if a
 * bin falls outside [0, nbins) (the engine's bounds error). */
int oracle_anti_join(uint64_t nb, const int32_t* b_key, const int32_t* b_order_day, const uint8_t* b_segment,
                     uint64_t np, const int32_t* p_fk, const int32_t* p_ship_day, const int64_t* p_price,
                     const int64_t* p_discount, int32_t seg, int32_t od_lt, int32_t ship_gt, int nbins,
                     int64_t* out_counts, oracle_i128* out_sums, int threads) {
    const int T = nthreads(threads);
    int64_t maxk = 0;
    for (uint64_t i = 0; i < nb; i++)
        if (b_key[i] > maxk) maxk = b_key[i];
    const uint64_t words = (uint64_t)maxk / 32 + 1;
    uint32_t* bm = calloc(words, 4);
    if (!bm || nbins < 1 || nbins > 4096) {
        free(bm);
        return -1;
    }
#pragma omp parallel for num_threads(T) schedule(static)
    for (int64_t i = 0; i < (int64_t)nb; i++) {
        if (b_segment[i] == seg && b_order_day[i] < od_lt && b_key[i] >= 0)
            __atomic_fetch_or(&bm[b_key[i] >> 5], 1u << (b_key[i] & 31), __ATOMIC_RELAXED);
    }
    int64_t cnt[4096];
    i128 sum[4096];
    memset(cnt, 0, sizeof(int64_t) * (size_t)nbins);
    memset(sum, 0, sizeof(i128) * (size_t)nbins);
    int bad = 0;
#pragma omp parallel num_threads(T)
    {
        int64_t lc[4096];
        i128 ls[4096];
        memset(lc, 0, sizeof(int64_t) * (size_t)nbins);
        memset(ls, 0, sizeof(i128) * (size_t)nbins);
        int lbad = 0;
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)np; i++) {
            if (p_ship_day[i] <= ship_gt) continue;
            const int64_t k = p_fk[i];
            const int in = k >= 0 && (uint64_t)(k >> 5) < words && ((bm[k >> 5] >> (k & 31)) & 1u);
            if (in) continue;
            const int64_t b = p_discount[i];
            if (b < 0 || b >= nbins) {
                lbad = 1;
                continue;
            }
            lc[b] += 1;
            ls[b] += p_price[i];
        }
#pragma omp critical
        {
            for (int b = 0; b < nbins; b++) {
                cnt[b] += lc[b];
                sum[b] += ls[b];
            }
            bad |= lbad;
        }
    }
    free(bm);
    for (int b = 0; b < nbins; b++) {
        out_counts[b] = cnt[b];
        out_sums[b] = to_pair(sum[b]);
    }
    return bad ? -1 : 0;
}

/* ---- histogram: Q13 operator chain, metal_plan_builder.cpp:1244-1299 —
 * AtomicCount of the probe rows passing ship_day > ship_gt per key (an
 * array indexed by key, sized by the largest build key), then for every
 * build row an ArrayLookup of its key's count (metal_operators.cpp:213-225)
 * and an AtomicCount histogram over the counts. out_hist[c] = build rows
 * whose key has c such probe rows. Returns 0, or -1 if a probe key lies
 * beyond the largest build key or a count reaches nbins (the engine's
 * bounds errors). */
int oracle_histogram(uint64_t nb, const int32_t* b_key, uint64_t np, const int32_t* p_fk, const int32_t* p_ship_day,
                     int32_t ship_gt, int nbins, int64_t* out_hist, int threads) {
    const int T = nthreads(threads);
    int64_t maxk = 0;
    for (uint64_t i = 0; i < nb; i++)
        if (b_key[i] > maxk) maxk = b_key[i];
    uint32_t* cnt = calloc((size_t)maxk + 1, 4);
    if (!cnt) return -1;
    int bad = 0;
#pragma omp parallel for num_threads(T) schedule(static) reduction(| : bad)
    for (int64_t i = 0; i < (int64_t)np; i++) {
        if (p_ship_day[i] <= ship_gt) continue;
        const int64_t k = p_fk[i];
        if (k < 0 || k > maxk) {
            bad = 1;
            continue;
        }
        __atomic_fetch_add(&cnt[k], 1u, __ATOMIC_RELAXED);
    }
    memset(out_hist, 0, sizeof(int64_t) * (size_t)nbins);
    for (uint64_t i = 0; i < nb; i++) {
        const int64_t k = b_key[i];
        if (k < 0 || k > maxk) continue;
        const uint32_t c = cnt[k];
        if (c >= (uint32_t)nbins) {
            bad = 1;
            continue;
        }
        out_hist[c] += 1;
    }
    free(cnt);
    return bad ? -1 : 0;
}
