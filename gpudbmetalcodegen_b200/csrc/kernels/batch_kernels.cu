// Batched mixed-query execution (include/gpudb_batch.h).
//
// Every query of a batch owns a slice of one zero-initialised device arena
// (outputs, hash table, bitmap, error word). Each pipeline shape runs as ONE
// persistent kernel: CTAs take work items — (query, tile of rows) — from a
// global counter, in the order of a per-shape prefix sum of tiles, so uneven
// table sizes balance across the GPU and a whole batch costs one memset and
// a handful of launches (build, agg, group, top-k, top-k merge), replayable
// as a CUDA graph.
//
// Hash tables are arrays of 16-byte slots {key + card (u32), count (u32),
// sum (u64)}: two slots per L2 sector, and the all-zero pattern is the empty
// slot (`int32 % card` lies in (-card, card), so key + card is never 0), so a
// single memset initialises the whole arena. Each CTA first aggregates into
// a shared-memory table of kSmemSlots entries (bounded probing; a row whose
// key finds no room goes to the global table directly) and flushes it at
// the end of every work item: few-group queries then cost a handful of
// global atomics per tile, and hot keys of skewed ones stay on chip.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/gpudb_batch.h"
#include "gpudb_device.cuh"

namespace gpudb {
void setThreadError(const std::string& message);
}

namespace {

constexpr int kTopK = 16;             // largest k a top-k query may ask for
constexpr long long kTkChunk = 4096;  // slot-list entries per top-k work item
constexpr int kUnroll = 4;            // independent rows in flight per thread
constexpr int kSmemSlots = 2048;      // per-CTA shared-memory aggregation table
constexpr int kSmemProbe = 4;         // probes into it before spilling to global

struct __align__(16) Slot {
    unsigned key;    // key + card, 0 = empty
    unsigned count;  // rows of the group (slices are < 2^32 rows)
    unsigned long long sum;
};

__host__ __device__ __forceinline__ unsigned encKey(long long key, long long card) {
    return (unsigned)(key + card);
}
__host__ __device__ __forceinline__ long long decKey(unsigned enc, long long card) { return (long long)enc - card; }

struct QDesc {
    int tmpl, thr, k, attr_lt;
    long long card, rows;
    unsigned cardMagic;  // key % card by multiply-high for keys >= 0
    int cardSh1, cardSh2;
    const int* key;
    const int* filter;
    const long long* value;
    const int* fk;
    const int* dim_key;
    const int* dim_attr;
    long long dim_rows, bitmap_words;
    unsigned long long* agg;  // [count, sum word 0, sum word 1]
    unsigned long long* topk_n;
    unsigned long long* nslots;
    unsigned* err;
    unsigned* bitmap;
    Slot* ht;
    int log2cap, maxProbe;
    int aggMode;  // GPUDB_AGG_SHARED / _GLOBAL_WARP / _GLOBAL / _SHARED_DIRECT
    int sharedWarp;  // SHARED: warp aggregation before the shared table
    unsigned* slots;
    long long* tk_part;  // [tk_chunks][kTopK] of (value, key)
    long long tk_chunks;
    long long* topk_out;  // [kTopK] of (key, value)
    // exact statistics
    unsigned long long* st_pass;
    unsigned long long* st_distinct;
    unsigned* st_bitmap;
    long long st_words;
};

// Group key = key % card. Non-negative keys use division by the invariant
// card via a multiply-high (Granlund & Montgomery, "Division by invariant
// integers using multiplication", PLDI 1994, Fig. 4.1): with
// l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0), t = mulhi(m, n).
void cardDivisor(long long card, unsigned* magic, int* sh1, int* sh2) {
    const unsigned long long d = (unsigned long long)card;
    int l = 0;
    while ((1ull << l) < d) l++;
    *magic = (unsigned)(((1ull << 32) * ((1ull << l) - d)) / d + 1ull);
    *sh1 = l < 1 ? l : 1;
    *sh2 = l - 1 > 0 ? l - 1 : 0;
}

__device__ __forceinline__ long long keyMod(int k, const QDesc& q) {
    if (k >= 0) {
        const unsigned n = (unsigned)k;
        const unsigned t = __umulhi(n, q.cardMagic);
        const unsigned quo = (t + ((n - t) >> q.cardSh1)) >> q.cardSh2;
        return (long long)(n - quo * (unsigned)q.card);
    }
    return (long long)k % q.card;
}

// A work list: queries (indices into the descriptor array) and the prefix
// sum of their work items.
struct WorkList {
    const int* q;
    const long long* prefix;  // nq + 1 entries
    int nq;
};

__device__ __forceinline__ int findQuery(const WorkList& wl, long long w) {
    int lo = 0, hi = wl.nq - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(wl.prefix + mid) <= w) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Filter words of rows b, b + step, ... (kUnroll of them); rows at or past
// r1 read as `thr`, which no row passes.
template <int N>
__device__ __forceinline__ void loadFilters(const int* __restrict__ filter, long long b, long long step, long long r1,
                                            int thr, int (&f)[N]) {
#pragma unroll
    for (int u = 0; u < N; ++u) f[u] = b + u * step < r1 ? __ldcs(filter + b + u * step) : thr;
}

// Words of rows b, b + step, ... (kUnroll of them) whatever the filter
// says; rows at or past r1 read as 0.
template <typename T, int N>
__device__ __forceinline__ void loadAhead(const T* __restrict__ col, long long b, long long step, long long r1,
                                          T (&x)[N]) {
#pragma unroll
    for (int u = 0; u < N; ++u) x[u] = b + u * step < r1 ? __ldcs(col + b + u * step) : (T)0;
}

// A warp whose first kUnroll x 32 rows of a work item pass the filter at
// least one time in four reads its dependent columns unconditionally, one
// iteration ahead with the filter words: at that selectivity nearly every
// 32-byte sector of those columns is needed anyway (each holds 4-8 rows),
// and the loads no longer wait for the filter. Sparser warps keep
// filter-guarded loads. Called by whole warps.
template <int N>
__device__ __forceinline__ bool denseWarp(const int (&f)[N], int thr) {
    int pass = 0;
#pragma unroll
    for (int u = 0; u < N; ++u) pass += __popc(__ballot_sync(0xffffffffu, f[u] < thr));
    return 4 * pass >= 32 * N;
}

// CTA-wide work pull; returns -1 when the list is exhausted.
__device__ __forceinline__ long long pullWork(unsigned long long* counter, long long total, long long* s_item) {
    __syncthreads();
    if (threadIdx.x == 0) *s_item = (long long)atomicAdd(counter, 1ull);
    __syncthreads();
    const long long w = *s_item;
    return w < total ? w : -1;
}

__device__ __forceinline__ void blockAdd2(long long c, long long s, unsigned long long* out, long long* red) {
    c = gpudb_warp_sum_i64(c);
    s = gpudb_warp_sum_i64(s);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) {
        red[2 * warp] = c;
        red[2 * warp + 1] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        long long tc = 0, ts = 0;
        for (int w = 0; w < nw; ++w) {
            tc += red[2 * w];
            ts += red[2 * w + 1];
        }
        if (tc) atomicAdd(out, (unsigned long long)tc);
        if (ts) gpudb_acc128_add(out + 1, ts);
    }
}

// Linear probing from slot `s`, whose key word `cur` is already loaded.
__device__ __forceinline__ long long slotFrom(Slot* ht, int log2cap, unsigned enc, unsigned long long s, unsigned cur,
                                              unsigned maxProbe, unsigned* err, bool* fresh) {
    const unsigned long long mask = (1ull << log2cap) - 1ull;
    for (unsigned p = 0; p < maxProbe; ++p) {
        if (p) cur = *((volatile unsigned*)&ht[s].key);
        if (cur == enc) return (long long)s;
        if (cur == 0u) {
            const unsigned prev = atomicCAS(&ht[s].key, 0u, enc);
            if (prev == 0u) {
                *fresh = true;
                return (long long)s;
            }
            if (prev == enc) return (long long)s;
        }
        s = (s + 1ull) & mask;
    }
    gpudb_set_error(err, GPUDB_ERR_HASH_OVERFLOW);
    return -1;
}

// Add (count, sum) to a group of the query's global table, starting from
// home slot `s0` whose key word `cur` is loaded; a group created here is
// appended to the slot list (one atomic per warp for the positions).
__device__ __forceinline__ void globalAddFrom(const QDesc& q, bool live, unsigned enc, unsigned long long s0,
                                              unsigned cur, unsigned long long c, unsigned long long v) {
    bool fresh = false;
    long long slot = -1;
    if (live) {
        slot = slotFrom(q.ht, q.log2cap, enc, s0, cur, (unsigned)q.maxProbe, q.err, &fresh);
        if (slot >= 0) {
            gpudb_red_add_u32(&q.ht[slot].count, (unsigned)c);
            gpudb_red_add_u64(&q.ht[slot].sum, v);
        }
    }
    const unsigned long long pos = gpudb_warp_reserve(q.nslots, fresh);
    if (fresh) q.slots[pos] = (unsigned)slot;
}

__device__ __forceinline__ void globalAdd(const QDesc& q, bool live, unsigned enc, unsigned long long c,
                                          unsigned long long v) {
    const unsigned long long s0 = gpudb_hash_slot((unsigned long long)enc, q.log2cap);
    const unsigned cur = live ? *((volatile unsigned*)&q.ht[s0].key) : 0u;
    globalAddFrom(q, live, enc, s0, cur, c, v);
}

// ---- JOIN build: bitmap of dim keys with attr < attr_lt -------------------
__global__ void __launch_bounds__(1024) kJoinBuild(const QDesc* __restrict__ qs, WorkList wl, long long tile, unsigned long long* counter) {
    __shared__ long long s_item;
    const long long total = __ldg(wl.prefix + wl.nq);
    for (long long w; (w = pullWork(counter, total, &s_item)) >= 0;) {
        const int qi = findQuery(wl, w);
        const QDesc& q = qs[__ldg(wl.q + qi)];
        const int* __restrict__ dk = q.dim_key;
        const int* __restrict__ da = q.dim_attr;
        unsigned* bm = q.bitmap;
        const long long words = q.bitmap_words;
        const int attrLt = q.attr_lt;
        const long long r0 = (w - __ldg(wl.prefix + qi)) * tile, r1 = min(q.dim_rows, r0 + tile);
        for (long long i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
            if (__ldcs(da + i) >= attrLt) continue;
            const long long k = __ldcs(dk + i);
            if (k >= 0 && (k >> 5) < words) gpudb_bitmap_set(bm, k);
            else gpudb_set_error(q.err, GPUDB_ERR_BOUNDS);
        }
    }
}

// ---- AGG / JOIN probe: filter [-> semi-join] -> count + sum ---------------
template <int U>
__global__ void __launch_bounds__(U == 4 ? 1024 : 512, U == 4 ? 1 : 4) kAgg(const QDesc* __restrict__ qs, WorkList wl, long long tile, unsigned long long* counter) {
    __shared__ long long s_item;
    __shared__ long long red[64];
    const long long total = __ldg(wl.prefix + wl.nq);
    for (long long w; (w = pullWork(counter, total, &s_item)) >= 0;) {
        const int qi = findQuery(wl, w);
        const QDesc& q = qs[__ldg(wl.q + qi)];
        const int* __restrict__ filter = q.filter;
        const long long* __restrict__ value = q.value;
        const int thr = q.thr;
        const long long r0 = (w - __ldg(wl.prefix + qi)) * tile, r1 = min(q.rows, r0 + tile);
        const long long step = (long long)blockDim.x;
        long long c = 0, s = 0;
        // the filter words of a thread's next U rows are loaded while
        // the current rows' dependent loads are in flight
        int fn[U];
        loadFilters(filter, r0 + threadIdx.x, step, r1, thr, fn);
        const bool dense = denseWarp(fn, thr);
        if (q.tmpl == GPUDB_TPL_JOIN && dense) {
            // most rows pass: fk and value ride along with the filter words
            const int* __restrict__ fk = q.fk;
            const unsigned* __restrict__ bm = q.bitmap;
            const long long words = q.bitmap_words;
            int kn[U];
            long long vn[U];
            loadAhead(fk, r0 + threadIdx.x, step, r1, kn);
            loadAhead(value, r0 + threadIdx.x, step, r1, vn);
            for (long long b = r0 + threadIdx.x; b < r1; b += U * step) {
                int f[U], key[U];
                long long v[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    f[u] = fn[u];
                    key[u] = kn[u];
                    v[u] = vn[u];
                }
                loadFilters(filter, b + U * step, step, r1, thr, fn);
                loadAhead(fk, b + U * step, step, r1, kn);
                loadAhead(value, b + U * step, step, r1, vn);
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const long long k = key[u];
                    if (f[u] < thr && k >= 0 && (k >> 5) < words && gpudb_bitmap_test(bm, k)) {
                        ++c;
                        s += v[u];
                    }
                }
            }
        } else if (q.tmpl == GPUDB_TPL_JOIN) {
            const int* __restrict__ fk = q.fk;
            const unsigned* __restrict__ bm = q.bitmap;
            const long long words = q.bitmap_words;
            for (long long b = r0 + threadIdx.x; b < r1; b += U * step) {
                int f[U];
#pragma unroll
                for (int u = 0; u < U; ++u) f[u] = fn[u];
                loadFilters(filter, b + U * step, step, r1, thr, fn);
                int key[U];
#pragma unroll
                for (int u = 0; u < U; ++u) key[u] = f[u] < thr ? __ldcs(fk + b + u * step) : -1;
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const long long k = key[u];
                    if (k >= 0 && (k >> 5) < words && gpudb_bitmap_test(bm, k)) {
                        ++c;
                        s += __ldcs(value + b + u * step);
                    }
                }
            }
        } else if (dense) {
            long long vn[U];
            loadAhead(value, r0 + threadIdx.x, step, r1, vn);
            for (long long b = r0 + threadIdx.x; b < r1; b += U * step) {
                int f[U];
                long long v[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    f[u] = fn[u];
                    v[u] = vn[u];
                }
                loadFilters(filter, b + U * step, step, r1, thr, fn);
                loadAhead(value, b + U * step, step, r1, vn);
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (f[u] < thr) {
                        ++c;
                        s += v[u];
                    }
            }
        } else {
            for (long long b = r0 + threadIdx.x; b < r1; b += U * step) {
                int f[U];
#pragma unroll
                for (int u = 0; u < U; ++u) f[u] = fn[u];
                loadFilters(filter, b + U * step, step, r1, thr, fn);
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (f[u] < thr) {
                        ++c;
                        s += __ldcs(value + b + u * step);
                    }
            }
        }
        blockAdd2(c, s, q.agg, red);
    }
}

// ---- GROUPBY / TOPK: filter -> key % card -> hash table (count, sum) -------
// Per query, the strategy the host picked from the expected group count and
// the sample's key repetition:
//   SHARED_DIRECT the CTA's shared table indexed by the key itself;
//   SHARED      warp aggregation, then the CTA's hashed shared table;
//   GLOBAL_WARP warp aggregation, then the global table;
//   GLOBAL      the global table directly.
// A CTA keeps its shared table across a query's work items and flushes it
// into the query's global table when it moves to another query or runs out
// of work. On the global path the home-slot key words of a thread's U rows
// are loaded together, so an existing group costs one L2 round trip per U
// rows, then fire-and-forget reductions. U = 1 row per thread at a
// 32-register cap (the default: every thread slot of the SM resident),
// U = 2 at 42 registers, U = 4 at 64 (U < 4: blocks of at most 512).
template <int U>
__global__ void __launch_bounds__(U == 4 ? 1024 : 512, U == 4 ? 1 : (U == 2 ? 3 : 4)) kGroup(const QDesc* __restrict__ qs, WorkList wl, long long tile,
                                               unsigned long long* counter) {
    __shared__ long long s_item;
    __shared__ unsigned sKey[kSmemSlots];
    __shared__ unsigned sCnt[kSmemSlots];
    __shared__ unsigned long long sSum[kSmemSlots];
    for (int i = threadIdx.x; i < kSmemSlots; i += blockDim.x) {
        sKey[i] = 0u;
        sCnt[i] = 0u;
        sSum[i] = 0ull;
    }
    volatile unsigned* vKey = sKey;
    const long long total = __ldg(wl.prefix + wl.nq);
    // the query whose groups the shared table holds (SHARED mode), -1 when
    // empty: the table is flushed into that query's global table only when
    // the CTA moves to another query's rows or runs out of work, so a query's
    // work items on one CTA share one table and one flush
    int heldQ = -1;
    auto flushShared = [&](const QDesc& q) {
        const bool direct = q.aggMode == GPUDB_AGG_SHARED_DIRECT;
        for (int i = threadIdx.x; i < kSmemSlots; i += blockDim.x) {
            // a direct slot i holds key i + 1 - card (encoded i + 1) once counted
            const unsigned k = direct ? (sCnt[i] ? (unsigned)i + 1u : 0u) : sKey[i];
            globalAdd(q, k != 0u, k, sCnt[i], sSum[i]);
            sKey[i] = 0u;
            sCnt[i] = 0u;
            sSum[i] = 0ull;
        }
    };
    for (long long w; (w = pullWork(counter, total, &s_item)) >= 0;) {
        const int qi = findQuery(wl, w);
        const int qd = __ldg(wl.q + qi);
        if (heldQ >= 0 && heldQ != qd) {
            // pullWork's barriers ordered every add of the held query before
            // this flush; the barrier after it orders the reset before the
            // next rows' adds
            flushShared(qs[heldQ]);
            heldQ = -1;
            __syncthreads();
        }
        const QDesc& q = qs[qd];
        const int* __restrict__ filter = q.filter;
        const int* __restrict__ keyc = q.key;
        const long long* __restrict__ value = q.value;
        const int thr = q.thr;
        const long long card = q.card;
        const int mode = q.aggMode;
        Slot* ht = q.ht;
        const int log2cap = q.log2cap;
        const long long r0 = (w - __ldg(wl.prefix + qi)) * tile, r1 = min(q.rows, r0 + tile);
        const long long step = (long long)blockDim.x;
        // (the dense-warp loads of kAgg measured no faster here: this
        // kernel's time goes to the aggregation, and the extra registers spill)
        int fn[U];
        loadFilters(filter, r0 + threadIdx.x, step, r1, thr, fn);
        for (long long b = r0 + threadIdx.x; b < r1; b += U * step) {
            int f[U], kr[U];
            long long v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) f[u] = fn[u];
            loadFilters(filter, b + U * step, step, r1, thr, fn);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const bool p = f[u] < thr;
                kr[u] = p ? __ldcs(keyc + b + u * step) : 0;
                v[u] = p ? __ldcs(value + b + u * step) : 0;
            }
            unsigned enc[U];
            bool live[U];
            unsigned c[U];  // rows a lane adds for its group: at most a warp's
            unsigned long long val[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                live[u] = f[u] < thr;
                enc[u] = live[u] ? encKey(keyMod(kr[u], q), card) : 0u;
                c[u] = 1u;
                val[u] = (unsigned long long)v[u];
            }
            if (mode == GPUDB_AGG_SHARED_DIRECT) {
                // keys in (-card, card): enc - 1 in [0, 2 card - 1) indexes
                // the table directly, no probing and no warp aggregation
                // (same-slot lanes of one warp serialise in the shared
                // atomic unit, cheaper than a match and two peer sums)
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (!live[u]) continue;
                    gpudb_red_add_shared_u32(&sCnt[enc[u] - 1u], 1u);
                    gpudb_red_add_shared_u64(&sSum[enc[u] - 1u], val[u]);
                }
                continue;
            }
            if (mode == GPUDB_AGG_GLOBAL_WARP || (mode == GPUDB_AGG_SHARED && q.sharedWarp)) {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (!live[u]) continue;
                    const unsigned am = __activemask();
                    const unsigned peers = __match_any_sync(am, enc[u]);
                    c[u] = (unsigned)__popc(peers);  // every peer is one live row
                    val[u] = gpudb_peer_sum(am, peers, val[u]);
                    live[u] = (int)(threadIdx.x & 31u) == __ffs(peers) - 1;
                }
            }
            if (mode == GPUDB_AGG_SHARED) {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (!live[u]) continue;
                    unsigned h = (unsigned)gpudb_hash_slot((unsigned long long)enc[u], 11);
                    bool done = false;
#pragma unroll 1
                    for (int p = 0; p < kSmemProbe; ++p) {
                        unsigned cur = vKey[h];
                        if (cur == 0u) cur = atomicCAS(&sKey[h], 0u, enc[u]) == 0u ? enc[u] : vKey[h];
                        if (cur == enc[u]) {
                            gpudb_red_add_shared_u32(&sCnt[h], c[u]);
                            gpudb_red_add_shared_u64(&sSum[h], val[u]);
                            done = true;
                            break;
                        }
                        h = (h + 1u) & (kSmemSlots - 1);
                    }
                    // (spills one at a time: batching their home-slot loads
                    // as the global path does measured slower, its extra
                    // registers spilling)
                    if (!done) globalAdd(q, true, enc[u], c[u], val[u]);
                }
            } else {
                unsigned long long s0[U];
                unsigned cur[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    s0[u] = gpudb_hash_slot((unsigned long long)enc[u], log2cap);
                    cur[u] = live[u] ? *((volatile unsigned*)&ht[s0[u]].key) : 0u;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (live[u] && cur[u] == enc[u]) {  // the group exists in its home slot
                        gpudb_red_add_u32(&ht[s0[u]].count, c[u]);
                        gpudb_red_add_u64(&ht[s0[u]].sum, val[u]);
                        live[u] = false;
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) globalAddFrom(q, live[u], enc[u], s0[u], cur[u], c[u], val[u]);
            }
        }
        if (mode == GPUDB_AGG_SHARED || mode == GPUDB_AGG_SHARED_DIRECT) heldQ = qd;
    }
    // pullWork's barriers ordered the last adds before this flush
    if (heldQ >= 0) flushShared(qs[heldQ]);
}

// Block-wide merge of per-thread sorted lists; warp 0 receives the result.
__device__ __forceinline__ void blockTopK(long long (&vv)[kTopK], long long (&kk)[kTopK], long long* sv, long long* sk,
                                          long long (&ov)[kTopK], long long (&ok)[kTopK]) {
    long long wv[kTopK], wk[kTopK];
    gpudb_topk_warp_merge<kTopK>(vv, kk, wv, wk);
    __syncthreads();
    if ((threadIdx.x & 31u) == 0u)
        for (int i = 0; i < kTopK; ++i) {
            sv[(threadIdx.x >> 5) * kTopK + i] = wv[i];
            sk[(threadIdx.x >> 5) * kTopK + i] = wk[i];
        }
    __syncthreads();
    if (threadIdx.x < 32u) {
#pragma unroll
        for (int i = 0; i < kTopK; ++i) {
            vv[i] = GPUDB_TOPK_NONE_VAL;
            kk[i] = GPUDB_TOPK_NONE_KEY;
        }
        for (int e = threadIdx.x; e < (int)(blockDim.x >> 5) * kTopK; e += 32) gpudb_topk_push<kTopK>(vv, kk, sv[e], sk[e]);
        gpudb_topk_warp_merge<kTopK>(vv, kk, ov, ok);
    }
}

// ---- TOPK, pass 1: per chunk of the slot list, the best kTopK groups -------
__global__ void __launch_bounds__(256) kTopKChunks(const QDesc* __restrict__ qs, WorkList wl,
                                                   unsigned long long* counter) {
    __shared__ long long s_item;
    __shared__ long long sv[8 * kTopK], sk[8 * kTopK];
    const long long total = __ldg(wl.prefix + wl.nq);
    for (long long w; (w = pullWork(counter, total, &s_item)) >= 0;) {
        const int qi = findQuery(wl, w);
        const QDesc& q = qs[__ldg(wl.q + qi)];
        const long long c = w - __ldg(wl.prefix + qi);
        const long long n = (long long)*q.nslots;
        const long long j0 = c * kTkChunk, j1 = min(n, j0 + kTkChunk);
        if (j0 >= n) continue;  // chunk past the groups this query created
        long long vv[kTopK], kk[kTopK];
#pragma unroll
        for (int i = 0; i < kTopK; ++i) {
            vv[i] = GPUDB_TOPK_NONE_VAL;
            kk[i] = GPUDB_TOPK_NONE_KEY;
        }
        for (long long j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
            const Slot& s = q.ht[q.slots[j]];
            gpudb_topk_push<kTopK>(vv, kk, (long long)s.sum, decKey(s.key, q.card));
        }
        long long ov[kTopK], ok[kTopK];
        blockTopK(vv, kk, sv, sk, ov, ok);
        if (threadIdx.x == 0) {
            long long* dst = q.tk_part + 2 * kTopK * c;
            for (int i = 0; i < kTopK; ++i) {
                dst[2 * i] = ov[i];
                dst[2 * i + 1] = ok[i];
            }
        }
    }
}

// ---- TOPK, pass 2: one CTA per query merges its chunks' lists --------------
__global__ void __launch_bounds__(256) kTopKMerge(const QDesc* __restrict__ qs, const int* __restrict__ qlist) {
    __shared__ long long sv[8 * kTopK], sk[8 * kTopK];
    const QDesc& q = qs[qlist[blockIdx.x]];
    const long long n = (long long)*q.nslots;
    const long long chunks = min(q.tk_chunks, (n + kTkChunk - 1) / kTkChunk);
    long long vv[kTopK], kk[kTopK];
#pragma unroll
    for (int i = 0; i < kTopK; ++i) {
        vv[i] = GPUDB_TOPK_NONE_VAL;
        kk[i] = GPUDB_TOPK_NONE_KEY;
    }
    for (long long e = threadIdx.x; e < chunks * kTopK; e += blockDim.x)
        gpudb_topk_push<kTopK>(vv, kk, q.tk_part[2 * e], q.tk_part[2 * e + 1]);
    long long ov[kTopK], ok[kTopK];
    blockTopK(vv, kk, sv, sk, ov, ok);
    if (threadIdx.x == 0) {
        const long long m = min((long long)q.k, n);
        for (long long i = 0; i < m; ++i) {
            q.topk_out[2 * i] = ok[i];
            q.topk_out[2 * i + 1] = ov[i];
        }
        *q.topk_n = (unsigned long long)m;
    }
}

// ---- exact statistics: passing rows and distinct keys ----------------------
__global__ void __launch_bounds__(1024) kStats(const QDesc* __restrict__ qs, WorkList wl, long long tile, unsigned long long* counter) {
    __shared__ long long s_item;
    const long long total = __ldg(wl.prefix + wl.nq);
    for (long long w; (w = pullWork(counter, total, &s_item)) >= 0;) {
        const int qi = findQuery(wl, w);
        const QDesc& q = qs[__ldg(wl.q + qi)];
        const int* __restrict__ filter = q.filter;
        const int* __restrict__ keyc = q.key;
        const int thr = q.thr;
                unsigned* bm = q.st_bitmap;
        const long long words = q.st_words;
        const long long r0 = (w - __ldg(wl.prefix + qi)) * tile, r1 = min(q.rows, r0 + tile);
        const bool grouped = q.tmpl == GPUDB_TPL_GROUPBY || q.tmpl == GPUDB_TPL_TOPK;
        const long long step = (long long)blockDim.x;
        long long pass = 0, fresh = 0;
        for (long long b = r0 + threadIdx.x; b < r1; b += kUnroll * step) {
            int f[kUnroll], kr[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) f[u] = b + u * step < r1 ? __ldcs(filter + b + u * step) : thr;
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) kr[u] = (grouped && f[u] < thr) ? __ldcs(keyc + b + u * step) : 0;
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) {
                if (f[u] >= thr) continue;
                ++pass;
                if (!grouped) continue;
                const long long k = keyMod(kr[u], q);
                const long long wd = k >> 5;
                const unsigned bit = 1u << (unsigned)(k & 31);
                if (k < 0 || wd >= words) {
                    gpudb_set_error(q.err, GPUDB_ERR_BOUNDS);
                    continue;
                }
                if ((bm[wd] & bit) == 0u && (atomicOr(bm + wd, bit) & bit) == 0u) ++fresh;
            }
        }
        pass = gpudb_warp_sum_i64(pass);
        fresh = gpudb_warp_sum_i64(fresh);
        if ((threadIdx.x & 31) == 0) {
            if (pass) atomicAdd(q.st_pass, (unsigned long long)pass);
            if (fresh) atomicAdd(q.st_distinct, (unsigned long long)fresh);
        }
    }
}

// ---- 4096-row feature sample: one CTA per query ----------------------------
// Evenly spaced rows of the slice: rows sampled, rows passing the filter,
// distinct group keys among them and the multiplicity of the most frequent
// key (the skew signal that picks the aggregation strategy).
constexpr int kSample = 4096, kSampleSlots = 8192;
constexpr int kSampleSmem = kSampleSlots * (8 + 4);
__global__ void kSampleStats(const QDesc* __restrict__ qs, unsigned long long* out /* [n][4] */) {
    extern __shared__ unsigned long long setKeys[];
    unsigned* setCnt = reinterpret_cast<unsigned*>(setKeys + kSampleSlots);
    __shared__ unsigned long long s_pass, s_distinct;
    __shared__ unsigned s_top;
    const QDesc& q = qs[blockIdx.x];
    for (int i = threadIdx.x; i < kSampleSlots; i += blockDim.x) {
        setKeys[i] = GPUDB_EMPTY64;
        setCnt[i] = 0u;
    }
    if (threadIdx.x == 0) {
        s_pass = 0;
        s_distinct = 0;
        s_top = 0;
    }
    __syncthreads();
    const long long m = q.rows < kSample ? q.rows : kSample;
    const bool grouped = q.tmpl == GPUDB_TPL_GROUPBY || q.tmpl == GPUDB_TPL_TOPK;
    for (long long j = threadIdx.x; j < m; j += blockDim.x) {
        const long long r = (j * q.rows) / m;  // evenly spaced rows of the slice
        if (q.filter[r] >= q.thr) continue;
        atomicAdd(&s_pass, 1ull);
        if (!grouped) continue;
        const unsigned long long k = (unsigned long long)keyMod(q.key[r], q);
        unsigned h = (unsigned)gpudb_hash_slot(k, 13);
        for (int p = 0; p < kSampleSlots; ++p) {
            const unsigned long long cur = setKeys[h];
            bool mine = cur == k;
            if (cur == GPUDB_EMPTY64) {
                const unsigned long long prev = atomicCAS(setKeys + h, GPUDB_EMPTY64, k);
                if (prev == GPUDB_EMPTY64) atomicAdd(&s_distinct, 1ull);
                mine = prev == GPUDB_EMPTY64 || prev == k;
            }
            if (mine) {
                atomicAdd(setCnt + h, 1u);
                break;
            }
            h = (h + 1) & (kSampleSlots - 1);
        }
    }
    __syncthreads();
    unsigned top = 0;
    for (int i = threadIdx.x; i < kSampleSlots; i += blockDim.x) top = max(top, setCnt[i]);
    for (int o = 16; o > 0; o >>= 1) top = max(top, __shfl_xor_sync(0xffffffffu, top, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&s_top, top);
    __syncthreads();
    if (threadIdx.x == 0) {
        out[4 * blockIdx.x] = (unsigned long long)m;
        out[4 * blockIdx.x + 1] = s_pass;
        out[4 * blockIdx.x + 2] = s_distinct;
        out[4 * blockIdx.x + 3] = s_top;
    }
}

// ---- collect: per-query result rows and their exclusive prefix (one CTA) ---
__global__ void kResultRows(const QDesc* __restrict__ qs, int n, unsigned long long* rows, unsigned long long* offs) {
    __shared__ unsigned long long carry;
    __shared__ unsigned long long wsum[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + threadIdx.x;
        unsigned long long r = 0;
        if (i < n) {
            const QDesc& q = qs[i];
            r = q.tmpl == GPUDB_TPL_GROUPBY ? *q.nslots : q.tmpl == GPUDB_TPL_TOPK ? *q.topk_n : 1ull;
            rows[i] = r;
        }
        unsigned long long x = r;  // inclusive warp scan
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
            if ((int)(threadIdx.x & 31) >= o) x += y;
        }
        if ((threadIdx.x & 31) == 31) wsum[threadIdx.x >> 5] = x;
        __syncthreads();
        unsigned long long before = carry;
        for (int w = 0; w < (int)(threadIdx.x >> 5); ++w) before += wsum[w];
        if (i < n) offs[i] = before + x - r;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = before + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) offs[n] = carry;
}

// ---- collect: compaction of every query's rows into one packed buffer ------
__global__ void kCollect(const QDesc* __restrict__ qs, WorkList wl, long long chunk, unsigned long long* counter,
                         const unsigned long long* __restrict__ offs, long long* __restrict__ out) {
    __shared__ long long s_item;
    const long long total = __ldg(wl.prefix + wl.nq);
    for (long long w; (w = pullWork(counter, total, &s_item)) >= 0;) {
        const int qi = findQuery(wl, w);
        const int id = __ldg(wl.q + qi);
        const QDesc& q = qs[id];
        long long* dst = out + 3 * (long long)offs[id];
        const long long c = w - __ldg(wl.prefix + qi);
        if (q.tmpl == GPUDB_TPL_AGG || q.tmpl == GPUDB_TPL_JOIN) {
            if (threadIdx.x == 0) {
                dst[0] = (long long)q.agg[0];
                // exact 128-bit sum = (int64)w1 * 2^32 + w0, split into (lo, hi)
                const __int128 s = (__int128)(long long)q.agg[2] * ((__int128)1 << 32) + (__int128)q.agg[1];
                dst[1] = (long long)(unsigned long long)s;
                dst[2] = (long long)(s >> 64);
            }
        } else if (q.tmpl == GPUDB_TPL_TOPK) {
            const long long m = (long long)*q.topk_n;
            for (long long i = threadIdx.x; i < m; i += blockDim.x) {
                dst[3 * i] = q.topk_out[2 * i];
                dst[3 * i + 1] = q.topk_out[2 * i + 1];
                dst[3 * i + 2] = 0;
            }
        } else {
            const long long n = (long long)*q.nslots;
            const long long j1 = min(n, (c + 1) * chunk);
            for (long long j = c * chunk + threadIdx.x; j < j1; j += blockDim.x) {
                const Slot& s = q.ht[q.slots[j]];
                dst[3 * j] = decKey(s.key, q.card);
                dst[3 * j + 1] = (long long)s.count;
                dst[3 * j + 2] = (long long)s.sum;
            }
        }
    }
}

unsigned long long pow2ceil(unsigned long long v) {
    unsigned long long p = 16;
    while (p < v) p <<= 1;
    return p;
}
int log2u(unsigned long long v) {
    int l = 0;
    while ((1ull << l) < v) l++;
    return l;
}
bool grouped(int tmpl) { return tmpl == GPUDB_TPL_GROUPBY || tmpl == GPUDB_TPL_TOPK; }

#define B_CHECK(call, code)                                                                        \
    do {                                                                                           \
        const cudaError_t _e = (call);                                                             \
        if (_e != cudaSuccess) {                                                                   \
            gpudb::setThreadError(std::string("batch: ") + #call + ": " + cudaGetErrorString(_e)); \
            return code;                                                                           \
        }                                                                                          \
    } while (0)

// Grow-only device buffer from the stream-ordered pool allocator: growing
// it never synchronises the device (cudaFree would), so batches of other
// streams keep running while this one resizes; 25 % headroom on growth.
struct DeviceBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int reserve(size_t want, cudaStream_t st) {
        if (want <= bytes) return GPUDB_OK;
        release(st);
        const size_t cap = want + want / 4 + 256;
        B_CHECK(cudaMallocAsync(&p, cap, st), GPUDB_E_ALLOC);
        bytes = cap;
        return GPUDB_OK;
    }
    void release(cudaStream_t st) {
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
        bytes = 0;
    }
};

size_t al256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

struct gpudb_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    int numSMs = 148;
    int block = 512, maxProbe = 128, warpAgg = 1;
    // rows in flight per thread of the group-by kernel: 1 (measured fastest
    // on the mixed batch: its latency-bound aggregation gains more from
    // twice the resident threads than it loses to a few spilled
    // registers), 2 or 4
    int groupRows = 1;
    int sharedWarp = 1;  // SHARED strategy: warp aggregation before the shared table (1) or not (0)
    // rows in flight per thread of the agg / join kernel: 2 (32 registers,
    // every thread slot resident; measured 9.9 ms against 10.6 ms per
    // mixed batch) or 4 (64 registers)
    int aggRows = 2;
    long long tile = 32768;  // rows per work item (measured: 16K 5.31k, 32K 5.45k mixed queries/s)
    std::vector<gpudb_batch_query> queries;
    std::vector<QDesc> desc;
    DeviceBuf arena;  // zero-initialised per execution
    size_t zeroBytes = 0;
    DeviceBuf scratch;  // never initialised: slot lists, top-k partials
    DeviceBuf meta;     // descriptors + work lists
    DeviceBuf stats, sample, collect;
    QDesc* dDesc = nullptr;
    WorkList wlBuild{}, wlAgg{}, wlGroup{}, wlTopk{}, wlStats{}, wlCollect{};
    int* dTopk = nullptr;
    int nTopk = 0;
    long long collectChunk = 1 << 16;
    unsigned long long* counters = nullptr;  // work counters (first words of the arena)
    unsigned* errHost = nullptr;             // pinned, one word per query
    size_t errCap = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graphExec = nullptr;
    bool dirty = true;
    long long lastLaunches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t evStage[GPUDB_BATCH_STAGES + 1] = {};
    double stageMs[GPUDB_BATCH_STAGES] = {};
    bool stagesValid = false;
};

namespace {

void dropGraph(gpudb_batch* b) {
    if (b->graphExec) cudaGraphExecDestroy(b->graphExec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->graphExec = nullptr;
    b->graph = nullptr;
}

// Lay out the arena and the work lists for the current queries.
int plan(gpudb_batch* b) {
    const int n = (int)b->queries.size();
    size_t z = al256(8 * 8);  // work counters
    size_t sc = 0;
    std::vector<size_t> zOff(n), sOff(n);
    std::vector<unsigned long long> caps(n, 0);
    std::vector<long long> tkChunks(n, 0);
    for (int i = 0; i < n; i++) {
        const auto& q = b->queries[i];
        zOff[i] = z;
        z += 64;  // agg[3], topk_n, nslots, err
        if (q.tmpl == GPUDB_TPL_JOIN) z += 4 * ((size_t)q.dim_max_key / 32 + 1);
        if (grouped(q.tmpl)) {
            caps[i] = pow2ceil(2 * std::max<uint64_t>(q.groups, 1));
            z = al256(z);
            z += sizeof(Slot) * caps[i];
            sOff[i] = sc;
            sc += al256(4 * caps[i]);
            if (q.tmpl == GPUDB_TPL_TOPK) {
                tkChunks[i] = (long long)((caps[i] + kTkChunk - 1) / kTkChunk);
                sc += al256(16 * kTopK * (size_t)tkChunks[i] + 16 * kTopK);
            }
        }
        z = al256(z);
    }
    if (int st = b->arena.reserve(z, b->stream)) return st;
    if (int st = b->scratch.reserve(std::max<size_t>(sc, 256), b->stream)) return st;
    b->zeroBytes = z;
    char* zb = static_cast<char*>(b->arena.p);
    char* sb = static_cast<char*>(b->scratch.p);
    b->counters = reinterpret_cast<unsigned long long*>(zb);
    b->desc.assign(n, QDesc{});
    std::vector<int> lBuild, lAgg, lGroup, lTopk, lAll(n), lCollect;
    std::vector<long long> pBuild{0}, pAgg{0}, pGroup{0}, pTopk{0}, pAll{0}, pCollect{0};
    for (int i = 0; i < n; i++) {
        const auto& q = b->queries[i];
        QDesc& d = b->desc[i];
        d.tmpl = q.tmpl;
        d.thr = q.thr;
        d.k = q.k;
        d.attr_lt = q.attr_lt;
        d.card = q.card > 0 ? q.card : 1;
        cardDivisor(d.card, &d.cardMagic, &d.cardSh1, &d.cardSh2);
        d.rows = (long long)q.rows;
        d.key = q.key;
        d.filter = q.filter;
        d.value = reinterpret_cast<const long long*>(q.value);
        d.fk = q.fk;
        d.dim_key = q.dim_key;
        d.dim_attr = q.dim_attr;
        d.dim_rows = (long long)q.dim_rows;
        d.maxProbe = b->maxProbe;
        // aggregation strategy: the caller's choice, else the shared-memory
        // table (with spill to the global one), which is never far off
        d.aggMode = q.agg_mode != GPUDB_AGG_AUTO ? q.agg_mode : GPUDB_AGG_SHARED;
        if (!b->warpAgg && d.aggMode == GPUDB_AGG_GLOBAL_WARP) d.aggMode = GPUDB_AGG_GLOBAL;
        // the direct table holds the 2 card - 1 encoded keys of (-card, card)
        if (d.aggMode == GPUDB_AGG_SHARED_DIRECT && 2 * d.card - 1 > kSmemSlots) d.aggMode = GPUDB_AGG_SHARED;
        d.sharedWarp = b->sharedWarp;
        char* p = zb + zOff[i];
        d.agg = reinterpret_cast<unsigned long long*>(p);
        d.topk_n = d.agg + 3;
        d.nslots = d.agg + 4;
        d.err = reinterpret_cast<unsigned*>(p + 40);
        p += 64;
        if (q.tmpl == GPUDB_TPL_JOIN) {
            d.bitmap = reinterpret_cast<unsigned*>(p);
            d.bitmap_words = q.dim_max_key / 32 + 1;
            p += 4 * (size_t)d.bitmap_words;
        }
        if (grouped(q.tmpl)) {
            p = zb + al256((size_t)(p - zb));
            d.ht = reinterpret_cast<Slot*>(p);
            d.log2cap = log2u(caps[i]);
            d.slots = reinterpret_cast<unsigned*>(sb + sOff[i]);
            if (q.tmpl == GPUDB_TPL_TOPK) {
                d.tk_part = reinterpret_cast<long long*>(sb + sOff[i] + al256(4 * caps[i]));
                d.tk_chunks = tkChunks[i];
                d.topk_out = d.tk_part + 2 * kTopK * tkChunks[i];
            }
        }
        const long long tiles = (d.rows + b->tile - 1) / b->tile;
        lAll[i] = i;
        pAll.push_back(pAll.back() + tiles);
        if (q.tmpl == GPUDB_TPL_JOIN) {
            lBuild.push_back(i);
            pBuild.push_back(pBuild.back() + (d.dim_rows + b->tile - 1) / b->tile);
        }
        if (q.tmpl == GPUDB_TPL_AGG || q.tmpl == GPUDB_TPL_JOIN) {
            lAgg.push_back(i);
            pAgg.push_back(pAgg.back() + tiles);
        }
        if (grouped(q.tmpl)) {
            lGroup.push_back(i);
            pGroup.push_back(pGroup.back() + tiles);
        }
        if (q.tmpl == GPUDB_TPL_TOPK) {
            lTopk.push_back(i);
            pTopk.push_back(pTopk.back() + tkChunks[i]);
        }
        lCollect.push_back(i);
        const long long cchunks = q.tmpl == GPUDB_TPL_GROUPBY
                                      ? (long long)((caps[i] + b->collectChunk - 1) / b->collectChunk)
                                      : 1;
        pCollect.push_back(pCollect.back() + std::max<long long>(1, cchunks));
    }
    std::vector<char> host;
    auto put = [&](const void* src, size_t bytes) {
        const size_t off = al256(host.size());
        host.resize(off + std::max<size_t>(bytes, 8));
        if (bytes) std::memcpy(host.data() + off, src, bytes);
        return off;
    };
    const size_t oDesc = put(b->desc.data(), sizeof(QDesc) * n);
    auto putList = [&](const std::vector<int>& l, const std::vector<long long>& pf) {
        const size_t a = put(l.data(), 4 * l.size());
        const size_t c = put(pf.data(), 8 * pf.size());
        return std::make_pair(a, c);
    };
    const auto oB = putList(lBuild, pBuild), oA = putList(lAgg, pAgg), oG = putList(lGroup, pGroup),
               oT = putList(lTopk, pTopk), oS = putList(lAll, pAll), oC = putList(lCollect, pCollect);
    if (int st = b->meta.reserve(host.size(), b->stream)) return st;
    B_CHECK(cudaMemcpyAsync(b->meta.p, host.data(), host.size(), cudaMemcpyHostToDevice, b->stream), GPUDB_E_CUDA);
    char* m = static_cast<char*>(b->meta.p);
    auto wl = [&](std::pair<size_t, size_t> o, size_t nq) {
        return WorkList{reinterpret_cast<int*>(m + o.first), reinterpret_cast<long long*>(m + o.second), (int)nq};
    };
    b->dDesc = reinterpret_cast<QDesc*>(m + oDesc);
    b->wlBuild = wl(oB, lBuild.size());
    b->wlAgg = wl(oA, lAgg.size());
    b->wlGroup = wl(oG, lGroup.size());
    b->wlTopk = wl(oT, lTopk.size());
    b->wlStats = wl(oS, n);
    b->wlCollect = wl(oC, lCollect.size());
    b->dTopk = reinterpret_cast<int*>(m + oT.first);
    b->nTopk = (int)lTopk.size();
    if ((size_t)n > b->errCap) {
        if (b->errHost) cudaFreeHost(b->errHost);
        b->errHost = nullptr;
        b->errCap = 0;
        const size_t cap = std::max<size_t>(4096, 2 * (size_t)n);
        B_CHECK(cudaHostAlloc((void**)&b->errHost, sizeof(unsigned) * cap, cudaHostAllocDefault), GPUDB_E_ALLOC);
        b->errCap = cap;
    }
    B_CHECK(cudaStreamSynchronize(b->stream), GPUDB_E_CUDA);
    dropGraph(b);
    b->dirty = false;
    return GPUDB_OK;
}

int gridFor(gpudb_batch* b, const void* fn, int block) {
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, block, 0);
    return std::max(1, occ) * b->numSMs;
}

// Enqueue the memset + kernels of one execution on b->stream; with `stages`
// an event follows every step (not inside a graph capture).
int enqueue(gpudb_batch* b, bool stages) {
    const int n = (int)b->queries.size();
    long long launches = 0;
    auto mark = [&](int i) { if (stages) cudaEventRecord(b->evStage[i], b->stream); };
    mark(0);
    B_CHECK(cudaMemsetAsync(b->arena.p, 0, b->zeroBytes, b->stream), GPUDB_E_CUDA);
    mark(1);
    if (b->wlBuild.nq) {
        kJoinBuild<<<gridFor(b, (const void*)kJoinBuild, b->block), b->block, 0, b->stream>>>(b->dDesc, b->wlBuild,
                                                                                              b->tile, b->counters + 0);
        launches++;
    }
    mark(2);
    if (b->wlAgg.nq) {
        if (b->aggRows == 2 && b->block <= 512)  // the 2-row form is built for blocks of <= 512
            kAgg<2><<<gridFor(b, (const void*)kAgg<2>, b->block), b->block, 0, b->stream>>>(
                b->dDesc, b->wlAgg, b->tile, b->counters + 1);
        else
            kAgg<4><<<gridFor(b, (const void*)kAgg<4>, b->block), b->block, 0, b->stream>>>(
                b->dDesc, b->wlAgg, b->tile, b->counters + 1);
        launches++;
    }
    mark(3);
    if (b->wlGroup.nq) {
        // the 1- and 2-row forms are built for blocks of at most 512 threads
        if (b->groupRows == 2 && b->block <= 512)
            kGroup<2><<<gridFor(b, (const void*)kGroup<2>, b->block), b->block, 0, b->stream>>>(
                b->dDesc, b->wlGroup, b->tile, b->counters + 2);
        else if (b->groupRows == 1 && b->block <= 512)
            kGroup<1><<<gridFor(b, (const void*)kGroup<1>, b->block), b->block, 0, b->stream>>>(
                b->dDesc, b->wlGroup, b->tile, b->counters + 2);
        else
            kGroup<4><<<gridFor(b, (const void*)kGroup<4>, b->block), b->block, 0, b->stream>>>(
                b->dDesc, b->wlGroup, b->tile, b->counters + 2);
        launches++;
    }
    mark(4);
    if (b->nTopk) {
        kTopKChunks<<<gridFor(b, (const void*)kTopKChunks, 256), 256, 0, b->stream>>>(b->dDesc, b->wlTopk,
                                                                                      b->counters + 3);
        mark(5);
        kTopKMerge<<<b->nTopk, 256, 0, b->stream>>>(b->dDesc, b->dTopk);
        launches += 2;
    } else {
        mark(5);
    }
    mark(6);
    B_CHECK(cudaGetLastError(), GPUDB_E_LAUNCH);
    // per-query error words -> pinned host copy
    for (int i = 0; i < n; i++)
        B_CHECK(cudaMemcpyAsync(b->errHost + i, b->desc[i].err, sizeof(unsigned), cudaMemcpyDeviceToHost, b->stream),
                GPUDB_E_CUDA);
    b->lastLaunches = launches;
    return GPUDB_OK;
}

float elapsed(gpudb_batch* b) {
    float t = 0;
    cudaEventElapsedTime(&t, b->ev0, b->ev1);
    return t;
}

// Zone-map statistics of a resident column: min and max of n int32 or
// int64 values (the sizer's column features). One grid-stride pass, warp
// shuffle reduction, one signed 64-bit atomicMin / atomicMax per warp.
template <typename T>
__global__ void __launch_bounds__(256) kColumnMinMax(const T* __restrict__ v, unsigned long long n,
                                                     long long* __restrict__ out) {
    long long lo = LLONG_MAX, hi = LLONG_MIN;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const long long x = (long long)__ldcs(v + i);
        lo = x < lo ? x : lo;
        hi = x > hi ? x : hi;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const long long a = __shfl_xor_sync(0xffffffffu, lo, o), b = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if ((threadIdx.x & 31u) == 0u) {
        atomicMin(out, lo);
        atomicMax(out + 1, hi);
    }
}

}  // namespace

extern "C" {

int gpudb_batch_create(gpudb_ctx* ctx, gpudb_batch** out) {
    if (!out) return GPUDB_E_INVALID;
    *out = nullptr;
    (void)ctx;  // the batch runs on the calling thread's current device
    auto b = std::make_unique<gpudb_batch>();
    int dev = 0;
    B_CHECK(cudaGetDevice(&dev), GPUDB_E_NOGPU);
    b->device = dev;
    B_CHECK(cudaDeviceGetAttribute(&b->numSMs, cudaDevAttrMultiProcessorCount, dev), GPUDB_E_CUDA);
    B_CHECK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), GPUDB_E_CUDA);
    B_CHECK(cudaEventCreate(&b->ev0), GPUDB_E_CUDA);
    B_CHECK(cudaEventCreate(&b->ev1), GPUDB_E_CUDA);
    for (auto& e : b->evStage) B_CHECK(cudaEventCreate(&e), GPUDB_E_CUDA);
    B_CHECK(cudaFuncSetAttribute(kSampleStats, cudaFuncAttributeMaxDynamicSharedMemorySize, kSampleSmem),
            GPUDB_E_LAUNCH);
    *out = b.release();
    return GPUDB_OK;
}

void gpudb_batch_free(gpudb_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    dropGraph(b);
    for (DeviceBuf* d : {&b->arena, &b->scratch, &b->meta, &b->stats, &b->sample, &b->collect}) d->release(b->stream);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->errHost) cudaFreeHost(b->errHost);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    for (auto& e : b->evStage)
        if (e) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int gpudb_batch_set_queries(gpudb_batch* b, const gpudb_batch_query* q, int n) {
    if (!b || (n > 0 && !q) || n < 0) return GPUDB_E_INVALID;
    for (int i = 0; i < n; i++) {
        const auto& x = q[i];
        const std::string who = "batch: query " + std::to_string(i);
        if (x.tmpl < 0 || x.tmpl > GPUDB_TPL_TOPK || (x.rows && (!x.filter || !x.value))) {
            gpudb::setThreadError(who + " is malformed");
            return GPUDB_E_INVALID;
        }
        if (grouped(x.tmpl) && ((x.rows && !x.key) || x.card < 1 || x.card >= (1ll << 31) || x.rows >= (1ull << 32))) {
            gpudb::setThreadError(who + " needs a key column, 1 <= card < 2^31 and fewer than 2^32 rows");
            return GPUDB_E_INVALID;
        }
        if (grouped(x.tmpl) && x.groups > (1ull << 30)) {
            gpudb::setThreadError(who + " asks for more than 2^30 groups");
            return GPUDB_E_INVALID;
        }
        if (x.agg_mode < GPUDB_AGG_AUTO || x.agg_mode > GPUDB_AGG_SHARED_DIRECT) {
            gpudb::setThreadError(who + " has an unknown agg_mode");
            return GPUDB_E_INVALID;
        }
        if (x.tmpl == GPUDB_TPL_TOPK && (x.k < 1 || x.k > kTopK)) {
            gpudb::setThreadError(who + " needs 1 <= k <= 16");
            return GPUDB_E_INVALID;
        }
        if (x.tmpl == GPUDB_TPL_JOIN &&
            ((x.rows && !x.fk) || (x.dim_rows && (!x.dim_key || !x.dim_attr)) || x.dim_max_key < 0)) {
            gpudb::setThreadError(who + " needs fk, the dim columns and dim_max_key >= 0");
            return GPUDB_E_INVALID;
        }
    }
    cudaSetDevice(b->device);
    b->queries.assign(q, q + n);
    b->dirty = true;
    return plan(b);
}

int gpudb_batch_set_groups(gpudb_batch* b, int qi, uint64_t groups) {
    if (!b || qi < 0 || qi >= (int)b->queries.size() || groups > (1ull << 30)) return GPUDB_E_INVALID;
    if (b->queries[qi].groups != groups) {
        b->queries[qi].groups = groups;
        b->dirty = true;
    }
    return GPUDB_OK;
}

int gpudb_batch_set_agg_mode(gpudb_batch* b, int qi, int mode) {
    if (!b || qi < 0 || qi >= (int)b->queries.size() || mode < GPUDB_AGG_AUTO || mode > GPUDB_AGG_SHARED_DIRECT)
        return GPUDB_E_INVALID;
    if (b->queries[qi].agg_mode != mode) {
        b->queries[qi].agg_mode = mode;
        b->dirty = true;
    }
    return GPUDB_OK;
}

int gpudb_batch_set_option(gpudb_batch* b, const char* name, long long value) {
    if (!b || !name) return GPUDB_E_INVALID;
    const std::string n(name);
    if (n == "group_rows") {
        if (value != 1 && value != 2 && value != 4) {
            gpudb::setThreadError("group_rows must be 1, 2 or 4");
            return GPUDB_E_INVALID;
        }
        b->groupRows = (int)value;
        b->dirty = true;
        return GPUDB_OK;
    }
    if (n == "shared_warp") {
        if (value != 0 && value != 1) {
            gpudb::setThreadError("shared_warp must be 0 or 1");
            return GPUDB_E_INVALID;
        }
        b->sharedWarp = (int)value;
        b->dirty = true;
        return GPUDB_OK;
    }
    if (n == "agg_rows") {
        if (value != 2 && value != 4) {
            gpudb::setThreadError("agg_rows must be 2 or 4");
            return GPUDB_E_INVALID;
        }
        b->aggRows = (int)value;
        b->dirty = true;
        return GPUDB_OK;
    }
    gpudb::setThreadError("unknown batch option '" + n + "'");
    return GPUDB_E_INVALID;
}

int gpudb_batch_set_tuning(gpudb_batch* b, int block, int tile_rows, int warp_aggregate, int max_probe) {
    if (!b || block < 64 || block > 1024 || block % 32 || tile_rows < 256 || max_probe < 1) return GPUDB_E_INVALID;
    b->block = block;
    b->tile = tile_rows;
    b->warpAgg = warp_aggregate ? 1 : 0;
    b->maxProbe = max_probe;
    b->dirty = true;
    return GPUDB_OK;
}

int gpudb_batch_execute(gpudb_batch* b, int use_graph, double* ms, uint32_t* errors) {
    if (!b) return GPUDB_E_INVALID;
    cudaSetDevice(b->device);
    if (b->dirty)
        if (int st = plan(b)) return st;
    const int n = (int)b->queries.size();
    B_CHECK(cudaEventRecord(b->ev0, b->stream), GPUDB_E_CUDA);
    if (use_graph) {
        if (!b->graphExec) {
            B_CHECK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), GPUDB_E_CUDA);
            const int st = enqueue(b, false);
            cudaGraph_t g = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
            if (st != GPUDB_OK) {
                if (g) cudaGraphDestroy(g);
                return st;
            }
            B_CHECK(ce, GPUDB_E_CUDA);
            b->graph = g;
            B_CHECK(cudaGraphInstantiate(&b->graphExec, g, 0), GPUDB_E_CUDA);
        }
        B_CHECK(cudaGraphLaunch(b->graphExec, b->stream), GPUDB_E_CUDA);
        b->stagesValid = false;
    } else {
        if (int st = enqueue(b, true)) return st;
    }
    B_CHECK(cudaEventRecord(b->ev1, b->stream), GPUDB_E_CUDA);
    B_CHECK(cudaEventSynchronize(b->ev1), GPUDB_E_CUDA);
    if (ms) *ms = elapsed(b);
    if (!use_graph) {
        for (int i = 0; i < GPUDB_BATCH_STAGES; i++) {
            float t = 0;
            cudaEventElapsedTime(&t, b->evStage[i], b->evStage[i + 1]);
            b->stageMs[i] = t;
        }
        b->stagesValid = true;
    }
    if (errors && n) std::memcpy(errors, b->errHost, sizeof(unsigned) * n);
    return GPUDB_OK;
}

int gpudb_batch_exact_stats(gpudb_batch* b, uint64_t* passing, uint64_t* distinct, double* ms) {
    if (!b) return GPUDB_E_INVALID;
    cudaSetDevice(b->device);
    if (b->dirty)
        if (int st = plan(b)) return st;
    const int n = (int)b->queries.size();
    if (n == 0) return GPUDB_OK;
    // counter, pass[n], distinct[n], one distinct bitmap per grouped query
    size_t words = 0;
    for (const auto& q : b->queries)
        if (grouped(q.tmpl)) words += (size_t)q.card / 32 + 1;
    const size_t bytes = 8 + 16 * (size_t)n + 4 * words;
    if (int st = b->stats.reserve(bytes, b->stream)) return st;
    unsigned long long* counter = static_cast<unsigned long long*>(b->stats.p);
    unsigned long long* pass = counter + 1;
    unsigned long long* dist = pass + n;
    unsigned* bm = reinterpret_cast<unsigned*>(dist + n);
    std::vector<QDesc> d = b->desc;
    size_t w = 0;
    for (int i = 0; i < n; i++) {
        d[i].st_pass = pass + i;
        d[i].st_distinct = dist + i;
        if (grouped(b->queries[i].tmpl)) {
            d[i].st_bitmap = bm + w;
            d[i].st_words = d[i].card / 32 + 1;
            w += (size_t)d[i].st_words;
        }
    }
    // the pass runs on descriptors that carry the statistics buffers; the
    // execution's descriptors are put back behind it
    B_CHECK(cudaMemcpyAsync(b->dDesc, d.data(), sizeof(QDesc) * n, cudaMemcpyHostToDevice, b->stream), GPUDB_E_CUDA);
    B_CHECK(cudaEventRecord(b->ev0, b->stream), GPUDB_E_CUDA);
    B_CHECK(cudaMemsetAsync(b->stats.p, 0, bytes, b->stream), GPUDB_E_CUDA);
    kStats<<<gridFor(b, (const void*)kStats, b->block), b->block, 0, b->stream>>>(b->dDesc, b->wlStats, b->tile,
                                                                                  counter);
    B_CHECK(cudaGetLastError(), GPUDB_E_LAUNCH);
    B_CHECK(cudaEventRecord(b->ev1, b->stream), GPUDB_E_CUDA);
    std::vector<unsigned long long> h(2 * (size_t)n);
    B_CHECK(cudaMemcpyAsync(h.data(), pass, 16 * (size_t)n, cudaMemcpyDeviceToHost, b->stream), GPUDB_E_CUDA);
    B_CHECK(cudaMemcpyAsync(b->dDesc, b->desc.data(), sizeof(QDesc) * n, cudaMemcpyHostToDevice, b->stream),
            GPUDB_E_CUDA);
    B_CHECK(cudaStreamSynchronize(b->stream), GPUDB_E_CUDA);
    if (ms) *ms = elapsed(b);
    for (int i = 0; i < n; i++) {
        if (passing) passing[i] = h[i];
        if (distinct) distinct[i] = h[n + i];
    }
    return GPUDB_OK;
}

int gpudb_batch_features(gpudb_batch* b, float* f, double* ms) {
    if (!b || !f) return GPUDB_E_INVALID;
    cudaSetDevice(b->device);
    if (b->dirty)
        if (int st = plan(b)) return st;
    const int n = (int)b->queries.size();
    if (n == 0) return GPUDB_OK;
    if (int st = b->sample.reserve(32 * (size_t)n, b->stream)) return st;
    unsigned long long* out = static_cast<unsigned long long*>(b->sample.p);
    B_CHECK(cudaEventRecord(b->ev0, b->stream), GPUDB_E_CUDA);
    kSampleStats<<<n, 256, kSampleSmem, b->stream>>>(b->dDesc, out);
    B_CHECK(cudaGetLastError(), GPUDB_E_LAUNCH);
    B_CHECK(cudaEventRecord(b->ev1, b->stream), GPUDB_E_CUDA);
    std::vector<unsigned long long> h(4 * (size_t)n);
    B_CHECK(cudaMemcpyAsync(h.data(), out, 32 * (size_t)n, cudaMemcpyDeviceToHost, b->stream), GPUDB_E_CUDA);
    B_CHECK(cudaStreamSynchronize(b->stream), GPUDB_E_CUDA);
    if (ms) *ms = elapsed(b);
    for (int i = 0; i < n; i++) {
        const auto& q = b->queries[i];
        const double m = (double)h[4 * i], pass = (double)h[4 * i + 1], dist = (double)h[4 * i + 2],
                     top = (double)h[4 * i + 3];
        const double rows = (double)q.rows;
        // key domain under the modulus, from the key column's min / max
        const double span = (double)q.key_max - (double)q.key_min + 1.0;
        const double card = std::max(1.0, std::min((double)std::max<int64_t>(q.card, 1), span > 0 ? span : 1.0));
        // predicate position inside the filter column's [min, max]
        const double frange = (double)q.filter_max - (double)q.filter_min + 1.0;
        const double predPos =
            frange > 0 ? std::min(1.0, std::max(0.0, ((double)q.thr - (double)q.filter_min) / frange)) : 0.0;
        const double sel = m > 0 ? pass / m : 0.0;
        const double expPass = rows * sel;
        const double uniformDistinct = card * (1.0 - std::exp(-expPass / card));
        float* x = f + (size_t)i * GPUDB_SIZER_FEATURES;
        for (int j = 0; j < GPUDB_SIZER_FEATURES; j++) x[j] = 0.0f;
        x[q.tmpl & 3] = 1.0f;                                      // template id, one-hot
        x[4] = (float)(std::log2(rows + 1.0) / 27.0);              // slice rows
        x[5] = (float)predPos;                                     // predicate constant vs column min / max
        x[6] = (float)(std::log2(card) / 24.0);                    // group-key domain
        x[7] = (float)sel;                                         // sample selectivity
        x[8] = (float)(pass > 0 ? dist / pass : 0.0);              // sample distinct / sample passing
        x[9] = (float)(std::log2(dist + 1.0) / 12.0);              // sample distinct count
        x[10] = (float)(std::log2(expPass + 1.0) / 27.0);          // estimated passing rows
        x[11] = (float)(std::log2((expPass + 1.0) / card) / 30.0);
        x[12] = (float)(pass > 0 ? top / pass : 0.0);              // share of the most frequent sample key
        x[13] = (float)(std::log2(pass + 1.0) / 12.0);             // sample passing count
        x[14] = (float)(std::log2(uniformDistinct + 1.0) / 24.0);  // uniform-key estimate of the groups
        x[15] = 1.0f;
    }
    return GPUDB_OK;
}

int gpudb_batch_collect(gpudb_batch* b, uint64_t* rows, void* host, uint64_t host_bytes, uint64_t* bytes_needed,
                        double* ms) {
    if (!b) return GPUDB_E_INVALID;
    cudaSetDevice(b->device);
    if (b->dirty) {
        gpudb::setThreadError("batch: collect before execute");
        return GPUDB_E_INVALID;
    }
    const int n = (int)b->queries.size();
    if (n == 0) {
        if (bytes_needed) *bytes_needed = 0;
        return GPUDB_OK;
    }
    // rows[n] + offsets[n+1] + counter, then the packed result rows
    const size_t head = al256(8 * (2 * (size_t)n + 2));
    size_t maxRows = 0;
    for (int i = 0; i < n; i++) {
        const auto& q = b->queries[i];
        maxRows += q.tmpl == GPUDB_TPL_GROUPBY ? (size_t)pow2ceil(2 * std::max<uint64_t>(q.groups, 1))
                   : q.tmpl == GPUDB_TPL_TOPK  ? (size_t)kTopK
                                               : 1;
    }
    if (int st = b->collect.reserve(head + 24 * maxRows, b->stream)) return st;
    unsigned long long* dRows = static_cast<unsigned long long*>(b->collect.p);
    unsigned long long* dOffs = dRows + n;
    unsigned long long* counter = dOffs + n + 1;
    long long* out = reinterpret_cast<long long*>(static_cast<char*>(b->collect.p) + head);
    B_CHECK(cudaEventRecord(b->ev0, b->stream), GPUDB_E_CUDA);
    B_CHECK(cudaMemsetAsync(counter, 0, 8, b->stream), GPUDB_E_CUDA);
    kResultRows<<<1, 1024, 0, b->stream>>>(b->dDesc, n, dRows, dOffs);
    kCollect<<<gridFor(b, (const void*)kCollect, 256), 256, 0, b->stream>>>(b->dDesc, b->wlCollect, b->collectChunk,
                                                                           counter, dOffs, out);
    B_CHECK(cudaGetLastError(), GPUDB_E_LAUNCH);
    std::vector<unsigned long long> h(2 * (size_t)n + 1);
    B_CHECK(cudaMemcpyAsync(h.data(), dRows, 8 * (2 * (size_t)n + 1), cudaMemcpyDeviceToHost, b->stream),
            GPUDB_E_CUDA);
    B_CHECK(cudaStreamSynchronize(b->stream), GPUDB_E_CUDA);
    const unsigned long long total = h[2 * (size_t)n];
    if (rows)
        for (int i = 0; i < n; i++) rows[i] = h[i];
    if (bytes_needed) *bytes_needed = 24 * total;
    if (host) {
        if (host_bytes < 24 * total) {
            gpudb::setThreadError("batch: collect buffer too small");
            return GPUDB_E_INVALID;
        }
        if (total) B_CHECK(cudaMemcpyAsync(host, out, 24 * total, cudaMemcpyDeviceToHost, b->stream), GPUDB_E_CUDA);
    }
    B_CHECK(cudaEventRecord(b->ev1, b->stream), GPUDB_E_CUDA);
    B_CHECK(cudaEventSynchronize(b->ev1), GPUDB_E_CUDA);
    if (ms) *ms = elapsed(b);
    return GPUDB_OK;
}

int gpudb_batch_result_scalar(gpudb_batch* b, int qi, int64_t* count, uint64_t* sum_lo, int64_t* sum_hi) {
    if (!b || qi < 0 || qi >= (int)b->queries.size() || b->dirty) return GPUDB_E_INVALID;
    const QDesc& d = b->desc[qi];
    if (d.tmpl != GPUDB_TPL_AGG && d.tmpl != GPUDB_TPL_JOIN) return GPUDB_E_INVALID;
    cudaSetDevice(b->device);
    unsigned long long w[3];
    B_CHECK(cudaMemcpyAsync(w, d.agg, 24, cudaMemcpyDeviceToHost, b->stream), GPUDB_E_CUDA);
    B_CHECK(cudaStreamSynchronize(b->stream), GPUDB_E_CUDA);
    const __int128 s = (__int128)(int64_t)w[2] * ((__int128)1 << 32) + (__int128)w[1];
    if (count) *count = (int64_t)w[0];
    if (sum_lo) *sum_lo = (uint64_t)s;
    if (sum_hi) *sum_hi = (int64_t)(s >> 64);
    return GPUDB_OK;
}

int gpudb_batch_result_groups(gpudb_batch* b, int qi, uint64_t cap, uint64_t* ngroups, int64_t* keys, int64_t* counts,
                              int64_t* sums) {
    if (!b || qi < 0 || qi >= (int)b->queries.size() || !ngroups || b->dirty) return GPUDB_E_INVALID;
    const QDesc& d = b->desc[qi];
    if (!grouped(d.tmpl)) return GPUDB_E_INVALID;
    cudaSetDevice(b->device);
    unsigned long long n = 0;
    B_CHECK(cudaMemcpyAsync(&n, d.nslots, 8, cudaMemcpyDeviceToHost, b->stream), GPUDB_E_CUDA);
    B_CHECK(cudaStreamSynchronize(b->stream), GPUDB_E_CUDA);
    *ngroups = n;
    if (!keys || !counts || !sums || n == 0 || cap < n) return GPUDB_OK;
    std::vector<unsigned> slots(n);
    std::vector<Slot> table((size_t)1 << d.log2cap);
    B_CHECK(cudaMemcpyAsync(slots.data(), d.slots, 4 * n, cudaMemcpyDeviceToHost, b->stream), GPUDB_E_CUDA);
    B_CHECK(cudaMemcpyAsync(table.data(), d.ht, sizeof(Slot) * table.size(), cudaMemcpyDeviceToHost, b->stream),
            GPUDB_E_CUDA);
    B_CHECK(cudaStreamSynchronize(b->stream), GPUDB_E_CUDA);
    for (unsigned long long j = 0; j < n; j++) {
        const Slot& s = table[slots[j]];
        keys[j] = (int64_t)decKey(s.key, d.card);
        counts[j] = (int64_t)s.count;
        sums[j] = (int64_t)s.sum;
    }
    return GPUDB_OK;
}

int gpudb_batch_result_topk(gpudb_batch* b, int qi, int64_t* keys, int64_t* vals, int* n) {
    if (!b || qi < 0 || qi >= (int)b->queries.size() || !n || b->dirty) return GPUDB_E_INVALID;
    const QDesc& d = b->desc[qi];
    if (d.tmpl != GPUDB_TPL_TOPK) return GPUDB_E_INVALID;
    cudaSetDevice(b->device);
    unsigned long long cnt = 0;
    long long kv[2 * kTopK];
    B_CHECK(cudaMemcpyAsync(&cnt, d.topk_n, 8, cudaMemcpyDeviceToHost, b->stream), GPUDB_E_CUDA);
    B_CHECK(cudaMemcpyAsync(kv, d.topk_out, sizeof(kv), cudaMemcpyDeviceToHost, b->stream), GPUDB_E_CUDA);
    B_CHECK(cudaStreamSynchronize(b->stream), GPUDB_E_CUDA);
    *n = (int)cnt;
    for (unsigned long long i = 0; i < cnt; i++) {
        if (keys) keys[i] = kv[2 * i];
        if (vals) vals[i] = kv[2 * i + 1];
    }
    return GPUDB_OK;
}

long long gpudb_batch_last_launches(gpudb_batch* b) { return b ? b->lastLaunches : 0; }

int gpudb_batch_stage_ms(gpudb_batch* b, double* ms) {
    if (!b || !ms) return GPUDB_E_INVALID;
    if (!b->stagesValid) {
        gpudb::setThreadError("batch: stage times need an execute without a graph");
        return GPUDB_E_INVALID;
    }
    for (int i = 0; i < GPUDB_BATCH_STAGES; i++) ms[i] = b->stageMs[i];
    return GPUDB_OK;
}

int gpudb_column_minmax(const void* column, uint64_t n, int elem_bytes, int64_t* min_out, int64_t* max_out,
                        void* stream) {
    if (!min_out || !max_out || (n && !column) || (elem_bytes != 4 && elem_bytes != 8)) {
        gpudb::setThreadError("column_minmax: needs int32 / int64 elements and output pointers");
        return GPUDB_E_INVALID;
    }
    if (n == 0) {
        *min_out = 0;
        *max_out = 0;
        return GPUDB_OK;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 0;
    B_CHECK(cudaGetDevice(&dev), GPUDB_E_NOGPU);
    B_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), GPUDB_E_CUDA);
    long long* d = nullptr;
    B_CHECK(cudaMallocAsync((void**)&d, 2 * sizeof(long long), st), GPUDB_E_ALLOC);
    const long long init[2] = {LLONG_MAX, LLONG_MIN};
    long long host[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(d, init, sizeof init, cudaMemcpyHostToDevice, st);
    const unsigned long long want = (n + 255) / 256;
    const int blocks = (int)std::min<unsigned long long>(want, (unsigned long long)sms * 8);
    if (e == cudaSuccess) {
        if (elem_bytes == 4) kColumnMinMax<int><<<blocks, 256, 0, st>>>(static_cast<const int*>(column), n, d);
        else kColumnMinMax<long long><<<blocks, 256, 0, st>>>(static_cast<const long long*>(column), n, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, d, sizeof host, cudaMemcpyDeviceToHost, st);
    const cudaError_t f = cudaFreeAsync(d, st);
    if (e == cudaSuccess) e = f;
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        gpudb::setThreadError(std::string("column_minmax: ") + cudaGetErrorString(e));
        return GPUDB_E_CUDA;
    }
    *min_out = host[0];
    *max_out = host[1];
    return GPUDB_OK;
}

}  // extern "C"
