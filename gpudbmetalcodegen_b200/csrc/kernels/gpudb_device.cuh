// ===================================================================
// gpudb_device.cuh — hand-written sm_100a device template library.
//
// Prepended (by CudaCodegen::print) to every NVRTC translation unit the
// engine generates; also included by the nvcc-compiled kernels of the
// library. It plays the role of the reference's MSL common header
// (codegen/core/metal_common_header.h:43-202) but is written for B200:
//   * native 64-bit atomics; exact 128-bit sums kept as two 64-bit words
//     that are added WITHOUT carry propagation (gpudb_acc128_add);
//   * warp shuffles / redux for reductions, __match_any_sync for
//     warp-aggregated hash updates under key skew;
//   * cp.async.bulk (TMA bulk copy into the issuing CTA only) + mbarrier pipelines
//     for column staging into shared memory;
//   * open-addressing hash tables (linear probe and 8-slot buckets) with
//     64-bit atomicCAS inserts and a bounded probe length;
//   * every wait is bounded by %globaltimer and reports through the
//     device error word instead of trapping.
// ===================================================================
#pragma once

typedef long long gpudb_i64;
typedef unsigned long long gpudb_u64;
typedef unsigned int gpudb_u32;

// ---- device error word bits (read by the host after every run) ----
#define GPUDB_ERR_HASH_OVERFLOW 0x1u   // probe limit exceeded / table full
#define GPUDB_ERR_WAIT_TIMEOUT 0x2u    // an mbarrier / flag wait gave up
#define GPUDB_ERR_BOUNDS 0x4u          // index outside a direct-address buffer
#define GPUDB_ERR_SENTINEL_KEY 0x8u    // key equal to the empty-slot sentinel
#define GPUDB_ERR_CAPACITY 0x10u       // output capacity exceeded

#define GPUDB_EMPTY64 0xFFFFFFFFFFFFFFFFull
#define GPUDB_EMPTY32 0xFFFFFFFFu
#ifndef GPUDB_WAIT_NS
#define GPUDB_WAIT_NS 1000000000ull    // 1 s bound on any spin-wait
#endif

// Thread coordinates under the names the operator templates use
// (reference: thread_position_in_grid / threads_per_grid / ... in
// metal_codegen_base.cpp:357-387).
#define GPUDB_THREAD_VARS                                                       \
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;     \
    const long long tpg = (long long)gridDim.x * blockDim.x;                    \
    const unsigned lid = threadIdx.x;                                           \
    const unsigned tg_size = blockDim.x;                                        \
    const unsigned gid = blockIdx.x;                                            \
    const unsigned simd_lane = threadIdx.x & 31u;                               \
    const unsigned simd_id = threadIdx.x >> 5;                                  \
    (void)tid; (void)tpg; (void)lid; (void)tg_size; (void)gid;                  \
    (void)simd_lane; (void)simd_id;

__device__ __forceinline__ void gpudb_set_error(unsigned* err, unsigned code) { atomicOr(err, code); }

__device__ __forceinline__ gpudb_u64 gpudb_now_ns() {
    gpudb_u64 t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ------------------------------------------------------------------
// Reductions
// ------------------------------------------------------------------
__device__ __forceinline__ long long gpudb_warp_sum_i64(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ unsigned long long gpudb_warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ unsigned long long gpudb_warp_max_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, v, o);
        v = t > v ? t : v;
    }
    return v;
}

// Block-wide reduction of NACC per-thread accumulators. Each warp reduces
// with shuffles and lane 0 parks its partials in smem[warp*NACC + a];
// after the barrier, thread a (a < NACC, strided) owns the block total of
// accumulator a and returns it through *out. Returns true for owners.
// smem must hold (blockDim.x/32) * NACC values.
template <int NACC>
__device__ __forceinline__ void gpudb_block_partials(const long long (&acc)[NACC], long long* smem) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int a = 0; a < NACC; ++a) {
        const long long v = gpudb_warp_sum_i64(acc[a]);
        if (lane == 0) smem[warp * NACC + a] = v;
    }
    __syncthreads();
}

__device__ __forceinline__ long long gpudb_block_total(const long long* smem, int nacc, int a) {
    const int nw = (int)(blockDim.x >> 5);
    long long s = 0;
    for (int w = 0; w < nw; ++w) s += smem[w * nacc + a];
    return s;
}

// ------------------------------------------------------------------
// Exact 128-bit accumulation in two 64-bit words, no carry chain.
//   v = hi * 2^32 + lo,  lo = v & (2^32-1) in [0, 2^32),  hi = v >> 32 (signed)
//   word[0] += lo, word[1] += hi  (both plain u64 atomics; RED when unused)
// Exact for fewer than 2^32 additions: the host reconstructs
//   total = (int64)word[1] * 2^32 + word[0]   in 128-bit arithmetic.
// ------------------------------------------------------------------
__device__ __forceinline__ void gpudb_acc128_add(unsigned long long* pair, long long v) {
    atomicAdd(pair, (unsigned long long)(v & 0xFFFFFFFFll));
    atomicAdd(pair + 1, (unsigned long long)(v >> 32));
}

__device__ __forceinline__ void gpudb_acc64_add(unsigned long long* word, long long v) {
    atomicAdd(word, (unsigned long long)v);
}

// ------------------------------------------------------------------
// Remainder by a divisor known only at run time but the same for every
// row (a group key k % card with card a kernel argument): division by an
// invariant integer through a multiply-high (Granlund & Montgomery,
// "Division by invariant integers using multiplication", PLDI 1994,
// Fig. 4.1). With l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0), t = mulhi(m, n),
// exact for 32-bit n and 1 <= d < 2^32. Each thread derives (m, l) once.
// ------------------------------------------------------------------
struct gpudb_divmagic {
    unsigned magic;
    int sh1, sh2;
    long long d;
};

__device__ __forceinline__ gpudb_divmagic gpudb_divmagic_make(long long d) {
    gpudb_divmagic m;
    m.d = d < 1 ? 1 : d;
    const unsigned long long ud = (unsigned long long)m.d;
    int l = 0;
    while (l < 32 && (1ull << l) < ud) l++;
    m.magic = (unsigned)(((1ull << 32) * ((1ull << l) - ud)) / ud + 1ull);
    m.sh1 = l < 1 ? l : 1;
    m.sh2 = l - 1 > 0 ? l - 1 : 0;
    return m;
}

// k % d for a 32-bit key, with the sign of k (C semantics) for negative k.
__device__ __forceinline__ long long gpudb_mod_i32(int k, const gpudb_divmagic& m) {
    if (k >= 0 && m.d < (1ll << 32)) {
        const unsigned n = (unsigned)k;
        const unsigned t = __umulhi(n, m.magic);
        const unsigned quo = (t + ((n - t) >> m.sh1)) >> m.sh2;
        return (long long)(n - quo * (unsigned)m.d);
    }
    return (long long)k % m.d;
}

// ------------------------------------------------------------------
// Order of group rows in an ORDER BY value DESC, key ASC: a before b.
// ------------------------------------------------------------------
__device__ __forceinline__ bool gpudb_row_before(long long va, long long ka, long long vb, long long kb) {
    return va > vb || (va == vb && ka < kb);
}

// Merge passes a sort of n rows in chunks of `chunk` rows needs: the
// smallest q with chunk << q >= n.
__device__ __forceinline__ int gpudb_merge_passes(long long n, int chunk) {
    int q = 0;
    while (((long long)chunk << q) < n) q++;
    return q;
}

// The same split found by one warp together: each round its 32 lanes test
// 32 evenly spaced candidates (the test is monotone: true for every index
// below the split), so the range shrinks 32-fold per round of loads. All
// lanes of the warp call it and get the split.
__device__ __forceinline__ int gpudb_merge_path_warp(const long long* av, const long long* ak, int na,
                                                     const long long* bv, const long long* bk, int nb, int d) {
    const int lane = (int)(threadIdx.x & 31u);
    int lo = d > nb ? d - nb : 0, hi = d < na ? d : na;
    while (lo < hi) {
        const int step = (hi - lo + 31) / 32;
        const int i = lo + lane * step;
        const bool t = i < hi && !gpudb_row_before(bv[d - 1 - i], bk[d - 1 - i], av[i], ak[i]);
        const int c = __popc(__ballot_sync(0xffffffffu, t));
        if (c == 0) break;  // the split is lo
        const int nlo = lo + (c - 1) * step + 1, nhi = lo + c * step;
        lo = nlo;
        hi = nhi < hi ? nhi : hi;
    }
    return lo;
}

// Merge path split of diagonal d between sorted A[0..na) and B[0..nb)
// (arrays of value / key, row order gpudb_row_before): the number of A rows
// among the first d merged rows (ties take A first).
__device__ __forceinline__ int gpudb_merge_path(const long long* av, const long long* ak, int na, const long long* bv,
                                                const long long* bk, int nb, int d) {
    int lo = d > nb ? d - nb : 0, hi = d < na ? d : na;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        // A[mid] goes before B[d - 1 - mid]: more A rows belong to the prefix
        if (!gpudb_row_before(bv[d - 1 - mid], bk[d - 1 - mid], av[mid], ak[mid])) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// ------------------------------------------------------------------
// Bitmaps (semi / anti joins). Reference: bitmap_test / bitmap_set,
// metal_common_header.h:103-111.
// ------------------------------------------------------------------
__device__ __forceinline__ bool gpudb_bitmap_test(const unsigned* __restrict__ bm, long long key) {
    return (__ldg(bm + (key >> 5)) >> (unsigned)(key & 31)) & 1u;
}

__device__ __forceinline__ void gpudb_bitmap_set(unsigned* bm, long long key) {
    atomicOr(bm + (key >> 5), 1u << (unsigned)(key & 31));
}

// ------------------------------------------------------------------
// Warp helpers
// ------------------------------------------------------------------
// Sum x over the lanes of `peers` (all lanes of `active` call with the
// same `active`); the group's lowest lane (rank 0) ends with the total.
// Tree over ranks: each round even-ranked lanes absorb their nearest
// remaining peer above, odd-ranked lanes drop out, ranks halve.
template <typename T>
__device__ __forceinline__ T gpudb_peer_sum(unsigned active, unsigned peers, T x) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned rank = __popc(peers & ((1u << lane) - 1u));
    unsigned above = peers & ~((2u << lane) - 1u);
    while (__any_sync(active, above != 0u)) {
        const int nxt = __ffs(above) - 1;
        const T t = __shfl_sync(active, x, nxt < 0 ? (int)lane : nxt);
        if (nxt >= 0 && (rank & 1u) == 0u) x += t;
        const unsigned gone = __ballot_sync(active, (rank & 1u) != 0u);
        above &= ~gone;
        rank >>= 1;
    }
    return x;
}

// Reserve output positions for the lanes with take=true using one atomic
// per warp (ballot + popc); returns this lane's position.
__device__ __forceinline__ unsigned long long gpudb_warp_reserve(unsigned long long* counter, bool take) {
    const unsigned active = __activemask();
    const unsigned m = __ballot_sync(active, take);
    const unsigned lane = threadIdx.x & 31u;
    const int leader = __ffs(active) - 1;
    unsigned long long base = 0;
    if ((int)lane == leader && m) base = atomicAdd(counter, (unsigned long long)__popc(m));
    base = __shfl_sync(active, base, leader);
    return base + (unsigned long long)__popc(m & ((1u << lane) - 1u));
}

// ------------------------------------------------------------------
// V consecutive elements of a staged column (shared memory, aligned to
// sizeof(T) * V) into registers with as few wide loads as possible.
// ------------------------------------------------------------------
template <typename T, int V>
__device__ __forceinline__ void gpudb_vload(const void* src, T (&out)[V]) {
    constexpr int B = (int)sizeof(T) * V;
    if constexpr (B % 16 == 0) {
        union {
            int4 v[B / 16];
            T t[V];
        } u;
#pragma unroll
        for (int c = 0; c < B / 16; ++c) u.v[c] = reinterpret_cast<const int4*>(src)[c];
#pragma unroll
        for (int j = 0; j < V; ++j) out[j] = u.t[j];
    } else if constexpr (B == 8) {
        union {
            uint2 v;
            T t[V];
        } u;
        u.v = *reinterpret_cast<const uint2*>(src);
#pragma unroll
        for (int j = 0; j < V; ++j) out[j] = u.t[j];
    } else if constexpr (B == 4) {
        union {
            unsigned v;
            T t[V];
        } u;
        u.v = *reinterpret_cast<const unsigned*>(src);
#pragma unroll
        for (int j = 0; j < V; ++j) out[j] = u.t[j];
    } else {
#pragma unroll
        for (int j = 0; j < V; ++j) out[j] = reinterpret_cast<const T*>(src)[j];
    }
}

// ------------------------------------------------------------------
// TMA bulk copy (cp.async.bulk, 1-D, CTA-local destination) + mbarrier
// ------------------------------------------------------------------
__device__ __forceinline__ unsigned gpudb_smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

// ------------------------------------------------------------------
// Fire-and-forget reductions (PTX `red`): an add whose old value nobody
// reads, so the issuing thread never waits for the atomic unit's answer.
// Relaxed, GPU scope: the semantics of atomicAdd.
// ------------------------------------------------------------------
__device__ __forceinline__ void gpudb_red_add_u32(unsigned* p, unsigned v) {
    asm volatile("red.relaxed.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void gpudb_red_add_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void gpudb_red_add_shared_u32(unsigned* p, unsigned v) {
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(gpudb_smem_addr(p)), "r"(v) : "memory");
}
__device__ __forceinline__ void gpudb_red_add_shared_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("red.shared.add.u64 [%0], %1;" ::"r"(gpudb_smem_addr(p)), "l"(v) : "memory");
}

__device__ __forceinline__ void gpudb_mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(gpudb_smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void gpudb_mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void gpudb_fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void gpudb_mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(gpudb_smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Plain arrival (one count) on `bar`, e.g. a consumer warp releasing a stage.
__device__ __forceinline__ void gpudb_mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(gpudb_smem_addr(bar)) : "memory");
}

// Copy `bytes` (multiple of 16; both addresses 16-byte aligned) from
// global to this CTA's shared memory; completion is signalled on `bar`.
__device__ __forceinline__ void gpudb_bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            gpudb_smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(gpudb_smem_addr(bar))
        : "memory");
}

// Same, with an L2 evict-first hint (the scanned columns are read once).
__device__ __forceinline__ void gpudb_bulk_g2s_stream(void* dst, const void* src, unsigned bytes,
                                                      unsigned long long* bar, unsigned long long policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
        "%4;" ::"r"(gpudb_smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(gpudb_smem_addr(bar)), "l"(policy)
        : "memory");
}

// Bring `bytes` (multiple of 16, 16-byte aligned source) into L2 ahead of a
// later copy; no shared memory, no completion to wait for.
__device__ __forceinline__ void gpudb_bulk_prefetch_l2(const void* src, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ unsigned long long gpudb_policy_evict_first() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// Wait for phase `parity` of `bar`; bounded by GPUDB_WAIT_NS of wall time.
__device__ __forceinline__ bool gpudb_mbar_wait(unsigned long long* bar, unsigned parity, unsigned* err) {
    const unsigned addr = gpudb_smem_addr(bar);
    unsigned done = 0;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    const unsigned long long t0 = gpudb_now_ns();
    for (;;) {
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        if (gpudb_now_ns() - t0 > GPUDB_WAIT_NS) {
            gpudb_set_error(err, GPUDB_ERR_WAIT_TIMEOUT);
            return false;
        }
    }
}

// ------------------------------------------------------------------
// Open-addressing hash tables. Keys live in their own array; an empty
// slot holds all-ones (the 0xFF fill of the key buffer). Capacity is a
// power of two; slot = high bits of key * 2^64/phi (Fibonacci hashing).
// Reference: host-built linear-probe tables with load factor <= 0.5 and a
// 64-step probe bound (query_preprocessing.cpp:352-386, 443-479;
// metal_plan_builder.cpp:1598-1610, 1968-1982); here the build runs on the
// GPU with atomicCAS and the bound is a parameter.
// ------------------------------------------------------------------
// log2 of the slot count for `groups` expected groups (load factor <= 1/2,
// at least 16 slots), computed on the device from counters an earlier
// kernel produced; never above the allocation's log2max.
__device__ __forceinline__ int gpudb_device_log2cap(unsigned long long groups, int log2max) {
    const unsigned long long want = groups * 2ull > 16ull ? groups * 2ull : 16ull;
    int l = 4;
    while (l < log2max && (1ull << l) < want) ++l;
    return l;
}

__device__ __forceinline__ unsigned long long gpudb_hash_slot(unsigned long long key, int log2cap) {
    return (key * 0x9E3779B97F4A7C15ull) >> (64 - log2cap);
}

// Linear probing, 64-bit keys. Returns the slot holding `key` (inserted
// if absent) or -1 when `max_probe` slots were all taken. *fresh (when
// given) is set when this call claimed the slot, i.e. created the group.
__device__ __forceinline__ long long gpudb_ht_insert64(unsigned long long* keys, int log2cap,
                                                       unsigned long long key, unsigned max_probe,
                                                       unsigned* err, bool* fresh = nullptr) {
    if (key == GPUDB_EMPTY64) {
        gpudb_set_error(err, GPUDB_ERR_SENTINEL_KEY);
        return -1;
    }
    const unsigned long long mask = (1ull << log2cap) - 1ull;
    unsigned long long s = gpudb_hash_slot(key, log2cap);
    for (unsigned p = 0; p < max_probe; ++p) {
        const unsigned long long cur = keys[s];
        if (cur == key) return (long long)s;
        if (cur == GPUDB_EMPTY64) {
            const unsigned long long prev = atomicCAS(keys + s, GPUDB_EMPTY64, key);
            if (prev == GPUDB_EMPTY64) {
                if (fresh) *fresh = true;
                return (long long)s;
            }
            if (prev == key) return (long long)s;
        }
        s = (s + 1ull) & mask;
    }
    gpudb_set_error(err, GPUDB_ERR_HASH_OVERFLOW);
    return -1;
}

// Best-effort insert into a small table: the slot holding `key` or one it
// claimed within `max_probe` probes, else -1 (no error: the caller then
// uses its main table). The sentinel key is never placed here.
__device__ __forceinline__ long long gpudb_ht_try_insert64(unsigned long long* keys, int log2cap,
                                                           unsigned long long key, unsigned max_probe) {
    if (key == GPUDB_EMPTY64) return -1;
    const unsigned long long mask = (1ull << log2cap) - 1ull;
    unsigned long long s = gpudb_hash_slot(key, log2cap);
    for (unsigned p = 0; p < max_probe; ++p) {
        const unsigned long long cur = keys[s];
        if (cur == key) return (long long)s;
        if (cur == GPUDB_EMPTY64) {
            const unsigned long long prev = atomicCAS(keys + s, GPUDB_EMPTY64, key);
            if (prev == GPUDB_EMPTY64 || prev == key) return (long long)s;
        }
        s = (s + 1ull) & mask;
    }
    return -1;
}

// Packed group-by slots of 2^stride_log2 u64 words: word 0 holds ~key
// (0 = empty; the all-ones key stays reserved as in the other layouts) and
// the aggregates follow in the same sector. Returns the slot index, as
// gpudb_ht_insert64 does.
__device__ __forceinline__ long long gpudb_htp_insert64(unsigned long long* slots, int stride_log2, int log2cap,
                                                        unsigned long long key, unsigned max_probe, unsigned* err,
                                                        bool* fresh = nullptr) {
    if (key == GPUDB_EMPTY64) {
        gpudb_set_error(err, GPUDB_ERR_SENTINEL_KEY);
        return -1;
    }
    const unsigned long long want = ~key;
    const unsigned long long mask = (1ull << log2cap) - 1ull;
    unsigned long long s = gpudb_hash_slot(key, log2cap);
    for (unsigned p = 0; p < max_probe; ++p) {
        unsigned long long* w = slots + (s << stride_log2);
        const unsigned long long cur = *w;
        if (cur == want) return (long long)s;
        if (cur == 0ull) {
            const unsigned long long prev = atomicCAS(w, 0ull, want);
            if (prev == 0ull) {
                if (fresh) *fresh = true;
                return (long long)s;
            }
            if (prev == want) return (long long)s;
        }
        s = (s + 1ull) & mask;
    }
    gpudb_set_error(err, GPUDB_ERR_HASH_OVERFLOW);
    return -1;
}

__device__ __forceinline__ long long gpudb_ht_find64(const unsigned long long* __restrict__ keys, int log2cap,
                                                     unsigned long long key, unsigned max_probe) {
    const unsigned long long mask = (1ull << log2cap) - 1ull;
    unsigned long long s = gpudb_hash_slot(key, log2cap);
    for (unsigned p = 0; p < max_probe; ++p) {
        const unsigned long long cur = __ldg(keys + s);
        if (cur == key) return (long long)s;
        if (cur == GPUDB_EMPTY64) return -1;
        s = (s + 1ull) & mask;
    }
    return -1;
}

// 32-bit keys (dense integer join / group keys).
__device__ __forceinline__ long long gpudb_ht_insert32(unsigned* keys, int log2cap, unsigned key,
                                                       unsigned max_probe, unsigned* err, bool* fresh = nullptr) {
    if (key == GPUDB_EMPTY32) {
        gpudb_set_error(err, GPUDB_ERR_SENTINEL_KEY);
        return -1;
    }
    const unsigned long long mask = (1ull << log2cap) - 1ull;
    unsigned long long s = gpudb_hash_slot((unsigned long long)key, log2cap);
    for (unsigned p = 0; p < max_probe; ++p) {
        const unsigned cur = keys[s];
        if (cur == key) return (long long)s;
        if (cur == GPUDB_EMPTY32) {
            const unsigned prev = atomicCAS(keys + s, GPUDB_EMPTY32, key);
            if (prev == GPUDB_EMPTY32) {
                if (fresh) *fresh = true;
                return (long long)s;
            }
            if (prev == key) return (long long)s;
        }
        s = (s + 1ull) & mask;
    }
    gpudb_set_error(err, GPUDB_ERR_HASH_OVERFLOW);
    return -1;
}

__device__ __forceinline__ long long gpudb_ht_find32(const unsigned* __restrict__ keys, int log2cap, unsigned key,
                                                     unsigned max_probe) {
    const unsigned long long mask = (1ull << log2cap) - 1ull;
    unsigned long long s = gpudb_hash_slot((unsigned long long)key, log2cap);
    for (unsigned p = 0; p < max_probe; ++p) {
        const unsigned cur = __ldg(keys + s);
        if (cur == key) return (long long)s;
        if (cur == GPUDB_EMPTY32) return -1;
        s = (s + 1ull) & mask;
    }
    return -1;
}

// Bucketised layout: 8 x 64-bit keys per 64-byte bucket (two 32-byte
// sectors); the hash picks a bucket, buckets are probed linearly.
// Slot index = bucket * 8 + way. log2cap counts slots (>= 3).
__device__ __forceinline__ long long gpudb_htb_insert64(unsigned long long* keys, int log2cap,
                                                        unsigned long long key, unsigned max_buckets,
                                                        unsigned* err, bool* fresh = nullptr) {
    if (key == GPUDB_EMPTY64) {
        gpudb_set_error(err, GPUDB_ERR_SENTINEL_KEY);
        return -1;
    }
    const int lb = log2cap - 3;
    const unsigned long long bmask = (1ull << lb) - 1ull;
    unsigned long long b = lb > 0 ? gpudb_hash_slot(key, lb) : 0ull;
    for (unsigned p = 0; p < max_buckets; ++p) {
        unsigned long long* base = keys + b * 8ull;
        const ulonglong2* v = reinterpret_cast<const ulonglong2*>(base);
        unsigned long long k[8];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const ulonglong2 t = v[q];
            k[2 * q] = t.x;
            k[2 * q + 1] = t.y;
        }
#pragma unroll
        for (int w = 0; w < 8; ++w)
            if (k[w] == key) return (long long)(b * 8ull + w);
#pragma unroll 1
        for (int w = 0; w < 8; ++w) {
            if (k[w] != GPUDB_EMPTY64) continue;
            const unsigned long long prev = atomicCAS(base + w, GPUDB_EMPTY64, key);
            if (prev == GPUDB_EMPTY64) {
                if (fresh) *fresh = true;
                return (long long)(b * 8ull + w);
            }
            if (prev == key) return (long long)(b * 8ull + w);
            k[w] = prev;  // lost the race: slot now holds another key, keep scanning
        }
        b = (b + 1ull) & bmask;
    }
    gpudb_set_error(err, GPUDB_ERR_HASH_OVERFLOW);
    return -1;
}

__device__ __forceinline__ long long gpudb_htb_find64(const unsigned long long* __restrict__ keys, int log2cap,
                                                      unsigned long long key, unsigned max_buckets) {
    const int lb = log2cap - 3;
    const unsigned long long bmask = (1ull << lb) - 1ull;
    unsigned long long b = lb > 0 ? gpudb_hash_slot(key, lb) : 0ull;
    for (unsigned p = 0; p < max_buckets; ++p) {
        const ulonglong2* v = reinterpret_cast<const ulonglong2*>(keys + b * 8ull);
        bool any_empty = false;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const ulonglong2 t = __ldg(v + q);
            if (t.x == key) return (long long)(b * 8ull + 2 * q);
            if (t.y == key) return (long long)(b * 8ull + 2 * q + 1);
            any_empty |= (t.x == GPUDB_EMPTY64) | (t.y == GPUDB_EMPTY64);
        }
        if (any_empty) return -1;
        b = (b + 1ull) & bmask;
    }
    return -1;
}

// Per-block shared-memory pre-aggregation table (heavy hitters): linear
// probing over `cap` (power of two) slots of 64-bit keys; returns the slot
// or -1 when full within `max_probe` (caller then goes to global memory).
__device__ __forceinline__ int gpudb_smem_ht_slot64(unsigned long long* skeys, int log2cap, unsigned long long key,
                                                    int max_probe) {
    const unsigned mask = (1u << log2cap) - 1u;
    unsigned s = (unsigned)gpudb_hash_slot(key, log2cap);
    for (int p = 0; p < max_probe; ++p) {
        const unsigned long long cur = skeys[s];
        if (cur == key) return (int)s;
        if (cur == GPUDB_EMPTY64) {
            const unsigned long long prev = atomicCAS(skeys + s, GPUDB_EMPTY64, key);
            if (prev == GPUDB_EMPTY64 || prev == key) return (int)s;
        }
        s = (s + 1u) & mask;
    }
    return -1;
}

// ------------------------------------------------------------------
// Top-k: order is (value desc, key asc); "none" = (INT64_MIN, INT64_MAX).
// ------------------------------------------------------------------
#define GPUDB_TOPK_NONE_VAL (-0x7FFFFFFFFFFFFFFFll - 1ll)
#define GPUDB_TOPK_NONE_KEY 0x7FFFFFFFFFFFFFFFll

__device__ __forceinline__ bool gpudb_topk_better(long long va, long long ka, long long vb, long long kb) {
    return va > vb || (va == vb && ka < kb);
}

// Insert (v,k) into a register-resident sorted list of K (best first).
template <int K>
__device__ __forceinline__ void gpudb_topk_push(long long (&vv)[K], long long (&kk)[K], long long v, long long k) {
    if (!gpudb_topk_better(v, k, vv[K - 1], kk[K - 1])) return;
    vv[K - 1] = v;
    kk[K - 1] = k;
#pragma unroll
    for (int i = K - 1; i > 0; --i) {
        if (gpudb_topk_better(vv[i], kk[i], vv[i - 1], kk[i - 1])) {
            const long long tv = vv[i], tk = kk[i];
            vv[i] = vv[i - 1];
            kk[i] = kk[i - 1];
            vv[i - 1] = tv;
            kk[i - 1] = tk;
        }
    }
}

// Merge the 32 lanes' sorted lists into the warp's best K, in order, by K
// rounds of a shuffle arg-max over the lanes' list heads (any K). Every
// lane ends with the merged list in (ov, ok). Full warp must participate.
template <int K>
__device__ __forceinline__ void gpudb_topk_warp_merge_rounds(const long long (&vv)[K], const long long (&kk)[K],
                                                             long long (&ov)[K], long long (&ok)[K]) {
    const unsigned lane = threadIdx.x & 31u;
    int head = 0;
#pragma unroll 1
    for (int r = 0; r < K; ++r) {
        long long hv = GPUDB_TOPK_NONE_VAL, hk = GPUDB_TOPK_NONE_KEY;
#pragma unroll
        for (int i = 0; i < K; ++i)
            if (i == head) {
                hv = vv[i];
                hk = kk[i];
            }
        long long bv = hv, bk = hk;
        int bl = (int)lane;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const long long v2 = __shfl_xor_sync(0xffffffffu, bv, o);
            const long long k2 = __shfl_xor_sync(0xffffffffu, bk, o);
            const int l2 = __shfl_xor_sync(0xffffffffu, bl, o);
            if (gpudb_topk_better(v2, k2, bv, bk) || (v2 == bv && k2 == bk && l2 < bl)) {
                bv = v2;
                bk = k2;
                bl = l2;
            }
        }
#pragma unroll
        for (int i = 0; i < K; ++i)
            if (i == r) {
                ov[i] = bv;
                ok[i] = bk;
            }
        if ((int)lane == bl && head < K) head++;
    }
}

// Sort one entry per lane of a warp into (value desc, key asc) order, best
// at lane 0: a 32-wide bitonic sorting network of shuffles. Full warp.
__device__ __forceinline__ void gpudb_topk_warp_sort32(long long& v, long long& k) {
    const int lane = (int)(threadIdx.x & 31u);
#pragma unroll
    for (int w = 2; w <= 32; w <<= 1) {
#pragma unroll
        for (int j = w >> 1; j > 0; j >>= 1) {
            const long long pv = __shfl_xor_sync(0xffffffffu, v, j), pk = __shfl_xor_sync(0xffffffffu, k, j);
            const bool better = gpudb_topk_better(v, k, pv, pk);
            // descending runs keep the better entry at the lower lane
            const bool keep = (((lane & j) == 0) == ((lane & w) == 0)) ? better : !better;
            if (!keep) {
                v = pv;
                k = pk;
            }
        }
    }
}

// Merge a second sorted list (ov, ok: lane j holds its j-th best) into the
// warp's sorted list (rv, rk). Lane j takes the better of its own entry
// and the other list's (31-j)-th: of two descending sequences that keeps
// the best 32 of both as a bitonic sequence, which five half-cleaner
// stages sort. Lanes K..31 end as "none". Full warp.
template <int K>
__device__ __forceinline__ void gpudb_topk_warp_merge_list(long long& rv, long long& rk, long long ov, long long ok) {
    const int lane = (int)(threadIdx.x & 31u);
    long long v = rv, k = rk;
    {
        const long long bv = __shfl_sync(0xffffffffu, ov, 31 - lane), bk = __shfl_sync(0xffffffffu, ok, 31 - lane);
        if (gpudb_topk_better(bv, bk, v, k)) {
            v = bv;
            k = bk;
        }
    }
#pragma unroll
    for (int j = 16; j > 0; j >>= 1) {
        const long long pv = __shfl_xor_sync(0xffffffffu, v, j), pk = __shfl_xor_sync(0xffffffffu, k, j);
        // the lower lane of each pair keeps the better entry, the upper the worse
        if (((lane & j) == 0) == gpudb_topk_better(pv, pk, v, k)) {
            v = pv;
            k = pk;
        }
    }
    rv = lane < K ? v : GPUDB_TOPK_NONE_VAL;
    rk = lane < K ? k : GPUDB_TOPK_NONE_KEY;
}

// A warp's best K (K <= 32) held one entry per lane: lane j holds the
// j-th best, lanes K..31 hold "none". Offer one entry per lane: a ballot
// keeps those better than the current K-th best. A few are inserted one
// at a time (one more ballot gives each its rank, the lanes below it
// shift); more are sorted by a bitonic network and merged as a list.
// Returns the ballot of offered entries that beat the K-th best. Full warp.
template <int K>
__device__ __forceinline__ unsigned gpudb_topk_warp_offer(long long& rv, long long& rk, long long cv, long long ck) {
    static_assert(K >= 1 && K <= 32, "a warp holds at most 32 entries");
    const int lane = (int)(threadIdx.x & 31u);
    const long long tv = __shfl_sync(0xffffffffu, rv, K - 1), tk = __shfl_sync(0xffffffffu, rk, K - 1);
    const unsigned any = __ballot_sync(0xffffffffu, gpudb_topk_better(cv, ck, tv, tk));
    if (!any) return 0u;
    const long long hv = __shfl_sync(0xffffffffu, rv, 0), hk = __shfl_sync(0xffffffffu, rk, 0);
    const bool empty = hv == GPUDB_TOPK_NONE_VAL && hk == GPUDB_TOPK_NONE_KEY;
    if (__popc(any) > (empty ? 2 : 4)) {
        long long v = (any >> lane) & 1u ? cv : GPUDB_TOPK_NONE_VAL, k = (any >> lane) & 1u ? ck : GPUDB_TOPK_NONE_KEY;
        gpudb_topk_warp_sort32(v, k);
        if (empty) {
            rv = lane < K ? v : GPUDB_TOPK_NONE_VAL;
            rk = lane < K ? k : GPUDB_TOPK_NONE_KEY;
        } else {
            gpudb_topk_warp_merge_list<K>(rv, rk, v, k);
        }
        return any;
    }
    unsigned m = any;
    while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1u;
        const long long xv = __shfl_sync(0xffffffffu, cv, src), xk = __shfl_sync(0xffffffffu, ck, src);
        const int pos = __popc(__ballot_sync(0xffffffffu, lane < K && gpudb_topk_better(rv, rk, xv, xk)));
        if (pos >= K) continue;  // the K-th best rose past it meanwhile
        const long long uv = __shfl_up_sync(0xffffffffu, rv, 1), uk = __shfl_up_sync(0xffffffffu, rk, 1);
        if (lane == pos) {
            rv = xv;
            rk = xk;
        } else if (lane > pos && lane < K) {
            rv = uv;
            rk = uk;
        }
    }
    return any;
}

// Same result for K <= 32 with far fewer instructions when most entries
// cannot enter: round r offers every lane's r-th entry to the warp's
// one-entry-per-lane list; the lanes' lists are sorted, so the first round
// in which no entry beats the K-th best ends the merge.
template <int K>
__device__ __forceinline__ void gpudb_topk_warp_merge(const long long (&vv)[K], const long long (&kk)[K],
                                                      long long (&ov)[K], long long (&ok)[K]) {
    if constexpr (K > 32) {
        gpudb_topk_warp_merge_rounds<K>(vv, kk, ov, ok);
    } else {
        long long rv = GPUDB_TOPK_NONE_VAL, rk = GPUDB_TOPK_NONE_KEY;
#pragma unroll
        for (int r = 0; r < K; ++r)
            if (!gpudb_topk_warp_offer<K>(rv, rk, vv[r], kk[r])) break;
#pragma unroll
        for (int i = 0; i < K; ++i) {
            ov[i] = __shfl_sync(0xffffffffu, rv, i);
            ok[i] = __shfl_sync(0xffffffffu, rk, i);
        }
    }
}
