// msl_cpu_shim.h — runs Metal Shading Language compute kernels, emitted by
// the reference engine's own code generator, as C++ on the CPU.
//
// TEST INFRASTRUCTURE (oracle pinning): the reference's kernels are
// compiled as C++ against this header so their outputs on seeded inputs can
// be compared with the CPU oracle. Each GPU thread of a threadgroup is a
// cooperative fiber (ucontext); threadgroup barriers and SIMD-group
// operations (shuffle_down, sum) switch fibers until all participants
// arrive. Threadgroups run in parallel on OS threads; `threadgroup`
// variables declared in kernel bodies become thread_local statics (one
// threadgroup runs at a time per OS thread). Atomics map to std::atomic.
#pragma once

#include <ucontext.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <thread>
#include <vector>

namespace metal {

typedef unsigned int uint;
typedef unsigned long ulong;
typedef unsigned char uchar;
typedef unsigned short ushort;

typedef std::atomic<uint32_t> atomic_uint;
typedef std::atomic<int32_t> atomic_int;
typedef std::atomic<float> atomic_float;

enum memory_order { memory_order_relaxed };
enum class mem_flags { mem_none = 0, mem_device = 1, mem_threadgroup = 2, mem_texture = 4 };

template <typename T, typename U>
inline T as_type(U v) {
    static_assert(sizeof(T) == sizeof(U), "as_type size mismatch");
    T t;
    std::memcpy(&t, &v, sizeof(T));
    return t;
}

template <typename T, typename U>
inline T atomic_fetch_add_explicit(std::atomic<T>* a, U v, memory_order) {
    return a->fetch_add((T)v, std::memory_order_relaxed);
}
template <typename T, typename U>
inline T atomic_fetch_or_explicit(std::atomic<T>* a, U v, memory_order) {
    return a->fetch_or((T)v, std::memory_order_relaxed);
}
template <typename T, typename U>
inline T atomic_fetch_min_explicit(std::atomic<T>* a, U v, memory_order) {
    T cur = a->load(std::memory_order_relaxed);
    while ((T)v < cur && !a->compare_exchange_weak(cur, (T)v, std::memory_order_relaxed)) {
    }
    return cur;
}
template <typename T, typename U>
inline T atomic_fetch_max_explicit(std::atomic<T>* a, U v, memory_order) {
    T cur = a->load(std::memory_order_relaxed);
    while ((T)v > cur && !a->compare_exchange_weak(cur, (T)v, std::memory_order_relaxed)) {
    }
    return cur;
}
template <typename T>
inline T atomic_load_explicit(std::atomic<T>* a, memory_order) {
    return a->load(std::memory_order_relaxed);
}
template <typename T>
inline T atomic_load_explicit(const std::atomic<T>* a, memory_order) {
    return a->load(std::memory_order_relaxed);
}
template <typename T, typename U>
inline void atomic_store_explicit(std::atomic<T>* a, U v, memory_order) {
    a->store((T)v, std::memory_order_relaxed);
}
template <typename T, typename U>
inline bool atomic_compare_exchange_weak_explicit(std::atomic<T>* a, T* expected, U desired, memory_order,
                                                  memory_order) {
    return a->compare_exchange_weak(*expected, (T)desired, std::memory_order_relaxed);
}

// ---------------------------------------------------------------------------
// fiber runtime
// ---------------------------------------------------------------------------
namespace cpu {

struct Fiber {
    ucontext_t ctx;
    std::vector<char> stack;
    bool done = false;
    uint lid = 0;
};

struct Group {  // one threadgroup in flight on this OS thread
    ucontext_t sched;
    std::vector<Fiber> fibers;
    int current = -1;
    uint size = 0;
    // threadgroup barrier
    uint arrived = 0;
    uint64_t generation = 0;
    // per-SIMD-group exchange: 32 slots of 8 bytes + barrier state
    std::vector<uint64_t> slots;
    std::vector<uint> simdArrived;
    std::vector<uint64_t> simdGen;
    std::function<void(uint)> body;
};

inline thread_local Group* tlGroup = nullptr;

inline void yieldToScheduler() {
    Group* g = tlGroup;
    swapcontext(&g->fibers[g->current].ctx, &g->sched);
}

inline void barrierAll() {
    Group* g = tlGroup;
    const uint64_t gen = g->generation;
    if (++g->arrived == g->size) {
        g->arrived = 0;
        g->generation++;
        return;
    }
    while (g->generation == gen) yieldToScheduler();
}

inline uint simdWidth(uint simdId) {
    Group* g = tlGroup;
    const uint base = simdId * 32u;
    return (g->size - base) < 32u ? (g->size - base) : 32u;
}

inline void barrierSimd(uint simdId) {
    Group* g = tlGroup;
    const uint64_t gen = g->simdGen[simdId];
    if (++g->simdArrived[simdId] == simdWidth(simdId)) {
        g->simdArrived[simdId] = 0;
        g->simdGen[simdId]++;
        return;
    }
    while (g->simdGen[simdId] == gen) yieldToScheduler();
}

inline void trampoline(unsigned lo, unsigned hi) {
    const uintptr_t p = ((uintptr_t)hi << 32) | (uintptr_t)lo;
    Fiber* f = reinterpret_cast<Fiber*>(p);
    tlGroup->body(f->lid);
    f->done = true;
    swapcontext(&f->ctx, &tlGroup->sched);
}

// Run `body(lid)` for every thread of one threadgroup of `size` threads.
inline void runGroup(uint size, const std::function<void(uint)>& body) {
    Group g;
    g.size = size;
    g.body = body;
    g.fibers.resize(size);
    const uint nsimd = (size + 31u) / 32u;
    g.slots.assign(nsimd * 32u, 0);
    g.simdArrived.assign(nsimd, 0);
    g.simdGen.assign(nsimd, 0);
    Group* saved = tlGroup;
    tlGroup = &g;
    for (uint i = 0; i < size; i++) {
        Fiber& f = g.fibers[i];
        f.lid = i;
        f.stack.resize(128 * 1024);
        getcontext(&f.ctx);
        f.ctx.uc_stack.ss_sp = f.stack.data();
        f.ctx.uc_stack.ss_size = f.stack.size();
        f.ctx.uc_link = nullptr;
        const uintptr_t p = reinterpret_cast<uintptr_t>(&f);
        makecontext(&f.ctx, (void (*)())trampoline, 2, (unsigned)(p & 0xffffffffu), (unsigned)(p >> 32));
    }
    for (;;) {
        bool all = true, progressed = false;
        for (uint i = 0; i < size; i++) {
            Fiber& f = g.fibers[i];
            if (f.done) continue;
            all = false;
            const uint64_t before = g.generation;
            g.current = (int)i;
            swapcontext(&g.sched, &f.ctx);
            progressed |= f.done || g.generation != before;
        }
        if (all) break;
        (void)progressed;
    }
    tlGroup = saved;
}

// Dispatch numTG threadgroups of tgSize threads over host threads.
inline void dispatch(uint numTG, uint tgSize,
                     const std::function<void(uint tid, uint tpg, uint lid, uint tgs, uint gid, uint lane, uint sid)>& k,
                     unsigned hostThreads = 0) {
    unsigned T = hostThreads ? hostThreads : std::max(1u, std::thread::hardware_concurrency());
    if (T > numTG) T = numTG;
    std::atomic<uint> next{0};
    auto worker = [&]() {
        for (;;) {
            const uint gid = next.fetch_add(1);
            if (gid >= numTG) break;
            runGroup(tgSize, [&](uint lid) {
                k(gid * tgSize + lid, numTG * tgSize, lid, tgSize, gid, lid & 31u, lid >> 5);
            });
        }
    };
    std::vector<std::thread> ts;
    for (unsigned t = 0; t < T; t++) ts.emplace_back(worker);
    for (auto& t : ts) t.join();
}

inline uint currentLid() { return tlGroup->fibers[tlGroup->current].lid; }

}  // namespace cpu

inline void threadgroup_barrier(mem_flags) { cpu::barrierAll(); }
inline void simdgroup_barrier(mem_flags) { cpu::barrierSimd(cpu::currentLid() >> 5); }

template <typename T>
inline T simd_shuffle_down(T v, uint delta) {
    static_assert(sizeof(T) <= 8, "shuffle of a wide type");
    cpu::Group* g = cpu::tlGroup;
    const uint lid = cpu::currentLid(), sid = lid >> 5, lane = lid & 31u;
    uint64_t raw = 0;
    std::memcpy(&raw, &v, sizeof(T));
    g->slots[lid] = raw;
    cpu::barrierSimd(sid);
    T out = v;
    if (lane + delta < cpu::simdWidth(sid)) std::memcpy(&out, &g->slots[sid * 32u + lane + delta], sizeof(T));
    cpu::barrierSimd(sid);
    return out;
}

template <typename T>
inline T simd_sum(T v) {
    cpu::Group* g = cpu::tlGroup;
    const uint lid = cpu::currentLid(), sid = lid >> 5;
    uint64_t raw = 0;
    std::memcpy(&raw, &v, sizeof(T));
    g->slots[lid] = raw;
    cpu::barrierSimd(sid);
    T s = T(0);
    for (uint l = 0; l < cpu::simdWidth(sid); l++) {
        T x;
        std::memcpy(&x, &g->slots[sid * 32u + l], sizeof(T));
        s += x;
    }
    cpu::barrierSimd(sid);
    return s;
}

}  // namespace metal

// MSL address-space and function qualifiers have no CPU meaning.
#define kernel
#define device
#define constant
