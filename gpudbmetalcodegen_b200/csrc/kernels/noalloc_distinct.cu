// Allocation-free distinct count: gpudb_distinct_count_noalloc().
//
// Who needs it: callers that must not allocate device memory on the call
// path — hosts that hand the GPU to a strict memory
// budget or their own pool (database buffer managers, JNI/cgo hosts whose
// allocator owns all device memory), and latency-critical loops where a
// cudaMalloc/cudaFree round trip (and its implicit synchronisation) is not
// acceptable. They pass their own inputs and output; this function touches
// no allocator.
//
// What it computes: the number of distinct values of (key[i] % card) over
// the rows with filter[i] < thr — the same result as the "distinct"
// pipeline (gpudb_query_run with template=distinct), which sizes group
// tables. Its scratch bitmap is not allocated per call: it lives in the
// file-scope array below, sized for card <= GPUDB_NOALLOC_MAX_CARD (2^22
// keys: a 512 KiB bitmap plus one counter). Every GPU that loads this
// library holds that array until the process exits.
//
// Contract:
//   * card must be in [1, 2^22]; larger values are rejected with
//     GPUDB_E_INVALID and a message (gpudb_last_error(NULL)).
//   * keys must be non-negative; a negative key is skipped.
//   * all calls share the one scratch array; the call clears it first, so
//     back-to-back calls on one stream are independent, but calls that
//     overlap on the GPU (different streams, or different host threads)
//     race on it and produce wrong counts.
//   * the first call on a device looks up the scratch array's device
//     address (cudaGetSymbolAddress) with that device current. The address is kept
//     until the process exits: a device reset (cudaDeviceReset, or a
//     destroyed primary context) leaves it stale, so after one this entry
//     point must not be called on that device again.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../../include/gpudb_rt.h"

namespace gpudb {
void setThreadError(const std::string& message);  // gpudb_capi.cpp
}

#define GPUDB_NOALLOC_MAX_CARD (1u << 22)
#define GPUDB_NOALLOC_HEADER_WORDS 32u  // counter + padding: bitmap starts 256 B in

// Scratch: [0] distinct counter, [1..31] unused, then the bitmap.
static __device__ __align__(256) unsigned long long
    gpudb_noalloc_scratch[GPUDB_NOALLOC_HEADER_WORDS + GPUDB_NOALLOC_MAX_CARD / 64 + 1];

namespace {

constexpr int kMaxDevices = 64;
std::mutex gMu;
unsigned long long* gScratch[kMaxDevices] = {};
int gSMs[kMaxDevices] = {};

__global__ void noalloc_clear(unsigned long long* scratch, unsigned long long words64) {
    const unsigned long long n = GPUDB_NOALLOC_HEADER_WORDS + words64;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x)
        scratch[i] = 0ull;
}

__global__ void noalloc_count(const int* __restrict__ key, const int* __restrict__ filter, long long n, int thr,
                              long long card, unsigned long long* scratch) {
    unsigned* bitmap = reinterpret_cast<unsigned*>(scratch + GPUDB_NOALLOC_HEADER_WORDS);
    unsigned long long fresh = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (filter[i] >= thr) continue;
        const long long k = (long long)key[i] % card;
        if (k < 0) continue;
        const unsigned bit = 1u << (unsigned)(k & 31);
        if ((atomicOr(bitmap + (k >> 5), bit) & bit) == 0u) fresh++;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) fresh += __shfl_xor_sync(0xffffffffu, fresh, o);
    if ((threadIdx.x & 31u) == 0u && fresh) atomicAdd(scratch, fresh);
}

__global__ void noalloc_store(const unsigned long long* scratch, unsigned long long* out) { *out = scratch[0]; }

// Device address of the scratch array for the current device (looked up
// once per device, with that device current).
int scratchFor(unsigned long long** ptr, int* sms) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        gpudb::setThreadError(std::string("gpudb_distinct_count_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
        return GPUDB_E_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        gpudb::setThreadError("gpudb_distinct_count_noalloc: device index out of range");
        return GPUDB_E_INVALID;
    }
    std::lock_guard<std::mutex> g(gMu);
    if (!gScratch[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, gpudb_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            gpudb::setThreadError(std::string("gpudb_distinct_count_noalloc: cudaGetSymbolAddress: ") +
                                  cudaGetErrorString(e));
            return GPUDB_E_CUDA;
        }
        int n = 0;
        e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess || n <= 0) {
            gpudb::setThreadError("gpudb_distinct_count_noalloc: cannot query the SM count");
            return GPUDB_E_CUDA;
        }
        gScratch[dev] = static_cast<unsigned long long*>(p);
        gSMs[dev] = n;
    }
    *ptr = gScratch[dev];
    *sms = gSMs[dev];
    return GPUDB_OK;
}

}  // namespace

extern "C" int gpudb_distinct_count_noalloc(const int32_t* key, const int32_t* filter, uint64_t n, int32_t thr,
                                            int64_t card, uint64_t* out_count, void* stream) {
    if (card < 1 || card > (int64_t)GPUDB_NOALLOC_MAX_CARD) {
        gpudb::setThreadError("gpudb_distinct_count_noalloc: card must be in [1, 4194304] (the static scratch "
                              "bitmap holds 2^22 keys), got " + std::to_string(card));
        return GPUDB_E_INVALID;
    }
    if (!out_count || (n && (!key || !filter))) {
        gpudb::setThreadError("gpudb_distinct_count_noalloc: NULL input or output pointer");
        return GPUDB_E_INVALID;
    }
    unsigned long long* scratch = nullptr;
    int sms = 0;
    const int st = scratchFor(&scratch, &sms);
    if (st != GPUDB_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const unsigned long long words64 = (unsigned long long)card / 64 + 1;
    const int threads = 256;
    const int clearBlocks = (int)((GPUDB_NOALLOC_HEADER_WORDS + words64 + threads - 1) / threads);
    noalloc_clear<<<clearBlocks, threads, 0, s>>>(scratch, words64);
    long long want = ((long long)n + threads - 1) / threads;
    const long long cap = (long long)sms * 8;
    const int blocks = (int)(want < 1 ? 1 : (want > cap ? cap : want));
    noalloc_count<<<blocks, threads, 0, s>>>(key, filter, (long long)n, thr, (long long)card, scratch);
    noalloc_store<<<1, 1, 0, s>>>(scratch, reinterpret_cast<unsigned long long*>(out_count));
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        gpudb::setThreadError(std::string("gpudb_distinct_count_noalloc: launch: ") + cudaGetErrorString(e));
        return GPUDB_E_LAUNCH;
    }
    return GPUDB_OK;
}
