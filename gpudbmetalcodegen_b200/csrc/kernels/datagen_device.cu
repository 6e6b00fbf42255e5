// Device twins of the mixed-workload generators (include/gpudb_datagen.h):
// the same per-row functions as the host generators (datagen_core.h), run
// as grid-stride kernels that write straight into device columns, so large
// resident tables are made in HBM without a host copy or an upload.
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "../../../include/gpudb_datagen.h"
#include "../datagen/datagen_core.h"

namespace gpudb_gen {
const std::vector<double>& zipfCdf(uint64_t n, double s);
void setError(const std::string& message);  // datagen.cpp: gpudb_datagen_last_error
}  // namespace gpudb_gen

namespace {

using namespace gpudb_gen;

__global__ void kGenMix(uint64_t seed, uint64_t nranks, uint64_t dimRows, const double* __restrict__ cdf,
                        uint64_t row0, uint64_t n, int32_t* rankU, int32_t* rankZ, int32_t* filter, int64_t* value,
                        int32_t* fk) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const MixRow m = mixRow(seed, nranks, dimRows, cdf, row0 + i);
        rankU[i] = m.rank_u;
        rankZ[i] = m.rank_z;
        filter[i] = m.filter;
        value[i] = m.value;
        fk[i] = m.fk;
    }
}

__global__ void kGenMixdim(uint64_t seed, uint64_t row0, uint64_t n, int32_t* key, int32_t* attr) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        key[i] = (int32_t)(row0 + i + 1);
        attr[i] = mixdimAttr(seed, row0 + i);
    }
}

int gridFor(uint64_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (n + 255) / 256;
    return (int)(want < (uint64_t)sms * 8 ? (want ? want : 1) : (uint64_t)sms * 8);
}

#define G_CHECK(call)                                                                             \
    do {                                                                                          \
        const cudaError_t _e = (call);                                                            \
        if (_e != cudaSuccess) {                                                                  \
            gpudb_gen::setError(std::string("datagen: ") + #call + ": " + cudaGetErrorString(_e)); \
            return -1;                                                                            \
        }                                                                                         \
    } while (0)

}  // namespace

extern "C" {

int gpudb_gen_mix_device(uint64_t seed, uint64_t nranks, double s, uint64_t dim_rows, uint64_t row0, uint64_t n,
                         int32_t* rank_u, int32_t* rank_z, int32_t* filter, int64_t* value, int32_t* fk,
                         void* stream) {
    if ((n && (!rank_u || !rank_z || !filter || !value || !fk)) || nranks == 0 || nranks > 0x7FFFFFFFull ||
        dim_rows == 0 || !(s > 0.0))
        return -1;
    if (n == 0) return 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const std::vector<double>& cdf = gpudb_gen::zipfCdf(nranks, s);
    double* dcdf = nullptr;
    G_CHECK(cudaMallocAsync((void**)&dcdf, sizeof(double) * nranks, st));
    G_CHECK(cudaMemcpyAsync(dcdf, cdf.data(), sizeof(double) * nranks, cudaMemcpyHostToDevice, st));
    kGenMix<<<gridFor(n), 256, 0, st>>>(seed, nranks, dim_rows, dcdf, row0, n, rank_u, rank_z, filter, value, fk);
    G_CHECK(cudaGetLastError());
    G_CHECK(cudaFreeAsync(dcdf, st));
    G_CHECK(cudaStreamSynchronize(st));
    return 0;
}

int gpudb_gen_mixdim_device(uint64_t seed, uint64_t row0, uint64_t n, int32_t* key, int32_t* attr, void* stream) {
    if (n && (!key || !attr)) return -1;
    if (n == 0) return 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    kGenMixdim<<<gridFor(n), 256, 0, st>>>(seed, row0, n, key, attr);
    G_CHECK(cudaGetLastError());
    G_CHECK(cudaStreamSynchronize(st));
    return 0;
}

}  // extern "C"
