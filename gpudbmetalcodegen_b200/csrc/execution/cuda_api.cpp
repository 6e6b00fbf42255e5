#include "cuda_api.h"

#include <mutex>

namespace gpudb {

namespace {

template <typename F>
bool fetch(DriverApi& api, const char* name, F& fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    const cudaError_t e = cudaGetDriverEntryPointByVersion(name, &p, 12000, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p) {
        api.error = std::string("driver entry point '") + name + "' unavailable: " + cudaGetErrorString(e);
        return false;
    }
    fn = reinterpret_cast<F>(p);
    return true;
}

}  // namespace

const DriverApi& driverApi() {
    static DriverApi api;
    static std::once_flag once;
    std::call_once(once, []() {
        bool ok = fetch(api, "cuModuleLoadData", api.cuModuleLoadData) &&
                  fetch(api, "cuModuleUnload", api.cuModuleUnload) &&
                  fetch(api, "cuModuleGetFunction", api.cuModuleGetFunction) &&
                  fetch(api, "cuLaunchKernel", api.cuLaunchKernel) &&
                  fetch(api, "cuFuncSetAttribute", api.cuFuncSetAttribute) &&
                  fetch(api, "cuFuncGetAttribute", api.cuFuncGetAttribute) &&
                  fetch(api, "cuOccupancyMaxActiveBlocksPerMultiprocessor",
                        api.cuOccupancyMaxActiveBlocksPerMultiprocessor) &&
                  fetch(api, "cuGetErrorString", api.cuGetErrorString);
        api.loaded = ok;
    });
    return api;
}

std::string cuErrorString(CUresult r) {
    const DriverApi& api = driverApi();
    const char* s = nullptr;
    if (api.cuGetErrorString && api.cuGetErrorString(r, &s) == CUDA_SUCCESS && s) return s;
    return "CUresult " + std::to_string((int)r);
}

}  // namespace gpudb
