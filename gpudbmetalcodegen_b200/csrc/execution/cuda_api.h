#pragma once
// Driver-API entry points used by the runtime (module load, launch,
// occupancy, function attributes). They are fetched through the CUDA
// runtime's cudaGetDriverEntryPointByVersion, so the library links no
// libcuda and loads on hosts without a GPU driver (the first call then
// fails cleanly with a status).
#include <cuda.h>
#include <cuda_runtime.h>

#include <string>

namespace gpudb {

struct DriverApi {
    bool loaded = false;
    std::string error;
    CUresult (*cuModuleLoadData)(CUmodule*, const void*) = nullptr;
    CUresult (*cuModuleUnload)(CUmodule) = nullptr;
    CUresult (*cuModuleGetFunction)(CUfunction*, CUmodule, const char*) = nullptr;
    CUresult (*cuLaunchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                               CUstream, void**, void**) = nullptr;
    CUresult (*cuFuncSetAttribute)(CUfunction, CUfunction_attribute, int) = nullptr;
    CUresult (*cuFuncGetAttribute)(int*, CUfunction_attribute, CUfunction) = nullptr;
    CUresult (*cuOccupancyMaxActiveBlocksPerMultiprocessor)(int*, CUfunction, int, size_t) = nullptr;
    CUresult (*cuGetErrorString)(CUresult, const char**) = nullptr;
};

// Loads the table once per process; returns it (check .loaded / .error).
const DriverApi& driverApi();

std::string cuErrorString(CUresult r);

}  // namespace gpudb
