#pragma once
// ===================================================================
// RuntimeCompiler — generated CUDA C++ -> sm_100a cubin -> CUmodule.
//
// Replaces the reference's Metal RuntimeCompiler
// (codegen/execution/runtime_compiler.h:9-41): compile() returns nothing
// and records a numbered source dump in the error text on failure (the
// reference prints it to stderr); getPipeline() caches by kernel name.
// B200 design: NVRTC compiles straight to an sm_100a CUBIN (no PTX JIT on
// load); cubins are cached by a 64-bit hash of (source, options, NVRTC
// version) in memory and on disk, so a process that has seen a plan
// before — or a build that pre-compiled it — loads without compiling.
// Compilation needs no GPU; loading does.
// ===================================================================
#include <cuda.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace gpudb {

struct CubinArtifact {
    std::string key;           // cache key (hex)
    std::vector<char> cubin;
    std::string log;           // NVRTC log (includes ptxas -v resource lines)
    double compileMs = 0.0;    // 0 when served from a cache
    bool fromDiskCache = false;
    bool fromMemoryCache = false;
};

class RuntimeCompiler {
public:
    // Compile-only: returns false and fills `error` (with a numbered source
    // listing) on failure.
    static bool compileToCubin(const std::string& source, CubinArtifact& out, std::string& error,
                               const std::vector<std::string>& extraOptions = {});

    static void setCacheDir(const std::string& dir);
    static std::string cacheDir();
    static std::string nvrtcVersionString();
    static void setFastMathEnabled(bool on);
    static bool fastMathEnabled();

    struct CompiledQuery {
        CUmodule module = nullptr;
        std::vector<CUfunction> functions;
        std::vector<std::string> kernelNames;
        std::string key;
        std::string log;
        double compileMs = 0.0;
        bool cached = false;
        // Unique per load: a module unloaded and loaded again may reuse its
        // CUfunction handles, so per-function caches (shared-memory
        // attributes, captured graphs) are keyed by this, not by handles.
        uint64_t loadId = 0;
        ~CompiledQuery();
    };

    // Compile (or fetch) and load into the current context, resolving each
    // kernel name. Returns nullptr and fills `error` on failure.
    static std::shared_ptr<CompiledQuery> compileAndLoad(const std::string& source,
                                                         const std::vector<std::string>& kernelNames,
                                                         std::string& error);
};

}  // namespace gpudb
