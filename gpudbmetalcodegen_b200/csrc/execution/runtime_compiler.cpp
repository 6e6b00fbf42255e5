#include "runtime_compiler.h"

#include <atomic>

#include <dlfcn.h>
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include "cuda_api.h"

namespace gpudb {

namespace {

std::mutex gMu;
std::map<std::string, std::vector<char>> gMem;  // key -> cubin
std::map<std::string, std::string> gMemLog;      // key -> NVRTC log
std::string gCacheDir;
bool gCacheDirSet = false;
bool gFastMath = false;

uint64_t fnv1a(const std::string& s, uint64_t h = 1469598103934665603ull) {
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ull;
    }
    return h;
}

std::string hex64(uint64_t v) {
    char b[17];
    snprintf(b, sizeof b, "%016llx", (unsigned long long)v);
    return b;
}

std::string numbered(const std::string& src) {
    std::ostringstream o;
    std::istringstream in(src);
    std::string line;
    int n = 1;
    while (std::getline(in, line)) o << n++ << ": " << line << "\n";
    return o.str();
}

std::string defaultCacheDir() {
    if (const char* e = std::getenv("GPUDB_KCACHE")) return e;
    Dl_info info;
    if (dladdr((void*)&defaultCacheDir, &info) && info.dli_fname) {
        std::string p = info.dli_fname;  // .../gpudbmetalcodegen_b200/lib/libgpudb.so
        auto s = p.rfind('/');
        if (s != std::string::npos) {
            p = p.substr(0, s);
            s = p.rfind('/');
            if (s != std::string::npos) return p.substr(0, s) + "/_kcache";
        }
    }
    return "";
}

std::vector<std::string> baseOptions() {
    std::vector<std::string> o = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo", "--ptxas-options=-v",
                                  "-DGPUDB_NVRTC=1"};
    if (gFastMath) o.push_back("--use_fast_math");
    return o;
}

bool readFile(const std::string& path, std::vector<char>& out) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    out.assign(std::istreambuf_iterator<char>(f), {});
    return !out.empty();
}

void writeFileAtomic(const std::string& path, const std::vector<char>& data) {
    const std::string tmp = path + ".tmp" + std::to_string(getpid());
    {
        std::ofstream f(tmp, std::ios::binary);
        if (!f) return;
        f.write(data.data(), (std::streamsize)data.size());
        if (!f) return;
    }
    std::rename(tmp.c_str(), path.c_str());
}

}  // namespace

void RuntimeCompiler::setCacheDir(const std::string& dir) {
    std::lock_guard<std::mutex> g(gMu);
    gCacheDir = dir;
    gCacheDirSet = true;
}

std::string RuntimeCompiler::cacheDir() {
    std::lock_guard<std::mutex> g(gMu);
    if (!gCacheDirSet) {
        gCacheDir = defaultCacheDir();
        gCacheDirSet = true;
    }
    return gCacheDir;
}

void RuntimeCompiler::setFastMathEnabled(bool on) { gFastMath = on; }
bool RuntimeCompiler::fastMathEnabled() { return gFastMath; }

std::string RuntimeCompiler::nvrtcVersionString() {
    int major = 0, minor = 0;
    nvrtcVersion(&major, &minor);
    return std::to_string(major) + "." + std::to_string(minor);
}

bool RuntimeCompiler::compileToCubin(const std::string& source, CubinArtifact& out, std::string& error,
                                     const std::vector<std::string>& extraOptions) {
    std::vector<std::string> opts = baseOptions();
    for (const auto& o : extraOptions) opts.push_back(o);
    std::string keySrc = source + "\n//" + nvrtcVersionString();
    for (const auto& o : opts) keySrc += "\n//" + o;
    out.key = hex64(fnv1a(keySrc));
    {
        std::lock_guard<std::mutex> g(gMu);
        auto it = gMem.find(out.key);
        if (it != gMem.end()) {
            out.cubin = it->second;
            out.log = gMemLog[out.key];
            out.fromMemoryCache = true;
            return true;
        }
    }
    const std::string dir = cacheDir();
    if (!dir.empty() && readFile(dir + "/" + out.key + ".cubin", out.cubin)) {
        std::vector<char> log;
        if (readFile(dir + "/" + out.key + ".log", log)) out.log.assign(log.begin(), log.end());
        std::lock_guard<std::mutex> g(gMu);
        gMem[out.key] = out.cubin;
        gMemLog[out.key] = out.log;
        out.fromDiskCache = true;
        return true;
    }

    const auto t0 = std::chrono::steady_clock::now();
    nvrtcProgram prog;
    nvrtcResult r = nvrtcCreateProgram(&prog, source.c_str(), "gpudb_generated.cu", 0, nullptr, nullptr);
    if (r != NVRTC_SUCCESS) {
        error = std::string("nvrtcCreateProgram: ") + nvrtcGetErrorString(r);
        return false;
    }
    std::vector<const char*> copts;
    for (const auto& o : opts) copts.push_back(o.c_str());
    r = nvrtcCompileProgram(prog, (int)copts.size(), copts.data());
    size_t logSize = 0;
    nvrtcGetProgramLogSize(prog, &logSize);
    std::string log(logSize, '\0');
    if (logSize) nvrtcGetProgramLog(prog, log.data());
    while (!log.empty() && (log.back() == '\0' || log.back() == '\n')) log.pop_back();
    out.log = log;
    if (r != NVRTC_SUCCESS) {
        error = std::string("NVRTC compilation failed: ") + nvrtcGetErrorString(r) + "\n" + log + "\n--- source ---\n" +
                numbered(source);
        nvrtcDestroyProgram(&prog);
        return false;
    }
    size_t n = 0;
    r = nvrtcGetCUBINSize(prog, &n);
    if (r != NVRTC_SUCCESS || n == 0) {
        error = std::string("nvrtcGetCUBINSize: ") + nvrtcGetErrorString(r);
        nvrtcDestroyProgram(&prog);
        return false;
    }
    out.cubin.resize(n);
    nvrtcGetCUBIN(prog, out.cubin.data());
    nvrtcDestroyProgram(&prog);
    out.compileMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    {
        std::lock_guard<std::mutex> g(gMu);
        gMem[out.key] = out.cubin;
        gMemLog[out.key] = out.log;
    }
    if (!dir.empty()) {
        mkdir(dir.c_str(), 0755);
        writeFileAtomic(dir + "/" + out.key + ".log", std::vector<char>(out.log.begin(), out.log.end()));
        writeFileAtomic(dir + "/" + out.key + ".cubin", out.cubin);
    }
    return true;
}

RuntimeCompiler::CompiledQuery::~CompiledQuery() {
    if (module) {
        const DriverApi& api = driverApi();
        if (api.loaded) api.cuModuleUnload(module);
    }
}

std::shared_ptr<RuntimeCompiler::CompiledQuery> RuntimeCompiler::compileAndLoad(
    const std::string& source, const std::vector<std::string>& kernelNames, std::string& error) {
    CubinArtifact art;
    if (!compileToCubin(source, art, error)) return nullptr;
    const DriverApi& api = driverApi();
    if (!api.loaded) {
        error = "CUDA driver API unavailable: " + api.error;
        return nullptr;
    }
    static std::atomic<uint64_t> loads{0};
    auto cq = std::make_shared<CompiledQuery>();
    cq->loadId = ++loads;
    cq->key = art.key;
    cq->log = art.log;
    cq->compileMs = art.compileMs;
    cq->cached = art.fromDiskCache || art.fromMemoryCache;
    CUresult r = api.cuModuleLoadData(&cq->module, art.cubin.data());
    if (r != CUDA_SUCCESS) {
        cq->module = nullptr;
        error = "cuModuleLoadData: " + cuErrorString(r);
        return nullptr;
    }
    for (const auto& k : kernelNames) {
        CUfunction f = nullptr;
        r = api.cuModuleGetFunction(&f, cq->module, k.c_str());
        if (r != CUDA_SUCCESS) {
            error = "kernel function not found: " + k + " (" + cuErrorString(r) + ")";
            return nullptr;
        }
        cq->functions.push_back(f);
        cq->kernelNames.push_back(k);
    }
    return cq;
}

}  // namespace gpudb
