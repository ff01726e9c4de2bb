// Runtime compilation of integrator kernels for sm_100a.
//
// The step function of a system only exists as text at run time (the KRS body the
// session layer produced, or the right-hand side recognised in it), so — like the
// reference engine (parametric_engine.cpp:1530-1652, compile_*_if_needed) — kernels
// are compiled by NVRTC. Unlike the reference, which JITs generic compute_<cc> PTX,
// this emits an sm_100a CUBIN directly and keeps an in-memory module cache keyed by a
// 64-bit hash of the complete source and options.
//
// The CUDA driver API is reached through dlopen("libcuda.so.1") so that the library
// loads on machines without a driver (symbol checks, CPU-only tests).
#pragma once

#include <cuda.h>

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace ucb {

// Driver API entry points resolved at run time.
struct Driver {
    bool loaded = false;
    std::string load_error;
    CUresult (*cuInit)(unsigned int) = nullptr;
    CUresult (*cuModuleLoadDataEx)(CUmodule*, const void*, unsigned int, CUjit_option*, void**) = nullptr;
    CUresult (*cuModuleGetFunction)(CUfunction*, CUmodule, const char*) = nullptr;
    CUresult (*cuModuleUnload)(CUmodule) = nullptr;
    CUresult (*cuLaunchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                               unsigned, CUstream, void**, void**) = nullptr;
    CUresult (*cuFuncSetAttribute)(CUfunction, CUfunction_attribute, int) = nullptr;
    CUresult (*cuFuncGetAttribute)(int*, CUfunction_attribute, CUfunction) = nullptr;
    CUresult (*cuGetErrorString)(CUresult, const char**) = nullptr;
    CUresult (*cuCtxGetCurrent)(CUcontext*) = nullptr;
    CUresult (*cuCtxSetCurrent)(CUcontext) = nullptr;
    CUresult (*cuOccupancyMaxActiveBlocksPerMultiprocessor)(int*, CUfunction, int, size_t) = nullptr;
    CUresult (*cuModuleGetGlobal)(CUdeviceptr*, size_t*, CUmodule, const char*) = nullptr;
    CUresult (*cuMemcpyHtoD)(CUdeviceptr, const void*, size_t) = nullptr;
};

Driver& driver();
std::string cu_error_string(CUresult r);

// One compiled program: module + looked-up kernels.
struct Module {
    CUmodule module = nullptr;
    std::map<std::string, CUfunction> functions;
    std::string log;
    int registers = 0;
    ~Module();
};

struct CompileRequest {
    std::string name;                 // program name for diagnostics
    std::string source;               // main translation unit
    std::vector<std::pair<std::string, std::string>> headers;  // name -> text
    std::vector<std::string> options; // extra NVRTC options
    std::vector<std::string> kernels; // extern "C" kernel names to look up
};

// Compiles (NVRTC, --gpu-architecture=sm_100a) to a CUBIN. Works without a GPU.
bool nvrtc_compile_cubin(const CompileRequest& rq, std::string& cubin, std::string& log);

// Compiles into the on-disk CUBIN cache without loading (no GPU needed). Returns false
// with the compiler log on error.
bool precompile_to_disk(const CompileRequest& rq, std::string& err);

// Thread-safe cache of loaded modules (needs a current CUDA context to load).
class ModuleCache {
public:
    // Device address of the owner's run-control block (ucb_device.cuh UcbControl); every
    // module loaded afterwards that defines the global `ucb_control` gets it.
    void set_control(void* device_ptr) { control_ = device_ptr; }
    std::shared_ptr<Module> get(const CompileRequest& rq, std::string& err);
    // Already-loaded module for this request, or nullptr (never compiles or loads).
    std::shared_ptr<Module> find(const CompileRequest& rq) const;
    size_t size() const;
    void clear();

private:
    mutable std::mutex mu_;
    std::map<uint64_t, std::shared_ptr<Module>> cache_;
    void* control_ = nullptr;
};

uint64_t fnv1a64(const std::string& s, uint64_t h = 1469598103934665603ULL);

// Directory of the on-disk CUBIN cache ("" when unknown).
std::string cubin_cache_dir();

}  // namespace ucb
