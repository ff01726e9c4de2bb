#include "jit.h"

#include <dlfcn.h>
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace ucb {

uint64_t fnv1a64(const std::string& s, uint64_t h) {
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ULL;
    }
    return h;
}

Driver& driver() {
    static Driver d;
    static std::once_flag once;
    std::call_once(once, [] {
        void* lib = dlopen("libcuda.so.1", RTLD_NOW | RTLD_GLOBAL);
        if (!lib) lib = dlopen("libcuda.so", RTLD_NOW | RTLD_GLOBAL);
        if (!lib) {
            d.load_error = std::string("cannot load the CUDA driver (libcuda.so.1): ") + dlerror();
            return;
        }
        auto sym = [&](const char* versioned, const char* plain) -> void* {
            void* p = dlsym(lib, versioned);
            if (!p) p = dlsym(lib, plain);
            return p;
        };
#define UCB_LOAD(field, v, p) d.field = reinterpret_cast<decltype(d.field)>(sym(v, p))
        UCB_LOAD(cuInit, "cuInit", "cuInit");
        UCB_LOAD(cuModuleLoadDataEx, "cuModuleLoadDataEx", "cuModuleLoadDataEx");
        UCB_LOAD(cuModuleGetFunction, "cuModuleGetFunction", "cuModuleGetFunction");
        UCB_LOAD(cuModuleUnload, "cuModuleUnload", "cuModuleUnload");
        UCB_LOAD(cuLaunchKernel, "cuLaunchKernel", "cuLaunchKernel");
        UCB_LOAD(cuFuncSetAttribute, "cuFuncSetAttribute", "cuFuncSetAttribute");
        UCB_LOAD(cuFuncGetAttribute, "cuFuncGetAttribute", "cuFuncGetAttribute");
        UCB_LOAD(cuGetErrorString, "cuGetErrorString", "cuGetErrorString");
        UCB_LOAD(cuCtxGetCurrent, "cuCtxGetCurrent", "cuCtxGetCurrent");
        UCB_LOAD(cuCtxSetCurrent, "cuCtxSetCurrent", "cuCtxSetCurrent");
        UCB_LOAD(cuOccupancyMaxActiveBlocksPerMultiprocessor, "cuOccupancyMaxActiveBlocksPerMultiprocessor",
                 "cuOccupancyMaxActiveBlocksPerMultiprocessor");
        UCB_LOAD(cuModuleGetGlobal, "cuModuleGetGlobal_v2", "cuModuleGetGlobal");
        UCB_LOAD(cuMemcpyHtoD, "cuMemcpyHtoD_v2", "cuMemcpyHtoD");
#undef UCB_LOAD
        if (!d.cuInit || !d.cuModuleLoadDataEx || !d.cuModuleGetFunction || !d.cuLaunchKernel ||
            !d.cuModuleUnload || !d.cuGetErrorString) {
            d.load_error = "CUDA driver is missing required entry points";
            return;
        }
        d.loaded = true;
    });
    return d;
}

std::string cu_error_string(CUresult r) {
    const char* s = nullptr;
    if (driver().cuGetErrorString) driver().cuGetErrorString(r, &s);
    return s ? std::string(s) : ("CUresult " + std::to_string((int)r));
}

Module::~Module() {
    if (module && driver().loaded) driver().cuModuleUnload(module);
}

bool nvrtc_compile_cubin(const CompileRequest& rq, std::string& cubin, std::string& log) {
    std::vector<const char*> hsrc, hname;
    for (auto& h : rq.headers) {
        hname.push_back(h.first.c_str());
        hsrc.push_back(h.second.c_str());
    }
    nvrtcProgram prog = nullptr;
    nvrtcResult r = nvrtcCreateProgram(&prog, rq.source.c_str(), rq.name.c_str(), (int)hsrc.size(),
                                       hsrc.data(), hname.data());
    if (r != NVRTC_SUCCESS) {
        log = std::string("nvrtcCreateProgram: ") + nvrtcGetErrorString(r);
        return false;
    }
    std::vector<std::string> opts = {"--gpu-architecture=sm_100a", "--std=c++17", "-default-device",
                                     "--extra-device-vectorization", "-lineinfo"};
    for (auto& o : rq.options) opts.push_back(o);
    if (std::getenv("UCB_PTXAS_VERBOSE")) opts.push_back("--ptxas-options=-v");
    std::vector<const char*> copts;
    for (auto& o : opts) copts.push_back(o.c_str());
    r = nvrtcCompileProgram(prog, (int)copts.size(), copts.data());
    size_t logsz = 0;
    nvrtcGetProgramLogSize(prog, &logsz);
    if (logsz > 1) {
        log.resize(logsz);
        nvrtcGetProgramLog(prog, &log[0]);
        while (!log.empty() && log.back() == '\0') log.pop_back();
    }
    if (r != NVRTC_SUCCESS) {
        log = "NVRTC compile failed (" + rq.name + "):\n" + log;
        nvrtcDestroyProgram(&prog);
        return false;
    }
    if (std::getenv("UCB_PTXAS_VERBOSE") && !log.empty()) std::fprintf(stderr, "[ucb nvrtc %s]\n%s\n", rq.name.c_str(), log.c_str());
    size_t sz = 0;
    nvrtcGetCUBINSize(prog, &sz);
    cubin.assign(sz, '\0');
    nvrtcGetCUBIN(prog, &cubin[0]);
    nvrtcDestroyProgram(&prog);
    return true;
}

namespace {

uint64_t request_key(const CompileRequest& rq) {
    uint64_t h = fnv1a64(rq.source);
    for (auto& x : rq.headers) h = fnv1a64(x.second, fnv1a64(x.first, h));
    for (auto& o : rq.options) h = fnv1a64(o, h);
    int ver = 0;
    int maj = 0, min = 0;
    nvrtcVersion(&maj, &min);
    ver = maj * 100 + min;
    h = fnv1a64(std::to_string(ver), h);
    return h;
}

// Directory of the loaded libucb.so; the CUBIN disk cache defaults to <dir>/_cache.
std::string cache_dir() {
    const char* e = std::getenv("UCB_CUBIN_CACHE");
    if (e) return e;
    Dl_info info;
    if (dladdr(reinterpret_cast<void*>(&cache_dir), &info) && info.dli_fname) {
        std::string p(info.dli_fname);
        auto pos = p.find_last_of('/');
        if (pos != std::string::npos) return p.substr(0, pos) + "/_cache";
    }
    return "";
}

bool read_file(const std::string& path, std::string& out) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    std::ostringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return !out.empty();
}

void write_file_atomic(const std::string& path, const std::string& data) {
    const std::string tmp = path + ".tmp" + std::to_string(getpid());
    {
        std::ofstream f(tmp, std::ios::binary);
        if (!f) return;
        f.write(data.data(), (std::streamsize)data.size());
    }
    std::rename(tmp.c_str(), path.c_str());
}

}  // namespace

std::string cubin_cache_dir() { return cache_dir(); }

bool precompile_to_disk(const CompileRequest& rq, std::string& err) {
    const uint64_t key = request_key(rq);
    const std::string dir = cache_dir();
    char fname[64];
    std::snprintf(fname, sizeof fname, "/k_%016llx.cubin", (unsigned long long)key);
    const std::string path = dir.empty() ? "" : dir + fname;
    std::string cubin, log;
    if (!path.empty() && read_file(path, cubin)) return true;
    if (!nvrtc_compile_cubin(rq, cubin, log)) {
        err = log;
        return false;
    }
    if (!path.empty()) {
        mkdir(dir.c_str(), 0755);
        write_file_atomic(path, cubin);
    }
    return true;
}

std::shared_ptr<Module> ModuleCache::get(const CompileRequest& rq, std::string& err) {
    const uint64_t key = request_key(rq);
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = cache_.find(key);
        if (it != cache_.end()) return it->second;
    }
    Driver& d = driver();
    if (!d.loaded) {
        err = d.load_error;
        return nullptr;
    }
    std::string cubin, log;
    const std::string dir = cache_dir();
    char fname[64];
    std::snprintf(fname, sizeof fname, "/k_%016llx.cubin", (unsigned long long)key);
    const std::string path = dir.empty() ? "" : dir + fname;
    if (path.empty() || !read_file(path, cubin)) {
        if (!nvrtc_compile_cubin(rq, cubin, log)) {
            err = log;
            return nullptr;
        }
        if (!path.empty()) {
            mkdir(dir.c_str(), 0755);
            write_file_atomic(path, cubin);
        }
    }
    auto m = std::make_shared<Module>();
    m->log = log;
    CUresult r = d.cuModuleLoadDataEx(&m->module, cubin.data(), 0, nullptr, nullptr);
    if (r != CUDA_SUCCESS) {
        m->module = nullptr;
        err = "cuModuleLoadDataEx(" + rq.name + "): " + cu_error_string(r);
        return nullptr;
    }
    for (auto& k : rq.kernels) {
        CUfunction f = nullptr;
        r = d.cuModuleGetFunction(&f, m->module, k.c_str());
        if (r != CUDA_SUCCESS) {
            err = "cuModuleGetFunction(" + k + "): " + cu_error_string(r);
            return nullptr;
        }
        m->functions[k] = f;
        if (d.cuFuncGetAttribute) d.cuFuncGetAttribute(&m->registers, CU_FUNC_ATTRIBUTE_NUM_REGS, f);
    }
    if (control_ && d.cuModuleGetGlobal && d.cuMemcpyHtoD) {
        CUdeviceptr g = 0;
        size_t gsz = 0;
        if (d.cuModuleGetGlobal(&g, &gsz, m->module, "ucb_control") == CUDA_SUCCESS && gsz == sizeof(void*)) {
            r = d.cuMemcpyHtoD(g, &control_, sizeof(void*));
            if (r != CUDA_SUCCESS) {
                err = "binding the run-control block: " + cu_error_string(r);
                return nullptr;
            }
        }
    }
    std::lock_guard<std::mutex> lk(mu_);
    cache_[key] = m;
    return m;
}

std::shared_ptr<Module> ModuleCache::find(const CompileRequest& rq) const {
    const uint64_t key = request_key(rq);
    std::lock_guard<std::mutex> lk(mu_);
    auto it = cache_.find(key);
    return it == cache_.end() ? nullptr : it->second;
}

size_t ModuleCache::size() const {
    std::lock_guard<std::mutex> lk(mu_);
    return cache_.size();
}

void ModuleCache::clear() {
    std::lock_guard<std::mutex> lk(mu_);
    cache_.clear();
}

}  // namespace ucb
