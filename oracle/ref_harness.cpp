// TEST INFRASTRUCTURE (part of the oracle): launches the reference's own integrator
// kernels, compiled unchanged from its NVRTC templates by oracle/build_ref_kernels.py,
// with the host-side sizing, argument order and result unpacking of the reference's
// drivers. It never calls the engine (libucb); only tests load it, to pin the oracle and
// the engine to the reference's own code running on the GPU.
//
// Restated host logic (U-CUDA/parametric_engine.cpp):
//   run_lle_2d  :2587-2965  (step counts :2717-2718, block size :2848-2851, arguments
//                            :2854-2903, dynamic shared memory :2905-2906, flags :2930)
//   run_ls_2d   :3430-3786  (block size :3683-3688, shared memory :3714-3715, the
//                            per-cell N-exponent layout :3740-3755)
//   run_bif1d   :1674-2091  (record length :1795-1796, arguments :1960-2000, shared
//                            memory :2002, peakFinderCUDA launch :2007-2024, rows :2033-2083)
// The device type is the reference's `typedef float numb` (configCUDA.h:4): requests in
// double are narrowed to float where the reference narrows them (to_numb, `(numb)` casts).
// The memory budget chunking (nPtsLimiter from cudaMemGetInfo) always yields one chunk for
// the grids the tests use, so one launch covers the grid (amountOfCalculatedPoints = 0).
#include <cuda.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

typedef float numb;

namespace {

thread_local std::string g_err;

bool ck(CUresult r, const char* where) {
    if (r == CUDA_SUCCESS) return true;
    const char* s = nullptr;
    cuGetErrorString(r, &s);
    g_err = std::string(where) + ": " + (s ? s : "unknown CUDA error");
    return false;
}

// The primary context of device 0, current for the lifetime of one call (the same
// context the CUDA runtime and the engine use, so device memory stays in one place).
struct Scope {
    CUcontext ctx = nullptr;
    bool ok = false;
    Scope() {
        CUdevice dev;
        if (!ck(cuInit(0), "cuInit") || !ck(cuDeviceGet(&dev, 0), "cuDeviceGet") ||
            !ck(cuDevicePrimaryCtxRetain(&ctx, dev), "cuDevicePrimaryCtxRetain") ||
            !ck(cuCtxPushCurrent(ctx), "cuCtxPushCurrent"))
            return;
        ok = true;
    }
    ~Scope() {
        if (ok) {
            CUcontext c;
            cuCtxPopCurrent(&c);
            CUdevice dev;
            if (cuDeviceGet(&dev, 0) == CUDA_SUCCESS) cuDevicePrimaryCtxRelease(dev);
        }
    }
};

struct Module {
    CUmodule mod = nullptr;
    ~Module() { if (mod) cuModuleUnload(mod); }
    bool load(const char* path) {
        std::ifstream f(path, std::ios::binary);
        if (!f) { g_err = std::string("cannot read ") + path; return false; }
        std::vector<char> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
        return ck(cuModuleLoadData(&mod, bytes.data()), "cuModuleLoadData");
    }
    bool fn(const char* name, CUfunction* out) { return ck(cuModuleGetFunction(out, mod, name), name); }
};

// Device buffers freed at scope exit, like the reference's cleanup() lambdas.
struct Buffers {
    std::vector<CUdeviceptr> ptrs;
    ~Buffers() { for (CUdeviceptr p : ptrs) cuMemFree(p); }
    bool alloc(CUdeviceptr* p, size_t bytes, const char* what) {
        if (!ck(cuMemAlloc(p, bytes ? bytes : 4), what)) return false;
        ptrs.push_back(*p);
        return true;
    }
    template <class T>
    bool upload(CUdeviceptr* p, const std::vector<T>& v, const char* what) {
        return alloc(p, v.size() * sizeof(T), what) &&
               (v.empty() || ck(cuMemcpyHtoD(*p, v.data(), v.size() * sizeof(T)), what));
    }
};

std::vector<numb> to_numb(const double* p, int n) { return std::vector<numb>(p, p + n); }

bool timed_launch(CUfunction f, unsigned grid, unsigned block, unsigned shared, void** args,
                  float* ms, const char* what) {
    CUevent e0 = nullptr, e1 = nullptr;
    bool ok = ck(cuEventCreate(&e0, CU_EVENT_DEFAULT), "cuEventCreate") &&
              ck(cuEventCreate(&e1, CU_EVENT_DEFAULT), "cuEventCreate") &&
              ck(cuEventRecord(e0, nullptr), "cuEventRecord") &&
              ck(cuLaunchKernel(f, grid, 1, 1, block, 1, 1, shared, nullptr, args, nullptr), what) &&
              ck(cuEventRecord(e1, nullptr), "cuEventRecord") && ck(cuCtxSynchronize(), what);
    float t = 0.f;
    if (ok) ok = ck(cuEventElapsedTime(&t, e0, e1), "cuEventElapsedTime");
    if (ms) *ms += t;
    if (e0) cuEventDestroy(e0);
    if (e1) cuEventDestroy(e1);
    return ok;
}

}  // namespace

extern "C" {

const char* refh_last_error() { return g_err.c_str(); }

// LLEKernelCUDA (ls = 0) or LSKernelCUDA (ls = 1) over an nPts x nPts grid at kernel level
// (par_or_var is compiled into the module; ranges / indices are the kernel slots X, Y).
// out: nPts^2 values (ls = 0) or nPts^2 x nx values, cell-major (ls = 1), kernel order,
// widened from numb. Returns 0 on success.
int refh_lle2d(const char* cubin, const char* kernel, int ls, int nPts, double NT, double tMax,
               double transientTime, double h, double eps, double maxValue, const double* ranges4,
               const int* idx2, const double* ic, int nx, const double* values, int nvals, int hSweepAxis,
               int logAxisMask, double* out, float* kernel_ms) {
    Scope scope;
    if (!scope.ok) return 1;
    Module m;
    CUfunction f;
    if (!m.load(cubin) || !m.fn(kernel, &f)) return 1;

    const int N = nx;
    const int amountOfPointsInBlock = (int)(tMax / NT);
    const int amountOfPointsForSkip = (int)(transientTime / h);
    if (amountOfPointsInBlock <= 0) { g_err = "amountOfPointsInBlock <= 0"; return 1; }
    const size_t total = (size_t)nPts * (size_t)nPts;
    const size_t per_cell = ls ? (size_t)N : 1;

    Buffers b;
    CUdeviceptr d_ranges, d_idx, d_ic, d_values, d_result;
    std::vector<numb> ranges = to_numb(ranges4, 4);
    std::vector<int> idx(idx2, idx2 + 2);
    if (!b.upload(&d_ranges, ranges, "ranges") || !b.upload(&d_idx, idx, "indices") ||
        !b.upload(&d_ic, to_numb(ic, N), "initial conditions") ||
        !b.upload(&d_values, to_numb(values, nvals), "values") ||
        !b.alloc(&d_result, total * per_cell * sizeof(numb), "result"))
        return 1;

    int blockSize;
    unsigned shared;
    if (!ls) {
        blockSize = (int)std::ceil((1024.0 * 32.0) / ((double)(3 * N + nvals) * (double)sizeof(numb)));
        if (blockSize < 1) blockSize = 1;
        if (blockSize > 32) blockSize = 32;
        shared = (unsigned)((3 * N + nvals) * sizeof(numb) * blockSize);
    } else {
        blockSize = (int)(32000 / ((double)(3 * N + 2 * N * N + nvals) * (double)sizeof(numb)));
        if (blockSize > 32) blockSize = 32;
        if (blockSize < 1) blockSize = 1;
        shared = (unsigned)((3 * N + 2 * N * N + nvals) * sizeof(numb) * blockSize);
    }
    const int gridSize = (int)((total + blockSize - 1) / blockSize);

    int nPts_arg = nPts, nPtsLimiter_arg = (int)total;
    numb NT_arg = (numb)NT, tMax_arg = (numb)tMax;
    int sizeOfBlock_arg = amountOfPointsInBlock, amountOfCalculatedPoints = 0;
    int amountOfPointsForSkip_arg = amountOfPointsForSkip, dimension_arg = 2;
    numb h_arg = (numb)h, eps_arg = (numb)eps;
    int amountOfIC_arg = N, amountOfValues_arg = nvals, amountOfIterations_arg = (int)(tMax / NT);
    int preScaller_arg = 1, writableVar_arg = 0;
    numb maxValue_arg = (numb)maxValue;
    int hSweepAxis_arg = hSweepAxis;
    numb transientTime_arg = (numb)transientTime;
    int logAxisMask_arg = logAxisMask;
    void* args[] = {&nPts_arg, &nPtsLimiter_arg, &NT_arg, &tMax_arg, &sizeOfBlock_arg,
                    &amountOfCalculatedPoints, &amountOfPointsForSkip_arg, &dimension_arg, &d_ranges,
                    &h_arg, &eps_arg, &d_idx, &d_ic, &amountOfIC_arg, &d_values, &amountOfValues_arg,
                    &amountOfIterations_arg, &preScaller_arg, &writableVar_arg, &maxValue_arg, &d_result,
                    &hSweepAxis_arg, &transientTime_arg, &logAxisMask_arg};
    if (kernel_ms) *kernel_ms = 0.f;
    if (!timed_launch(f, gridSize, blockSize, shared, args, kernel_ms, "cuLaunchKernel")) return 1;

    std::vector<numb> host(total * per_cell);
    if (!ck(cuMemcpyDtoH(host.data(), d_result, host.size() * sizeof(numb)), "copy result")) return 1;
    for (size_t i = 0; i < host.size(); ++i) out[i] = host[i];
    return 0;
}

// calculateDiscreteModelCUDA + peakFinderCUDA over nPts points of one axis (run_bif1d,
// no continuation, no h sweep). counts[k] = the point's peak count as run_bif1d stores it
// in res.flags (-1 unusable, 0 none); peaks / intervals: the first min(count, cap) entries
// of the point's row, widened from numb, NaN beyond.
int refh_bif1d(const char* cubin, const char* kernel_traj, const char* kernel_peak, int nPts,
               int sweep_over_var, double lo, double hi, int index, const double* ic, int nx,
               const double* values, int nvals, double h, double transientTime, double tMax, int preScaller,
               int writableVar, double maxValue, int logAxisMask, int cap, int* counts, double* peaks,
               double* intervals, float* kernel_ms) {
    Scope scope;
    if (!scope.ok) return 1;
    Module m;
    CUfunction ft, fp;
    if (!m.load(cubin) || !m.fn(kernel_traj, &ft) || !m.fn(kernel_peak, &fp)) return 1;

    const int N = nx;
    const int amountOfPointsInBlock = (int)std::ceil(tMax / h / preScaller);
    const int amountOfPointsForSkip = (int)(transientTime / h);
    if (amountOfPointsInBlock <= 0) { g_err = "amountOfPointsInBlock <= 0"; return 1; }
    const size_t rows = (size_t)nPts * (size_t)amountOfPointsInBlock;

    Buffers b;
    CUdeviceptr d_data, d_ranges, d_idx, d_ic, d_values, d_npeaks, d_peaks, d_times, d_iters;
    std::vector<numb> ranges = {(numb)lo, (numb)hi};
    std::vector<int> idx = {index};
    if (!b.alloc(&d_data, rows * sizeof(numb), "data") || !b.upload(&d_ranges, ranges, "ranges") ||
        !b.upload(&d_idx, idx, "indices") || !b.upload(&d_ic, to_numb(ic, N), "initial conditions") ||
        !b.upload(&d_values, to_numb(values, nvals), "values") ||
        !b.alloc(&d_peaks, rows * sizeof(numb), "outPeaks") || !b.alloc(&d_times, rows * sizeof(numb), "timeOfPeaks") ||
        !b.alloc(&d_npeaks, (size_t)nPts * sizeof(int), "amountOfPeaks") ||
        !b.alloc(&d_iters, (size_t)nPts * sizeof(int), "actualIterations"))
        return 1;

    const int blockSize = 32;
    const int gridSize = (nPts + blockSize - 1) / blockSize;
    int nPts_int = nPts, nPtsLimiter_int = nPts;
    size_t sizeOfBlock_s = (size_t)amountOfPointsInBlock, amountOfCalculatedPoints = 0;
    size_t amountOfPointsForSkip_s = (size_t)amountOfPointsForSkip;
    int dimension = 1;
    numb h_arg = (numb)h;
    int amountOfIC_int = N, amountOfValues_int = nvals;
    size_t amountOfIterations_arg = (size_t)amountOfPointsInBlock;
    int preScaller_int = preScaller, writableVar_int = writableVar;
    numb maxValue_arg = (numb)maxValue;
    bool par_or_var_arg = !sweep_over_var;
    int hSweepAxis_arg = -1;
    numb transientTime_arg = (numb)transientTime, tMax_arg = (numb)tMax;
    int logAxisMask_arg = logAxisMask;
    void* args_traj[] = {&nPts_int, &nPtsLimiter_int, &sizeOfBlock_s, &amountOfCalculatedPoints,
                         &amountOfPointsForSkip_s, &dimension, &d_ranges, &h_arg, &d_idx, &d_ic,
                         &amountOfIC_int, &d_values, &amountOfValues_int, &amountOfIterations_arg,
                         &preScaller_int, &writableVar_int, &maxValue_arg, &d_data, &d_npeaks,
                         &par_or_var_arg, &hSweepAxis_arg, &transientTime_arg, &tMax_arg, &d_iters,
                         &logAxisMask_arg};
    const unsigned shared = (unsigned)((N + nvals) * sizeof(numb) * blockSize);
    if (kernel_ms) *kernel_ms = 0.f;
    if (!timed_launch(ft, gridSize, blockSize, shared, args_traj, kernel_ms, "cuLaunchKernel(traj)")) return 1;

    numb timeStep_arg = (numb)(h * (double)preScaller);
    void* args_peak[] = {&d_data, &sizeOfBlock_s, &nPtsLimiter_int, &d_npeaks, &d_peaks, &d_times,
                         &timeStep_arg, &d_iters};
    if (!timed_launch(fp, gridSize, blockSize, 0, args_peak, kernel_ms, "cuLaunchKernel(peak)")) return 1;

    std::vector<numb> hp(rows), ht(rows);
    std::vector<int> hn(nPts);
    if (!ck(cuMemcpyDtoH(hp.data(), d_peaks, rows * sizeof(numb)), "copy outPeaks") ||
        !ck(cuMemcpyDtoH(ht.data(), d_times, rows * sizeof(numb)), "copy timeOfPeaks") ||
        !ck(cuMemcpyDtoH(hn.data(), d_npeaks, (size_t)nPts * sizeof(int)), "copy amountOfPeaks"))
        return 1;
    for (int k = 0; k < nPts; ++k) {
        counts[k] = hn[k];
        int n = hn[k] < amountOfPointsInBlock ? hn[k] : amountOfPointsInBlock;
        for (int i = 0; i < cap; ++i) {
            bool have = i < n;
            peaks[(size_t)k * cap + i] = have ? (double)hp[(size_t)k * amountOfPointsInBlock + i] : NAN;
            intervals[(size_t)k * cap + i] = have ? (double)ht[(size_t)k * amountOfPointsInBlock + i] : NAN;
        }
    }
    return 0;
}

}  // extern "C"
