// LLE-map entry point that allocates no device memory.
//
// ucb_lle2d_device() keeps its scratch (work-queue counter, step counter, axis value
// tables) in an engine workspace obtained with cudaMalloc on first use. Some callers
// cannot allow that: applications that own all device memory through their own pool or a
// fixed, pre-reserved budget, and latency-critical loops that must not hit cudaMalloc /
// cudaFree (cudaFree synchronises the whole device). For them,
// ucb_lle2d_device_noalloc() runs the same kernel with its scratch in the file-scope
// device array below, which every GPU that loads this library holds until the process
// exits. The caller still provides the output buffers.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "engine_internal.h"

namespace {

// Layout used by the LLE kernel launch: [0, 8) work counter, [8, 16) step counter,
// [256, ...) axis-0 table, then the axis-1 table at the next 256-byte boundary.
constexpr size_t kNoAllocScratchBytes = 256 + 2 * (size_t)UCB_NOALLOC_MAX_PTS * sizeof(double);

__device__ __align__(256) unsigned char ucb_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Looks up (refresh = true, at prepare time) or returns the cached device address of the
// scratch array on `device`, which must be current. The array's host-side name is only a
// stand-in; the kernel needs this address.
int scratch_address(int device, bool refresh, void** out, std::string& err) {
    if (device < 0 || device >= kMaxDevices) {
        err = "device index out of range";
        return UCB_E_INVALID;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (refresh || !g_scratch_addr[device]) {
        void* ptr = nullptr;
        cudaError_t ce = cudaGetSymbolAddress(&ptr, ucb_noalloc_scratch);
        if (ce != cudaSuccess || !ptr) {
            err = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(ce);
            return UCB_E_CUDA;
        }
        g_scratch_addr[device] = ptr;
    }
    *out = g_scratch_addr[device];
    return UCB_OK;
}

// Axis tables travel to the scratch array as kernel parameters (at most ~31 KB per
// launch): no host memory has to outlive the call and no staging copy is made.
constexpr int kChunkWords = 7936;
struct TableChunk {
    unsigned int* dst;
    unsigned int count;
    unsigned int words[kChunkWords];
};

__global__ void ucb_noalloc_fill(const TableChunk c) {
    for (unsigned int i = threadIdx.x; i < c.count; i += blockDim.x) c.dst[i] = c.words[i];
}

int upload_by_parameters(void* dst, const void* src, size_t bytes, cudaStream_t stream, std::string& err) {
    const size_t words = bytes / 4;
    const unsigned int* s = static_cast<const unsigned int*>(src);
    unsigned int* d = static_cast<unsigned int*>(dst);
    TableChunk c;
    for (size_t off = 0; off < words; off += kChunkWords) {
        const size_t n = words - off < (size_t)kChunkWords ? words - off : (size_t)kChunkWords;
        c.dst = d + off;
        c.count = (unsigned int)n;
        std::memcpy(c.words, s + off, n * 4);
        ucb_noalloc_fill<<<1, 256, 0, stream>>>(c);
        cudaError_t ce = cudaGetLastError();
        if (ce != cudaSuccess) {
            err = std::string("axis-table upload: ") + cudaGetErrorString(ce);
            return UCB_E_CUDA;
        }
    }
    return UCB_OK;
}

int fail(ucb_engine* e, ucb_lle2d_result* res, int code, const std::string& msg) {
    e->last_error = msg;
    std::snprintf(res->error, sizeof res->error, "%s", msg.c_str());
    res->ok = 0;
    return code;
}

}  // namespace

extern "C" UCB_API int ucb_prepare_lle2d(ucb_engine* e, const ucb_lle2d_request* req) {
    if (!e || !req) return UCB_E_INVALID;
    std::string err;
    int rc = ucb::lle2d_pin(e, *req, err);
    if (rc != UCB_OK) {
        e->last_error = err;
        return rc;
    }
    void* ptr = nullptr;
    rc = scratch_address(e->device, true, &ptr, err);
    if (rc != UCB_OK) {
        e->last_error = err;
        return rc;
    }
    // Load the table-upload kernel now (with lazy module loading its first launch would
    // otherwise load it, and loading code allocates device memory).
    cudaFuncAttributes fa;
    cudaError_t ce = cudaFuncGetAttributes(&fa, ucb_noalloc_fill);
    if (ce != cudaSuccess) {
        e->last_error = std::string("loading the table-upload kernel: ") + cudaGetErrorString(ce);
        return UCB_E_CUDA;
    }
    return UCB_OK;
}

extern "C" UCB_API int ucb_lle2d_device_noalloc(ucb_engine* e, const ucb_lle2d_request* req, double* d_values,
                                                int32_t* d_flags, void* stream, ucb_lle2d_result* res) {
    if (!e || !req || !res) return UCB_E_INVALID;
    res->ok = 0;
    res->error[0] = 0;
    if (req->n_pts > UCB_NOALLOC_MAX_PTS)
        return fail(e, res, UCB_E_INVALID,
                    "n_pts " + std::to_string(req->n_pts) + " exceeds the scratch-array limit of " +
                        std::to_string(UCB_NOALLOC_MAX_PTS) + " points per axis");
    if (!d_values || !d_flags) return fail(e, res, UCB_E_INVALID, "output buffers are NULL");
    std::string err;
    void *plan = nullptr, *launch = nullptr;
    int rc = ucb::lle2d_find_pinned(e, *req, err, &plan, &launch);
    if (rc != UCB_OK) return fail(e, res, rc, err);
    void* scratch = nullptr;
    rc = scratch_address(e->device, false, &scratch, err);
    if (rc == UCB_OK)
        rc = ucb::lle2d_enqueue_with_scratch(e, *req, plan, launch, d_values, d_flags, (cudaStream_t)stream,
                                             static_cast<char*>(scratch), err, upload_by_parameters);
    ucb::lle2d_release(plan, launch);
    if (rc != UCB_OK) return fail(e, res, rc, err);
    res->n_pts = req->n_pts;
    res->ok = 1;
    return UCB_OK;
}
