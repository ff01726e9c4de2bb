// FMA-throughput probe used as the roofline denominator of the FP64 / FP32 integrator
// kernels (the measured-peaks file of the build pool only carries HBM and BF16 GEMM
// figures). Each thread runs 8 independent FMA chains so the pipe, not latency, bounds
// it; the result is 2 * FMAs / time.
#include <cuda_runtime.h>

#include <cstdio>

#include "../../include/ucb.h"

namespace {

template <class T>
__global__ void __launch_bounds__(256) fma_probe(T* out, int iters, T a, T b) {
    T x0 = (T)threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
      x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            x0 = fma(x0, a, b);
            x1 = fma(x1, a, b);
            x2 = fma(x2, a, b);
            x3 = fma(x3, a, b);
            x4 = fma(x4, a, b);
            x5 = fma(x5, a, b);
            x6 = fma(x6, a, b);
            x7 = fma(x7, a, b);
        }
    }
    const T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == (T)-1.2345) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

template <class T>
int run_probe(double* tflops, float* ms_out) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    T* out = nullptr;
    const int block = 256, blocks = sms * 8, iters = 4096;
    if (cudaMalloc(&out, sizeof(T) * block * blocks) != cudaSuccess) return UCB_E_CUDA;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_probe<T><<<blocks, block>>>(out, 64, (T)0.999999, (T)1e-7);  // warm-up
    cudaEventRecord(e0);
    fma_probe<T><<<blocks, block>>>(out, iters, (T)0.999999, (T)1e-7);
    cudaEventRecord(e1);
    cudaError_t ce = cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (ce != cudaSuccess) return UCB_E_CUDA;
    const double fmas = (double)blocks * block * iters * 16 * 8;
    *tflops = 2.0 * fmas / (ms * 1e-3) / 1e12;
    if (ms_out) *ms_out = ms;
    return UCB_OK;
}

}  // namespace

extern "C" UCB_API int ucb_measure_fma_peak(int precision, double* tflops) {
    if (!tflops) return UCB_E_INVALID;
    return precision == UCB_PREC_F64 ? run_probe<double>(tflops, nullptr) : run_probe<float>(tflops, nullptr);
}
