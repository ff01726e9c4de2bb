// FMA-throughput probe used as the roofline denominator of the FP64 / FP32 integrator
// kernels (the measured-peaks file of the build pool only carries HBM and BF16 GEMM
// figures). Each thread runs 8 independent FMA chains so the pipe, not latency, bounds
// it; the result is 2 * FMAs / time. UCB_PEAK_F32X2 measures packed FP32 pairs.
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

// The same with packed FP32 pairs (__ffma2_rn: two FMAs per instruction on sm_100).
__global__ void __launch_bounds__(256) fma2_probe(float2* out, int iters, float2 a, float2 b) {
    const float t = (float)threadIdx.x;
    float2 x0 = make_float2(t, t + 0.5f), x1 = make_float2(t + 1, t + 1.5f), x2 = make_float2(t + 2, t + 2.5f),
           x3 = make_float2(t + 3, t + 3.5f), x4 = make_float2(t + 4, t + 4.5f), x5 = make_float2(t + 5, t + 5.5f),
           x6 = make_float2(t + 6, t + 6.5f), x7 = make_float2(t + 7, t + 7.5f);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            x0 = __ffma2_rn(x0, a, b);
            x1 = __ffma2_rn(x1, a, b);
            x2 = __ffma2_rn(x2, a, b);
            x3 = __ffma2_rn(x3, a, b);
            x4 = __ffma2_rn(x4, a, b);
            x5 = __ffma2_rn(x5, a, b);
            x6 = __ffma2_rn(x6, a, b);
            x7 = __ffma2_rn(x7, a, b);
        }
    }
    const float s = ((x0.x + x1.x) + (x2.x + x3.x)) + ((x4.y + x5.y) + (x6.y + x7.y));
    if (s == -1.2345f) out[blockIdx.x * blockDim.x + threadIdx.x] = x0;  // keeps the chains live
}

template <class T>
struct Probe {
    static void launch(int blocks, int block, T* out, int iters) {
        fma_probe<T><<<blocks, block>>>(out, iters, (T)0.999999, (T)1e-7);
    }
    static constexpr int lanes = 1;
};

template <>
struct Probe<float2> {
    static void launch(int blocks, int block, float2* out, int iters) {
        fma2_probe<<<blocks, block>>>(out, iters, make_float2(0.999999f, 0.999998f), make_float2(1e-7f, 2e-7f));
    }
    static constexpr int lanes = 2;
};

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
    Probe<T>::launch(blocks, block, out, 64);  // warm-up
    cudaEventRecord(e0);
    Probe<T>::launch(blocks, block, out, iters);
    cudaEventRecord(e1);
    cudaError_t ce = cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (ce != cudaSuccess) return UCB_E_CUDA;
    const double fmas = (double)blocks * block * iters * 16 * 8 * Probe<T>::lanes;
    *tflops = 2.0 * fmas / (ms * 1e-3) / 1e12;
    if (ms_out) *ms_out = ms;
    return UCB_OK;
}

}  // namespace

extern "C" UCB_API int ucb_measure_fma_peak(int precision, double* tflops) {
    if (!tflops) return UCB_E_INVALID;
    if (precision == UCB_PEAK_F32X2) return run_probe<float2>(tflops, nullptr);
    return precision == UCB_PREC_F64 ? run_probe<double>(tflops, nullptr) : run_probe<float>(tflops, nullptr);
}
