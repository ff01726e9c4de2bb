// BF16 MLP surrogate: tcgen05 tensor-core GEMMs, the fused prediction kernel, elementwise
// kernels and the training / prediction host code (no reference counterpart).
//
// GEMM (training): C[M, N] = A[M, K] B[N, K]^T with A and B K-contiguous ("TN"),
// M % 128 == 0, N % 128 == 0, K % 64 == 0. A persistent kernel (one CTA of 576 threads per
// SM) walks tiles of 128 x 256 or 128 x 128 (the narrower tile when N is not a multiple of
// 256 or when the wide tiles would leave SMs idle) and K splits: warp 0 streams 64-wide K
// chunks of A and B with TMA (128-byte swizzle, no multicast) into a ring of shared-memory
// stages, warp 1 issues tcgen05.mma (CuTe SM100_MMA_F16BF16_SS, cta_group::1, BF16 x BF16
// -> FP32) from one elected lane into one of two TMEM accumulators, and warps 2-17 read a
// finished accumulator with tcgen05.ld (four warps per 32-lane TMEM quadrant, a quarter of
// the columns each; thread t of a quadrant owns row t) while the next tile's MMAs run,
// apply bias / GELU and store FP32, BF16 and / or transposed BF16 copies through a per-warp
// shared-memory staging buffer (whole 16-byte pieces per store instruction). Waits are
// bounded; on a timeout the kernel records an error, waits for its own copies and MMAs,
// frees TMEM and returns. A split-K launch stores each split's partial tile in its own
// slice of a buffer, and the optimiser kernel adds the slices in split order (so a
// training step gives the same bits every time it runs). Backward products are the same TN
// GEMM on transposed copies, which the forward and dL/dZ epilogues write as they go.
//
// Prediction: one fused kernel per call (mlp_infer_kernel) runs features, every hidden
// layer and the output transform of a 128-row tile inside one CTA, with the activations in
// shared memory; HBM sees the inputs and the two outputs per row only.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cute/tensor.hpp>
#include <cute/arch/tmem_allocator_sm100.hpp>
#include <cute/atom/mma_traits_sm100.hpp>
#include <cute/atom/copy_traits_sm100.hpp>
#include <cute/algorithm/cooperative_copy.hpp>
#include <cutlass/arch/barrier.h>
#include <cutlass/numeric_types.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "engine_internal.h"
#include "mlp.h"

namespace ucbmlp {

using namespace cute;
using bf16 = cutlass::bfloat16_t;

constexpr int kBM = 128;   // rows of a tile (UMMA M, one TMEM lane per row)
constexpr int kBK = 64;    // K per pipeline stage: one 128-byte swizzle row of BF16
constexpr long long kWaitLimit = 1LL << 22;  // try_wait polls before a wait gives up
constexpr int kEpiWarps = 16;     // four per 32-lane TMEM quadrant, a quarter of the columns each
constexpr int kGemmThreads = 64 + 32 * kEpiWarps;  // warp 0 TMA, warp 1 MMA, warps 2-17 epilogue
constexpr int kMaxLayers = 9;     // hidden layers + the output layer

// Shapes and shared-memory layout of the persistent GEMM for a tile width BN (128 or 256).
template <int BN>
struct GemmCfg {
    using MmaOp = SM100_MMA_F16BF16_SS<bf16, bf16, float, kBM, BN, UMMA::Major::K, UMMA::Major::K>;
    using TiledMma = decltype(make_tiled_mma(MmaOp{}));
    using LayoutA = decltype(UMMA::tile_to_mma_shape(
        UMMA::Layout_K_SW128_Atom<bf16>{}, partition_shape_A(TiledMma{}, make_shape(Int<kBM>{}, Int<kBK>{}))));
    using LayoutB = decltype(UMMA::tile_to_mma_shape(
        UMMA::Layout_K_SW128_Atom<bf16>{}, partition_shape_B(TiledMma{}, make_shape(Int<BN>{}, Int<kBK>{}))));
    static constexpr int kStages = BN == 256 ? 3 : 4;
    static constexpr int kABytes = kBM * kBK * 2;
    static constexpr int kBBytes = BN * kBK * 2;
    static constexpr int kStageBytes = kABytes + kBBytes;  // multiple of 1024: every stage stays 1024-aligned
    // barriers: full / empty per stage, accumulator full / empty per TMEM buffer, drain
    static constexpr int kBarriers = 2 * kStages + 2 + 2 + 1;
    static constexpr int kEpiStage = 4096;  // per epilogue warp: staging of one 32 x 32 chunk
    static constexpr int kSmem = 1024 + kStages * kStageBytes + kEpiWarps * kEpiStage + 8 * kBarriers + 16;
    static_assert(kSmem <= 232448, "GEMM shared memory above the per-CTA limit");
    static_assert(kStageBytes % 1024 == 0, "swizzled stages need 1024-byte alignment");
    static_assert(2 * BN <= 512, "two accumulators must fit in TMEM");
};

struct Epilogue {
    const float* bias;  // bias[n] for n < nb (0 beyond)
    int nb;
    int gelu;           // outh / outt receive GELU(v) instead of v
    float* outf;        // FP32 result (pre-activation), row stride ldf
    int ldf;
    int atomic;         // split-K: outf is a buffer of partial tiles, one slice per K split
    long long split_stride;  // floats between the slices of consecutive splits
    bf16* outh;         // BF16 copy, row stride ldh
    int ldh;
    bf16* outt;         // BF16 transposed copy outt[n * ldt + m]
    int ldt;
    int m_store, n_store;  // only rows m < m_store and columns n < n_store are stored
    // backward through GELU: the product is dL/dH of a hidden layer; outh / outt receive
    // dZ = dL/dH GELU'(Z) with Z = zin (FP32, row stride ldz)
    const float* zin;
    int ldz;
    // sums over each 32-row block of the BF16 values stored to outh / outt (the bias gradient
    // of dZ): colsum[(m / 32) ldc + n]
    float* colsum;
    int ldc;
    // output layer of a training batch (columns 0 = mean, 1 = log-variance): the beta-NLL
    // against the standardised targets yb of the first n_valid of `rows` rows -> dout (row
    // stride 64, columns 0 and 1), doutT (rows 0 and 1 of a [128, rows] matrix), and per
    // 32-row block the sums of the two BF16 gradients and of the loss in blk[3 (m / 32) + 0..2]
    int nll;
    const float* yb;
    int n_valid, rows;
    float beta;
    bf16* dout;
    bf16* doutT;
    float* blk;
};

// Work of one launch: items are (M tile, N tile, K split) triples, handed out round robin
// over the persistent grid (every role of a CTA walks the same sequence).
struct GemmWork {
    int tiles_n, splits, kt_total, kt_per_split;
    int items;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return cute::cast_smem_ptr_to_uint(p); }

// mbarrier phase wait with a poll limit (each try_wait itself suspends for a bounded time).
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// 2-D tiled TMA load of one box into this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
        : "memory");
}
// Programmatic dependent launch: a kernel launched with programmatic stream serialisation may
// start while its predecessor in the stream still runs. launch_dependents lets the next
// kernel's CTAs start their prologue once every CTA of this grid has issued it; wait blocks
// until the predecessor grid has completed and its memory is visible. Without the launch
// attribute both are no-ops.
__device__ __forceinline__ void griddep_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// GELU in its tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))) (Hendrycks and
// Gimpel, 2016), with the hardware tanh (tanh.approx.f32, relative error about 2^-11, far
// below the BF16 rounding that follows).
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float kGeluC0 = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float kGeluC1 = 0.044715f;
// Two GELUs in packed FP32 pairs (fma / mul .f32x2: half the FP32 issue slots), the form
// both training and prediction use: h + h tanh(c0 (z + c1 z^3)) with h = z / 2.
constexpr float kGeluC01 = kGeluC0 * kGeluC1;
// tanh's argument c0 (z + c1 z^3) as z (c0 + c0 c1 z^2): two packed operations.
__device__ __forceinline__ float2 gelu_arg2(float2 z) {
    return __fmul2_rn(__ffma2_rn(__fmul2_rn(z, z), make_float2(kGeluC01, kGeluC01), make_float2(kGeluC0, kGeluC0)),
                      z);
}
__device__ __forceinline__ float2 gelu2(float2 z) {
    const float2 w = gelu_arg2(z);
    const float2 t = make_float2(tanh_hw(w.x), tanh_hw(w.y));
    const float2 h = __fmul2_rn(z, make_float2(0.5f, 0.5f));
    return __ffma2_rn(h, t, h);
}
// 2 gelu(z) = z + z tanh(w), one packed operation fewer than gelu2. Scaling by two commutes
// with every rounding on the way (the BF16 packing and the FP32 accumulation of the next
// layer's MMA), so a consumer that multiplies by 0.5 sees the bits gelu2 would have given.
__device__ __forceinline__ float2 gelu2_twice(float2 z) {
    const float2 w = gelu_arg2(z);
    const float2 t = make_float2(tanh_hw(w.x), tanh_hw(w.y));
    return __ffma2_rn(z, t, z);
}
__device__ __forceinline__ float gelu_grad(float z) {
    const float z2 = z * z;
    const float t = tanh_hw(z * fmaf(kGeluC01, z2, kGeluC0));
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGeluC0 * fmaf(3.0f * kGeluC1, z2, 1.0f);
}

// Sums over the 32 lanes of a warp of each of the 32 values v[0..31] (lane = one row):
// five exchange rounds in a fixed order (each round hands half of a lane's partial sums to
// the partner lane), after which lane l holds the sum of column l in v[returned index].
__device__ __forceinline__ int column_sums32(float (&v)[32]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int w = 16; w >= 1; w >>= 1) {
        const bool upper = (lane & w) != 0;
#pragma unroll
        for (int j = 0; j < w; ++j) {
            const float send = upper ? v[j] : v[j + w];
            const float keep = upper ? v[j + w] : v[j];
            v[j] = keep + __shfl_xor_sync(0xffffffffu, send, w);
        }
    }
    return 0;
}

// Beta-NLL of one output row (mean mu, log-variance lv_raw) of a training batch, the
// gradients dout / doutT, and the fixed-order sums over the warp's 32 rows into blk.
__device__ __forceinline__ void nll_rows(const Epilogue& ep, int r, float mu, float lv_raw) {
    float g0 = 0.f, g1 = 0.f, l = 0.f;
    if (r < ep.rows && r < ep.n_valid) {
        const float lv = fminf(fmaxf(lv_raw, -16.f), 16.f);
        const float iv = expf(-lv);
        const float d = mu - ep.yb[r];
        const float w = ep.beta > 0.f ? expf(ep.beta * lv) : 1.f;  // constant weight sigma^(2 beta)
        const float inv_n = 1.f / (float)ep.n_valid;
        l = w * 0.5f * (lv + d * d * iv) * inv_n;
        g0 = w * d * iv * inv_n;
        g1 = (lv_raw == lv) ? w * 0.5f * (1.f - d * d * iv) * inv_n : 0.f;
    }
    const bf16 b0 = bf16(g0), b1 = bf16(g1);
    if (r < ep.rows) {
        ep.dout[(size_t)r * 64] = b0;
        ep.dout[(size_t)r * 64 + 1] = b1;
        ep.doutT[r] = b0;
        ep.doutT[(size_t)ep.rows + r] = b1;
    }
    float s0 = float(b0), s1 = float(b1), sl = l;
#pragma unroll
    for (int w = 16; w >= 1; w >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, w);
        s1 += __shfl_xor_sync(0xffffffffu, s1, w);
        sl += __shfl_xor_sync(0xffffffffu, sl, w);
    }
    if ((threadIdx.x & 31) == 0) {
        ep.blk[3 * (r >> 5)] = s0;
        ep.blk[3 * (r >> 5) + 1] = s1;
        ep.blk[3 * (r >> 5) + 2] = sl;
    }
}

// One 32-column chunk of one accumulator row (this thread's) through the epilogue: bias,
// the FP32 / BF16 / transposed BF16 stores. v: the raw accumulator values.
// Epilogue features compiled into a GEMM instantiation (a launch only runs the code of its
// own mode: with one tile per CTA, as in a training step, every CTA executes the epilogue
// once, so code it does not need costs instruction fetches from L2).
enum : int {
    kEpBias = 1, kEpGelu = 2, kEpOutF = 4, kEpOutH = 8, kEpOutT = 16, kEpZin = 32, kEpColsum = 64, kEpNll = 128,
    kEpAll = 255,
    kModeForward = kEpBias | kEpGelu | kEpOutF | kEpOutH | kEpOutT,  // hidden layer of a training batch
    kModeLoss = kEpBias | kEpOutF | kEpNll,                           // output layer of a training batch
    kModeDz = kEpZin | kEpOutH | kEpOutT | kEpColsum,                 // dL/dZ of a hidden layer
    kModeSplit = kEpOutF,                                             // split-K slices
    kModeHidden = kEpBias | kEpGelu | kEpOutH,                        // prediction, hidden layer
    kModeOut = kEpBias | kEpOutF,                                     // prediction, output layer
};

// Stores of a warp's 32 x 32 chunk (one row per lane) through the warp's 4 KB staging buffer
// in shared memory, so that each global store instruction writes whole 16-byte pieces of a
// few rows (or columns) instead of one scattered piece per lane.
//
// Row-major: 32 rows of W 32-bit words (lane r's row is vals) to g + r * stride (bytes; g is
// row 0 of the warp). 16-byte unit q of row r sits at unit q ^ swz(r) of the row in the
// buffer, which keeps both the writes (one row per lane) and the reads (whole rows) free of
// bank conflicts.
template <int W>
__device__ __forceinline__ void rows_staged(uint32_t* stage, const uint32_t (&vals)[W], char* g, size_t stride) {
    constexpr int U = W / 4;  // 16-byte units per row: 8 (FP32) or 4 (BF16)
    const int lane = threadIdx.x & 31;
    auto swz = [](int r) { return U == 8 ? (r & 7) : ((r >> 1) & 3); };
    uint4* s4 = reinterpret_cast<uint4*>(stage);
#pragma unroll
    for (int q = 0; q < U; ++q)
        s4[lane * U + (q ^ swz(lane))] = make_uint4(vals[4 * q], vals[4 * q + 1], vals[4 * q + 2], vals[4 * q + 3]);
    __syncwarp();
#pragma unroll
    for (int pass = 0; pass < U; ++pass) {
        const int r = pass * (32 / U) + lane / U, q = lane % U;
        *reinterpret_cast<uint4*>(g + (size_t)r * stride + q * 16) = s4[r * U + (q ^ swz(r))];
    }
    __syncwarp();
}
// Transposed BF16: column j of the chunk (its 32 rows) to outt + j * ld (elements; outt points
// at column 0, row 0 of the warp). The buffer holds the chunk column-major, so each column's
// 64 bytes are contiguous; a store instruction writes 16-byte pieces of eight columns.
__device__ __forceinline__ void cols_staged(uint32_t* stage, const float (&g)[32], bf16* outt, size_t ld) {
    const int lane = threadIdx.x & 31;
    unsigned short* s2 = reinterpret_cast<unsigned short*>(stage);
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        const bf16 b = bf16(g[j]);
        s2[j * 32 + lane] = *reinterpret_cast<const unsigned short*>(&b);
    }
    __syncwarp();
    const uint4* s4 = reinterpret_cast<const uint4*>(stage);
#pragma unroll
    for (int pass = 0; pass < 4; ++pass) {
        const int j = pass * 8 + lane / 4, q = lane % 4;
        *reinterpret_cast<uint4*>(outt + (size_t)j * ld + q * 8) = s4[j * 4 + q];
    }
    __syncwarp();
}

template <int MODE>
__device__ __forceinline__ void epilogue_chunk(const Epilogue& ep, float* outf, int m, int n0, float (&v)[32],
                                               uint32_t* stage) {
    if ((MODE & kEpBias) && ep.bias) {
        if (n0 + 32 <= ep.nb && (reinterpret_cast<uintptr_t>(ep.bias + n0) & 15) == 0) {
            // every lane reads the same 32 values: eight broadcast 16-byte loads
            const float4* b4 = reinterpret_cast<const float4*>(ep.bias + n0);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float4 b = __ldg(b4 + q);
                v[4 * q] += b.x;
                v[4 * q + 1] += b.y;
                v[4 * q + 2] += b.z;
                v[4 * q + 3] += b.w;
            }
        } else {
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (n0 + j < ep.nb) v[j] += __ldg(ep.bias + n0 + j);
        }
    }
    const bool row_ok = m < ep.m_store;
    const bool full = n0 + 32 <= ep.n_store;
    // the whole warp's 32 rows are stored: the staged (coalesced) paths apply
    const bool warp_rows = __all_sync(0xffffffffu, row_ok);
    const int m0 = m - (int)(threadIdx.x & 31);
    if ((MODE & kEpOutF) && outf && warp_rows && full && (ep.ldf & 3) == 0 &&
        (reinterpret_cast<uintptr_t>(outf) & 15) == 0) {
        uint32_t w[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) w[j] = __float_as_uint(v[j]);
        rows_staged<32>(stage, w, reinterpret_cast<char*>(outf + (size_t)m0 * ep.ldf + n0), (size_t)ep.ldf * 4);
    } else if ((MODE & kEpOutF) && outf && row_ok) {
        float* p = outf + (size_t)m * ep.ldf + n0;
        if (full && (ep.ldf & 3) == 0 && (reinterpret_cast<uintptr_t>(outf) & 15) == 0) {
#pragma unroll
            for (int j = 0; j < 32; j += 4)
                *reinterpret_cast<float4*>(p + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        } else {
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (n0 + j < ep.n_store) p[j] = v[j];
        }
    }
    if ((MODE & kEpNll) && ep.nll && n0 == 0) nll_rows(ep, m, v[0], v[1]);
    if (!(MODE & (kEpOutH | kEpOutT)) || (!ep.outh && !ep.outt)) return;
    float g[32];
    if ((MODE & kEpZin) && ep.zin) {
        if (row_ok && full && (ep.ldz & 3) == 0) {
            const float4* z4 = reinterpret_cast<const float4*>(ep.zin + (size_t)m * ep.ldz + n0);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float4 z = __ldg(z4 + q);
                g[4 * q] = v[4 * q] * gelu_grad(z.x);
                g[4 * q + 1] = v[4 * q + 1] * gelu_grad(z.y);
                g[4 * q + 2] = v[4 * q + 2] * gelu_grad(z.z);
                g[4 * q + 3] = v[4 * q + 3] * gelu_grad(z.w);
            }
        } else {
#pragma unroll
            for (int j = 0; j < 32; ++j)
                g[j] = (row_ok && n0 + j < ep.n_store) ? v[j] * gelu_grad(ep.zin[(size_t)m * ep.ldz + n0 + j]) : 0.f;
        }
    } else if ((MODE & kEpGelu) && ep.gelu) {
#pragma unroll
        for (int j = 0; j < 32; j += 2) {
            const float2 q = gelu2(make_float2(v[j], v[j + 1]));
            g[j] = q.x;
            g[j + 1] = q.y;
        }
    } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) g[j] = v[j];
    }
    if ((MODE & kEpOutH) && ep.outh && warp_rows && full && (ep.ldh & 7) == 0 &&
        (reinterpret_cast<uintptr_t>(ep.outh) & 15) == 0) {
        uint32_t w[16];
#pragma unroll
        for (int j = 0; j < 32; j += 2) {
            __nv_bfloat162 h = __floats2bfloat162_rn(g[j], g[j + 1]);
            w[j / 2] = *reinterpret_cast<uint32_t*>(&h);
        }
        rows_staged<16>(stage, w, reinterpret_cast<char*>(ep.outh + (size_t)m0 * ep.ldh + n0), (size_t)ep.ldh * 2);
    } else if ((MODE & kEpOutH) && ep.outh && row_ok) {
        bf16* p = ep.outh + (size_t)m * ep.ldh + n0;
        if (full && (ep.ldh & 7) == 0 && (reinterpret_cast<uintptr_t>(ep.outh) & 15) == 0) {
#pragma unroll
            for (int j = 0; j < 32; j += 8) {
                uint4 q;
                __nv_bfloat162 h0 = __floats2bfloat162_rn(g[j], g[j + 1]), h1 = __floats2bfloat162_rn(g[j + 2], g[j + 3]);
                __nv_bfloat162 h2 = __floats2bfloat162_rn(g[j + 4], g[j + 5]), h3 = __floats2bfloat162_rn(g[j + 6], g[j + 7]);
                q.x = *reinterpret_cast<uint32_t*>(&h0);
                q.y = *reinterpret_cast<uint32_t*>(&h1);
                q.z = *reinterpret_cast<uint32_t*>(&h2);
                q.w = *reinterpret_cast<uint32_t*>(&h3);
                *reinterpret_cast<uint4*>(p + j) = q;
            }
        } else {
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (n0 + j < ep.n_store) p[j] = bf16(g[j]);
        }
    }
    if ((MODE & kEpOutT) && ep.outt && warp_rows && full && (ep.ldt & 7) == 0 &&
        (reinterpret_cast<uintptr_t>(ep.outt) & 15) == 0) {
        cols_staged(stage, g, ep.outt + (size_t)n0 * ep.ldt + m0, (size_t)ep.ldt);
    } else if ((MODE & kEpOutT) && ep.outt && row_ok) {
        // consecutive threads own consecutive rows: each column's stores are contiguous
#pragma unroll
        for (int j = 0; j < 32; ++j)
            if (n0 + j < ep.n_store) ep.outt[(size_t)(n0 + j) * ep.ldt + m] = bf16(g[j]);
    }
    if ((MODE & kEpColsum) && ep.colsum) {
        // column sums over the warp's 32 rows of the BF16-rounded values (rows past m_store
        // add 0): a fixed butterfly that leaves column n0 + lane in lane `lane`
#pragma unroll
        for (int j = 0; j < 32; ++j) g[j] = row_ok ? float(bf16(g[j])) : 0.f;
        const int s = column_sums32(g);
        if (n0 + (threadIdx.x & 31) < ep.n_store)
            ep.colsum[(size_t)(m >> 5) * ep.ldc + n0 + (threadIdx.x & 31)] = g[s];
    }
}

// C = A B^T, A [M, K] and B [N, K] K-contiguous BF16, FP32 accumulation in TMEM.
// Persistent and warp-specialised: warp 0 streams K chunks of A and B into a ring of
// shared-memory stages with TMA (128-byte swizzle, the layout the MMA descriptors read),
// warp 1 issues tcgen05.mma from one elected lane into one of two TMEM accumulators and
// commits to the stage's and the accumulator's mbarriers, warps 2-17 (four per 32-lane TMEM
// quadrant) read finished accumulators with tcgen05.ld, run the epilogue and hand the
// accumulator back, so the epilogue of one tile overlaps the MMAs of the next. Every wait
// is bounded; on a timeout the CTA records an error, stops, waits (bounded) for its own
// copies and MMAs in flight, frees TMEM and returns.
template <int BN, int MODE>
__global__ void __launch_bounds__(kGemmThreads, 1)
    gemm_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmWork w,
                    Epilogue ep, int* err) {
    using Cfg = GemmCfg<BN>;
    constexpr int S = Cfg::kStages;
    typename Cfg::TiledMma tiled_mma;
    extern __shared__ char smem_raw[];
    char* base = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    char* epi_stage = base + S * Cfg::kStageBytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(epi_stage + kEpiWarps * Cfg::kEpiStage);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + Cfg::kBarriers);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    auto full_bar = [&](int s) { return smem_u32(bars + s); };
    auto empty_bar = [&](int s) { return smem_u32(bars + S + s); };
    auto accf_bar = [&](int b) { return smem_u32(bars + 2 * S + b); };
    auto acce_bar = [&](int b) { return smem_u32(bars + 2 * S + 2 + b); };
    const uint32_t drain_bar = smem_u32(bars + 2 * S + 4);

    const int warp = threadIdx.x / 32, lane = threadIdx.x & 31;
    cute::TMEM::Allocator1Sm tmem;
    if (warp == 0) tmem.allocate(2 * BN, tmem_slot);
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(accf_bar(b), 1);
            mbar_init(acce_bar(b), kEpiWarps);
        }
        mbar_init(drain_bar, 1);
        *abort_flag = 0;
        cutlass::arch::fence_barrier_init();
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    auto fail = [&]() {
        *abort_flag = 1;
        atomicExch(err, 1);
    };
    // prologue done: the next kernel may start its own; nothing of the predecessor's output is
    // read (operands, bias, Z) or overwritten before it has completed
    griddep_launch_dependents();
    griddep_wait();

    if (warp == 0) {
        // ---- TMA producer (lane 0)
        if (lane == 0) {
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmA)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmB)) : "memory");
            int stage = 0;
            uint32_t phase = 0;
            int issued[S];
#pragma unroll
            for (int s = 0; s < S; ++s) issued[s] = 0;
            for (int item = blockIdx.x; item < w.items && !*abort_flag; item += gridDim.x) {
                const int sp = item % w.splits, tile = item / w.splits;
                const int tn = tile % w.tiles_n, tm = tile / w.tiles_n;
                const int kt0 = sp * w.kt_per_split;
                const int nk = min(w.kt_total, kt0 + w.kt_per_split) - kt0;
                for (int i = 0; i < nk; ++i) {
                    if (*abort_flag || !mbar_wait_bounded(empty_bar(stage), phase ^ 1)) {
                        fail();
                        break;
                    }
                    const uint32_t a_dst = smem_u32(base + stage * Cfg::kStageBytes);
                    mbar_expect_tx(full_bar(stage), Cfg::kStageBytes);
                    tma_load_2d(a_dst, &tmA, full_bar(stage), (kt0 + i) * kBK, tm * kBM);
                    tma_load_2d(a_dst + Cfg::kABytes, &tmB, full_bar(stage), (kt0 + i) * kBK, tn * BN);
                    ++issued[stage];
                    if (++stage == S) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
            // copies in flight when stopping early: wait (bounded) until each stage's last
            // load has landed
            if (*abort_flag)
                for (int s = 0; s < S; ++s)
                    if (issued[s] > 0) mbar_wait_bounded(full_bar(s), (uint32_t)((issued[s] - 1) & 1));
        }
    } else if (warp == 1) {
        // ---- MMA issuer (the whole warp follows; one elected lane issues)
        int stage = 0, buf = 0;
        uint32_t phase = 0, acc_phase = 0;
        for (int item = blockIdx.x; item < w.items && !*abort_flag; item += gridDim.x) {
            const int sp = item % w.splits;
            const int kt0 = sp * w.kt_per_split;
            const int nk = min(w.kt_total, kt0 + w.kt_per_split) - kt0;
            if (!mbar_wait_bounded(acce_bar(buf), acc_phase ^ 1)) {
                fail();
                break;
            }
            tc_fence_after();
            ThrMMA cta_mma = tiled_mma.get_slice(0);
            Tensor tAcc = cta_mma.make_fragment_C(cta_mma.partition_C(
                make_identity_tensor(make_shape(Int<kBM>{}, Int<BN>{}))));
            tAcc.data() = tmem_base + (uint32_t)(buf * BN);
            tiled_mma.accumulate_ = UMMA::ScaleOut::Zero;
            bool ok = true;
            for (int i = 0; i < nk; ++i) {
                if (*abort_flag || !mbar_wait_bounded(full_bar(stage), phase)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                bf16* a_ptr = reinterpret_cast<bf16*>(base + stage * Cfg::kStageBytes);
                Tensor sA = make_tensor(make_smem_ptr(a_ptr), typename Cfg::LayoutA{});
                Tensor sB = make_tensor(make_smem_ptr(a_ptr + Cfg::kABytes / 2), typename Cfg::LayoutB{});
                Tensor fA = cta_mma.make_fragment_A(sA);
                Tensor fB = cta_mma.make_fragment_B(sB);
                CUTE_UNROLL
                for (int kb = 0; kb < size<2>(fA); ++kb) {
                    gemm(tiled_mma, fA(_, _, kb), fB(_, _, kb), tAcc);
                    tiled_mma.accumulate_ = UMMA::ScaleOut::One;
                }
                cutlass::arch::umma_arrive(bars + S + stage);  // the stage is free once these MMAs ran
                if (++stage == S) {
                    stage = 0;
                    phase ^= 1;
                }
            }
            if (!ok) {
                fail();
                break;
            }
            cutlass::arch::umma_arrive(bars + 2 * S + buf);  // accumulator complete
            if (++buf == 2) {
                buf = 0;
                acc_phase ^= 1;
            }
        }
        // every MMA this warp issued has completed before TMEM can be released
        cutlass::arch::umma_arrive(bars + 2 * S + 4);
        if (!mbar_wait_bounded(drain_bar, 0)) fail();
    } else {
        // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (the lanes its quadrant may
        // access) and, with (w - 2) / 4, one half of the columns
        const int quad = warp & 3, part = (warp - 2) >> 2;
        const int row = quad * 32 + lane;
        int buf = 0;
        uint32_t acc_phase = 0;
        for (int item = blockIdx.x; item < w.items && !*abort_flag; item += gridDim.x) {
            const int sp = item % w.splits, tile = item / w.splits;
            const int tn = tile % w.tiles_n, tm = tile / w.tiles_n;
            if ((MODE & kEpZin) && ep.zin && tm * kBM + row < ep.m_store) {
                // this thread's Z row segment is independent of the MMAs: start its loads now
                const char* zr = reinterpret_cast<const char*>(ep.zin + (size_t)(tm * kBM + row) * ep.ldz +
                                                               tn * BN + part * (BN / 4));
#pragma unroll
                for (int b = 0; b < (BN / 4) * 4; b += 128)
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(zr + b));
            }
            if (!mbar_wait_bounded(accf_bar(buf), acc_phase)) {
                fail();
                break;
            }
            tc_fence_after();
            float* outf = ep.outf ? ep.outf + (size_t)sp * ep.split_stride : nullptr;
            const int m = tm * kBM + row;
            const uint32_t taddr = tmem_base + (uint32_t)(buf * BN) + ((uint32_t)(quad * 32) << 16);
#pragma unroll 1
            for (int c0 = part * (BN / 4); c0 < (part + 1) * (BN / 4); c0 += 32) {
                uint32_t r[32];
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
                             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                             : "r"(taddr + (uint32_t)c0));
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                float v[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
                epilogue_chunk<MODE>(ep, outf, m, tn * BN + c0, v,
                                     reinterpret_cast<uint32_t*>(epi_stage + (warp - 2) * Cfg::kEpiStage));
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(acce_bar(buf));
            if (++buf == 2) {
                buf = 0;
                acc_phase ^= 1;
            }
        }
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem.release_allocation_lock();
        tmem.free(tmem_base, 2 * BN);
    }
}

// ------------------------------------------------------------------ elementwise kernels
struct FeatureArgs {
    const float* u;            // n x 2, or nullptr: points from cells / grid
    const long long* cells;    // optional kernel-order cells
    long long n;
    int grid_n;
    long long row0;            // first input row of this chunk
    // mini-batch mode: rows drawn at random from the n inputs with a per-step hash
    const unsigned long long* step;  // device step counter (nullptr: sequential rows)
    unsigned long long seed;
    const float* y;            // targets of the n inputs (training)
    float y_mean, y_inv_std;
    float* yb;                 // standardised targets of the batch rows
    const float* Bf;           // fourier x 2
    int fourier;
    int rows;                  // rows of this chunk (multiple of 128)
    bf16* X;                   // rows x 2 fourier
    bf16* Xt;                  // 2 fourier x rows (optional)
};

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__device__ __forceinline__ void input_point(const float* u, const long long* cells, int grid_n, long long i,
                                            float& u0, float& u1) {
    if (u) {
        u0 = u[2 * i];
        u1 = u[2 * i + 1];
    } else {
        const long long c = cells ? cells[i] : i;
        const float inv = grid_n > 1 ? 1.0f / (float)(grid_n - 1) : 0.0f;
        u0 = (float)(c % grid_n) * inv;
        u1 = (float)(c / grid_n) * inv;
    }
}
__device__ __forceinline__ void input_point(const FeatureArgs& a, long long i, float& u0, float& u1) {
    input_point(a.u, a.cells, a.grid_n, i, u0, u1);
}

// sin and cos of the phase 2 pi (u0 B[2j] + u1 B[2j+1]) of frequency j. The phase in turns
// is reduced to [-1/2, 1/2] exactly (x - rint(x)); the hardware sine and cosine on [-pi, pi]
// then err by less than 2^-21, far below the BF16 resolution the features are stored in.
// Every step rounds in one fixed order (no contraction left to the compiler), so the
// training batches and the fused prediction see the same features.
__device__ __forceinline__ void feature_sincos(float u0, float u1, const float* Bf, int j, float& s, float& c) {
    const float x = __fmaf_rn(u0, __ldg(Bf + 2 * j), __fmul_rn(u1, __ldg(Bf + 2 * j + 1)));
    __sincosf(__fmul_rn(6.283185307179586f, __fsub_rn(x, rintf(x))), &s, &c);
}

// X[r, j] = sin(2 pi u.B_j), X[r, fourier + j] = cos(...). One thread per (row, group of
// 8 frequencies); consecutive threads take consecutive rows of one group, so the transposed
// copy's stores are contiguous across a warp and each row's 8 values go out as 16 bytes.
__global__ void features_kernel(FeatureArgs a) {
    griddep_launch_dependents();
    griddep_wait();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int groups = a.fourier / 8;
    if (t >= (long long)a.rows * groups) return;
    const int r = (int)(t % a.rows);
    const int j0 = 8 * (int)(t / a.rows);
    long long i;
    bool valid;
    if (a.step) {
        const unsigned long long h = mix64(a.seed ^ mix64(*a.step * 0x100000001B3ULL + (unsigned long long)r));
        i = (long long)(h % (unsigned long long)a.n);
        valid = a.n > 0;
    } else {
        i = a.row0 + r;
        valid = i < a.n;
    }
    float u0 = 0.f, u1 = 0.f;
    if (valid) input_point(a, i, u0, u1);
    float sv[8], cv[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        sv[q] = cv[q] = 0.f;
        if (valid) feature_sincos(u0, u1, a.Bf, j0 + q, sv[q], cv[q]);
    }
    const int F = 2 * a.fourier;
    uint4 ps, pc;
    __nv_bfloat162 h;
#define UCB_PACK(dst, v, k)                               \
    h = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]); \
    dst = *reinterpret_cast<uint32_t*>(&h);
    UCB_PACK(ps.x, sv, 0) UCB_PACK(ps.y, sv, 1) UCB_PACK(ps.z, sv, 2) UCB_PACK(ps.w, sv, 3)
    UCB_PACK(pc.x, cv, 0) UCB_PACK(pc.y, cv, 1) UCB_PACK(pc.z, cv, 2) UCB_PACK(pc.w, cv, 3)
#undef UCB_PACK
    *reinterpret_cast<uint4*>(a.X + (size_t)r * F + j0) = ps;
    *reinterpret_cast<uint4*>(a.X + (size_t)r * F + a.fourier + j0) = pc;
    if (a.Xt) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            a.Xt[(size_t)(j0 + q) * a.rows + r] = bf16(sv[q]);
            a.Xt[(size_t)(a.fourier + j0 + q) * a.rows + r] = bf16(cv[q]);
        }
    }
    if (j0 == 0 && a.yb) a.yb[r] = valid ? (a.y[i] - a.y_mean) * a.y_inv_std : 0.f;
}

// Gradient of a run of parameters as fixed-order sums of partial results: parameter off + e
// (row o = e / cols, column c = e % cols) has the gradient
//   sum over sp = 0 .. slices - 1 of part[sp * slice_stride + o * ld + c],
// added in a fixed order. Weight runs read the split-K slices of their weight-gradient GEMM
// (a few; one thread per parameter adds them in slice order), bias runs the per-32-row block
// sums of the epilogues (hundreds, rows = 1: one warp per parameter, lane l adding slices
// l, l + 32, ... in order, then a fixed five-round shuffle tree whose lane-0 result is used).
// layer >= 0: a weight run whose BF16 copies (W, W^T) are rewritten after the update.
// base: the run's first index within its section (threads for weight runs, warps for bias
// runs).
struct GradRun {
    long long off, count, base;
    int cols, ld;
    const float* part;
    long long slice_stride;
    int slices, layer;
};

// One training step's optimiser: every parameter's gradient from its partial sums (the same
// bits whatever the launch order of the backward kernels), Adam with cosine learning-rate
// decay, and the BF16 copies of the updated weights (W for the forward products, W^T for the
// backward ones). The grid's first `thread_blocks` blocks take the weight runs, one thread
// per parameter; the rest take the bias runs, one warp per parameter, and one more warp adds
// up the loss. update = 0: only the gradient is written (to grad) and the loss; nothing
// else changes. The step counter lives on the device so that a captured step replays
// unchanged; the last block to finish advances it, after every block has read it.
struct AdamArgs {
    float* w;
    float* m;
    float* v;
    float* grad;  // optional copy of the gradient
    GradRun run[2 * kMaxLayers];
    int n_wruns, n_runs;  // runs [0, n_wruns) weights, [n_wruns, n_runs) biases
    long long n_wparams, n_bparams;
    int thread_blocks;
    const float* blk;  // loss partials: blk[3 sp + 2], sp < n_blk
    int n_blk;
    float* loss;
    unsigned long long* step;
    unsigned int* done;  // block tickets (zero between launches)
    int update;
    int total_steps;
    float lr0, lr1, b1, b2, eps;
    bf16* W[kMaxLayers];
    bf16* Wt[kMaxLayers];
    int in[kMaxLayers], outk[kMaxLayers];
};

__device__ __forceinline__ void adam_update(const AdamArgs& a, const GradRun& r, long long e, float gi,
                                            unsigned long long t) {
    const long long i = r.off + e;
    if (a.grad) a.grad[i] = gi;
    if (!a.update) return;
    const float frac = a.total_steps > 1 ? fminf((float)t / (float)(a.total_steps - 1), 1.f) : 1.f;
    const float lr = a.lr1 + 0.5f * (a.lr0 - a.lr1) * (1.f + cospif(frac));
    const float c1 = 1.f - powf(a.b1, (float)(t + 1));
    const float c2 = 1.f - powf(a.b2, (float)(t + 1));
    const float mi = a.b1 * a.m[i] + (1.f - a.b1) * gi;
    const float vi = a.b2 * a.v[i] + (1.f - a.b2) * gi * gi;
    a.m[i] = mi;
    a.v[i] = vi;
    const float wi = a.w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + a.eps);
    a.w[i] = wi;
    if (r.layer >= 0) {
        const int l = r.layer;
        const int o = (int)(e / r.cols), c = (int)(e % r.cols);
        a.W[l][(size_t)o * a.in[l] + c] = bf16(wi);
        if (a.Wt[l] && o < a.outk[l]) a.Wt[l][(size_t)c * a.outk[l] + o] = bf16(wi);
    }
}

__global__ void adam_kernel(AdamArgs a) {
    griddep_wait();
    const unsigned long long t = *a.step;  // 0-based
    if ((int)blockIdx.x < a.thread_blocks) {
        const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        if (i < a.n_wparams) {
            int k = 0;
            while (k + 1 < a.n_wruns && i >= a.run[k + 1].base) ++k;
            const GradRun& r = a.run[k];
            const long long e = i - r.base;
            const float* p = r.part + (size_t)(e / r.cols) * r.ld + (e % r.cols);
            float gi = 0.f;
            int sp = 0;
            for (; sp + 4 <= r.slices; sp += 4) {
                float q[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) q[u] = p[(size_t)(sp + u) * r.slice_stride];
#pragma unroll
                for (int u = 0; u < 4; ++u) gi += q[u];
            }
            for (; sp < r.slices; ++sp) gi += p[(size_t)sp * r.slice_stride];
            adam_update(a, r, e, gi, t);
        }
    } else {
        const long long wi = ((long long)(blockIdx.x - a.thread_blocks) * blockDim.x + threadIdx.x) / 32;
        const int lane = threadIdx.x & 31;
        if (wi < a.n_bparams) {
            int k = a.n_wruns;
            while (k + 1 < a.n_runs && wi >= a.run[k + 1].base) ++k;
            const GradRun& r = a.run[k];
            const long long e = wi - r.base;
            float part = 0.f;
            for (int sp = lane; sp < r.slices; sp += 32) part += r.part[(size_t)sp * r.slice_stride + e];
#pragma unroll
            for (int w = 16; w >= 1; w >>= 1) part += __shfl_xor_sync(0xffffffffu, part, w);
            const float gi = __shfl_sync(0xffffffffu, part, 0);
            if (lane == 0) adam_update(a, r, e, gi, t);
        } else if (wi == a.n_bparams) {
            float part = 0.f;
            for (int b = lane; b < a.n_blk; b += 32) part += a.blk[3 * b + 2];
#pragma unroll
            for (int w = 16; w >= 1; w >>= 1) part += __shfl_xor_sync(0xffffffffu, part, w);
            if (lane == 0) *a.loss = part;
        }
    }
    if (!a.update) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(a.done, 1u) == gridDim.x - 1) {
            *a.step = t + 1;
            *a.done = 0;
        }
    }
}

// BF16 copies of every layer's weights: W (out_pad x in, rows >= out zero) for the
// forward product and W^T (in x outk, columns >= out zero) for the backward product.
struct RefreshArgs {
    int n_layers;
    const float* p;
    long long w_off[kMaxLayers];
    int out[kMaxLayers], in[kMaxLayers], out_pad[kMaxLayers], outk[kMaxLayers];
    bf16* W[kMaxLayers];
    bf16* Wt[kMaxLayers];
    long long start[kMaxLayers + 1];  // prefix sums of out_pad * in
};

__global__ void refresh_kernel(RefreshArgs a) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.start[a.n_layers]) return;
    int l = 0;
    while (t >= a.start[l + 1]) ++l;
    const long long k = t - a.start[l];
    const int o = (int)(k / a.in[l]), c = (int)(k % a.in[l]);
    const float val = o < a.out[l] ? a.p[a.w_off[l] + (long long)o * a.in[l] + c] : 0.f;
    a.W[l][(size_t)o * a.in[l] + c] = bf16(val);
    if (a.Wt[l] && o < a.outk[l]) a.Wt[l][(size_t)c * a.outk[l] + o] = bf16(val);
}

// Undoes the target standardisation: mean = mu * std_y + mean_y, std = exp(lv / 2) std_y.
__global__ void unscale_kernel(const float* out, int rows, long long n_left, float y_mean, float y_std, float* mean,
                               float* sd) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows || r >= n_left) return;
    mean[r] = __fmaf_rn(out[2 * r], y_std, y_mean);
    sd[r] = __fmul_rn(expf(0.5f * fminf(fmaxf(out[2 * r + 1], -16.f), 16.f)), y_std);
}

// ------------------------------------------------------------------ fused prediction
// Prediction of every input row in one launch. A CTA takes 128-row tiles and runs, for
// each, the Fourier features, the L hidden layers (bias + GELU) and the output transform
// back to back with the tile's activations in shared memory (BF16, in the 64-column,
// 128-byte-swizzled K-major chunks the MMA descriptors read), so HBM carries the two input
// coordinates and the two outputs of a row and nothing else. Each CTA keeps two tiles in
// flight (slots 0 and 1, one TMEM accumulator of H columns each): while warps 2-17 (four per
// TMEM lane quadrant, a quarter of the columns each) turn one slot's accumulator into its
// next activations, warp 1 runs the other slot's layer on the tensor cores. Warp 0 streams
// every layer's weights (64-wide K chunks, TMA with the 128-byte swizzle) through a ring of
// stages, once per tile and layer; they stay in L2.
// The epilogue writes a layer's output over the activations its MMAs have finished
// reading, so one activation buffer per slot suffices. Waits are bounded as in the GEMM.
struct InferMaps {
    CUtensorMap w[kMaxLayers];  // layer l's BF16 weights [rows, K]: boxes of 64 (K) x H rows (16 for the output layer)
};

struct InferArgs {
    const float* u;          // n x 2 inputs, or nullptr: points from cells / grid (input_point)
    const long long* cells;
    long long n;
    int grid_n;
    const float* Bf;         // fourier x 2 frequency matrix
    int fourier;
    int layers;              // hidden layers L (the output layer is layer L)
    const float* params;     // FP32 parameters; layer l's bias at params + b_off[l]
    long long b_off[kMaxLayers];
    float y_mean, y_std;
    float* mean;             // n predictions of the mean
    float* sd;               // n predictions of the standard deviation
    long long tiles;         // ceil(n / 128)
};

constexpr int kInferEpiWarps = 16;  // four per 32-lane TMEM quadrant, a quarter of the columns each
constexpr int kInferThreads = 64 + 32 * kInferEpiWarps;

template <int H>
struct InferCfg {
    static constexpr int kOutN = 16;                         // MMA width of the output layer (2 used)
    static constexpr int kChunkBytes = kBM * kBK * 2;        // one 128 x 64 operand chunk (16 KB)
    static constexpr int kActBytes = (H / kBK) * kChunkBytes; // one slot's activations
    static constexpr int kWBytes = H * kBK * 2;              // one weight stage: H rows x 64 K
    static constexpr int kWStages = H == 256 ? 3 : 6;
    // barriers: weight full / empty per stage, accumulator full and epilogue done per slot, drain
    static constexpr int kBarriers = 2 * kWStages + 4 + 1;
    static constexpr int kSmem = 1024 + 2 * kActBytes + kWStages * kWBytes + 8 * kBarriers + 16;
    using MmaH = SM100_MMA_F16BF16_SS<bf16, bf16, float, kBM, H, UMMA::Major::K, UMMA::Major::K>;
    using MmaO = SM100_MMA_F16BF16_SS<bf16, bf16, float, kBM, kOutN, UMMA::Major::K, UMMA::Major::K>;
    using TiledH = decltype(make_tiled_mma(MmaH{}));
    using TiledO = decltype(make_tiled_mma(MmaO{}));
    using LayoutA = decltype(UMMA::tile_to_mma_shape(
        UMMA::Layout_K_SW128_Atom<bf16>{}, partition_shape_A(TiledH{}, make_shape(Int<kBM>{}, Int<kBK>{}))));
    using LayoutAO = decltype(UMMA::tile_to_mma_shape(
        UMMA::Layout_K_SW128_Atom<bf16>{}, partition_shape_A(TiledO{}, make_shape(Int<kBM>{}, Int<kBK>{}))));
    using LayoutBH = decltype(UMMA::tile_to_mma_shape(
        UMMA::Layout_K_SW128_Atom<bf16>{}, partition_shape_B(TiledH{}, make_shape(Int<H>{}, Int<kBK>{}))));
    using LayoutBO = decltype(UMMA::tile_to_mma_shape(
        UMMA::Layout_K_SW128_Atom<bf16>{}, partition_shape_B(TiledO{}, make_shape(Int<kOutN>{}, Int<kBK>{}))));
    static_assert(H == 128 || H == 256, "fused prediction: hidden width 128 or 256");
    static_assert(kSmem <= 232448, "fused prediction: shared memory above the per-CTA limit");
    static_assert(kWBytes % 1024 == 0 && kChunkBytes % 1024 == 0, "swizzled operands need 1024-byte alignment");
};

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&h);
}
// Shared-memory byte offset of the 8-column segment holding column `col` (a multiple of 8)
// of row r in a K-major 128-row BF16 operand stored as 64-column chunks of 16 KB with the
// 128-byte swizzle (16-byte unit u of a row's 128 bytes sits at unit u ^ (r mod 8)), the
// layout TMA's SWIZZLE_128B writes and the UMMA descriptors of the GEMM read.
__device__ __forceinline__ uint32_t act_offset(int r, int col) {
    return (uint32_t)((col >> 6) * (kBM * kBK * 2) + r * 128 + ((((col & 63) >> 3) ^ (r & 7)) << 4));
}
__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(x), "r"(y), "r"(z), "r"(w) : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

template <int H>
__global__ void __launch_bounds__(kInferThreads, 1)
    mlp_infer_kernel(const __grid_constant__ InferMaps maps, const InferArgs a, int* err) {
    using Cfg = InferCfg<H>;
    constexpr int S = Cfg::kWStages;
    typename Cfg::TiledH mma_h;
    typename Cfg::TiledO mma_o;
    extern __shared__ char smem_raw[];
    char* base = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    char* wst = base + 2 * Cfg::kActBytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(wst + S * Cfg::kWBytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + Cfg::kBarriers);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    auto wfull = [&](int i) { return smem_u32(bars + i); };
    auto wempty = [&](int i) { return smem_u32(bars + S + i); };
    auto accf = [&](int t) { return smem_u32(bars + 2 * S + t); };
    auto epid = [&](int t) { return smem_u32(bars + 2 * S + 2 + t); };
    const uint32_t drain_bar = smem_u32(bars + 2 * S + 4);

    const int warp = threadIdx.x / 32, lane = threadIdx.x & 31;
    cute::TMEM::Allocator1Sm tmem;
    if (warp == 0) tmem.allocate(2 * H, tmem_slot);
    if (threadIdx.x == 0) {
        for (int i = 0; i < S; ++i) {
            mbar_init(wfull(i), 1);
            mbar_init(wempty(i), 1);
        }
        for (int t = 0; t < 2; ++t) {
            mbar_init(accf(t), 1);
            mbar_init(epid(t), kInferEpiWarps);
        }
        mbar_init(drain_bar, 1);
        *abort_flag = 0;
        cutlass::arch::fence_barrier_init();
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    auto fail = [&]() {
        *abort_flag = 1;
        atomicExch(err, 1);
    };

    const int L = a.layers, F = 2 * a.fourier;
    // slot s of this CTA takes tiles 2 blockIdx.x + s + 2 gridDim.x i, i = 0, 1, ...; every
    // role walks the same (i, layer, slot) sequence and skips a slot whose tile is past the end
    const long long stride = 2LL * gridDim.x;
    auto tile_of = [&](int s, long long i) { return 2LL * blockIdx.x + s + i * stride; };
    const long long iters = (a.tiles - 2LL * blockIdx.x + stride - 1) / stride;

    if (warp == 0) {
        // ---- weight producer (lane 0)
        if (lane == 0) {
            for (int l = 0; l <= L; ++l)
                asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.w[l])) : "memory");
            int stage = 0;
            uint32_t phase = 0;
            int issued[S];
#pragma unroll
            for (int i = 0; i < S; ++i) issued[i] = 0;
            bool stop = false;
            for (long long i = 0; i < iters && !stop; ++i)
                for (int l = 0; l <= L && !stop; ++l)
                    for (int s = 0; s < 2 && !stop; ++s) {
                        if (tile_of(s, i) >= a.tiles) continue;
                        const int nk = (l == 0 ? F : H) / kBK;
                        const uint32_t bytes = (uint32_t)((l == L ? Cfg::kOutN : H) * kBK * 2);
                        for (int kc = 0; kc < nk; ++kc) {
                            if (*abort_flag || !mbar_wait_bounded(wempty(stage), phase ^ 1)) {
                                fail();
                                stop = true;
                                break;
                            }
                            mbar_expect_tx(wfull(stage), bytes);
                            tma_load_2d(smem_u32(wst + stage * Cfg::kWBytes), &maps.w[l], wfull(stage), kc * kBK, 0);
                            ++issued[stage];
                            if (++stage == S) {
                                stage = 0;
                                phase ^= 1;
                            }
                        }
                    }
            if (*abort_flag)
                for (int i = 0; i < S; ++i)
                    if (issued[i] > 0) mbar_wait_bounded(wfull(i), (uint32_t)((issued[i] - 1) & 1));
        }
    } else if (warp == 1) {
        // ---- MMA issuer (the whole warp follows; one elected lane issues)
        ThrMMA th = mma_h.get_slice(0);
        ThrMMA to = mma_o.get_slice(0);
        int stage = 0;
        uint32_t phase = 0, ep_phase[2] = {0, 0};
        bool stop = false;
        for (long long i = 0; i < iters && !stop; ++i)
            for (int l = 0; l <= L && !stop; ++l)
                for (int s = 0; s < 2 && !stop; ++s) {
                    if (tile_of(s, i) >= a.tiles) continue;
                    // the slot's activations for this layer are written and its accumulator is free
                    if (*abort_flag || !mbar_wait_bounded(epid(s), ep_phase[s])) {
                        fail();
                        stop = true;
                        break;
                    }
                    ep_phase[s] ^= 1;
                    tc_fence_after();
                    const int nk = (l == 0 ? F : H) / kBK;
                    char* act = base + s * Cfg::kActBytes;
                    const uint32_t acc = tmem_base + (uint32_t)(s * H);
                    for (int kc = 0; kc < nk; ++kc) {
                        if (*abort_flag || !mbar_wait_bounded(wfull(stage), phase)) {
                            fail();
                            stop = true;
                            break;
                        }
                        tc_fence_after();
                        bf16* a_ptr = reinterpret_cast<bf16*>(act + kc * Cfg::kChunkBytes);
                        bf16* b_ptr = reinterpret_cast<bf16*>(wst + stage * Cfg::kWBytes);
                        if (l < L) {
                            Tensor tAcc = th.make_fragment_C(
                                th.partition_C(make_identity_tensor(make_shape(Int<kBM>{}, Int<H>{}))));
                            tAcc.data() = acc;
                            Tensor fA = th.make_fragment_A(make_tensor(make_smem_ptr(a_ptr), typename Cfg::LayoutA{}));
                            Tensor fB = th.make_fragment_B(make_tensor(make_smem_ptr(b_ptr), typename Cfg::LayoutBH{}));
                            mma_h.accumulate_ = kc == 0 ? UMMA::ScaleOut::Zero : UMMA::ScaleOut::One;
                            CUTE_UNROLL
                            for (int kb = 0; kb < size<2>(fA); ++kb) {
                                gemm(mma_h, fA(_, _, kb), fB(_, _, kb), tAcc);
                                mma_h.accumulate_ = UMMA::ScaleOut::One;
                            }
                        } else {
                            Tensor tAcc = to.make_fragment_C(
                                to.partition_C(make_identity_tensor(make_shape(Int<kBM>{}, Int<Cfg::kOutN>{}))));
                            tAcc.data() = acc;
                            Tensor fA = to.make_fragment_A(make_tensor(make_smem_ptr(a_ptr), typename Cfg::LayoutAO{}));
                            Tensor fB = to.make_fragment_B(make_tensor(make_smem_ptr(b_ptr), typename Cfg::LayoutBO{}));
                            mma_o.accumulate_ = kc == 0 ? UMMA::ScaleOut::Zero : UMMA::ScaleOut::One;
                            CUTE_UNROLL
                            for (int kb = 0; kb < size<2>(fA); ++kb) {
                                gemm(mma_o, fA(_, _, kb), fB(_, _, kb), tAcc);
                                mma_o.accumulate_ = UMMA::ScaleOut::One;
                            }
                        }
                        cutlass::arch::umma_arrive(bars + S + stage);  // the weight stage is free once these ran
                        if (++stage == S) {
                            stage = 0;
                            phase ^= 1;
                        }
                    }
                    if (stop) break;
                    cutlass::arch::umma_arrive(bars + 2 * S + s);  // the slot's accumulator is complete
                }
        cutlass::arch::umma_arrive(bars + 2 * S + 4);  // every MMA issued here has completed
        if (!mbar_wait_bounded(drain_bar, 0)) fail();
    } else {
        // ---- features and epilogues: warp w owns TMEM lanes / tile rows 32 (w % 4) .. + 31
        // and, with (w - 2) / 4, one quarter of the columns
        const int quad = warp & 3, part = (warp - 2) >> 2;
        const int r = quad * 32 + lane;
        uint32_t acc_phase[2] = {0, 0};
        auto signal = [&](int s) {
            // generic-proxy stores to shared memory become visible to the MMAs (async proxy)
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(epid(s));
        };
        // X[r, j] = sin(phase_j), X[r, fourier + j] = cos(phase_j), zero past the last input
        auto features = [&](int s, long long t) {
            const uint32_t act = smem_u32(base + s * Cfg::kActBytes);
            const long long i = t * kBM + r;
            const bool valid = i < a.n;
            float u0 = 0.f, u1 = 0.f;
            if (valid) input_point(a.u, a.cells, a.grid_n, i, u0, u1);
            const int fq = a.fourier / 4;
            for (int g = 0; g < fq; g += 8) {
                const int j0 = part * fq + g;
                uint32_t ps[4], pc[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    float s0 = 0.f, c0 = 0.f, s1 = 0.f, c1 = 0.f;
                    if (valid) {
                        feature_sincos(u0, u1, a.Bf, j0 + 2 * q, s0, c0);
                        feature_sincos(u0, u1, a.Bf, j0 + 2 * q + 1, s1, c1);
                    }
                    ps[q] = pack_bf16x2(s0, s1);
                    pc[q] = pack_bf16x2(c0, c1);
                }
                st_shared_v4(act + act_offset(r, j0), ps[0], ps[1], ps[2], ps[3]);
                st_shared_v4(act + act_offset(r, a.fourier + j0), pc[0], pc[1], pc[2], pc[3]);
            }
        };
        for (int s = 0; s < 2; ++s)
            if (tile_of(s, 0) < a.tiles) {
                features(s, tile_of(s, 0));
                signal(s);
            }
        bool stop = false;
        for (long long i = 0; i < iters && !stop; ++i)
            for (int l = 0; l <= L && !stop; ++l)
                for (int s = 0; s < 2; ++s) {
                    const long long t = tile_of(s, i);
                    if (t >= a.tiles) continue;
                    if (*abort_flag || !mbar_wait_bounded(accf(s), acc_phase[s])) {
                        fail();
                        stop = true;
                        break;
                    }
                    acc_phase[s] ^= 1;
                    tc_fence_after();
                    const uint32_t tq = tmem_base + (uint32_t)(s * H) + ((uint32_t)(quad * 32) << 16);
                    if (l < L) {
                        // bias + GELU -> BF16 activations of layer l + 1, over this slot's buffer
                        const uint32_t act = smem_u32(base + s * Cfg::kActBytes);
                        const float4* b4 = reinterpret_cast<const float4*>(a.params + a.b_off[l]);
                        // hidden activations are stored doubled (gelu2_twice): layers after the
                        // first take half their accumulator
                        const float in_scale = l == 0 ? 1.0f : 0.5f;
                        const float2 sc = make_float2(in_scale, in_scale);
#pragma unroll 1
                        for (int c0 = part * (H / 4); c0 < (part + 1) * (H / 4); c0 += 32) {
                            uint32_t rv[32];
                            tmem_ld32(tq + (uint32_t)c0, rv);
                            uint32_t pk[16];
#pragma unroll
                            for (int q = 0; q < 8; ++q) {
                                const float4 b = __ldg(b4 + c0 / 4 + q);
                                const float2 g0 = gelu2_twice(__ffma2_rn(
                                    make_float2(__uint_as_float(rv[4 * q]), __uint_as_float(rv[4 * q + 1])), sc,
                                    make_float2(b.x, b.y)));
                                const float2 g1 = gelu2_twice(__ffma2_rn(
                                    make_float2(__uint_as_float(rv[4 * q + 2]), __uint_as_float(rv[4 * q + 3])), sc,
                                    make_float2(b.z, b.w)));
                                pk[2 * q] = pack_bf16x2(g0.x, g0.y);
                                pk[2 * q + 1] = pack_bf16x2(g1.x, g1.y);
                            }
#pragma unroll
                            for (int q = 0; q < 4; ++q)
                                st_shared_v4(act + act_offset(r, c0 + 8 * q), pk[4 * q], pk[4 * q + 1], pk[4 * q + 2],
                                             pk[4 * q + 3]);
                        }
                        signal(s);
                    } else {
                        // output layer: mean = mu std_y + mean_y, sd = exp(clamp(lv) / 2) std_y
                        if (part == 0) {
                            uint32_t o0, o1;
                            asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];\n"
                                         : "=r"(o0), "=r"(o1)
                                         : "r"(tq));
                            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                            const float* bo = a.params + a.b_off[L];
                            const float mu = __fmaf_rn(__uint_as_float(o0), 0.5f, __ldg(bo));
                            const float lv = __fmaf_rn(__uint_as_float(o1), 0.5f, __ldg(bo + 1));
                            const long long row = t * kBM + r;
                            if (row < a.n) {
                                a.mean[row] = __fmaf_rn(mu, a.y_std, a.y_mean);
                                a.sd[row] = __fmul_rn(expf(0.5f * fminf(fmaxf(lv, -16.f), 16.f)), a.y_std);
                            }
                        }
                        const long long tn = tile_of(s, i + 1);
                        if (tn < a.tiles) {
                            features(s, tn);
                            signal(s);
                        }
                    }
                }
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem.release_allocation_lock();
        tmem.free(tmem_base, 2 * H);
    }
}

}  // namespace ucbmlp

// ====================================================================== host side
namespace ucb {

using ucbmlp::bf16;

namespace {

constexpr int kMaxSplits = 16;  // split-K slices per weight-gradient tile

bool cu_ok(cudaError_t e, std::string& err, const char* what) {
    if (e == cudaSuccess) return true;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}

// Kernel launch, with programmatic stream serialisation when pdl is set (the kernel may start
// while its predecessor in the stream finishes; the kernels wait with griddepcontrol before
// touching memory).
template <typename... KArgs, typename... Args>
bool launch(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
            std::string& err, const char* what, Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cu_ok(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...), err, what);
}

template <class T>
T* dalloc(size_t count, std::vector<void*>& owned, std::string& err, const char* what) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
        err = std::string("cudaMalloc(") + what + ") failed";
        return nullptr;
    }
    cudaMemset(p, 0, std::max<size_t>(count, 1) * sizeof(T));
    owned.push_back(p);
    return static_cast<T*>(p);
}

}  // namespace

struct Mlp {
    ucb_engine* e = nullptr;
    ucb_mlp_config cfg{};
    int F = 0, H = 0, L = 0;
    std::vector<int> in, out, out_pad, outk;
    std::vector<long long> w_off, b_off;
    long long n_params = 0;
    std::vector<void*> owned;      // device allocations of the network
    std::vector<void*> act_owned;  // batch-size dependent
    float *p = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr, *Bf = nullptr;
    std::vector<bf16*> W, Wt;
    unsigned long long* step = nullptr;
    int* err = nullptr;
    float* loss = nullptr;
    float y_mean = 0.f, y_std = 1.f;
    int rows = 0;                  // activation capacity (rows)
    bf16 *X = nullptr, *Xt = nullptr;
    std::vector<float*> Z;
    std::vector<bf16*> Hb, Ht;
    float* outp = nullptr;         // rows x 2
    float* yb = nullptr;
    bf16 *dout = nullptr, *doutT = nullptr;
    std::vector<bf16*> dZ, dZt;    // dL/dZ of each hidden layer and its transposed copy
    // training-step launches: programmatic dependent launch on, and a second stream for the
    // weight-gradient products (forked from / joined to the caller's stream with events)
    bool pdl = false;
    cudaStream_t side = nullptr;
    std::vector<cudaEvent_t> ev;
    // partial sums that the optimiser kernel adds in a fixed order: per layer the split-K
    // slices of the weight gradient, per hidden layer the bias-gradient sums of 32-row
    // blocks, and the output layer's per-block NLL sums
    std::vector<float*> part;
    std::vector<long long> part_cap;
    std::vector<int> splits;
    std::vector<float*> dbp;
    float* blk = nullptr;
    unsigned int* done = nullptr;
    // prediction buffers (ping-pong activations, no backward copies)
    std::vector<void*> pred_owned;
    int pred_rows = 0;
    bf16* pX = nullptr;
    bf16* pH[2] = {nullptr, nullptr};
    float* pOut = nullptr;
    cudaGraphExec_t graph = nullptr;
    long long graph_nodes = 0;
    MlpInputs graph_in;
    const float* graph_y = nullptr;
    float graph_y_mean = 0.f, graph_y_std = 0.f;

    ~Mlp() {
        if (graph) cudaGraphExecDestroy(graph);
        for (cudaEvent_t x : ev) cudaEventDestroy(x);
        if (side) cudaStreamDestroy(side);
        for (void* q : act_owned) cudaFree(q);
        for (void* q : pred_owned) cudaFree(q);
        for (void* q : owned) cudaFree(q);
    }
};

namespace {

std::mutex g_attr_mu;
std::vector<int> g_attr_devices;

// Every compiled GEMM instantiation: tile width x epilogue mode (the modes a training step
// and the layer-by-layer prediction use, and one with every feature for anything else).
constexpr int kGemmModes[] = {ucbmlp::kModeForward, ucbmlp::kModeLoss, ucbmlp::kModeDz, ucbmlp::kModeSplit,
                              ucbmlp::kModeHidden,  ucbmlp::kModeOut,  ucbmlp::kEpAll};
template <int BN, int I = 0, class F>
void for_each_mode(F&& f) {
    if constexpr (I < (int)(sizeof(kGemmModes) / sizeof(kGemmModes[0]))) {
        f(ucbmlp::gemm_tma_kernel<BN, kGemmModes[I]>, ucbmlp::GemmCfg<BN>::kSmem, kGemmModes[I]);
        for_each_mode<BN, I + 1>(f);
    }
}
template <class F>
void for_each_gemm(F&& f) {
    for_each_mode<128>([&](auto k, int smem, int) { f(k, smem); });
    for_each_mode<256>([&](auto k, int smem, int) { f(k, smem); });
}
// The epilogue mode of a launch: the smallest compiled one that covers the features it uses.
int gemm_mode(const ucbmlp::Epilogue& ep) {
    int need = 0;
    if (ep.bias) need |= ucbmlp::kEpBias;
    if (ep.gelu) need |= ucbmlp::kEpGelu;
    if (ep.outf) need |= ucbmlp::kEpOutF;
    if (ep.outh) need |= ucbmlp::kEpOutH;
    if (ep.outt) need |= ucbmlp::kEpOutT;
    if (ep.zin) need |= ucbmlp::kEpZin;
    if (ep.colsum) need |= ucbmlp::kEpColsum;
    if (ep.nll) need |= ucbmlp::kEpNll;
    int best = ucbmlp::kEpAll;
    for (int md : kGemmModes)
        if ((need & ~md) == 0 && __builtin_popcount(md) < __builtin_popcount(best)) best = md;
    return best;
}

// Dynamic shared memory above 48 KB is opted in once per device, before launches and
// before any stream capture.
bool set_gemm_attributes(int device, std::string& err) {
    std::lock_guard<std::mutex> lk(g_attr_mu);
    if (std::find(g_attr_devices.begin(), g_attr_devices.end(), device) != g_attr_devices.end()) return true;
    cudaError_t ce = cudaSuccess;
    for_each_gemm([&](auto kernel, int smem) {
        if (ce == cudaSuccess) ce = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    });
    if (!cu_ok(ce, err, "cudaFuncSetAttribute(gemm)")) return false;
    ce = cudaFuncSetAttribute(ucbmlp::mlp_infer_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              ucbmlp::InferCfg<128>::kSmem);
    if (!cu_ok(ce, err, "cudaFuncSetAttribute(infer 128)")) return false;
    ce = cudaFuncSetAttribute(ucbmlp::mlp_infer_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              ucbmlp::InferCfg<256>::kSmem);
    if (!cu_ok(ce, err, "cudaFuncSetAttribute(infer 256)")) return false;
    g_attr_devices.push_back(device);
    return true;
}

// cuTensorMapEncodeTiled from the driver the runtime has loaded (no link-time dependency on
// libcuda, so the library still loads on machines without a driver).
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_tiled(std::string& err) {
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    if (!fn) err = "cuTensorMapEncodeTiled is not available from the CUDA driver";
    return fn;
}

// Tensor map of a K-contiguous BF16 matrix [rows, K]: boxes of 64 (K) x box_rows with the
// 128-byte swizzle the MMA's shared-memory descriptors expect.
bool tensor_map(CUtensorMap* map, const bf16* ptr, int rows, int K, int box_rows, std::string& err) {
    EncodeTiled fn = encode_tiled(err);
    if (!fn) return false;
    if ((reinterpret_cast<uintptr_t>(ptr) & 15) != 0 || K % ucbmlp::kBK) {
        err = "gemm: operand not 16-byte aligned or K not a multiple of 64";
        return false;
    }
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)K * sizeof(bf16)};
    const cuuint32_t box[2] = {(cuuint32_t)ucbmlp::kBK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(ptr), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
        return false;
    }
    return true;
}

// C = A B^T (+ epilogue). ep.atomic: K is split into up to kMaxSplits slices per tile and
// each slice's partial tile (rows < m_store, columns < n_store) is stored at
// ep.outf + slice * m_eff * ep.ldf (m_eff = min(M, m_store)); *splits_out receives the
// number of slices and part_cap bounds the buffer (floats). The slices are added later, in
// slice order, by the optimiser kernel.
bool gemm(Mlp& m, const bf16* A, const bf16* B, int M, int N, int K, const ucbmlp::Epilogue& ep_in, cudaStream_t st,
          std::string& err, int* splits_out = nullptr, long long part_cap = 0) {
    ucbmlp::Epilogue ep = ep_in;
    if (M <= 0 || N <= 0 || K <= 0 || M % ucbmlp::kBM || N % 128 || K % ucbmlp::kBK) {
        err = "gemm: unsupported shape " + std::to_string(M) + "x" + std::to_string(N) + "x" + std::to_string(K);
        return false;
    }
    const int sms = std::max(m.e->sm_count, 1);
    // 256-wide tiles read A once; below one wide tile per SM the 128-wide tiles keep twice
    // as many SMs busy (and halve each CTA's epilogue)
    const int bn = (N % 256 == 0 && (M / ucbmlp::kBM) * (N / 256) >= sms) ? 256 : 128;
    const int tiles = (M / ucbmlp::kBM) * (N / bn);
    const int kt = K / ucbmlp::kBK;
    int per = kt;
    if (ep.atomic) {
        // about one (tile, slice) item per SM: more slices only add partial-tile traffic
        const int want = std::max(1, std::min({kt, kMaxSplits, sms / tiles}));
        per = (kt + want - 1) / want;
    }
    const int splits = (kt + per - 1) / per;
    const long long m_eff = std::min(M, ep.m_store), n_eff = std::min(N, ep.n_store);
    if (ep.atomic) {
        if (!splits_out || ep.ldf < n_eff || (long long)splits * m_eff * ep.ldf > part_cap) {
            err = "gemm: split-K partial buffer too small";
            return false;
        }
        ep.split_stride = m_eff * ep.ldf;
        *splits_out = splits;
    } else {
        ep.split_stride = 0;
    }
    CUtensorMap ta, tb;
    if (!tensor_map(&ta, A, M, K, ucbmlp::kBM, err) || !tensor_map(&tb, B, N, K, bn, err)) return false;
    ucbmlp::GemmWork w{N / bn, splits, kt, per, tiles * splits};
    const int grid = std::min(w.items, sms);
    m.e->launches += 1;
    const int mode = gemm_mode(ep);
    bool ok = false, found = false;
    auto go = [&](auto kernel, int smem, int md) {
        if (found || md != mode) return;
        found = true;
        ok = launch(m.pdl, kernel, dim3(grid), dim3(ucbmlp::kGemmThreads), smem, st, err, "gemm launch", ta, tb, w,
                    ep, m.err);
    };
    if (bn == 256)
        for_each_mode<256>(go);
    else
        for_each_mode<128>(go);
    if (!found) err = "gemm: no compiled epilogue mode";
    return ok;
}

ucbmlp::Epilogue epi() {
    ucbmlp::Epilogue ep{};
    ep.m_store = 1 << 30;
    ep.n_store = 1 << 30;
    return ep;
}

bool ensure_rows(Mlp& m, int rows, std::string& err) {
    if (rows <= m.rows) return true;
    if (m.graph) {
        cudaGraphExecDestroy(m.graph);
        m.graph = nullptr;
    }
    for (void* q : m.act_owned) cudaFree(q);
    m.act_owned.clear();
    m.Z.clear();
    m.Hb.clear();
    m.Ht.clear();
    m.rows = 0;
    auto& o = m.act_owned;
    const size_t R = rows;
    if (!(m.X = dalloc<bf16>(R * m.F, o, err, "features")) || !(m.Xt = dalloc<bf16>(R * m.F, o, err, "features^T")))
        return false;
    for (int l = 0; l < m.L; ++l) {
        float* z = dalloc<float>(R * m.H, o, err, "Z");
        bf16* h = dalloc<bf16>(R * m.H, o, err, "H");
        bf16* ht = dalloc<bf16>(R * m.H, o, err, "H^T");
        if (!z || !h || !ht) return false;
        m.Z.push_back(z);
        m.Hb.push_back(h);
        m.Ht.push_back(ht);
    }
    if (!(m.outp = dalloc<float>(R * 2, o, err, "out")) || !(m.yb = dalloc<float>(R, o, err, "y batch")) ||
        !(m.dout = dalloc<bf16>(R * 64, o, err, "dOut")) || !(m.doutT = dalloc<bf16>(R * 128, o, err, "dOut^T")))
        return false;
    m.dZ.assign(m.L, nullptr);
    m.dZt.assign(m.L, nullptr);
    for (int l = 0; l < m.L; ++l)
        if (!(m.dZ[l] = dalloc<bf16>(R * m.H, o, err, "dZ")) || !(m.dZt[l] = dalloc<bf16>(R * m.H, o, err, "dZ^T")))
            return false;
    m.part.assign(m.L + 1, nullptr);
    m.part_cap.assign(m.L + 1, 0);
    m.splits.assign(m.L + 1, 0);
    m.dbp.assign(m.L, nullptr);
    for (int l = 0; l <= m.L; ++l) {
        // split-K slices of layer l's weight gradient: [splits][rows of W][in]
        m.part_cap[l] = (long long)kMaxSplits * (l == m.L ? 2 : m.H) * m.in[l];
        if (!(m.part[l] = dalloc<float>((size_t)m.part_cap[l], o, err, "split-K partials"))) return false;
    }
    for (int l = 0; l < m.L; ++l)
        if (!(m.dbp[l] = dalloc<float>((R + 31) / 32 * m.H, o, err, "bias-gradient partials"))) return false;
    if (!(m.blk = dalloc<float>((R + 31) / 32 * 3, o, err, "NLL block sums")) ||
        !(m.done = dalloc<unsigned int>(1, o, err, "block tickets")))
        return false;
    m.rows = rows;
    return true;
}

bool ensure_pred_rows(Mlp& m, int rows, std::string& err) {
    if (rows <= m.pred_rows) return true;
    for (void* q : m.pred_owned) cudaFree(q);
    m.pred_owned.clear();
    m.pred_rows = 0;
    auto& o = m.pred_owned;
    const size_t R = rows;
    if (!(m.pX = dalloc<bf16>(R * m.F, o, err, "features")) || !(m.pH[0] = dalloc<bf16>(R * m.H, o, err, "H")) ||
        !(m.pH[1] = dalloc<bf16>(R * m.H, o, err, "H")) || !(m.pOut = dalloc<float>(R * 2, o, err, "out")))
        return false;
    m.pred_rows = rows;
    return true;
}

bool refresh(Mlp& m, cudaStream_t st, std::string& err) {
    ucbmlp::RefreshArgs a{};
    a.n_layers = m.L + 1;
    a.p = m.p;
    a.start[0] = 0;
    for (int l = 0; l <= m.L; ++l) {
        a.w_off[l] = m.w_off[l];
        a.out[l] = m.out[l];
        a.in[l] = m.in[l];
        a.out_pad[l] = m.out_pad[l];
        a.outk[l] = m.outk[l];
        a.W[l] = m.W[l];
        a.Wt[l] = m.Wt[l];
        a.start[l + 1] = a.start[l] + (long long)m.out_pad[l] * m.in[l];
    }
    const long long total = a.start[a.n_layers];
    ucbmlp::refresh_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(a);
    m.e->launches += 1;
    return cu_ok(cudaPeekAtLastError(), err, "refresh launch");
}

ucbmlp::FeatureArgs feature_args(Mlp& m, const MlpInputs& in, long long row0, int rows, bool train) {
    ucbmlp::FeatureArgs a{};
    a.u = in.u;
    a.cells = in.cells;
    a.n = in.n;
    a.grid_n = in.grid_n;
    a.row0 = row0;
    a.step = train ? m.step : nullptr;
    a.seed = m.cfg.seed * 0x9E3779B97F4A7C15ULL + 12345;
    a.y_mean = m.y_mean;
    a.y_inv_std = 1.f / m.y_std;
    a.Bf = m.Bf;
    a.fourier = m.cfg.fourier;
    a.rows = rows;
    a.X = m.X;
    a.Xt = train ? m.Xt : nullptr;
    return a;
}

bool features(Mlp& m, const ucbmlp::FeatureArgs& a, cudaStream_t st, std::string& err) {
    const long long t = (long long)a.rows * (a.fourier / 8);
    m.e->launches += 1;
    return launch(m.pdl, ucbmlp::features_kernel, dim3((unsigned)((t + 255) / 256)), dim3(256), 0, st, err,
                  "features launch", a);
}

// Forward pass over `rows` rows of m.X. keep: store Z and H^T for the backward pass and
// evaluate the loss of the first n_valid rows against m.yb (dOut, dOut^T, block sums).
bool forward(Mlp& m, int rows, bool keep, cudaStream_t st, std::string& err, int n_valid = 0) {
    const bf16* x = m.X;
    int k = m.F;
    for (int l = 0; l < m.L; ++l) {
        ucbmlp::Epilogue ep = epi();
        ep.bias = m.p + m.b_off[l];
        ep.nb = m.H;
        ep.gelu = 1;
        ep.outf = keep ? m.Z[l] : nullptr;
        ep.ldf = m.H;
        ep.outh = m.Hb[l];
        ep.ldh = m.H;
        ep.outt = keep ? m.Ht[l] : nullptr;
        ep.ldt = rows;
        if (!gemm(m, x, m.W[l], rows, m.H, k, ep, st, err)) return false;
        x = m.Hb[l];
        k = m.H;
    }
    ucbmlp::Epilogue ep = epi();
    ep.bias = m.p + m.b_off[m.L];
    ep.nb = 2;
    ep.outf = m.outp;
    ep.ldf = 2;
    ep.n_store = 2;
    if (keep) {
        ep.nll = 1;
        ep.yb = m.yb;
        ep.n_valid = n_valid;
        ep.rows = rows;
        ep.beta = m.cfg.beta_nll;
        ep.dout = m.dout;
        ep.doutT = m.doutT;
        ep.blk = m.blk;
    }
    return gemm(m, x, m.W[m.L], rows, m.out_pad[m.L], m.H, ep, st, err);
}

// Inference forward pass over `rows` rows of m.pX (activations ping-pong in m.pH).
bool forward_infer(Mlp& m, int rows, cudaStream_t st, std::string& err) {
    const bf16* x = m.pX;
    int k = m.F;
    for (int l = 0; l < m.L; ++l) {
        ucbmlp::Epilogue ep = epi();
        ep.bias = m.p + m.b_off[l];
        ep.nb = m.H;
        ep.gelu = 1;
        ep.outh = m.pH[l & 1];
        ep.ldh = m.H;
        if (!gemm(m, x, m.W[l], rows, m.H, k, ep, st, err)) return false;
        x = m.pH[l & 1];
        k = m.H;
    }
    ucbmlp::Epilogue ep = epi();
    ep.bias = m.p + m.b_off[m.L];
    ep.nb = 2;
    ep.outf = m.pOut;
    ep.ldf = 2;
    ep.n_store = 2;
    return gemm(m, x, m.W[m.L], rows, m.out_pad[m.L], m.H, ep, st, err);
}

// Backward pass for the batch of the last forward(keep) (which already left dL/dOut in
// dOut / dOut^T and the NLL block sums in blk): every product stores partial results only
// (split-K slices of the weight gradients, 32-row block sums of the bias gradients); the
// optimiser kernel adds them. dL/dZ of a hidden layer comes straight out of the epilogue of
// the product that gives dL/dH (GELU backward fused). The weight-gradient products run on a
// second stream beside that chain (each one forked when its dL/dZ is written, all joined
// before the caller's stream goes on), so only the dL/dZ chain is on the critical path.
bool backward(Mlp& m, int rows, cudaStream_t st, std::string& err) {
    const int Lo = m.L;
    int evi = 0;
    auto fork = [&]() {
        cudaEvent_t e = m.ev[evi++];
        return cu_ok(cudaEventRecord(e, st), err, "fork record") &&
               cu_ok(cudaStreamWaitEvent(m.side, e, 0), err, "fork wait");
    };
    auto weight_grad = [&](int l, const bf16* At, const bf16* prevT) {
        ucbmlp::Epilogue eg = epi();
        eg.outf = m.part[l];
        eg.ldf = m.in[l];
        eg.atomic = 1;
        int M = m.H;
        if (l == Lo) {  // dOut^T H: M padded to 128, rows 0 and 1 stored
            eg.m_store = 2;
            M = 128;
        }
        return gemm(m, At, prevT, M, m.in[l], rows, eg, m.side, err, &m.splits[l], m.part_cap[l]);
    };
    auto dz = [&](int l, const bf16* A, const bf16* Bt, int K) {  // dL/dZ of hidden layer l
        ucbmlp::Epilogue ep = epi();
        ep.zin = m.Z[l];
        ep.ldz = m.H;
        ep.outh = m.dZ[l];
        ep.ldh = m.H;
        ep.outt = m.dZt[l];
        ep.ldt = rows;
        ep.colsum = m.dbp[l];
        ep.ldc = m.H;
        return gemm(m, A, Bt, rows, m.H, K, ep, st, err);
    };
    // output layer: its weight gradient needs only dOut^T; dL/dZ of the last hidden layer is
    // (dOut W_out) GELU'(Z), K padded to 64
    if (!fork() || !weight_grad(Lo, m.doutT, m.Ht[Lo - 1]) || !dz(Lo - 1, m.dout, m.Wt[Lo], 64)) return false;
    for (int l = Lo - 1; l >= 0; --l) {
        if (!fork() || !weight_grad(l, m.dZt[l], l > 0 ? m.Ht[l - 1] : m.Xt)) return false;
        if (l > 0 && !dz(l - 1, m.dZ[l], m.Wt[l], m.H)) return false;
    }
    cudaEvent_t j = m.ev[evi++];
    return cu_ok(cudaEventRecord(j, m.side), err, "join record") && cu_ok(cudaStreamWaitEvent(st, j, 0), err, "join wait");
}

// The optimiser kernel over the partial results of the last backward(rows): update = true
// runs Adam and refreshes the BF16 weights; false only writes the gradient to m.g. Both
// write the loss.
bool adam(Mlp& m, int rows, bool update, cudaStream_t st, std::string& err) {
    ucbmlp::AdamArgs a{};
    a.w = m.p;
    a.m = m.m1;
    a.v = m.m2;
    a.grad = update ? nullptr : m.g;
    const int nblk = (rows + 31) / 32;
    int k = 0;
    long long base = 0;
    for (int l = 0; l <= m.L; ++l) {  // weight runs: one thread per parameter
        ucbmlp::GradRun w{};
        w.off = m.w_off[l];
        w.count = (long long)m.out[l] * m.in[l];
        w.base = base;
        w.cols = m.in[l];
        w.ld = m.in[l];
        w.part = m.part[l];
        w.slice_stride = (long long)(l == m.L ? 2 : m.H) * m.in[l];
        w.slices = m.splits[l];
        w.layer = l;
        a.run[k++] = w;
        base += w.count;
    }
    a.n_wruns = k;
    a.n_wparams = base;
    base = 0;
    for (int l = 0; l <= m.L; ++l) {  // bias runs: one warp per parameter
        const bool out = l == m.L;
        ucbmlp::GradRun b{};
        b.off = m.b_off[l];
        b.count = m.out[l];
        b.base = base;
        b.cols = m.out[l];
        b.ld = 0;
        b.part = out ? m.blk : m.dbp[l];
        b.slice_stride = out ? 3 : m.H;
        b.slices = nblk;
        b.layer = -1;
        a.run[k++] = b;
        base += b.count;
    }
    a.n_runs = k;
    a.n_bparams = base;
    a.thread_blocks = (int)((a.n_wparams + 255) / 256);
    const long long warp_blocks = ((a.n_bparams + 1) * 32 + 255) / 256;  // + the loss warp
    a.blk = m.blk;
    a.n_blk = nblk;
    a.loss = m.loss;
    a.step = m.step;
    a.done = m.done;
    a.update = update ? 1 : 0;
    a.total_steps = m.cfg.train_steps;
    a.lr0 = m.cfg.lr;
    a.lr1 = m.cfg.lr_final;
    a.b1 = 0.9f;
    a.b2 = 0.999f;
    a.eps = 1e-8f;
    for (int l = 0; l <= m.L; ++l) {
        a.W[l] = m.W[l];
        a.Wt[l] = m.Wt[l];
        a.in[l] = m.in[l];
        a.outk[l] = m.outk[l];
    }
    m.e->launches += 1;
    return launch(m.pdl, ucbmlp::adam_kernel, dim3((unsigned)(a.thread_blocks + warp_blocks)), dim3(256), 0, st,
                  err, "adam launch", a);
}

bool check_kernel_error(Mlp& m, cudaStream_t st, std::string& err) {
    int h = 0;
    if (!cu_ok(cudaMemcpyAsync(&h, m.err, sizeof(int), cudaMemcpyDeviceToHost, st), err, "read error flag") ||
        !cu_ok(cudaStreamSynchronize(st), err, "mlp"))
        return false;
    if (h) {
        err = "tensor-core GEMM timed out waiting for its MMAs";
        return false;
    }
    return true;
}

// One training step (features of a random batch, forward with the loss in the output
// layer's epilogue, backward, and the optimiser kernel: gradient sums, Adam, BF16 weights,
// step count): the sequence that is captured into a CUDA graph, 16 kernels for 4 hidden
// layers.
bool train_step(Mlp& m, const MlpInputs& in, const float* d_y, cudaStream_t st, std::string& err) {
    const int rows = m.cfg.batch;
    ucbmlp::FeatureArgs fa = feature_args(m, in, 0, rows, true);
    fa.y = d_y;
    fa.yb = m.yb;
    return features(m, fa, st, err) && forward(m, rows, true, st, err, rows) && backward(m, rows, st, err) &&
           adam(m, rows, true, st, err);
}

}  // namespace

Mlp* mlp_create(ucb_engine* e, const ucb_mlp_config& c, std::string& err) {
    if (c.fourier <= 0 || (2 * c.fourier) % 128 || c.hidden <= 0 || c.hidden % 128 || c.layers < 1 ||
        c.layers > ucbmlp::kMaxLayers - 1 || c.batch <= 0 || c.batch % 128 || c.train_steps < 0 ||
        !(c.fourier_scale >= 0.f)) {
        err = "invalid MLP configuration (2*fourier % 128 == 0, hidden % 128 == 0, 1 <= layers <= 8, "
              "batch % 128 == 0, train_steps >= 0)";
        return nullptr;
    }
    if (!ensure_init(e, err)) return nullptr;
    if (!set_gemm_attributes(e->device, err)) return nullptr;
    auto m = std::make_unique<Mlp>();
    m->e = e;
    m->cfg = c;
    m->F = 2 * c.fourier;
    m->H = c.hidden;
    m->L = c.layers;
    long long off = 0;
    for (int l = 0; l <= m->L; ++l) {
        const int i = l == 0 ? m->F : m->H;
        const int o = l == m->L ? 2 : m->H;
        m->in.push_back(i);
        m->out.push_back(o);
        m->out_pad.push_back(l == m->L ? 128 : o);
        m->outk.push_back(l == m->L ? 64 : o);
        m->w_off.push_back(off);
        off += (long long)o * i;
        m->b_off.push_back(off);
        off += o;
    }
    m->n_params = off;
    auto& ow = m->owned;
    if (!(m->p = dalloc<float>(off, ow, err, "params")) || !(m->g = dalloc<float>(off, ow, err, "grad")) ||
        !(m->m1 = dalloc<float>(off, ow, err, "adam m")) || !(m->m2 = dalloc<float>(off, ow, err, "adam v")) ||
        !(m->Bf = dalloc<float>(2 * c.fourier, ow, err, "fourier")) ||
        !(m->step = dalloc<unsigned long long>(1, ow, err, "step")) || !(m->err = dalloc<int>(1, ow, err, "err")) ||
        !(m->loss = dalloc<float>(1, ow, err, "loss")))
        return nullptr;
    for (int l = 0; l <= m->L; ++l) {
        bf16* w = dalloc<bf16>((size_t)m->out_pad[l] * m->in[l], ow, err, "W bf16");
        bf16* wt = l > 0 ? dalloc<bf16>((size_t)m->in[l] * m->outk[l], ow, err, "W^T bf16") : nullptr;
        if (!w || (l > 0 && !wt)) return nullptr;
        m->W.push_back(w);
        m->Wt.push_back(wt);
    }
    if (!cu_ok(cudaStreamCreateWithFlags(&m->side, cudaStreamNonBlocking), err, "weight-gradient stream"))
        return nullptr;
    m->ev.assign(m->L + 2, nullptr);
    for (auto& x : m->ev)
        if (!cu_ok(cudaEventCreateWithFlags(&x, cudaEventDisableTiming), err, "event")) return nullptr;
    if (!mlp_reinit(m.get(), err)) return nullptr;
    return m.release();
}

bool mlp_reinit(Mlp* m, std::string& err) {
    // Initialisation: W ~ N(0, 2 / in) for hidden layers (GELU), N(0, 0.1 / in) for the
    // output layer, biases 0; frequency matrix ~ N(0, fourier_scale^2).
    const ucb_mlp_config& c = m->cfg;
    std::mt19937_64 rng(c.seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    std::vector<float> hp(m->n_params, 0.f);
    for (int l = 0; l <= m->L; ++l) {
        const float sd = std::sqrt((l == m->L ? 0.1f : 2.0f) / (float)m->in[l]);
        for (long long k = 0; k < (long long)m->out[l] * m->in[l]; ++k) hp[m->w_off[l] + k] = sd * nd(rng);
    }
    std::vector<float> hb(2 * c.fourier);
    for (auto& v : hb) v = c.fourier_scale * nd(rng);
    m->y_mean = 0.f;
    m->y_std = 1.f;
    if (!cu_ok(cudaMemcpy(m->p, hp.data(), m->n_params * sizeof(float), cudaMemcpyHostToDevice), err,
               "upload params") ||
        !cu_ok(cudaMemcpy(m->Bf, hb.data(), hb.size() * sizeof(float), cudaMemcpyHostToDevice), err, "upload B"))
        return false;
    return refresh(*m, m->e->stream, err) && cu_ok(cudaStreamSynchronize(m->e->stream), err, "init");
}

const ucb_mlp_config& mlp_config(const Mlp* m) { return m->cfg; }

void mlp_destroy(Mlp* m) {
    if (!m) return;
    cudaDeviceSynchronize();
    delete m;
}

long long mlp_param_count(const Mlp* m) { return m ? m->n_params : 0; }
int mlp_features(const Mlp* m) { return m ? m->F : 0; }

// Whether the fused prediction kernel covers this network (hidden width 128 or 256, features
// no wider than a hidden layer).
static bool fused_predict_supported(const Mlp& m) {
    return (m.H == 128 || m.H == 256) && m.F <= m.H && m.F % ucbmlp::kBK == 0 && (m.F / 2) % 32 == 0 &&
           m.L + 1 <= ucbmlp::kMaxLayers;
}

static bool predict_fused(Mlp& m, const MlpInputs& in, float* d_mean, float* d_std, cudaStream_t st, std::string& err) {
    ucbmlp::InferMaps maps;
    std::memset(&maps, 0, sizeof maps);
    for (int l = 0; l < m.L; ++l)
        if (!tensor_map(&maps.w[l], m.W[l], m.H, m.in[l], m.H, err)) return false;
    if (!tensor_map(&maps.w[m.L], m.W[m.L], m.out_pad[m.L], m.H, ucbmlp::InferCfg<256>::kOutN, err)) return false;
    ucbmlp::InferArgs a{};
    a.u = in.u;
    a.cells = in.cells;
    a.n = in.n;
    a.grid_n = in.grid_n;
    a.Bf = m.Bf;
    a.fourier = m.cfg.fourier;
    a.layers = m.L;
    a.params = m.p;
    for (int l = 0; l <= m.L; ++l) {
        if (m.b_off[l] % 4) {
            err = "fused prediction: bias not 16-byte aligned";
            return false;
        }
        a.b_off[l] = m.b_off[l];
    }
    a.y_mean = m.y_mean;
    a.y_std = m.y_std;
    a.mean = d_mean;
    a.sd = d_std;
    a.tiles = (in.n + ucbmlp::kBM - 1) / ucbmlp::kBM;
    const long long pairs = (a.tiles + 1) / 2;
    const int grid = (int)std::min<long long>(pairs, std::max(m.e->sm_count, 1));
    if (m.H == 256)
        ucbmlp::mlp_infer_kernel<256><<<grid, ucbmlp::kInferThreads, ucbmlp::InferCfg<256>::kSmem, st>>>(maps, a, m.err);
    else
        ucbmlp::mlp_infer_kernel<128><<<grid, ucbmlp::kInferThreads, ucbmlp::InferCfg<128>::kSmem, st>>>(maps, a, m.err);
    m.e->launches += 1;
    return cu_ok(cudaPeekAtLastError(), err, "fused prediction launch");
}

bool mlp_predict(Mlp* m, const MlpInputs& in, float* d_mean, float* d_std, cudaStream_t st, std::string& err) {
    if (in.n <= 0) return true;
    if (fused_predict_supported(*m)) return predict_fused(*m, in, d_mean, d_std, st, err);
    const long long chunk = 1 << 18;
    const long long rows_needed = std::min<long long>(chunk, ((in.n + 127) / 128) * 128);
    if (!ensure_pred_rows(*m, (int)rows_needed, err)) return false;
    for (long long r0 = 0; r0 < in.n; r0 += chunk) {
        const long long left = in.n - r0;
        const int rows = (int)std::min<long long>(chunk, ((left + 127) / 128) * 128);
        ucbmlp::FeatureArgs fa = feature_args(*m, in, r0, rows, false);
        fa.X = m->pX;
        if (!features(*m, fa, st, err) || !forward_infer(*m, rows, st, err)) return false;
        ucbmlp::unscale_kernel<<<(rows + 255) / 256, 256, 0, st>>>(m->pOut, rows, left, m->y_mean, m->y_std,
                                                                   d_mean + r0, d_std + r0);
        m->e->launches += 1;
        if (!cu_ok(cudaPeekAtLastError(), err, "unscale launch")) return false;
    }
    return true;
}

bool mlp_fit(Mlp* m, const MlpInputs& in, const float* d_y, cudaStream_t st, float* loss_out, std::string& err) {
    if (in.n <= 0) {
        err = "no training rows";
        return false;
    }
    // target standardisation from the training targets
    std::vector<float> hy(in.n);
    if (!cu_ok(cudaMemcpyAsync(hy.data(), d_y, in.n * sizeof(float), cudaMemcpyDeviceToHost, st), err, "read y") ||
        !cu_ok(cudaStreamSynchronize(st), err, "read y"))
        return false;
    double s = 0, s2 = 0;
    for (float v : hy) {
        s += v;
        s2 += (double)v * v;
    }
    const double mean = s / in.n;
    const double var = std::max(s2 / in.n - mean * mean, 1e-12);
    m->y_mean = (float)mean;
    m->y_std = (float)std::sqrt(var);
    if (!ensure_rows(*m, m->cfg.batch, err)) return false;
    if (!cu_ok(cudaMemsetAsync(m->step, 0, sizeof(unsigned long long), st), err, "reset step") ||
        !cu_ok(cudaMemsetAsync(m->m1, 0, m->n_params * sizeof(float), st), err, "reset adam") ||
        !cu_ok(cudaMemsetAsync(m->m2, 0, m->n_params * sizeof(float), st), err, "reset adam") ||
        !cu_ok(cudaMemsetAsync(m->err, 0, sizeof(int), st), err, "reset err"))
        return false;
    if (m->cfg.train_steps == 0) return true;
    // The captured step bakes in the inputs and the target scale.
    const bool same = m->graph && m->graph_in.u == in.u && m->graph_in.cells == in.cells && m->graph_in.n == in.n &&
                      m->graph_in.grid_n == in.grid_n && m->graph_y == d_y && m->graph_y_mean == m->y_mean &&
                      m->graph_y_std == m->y_std;
    if (!same) {
        if (m->graph) {
            cudaGraphExecDestroy(m->graph);
            m->graph = nullptr;
        }
        // Capture one step on a private stream (capture does not run the kernels, so the
        // launch counter is restored and advanced per replay instead).
        cudaStream_t cs;
        if (!cu_ok(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), err, "capture stream")) return false;
        const long long l0 = m->e->launches;
        cudaGraph_t g = nullptr;
        bool ok = cu_ok(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), err, "begin capture");
        if (ok) {
            m->pdl = true;
            ok = train_step(*m, in, d_y, cs, err);
            m->pdl = false;
            const cudaError_t ce = cudaStreamEndCapture(cs, &g);
            ok = ok && cu_ok(ce, err, "end capture");
        }
        m->graph_nodes = m->e->launches - l0;
        m->e->launches = l0;
        if (ok) ok = cu_ok(cudaGraphInstantiate(&m->graph, g, 0), err, "graph instantiate");
        if (g) cudaGraphDestroy(g);
        cudaStreamDestroy(cs);
        if (!ok) return false;
        m->graph_in = in;
        m->graph_y = d_y;
        m->graph_y_mean = m->y_mean;
        m->graph_y_std = m->y_std;
    }
    for (int t = 0; t < m->cfg.train_steps; ++t) {
        if (!cu_ok(cudaGraphLaunch(m->graph, st), err, "graph launch")) return false;
    }
    m->e->launches += m->graph_nodes * m->cfg.train_steps;
    if (!check_kernel_error(*m, st, err)) return false;
    if (loss_out && !cu_ok(cudaMemcpy(loss_out, m->loss, sizeof(float), cudaMemcpyDeviceToHost), err, "read loss"))
        return false;
    return true;
}

}  // namespace ucb

// ====================================================================== C ABI
using namespace ucb;

struct ucb_mlp {
    ucb_engine* e;
    Mlp* m;
};

extern "C" {

void ucb_mlp_default_config(ucb_mlp_config* c) {
    std::memset(c, 0, sizeof *c);
    c->fourier = 64;
    c->hidden = 256;
    c->layers = 4;
    c->fourier_scale = 3.0f;
    c->seed = 0;
    c->batch = 8192;
    c->train_steps = 1500;
    c->lr = 2e-3f;
    c->lr_final = 2e-5f;
    c->beta_nll = 0.5f;
}

ucb_mlp* ucb_mlp_create(ucb_engine* e, const ucb_mlp_config* cfg) {
    if (!e || !cfg) return nullptr;
    std::string err;
    cudaSetDevice(e->device);
    Mlp* m = mlp_create(e, *cfg, err);
    if (!m) {
        e->last_error = err;
        return nullptr;
    }
    return new ucb_mlp{e, m};
}

void ucb_mlp_destroy(ucb_mlp* m) {
    if (!m) return;
    cudaSetDevice(m->e->device);
    mlp_destroy(m->m);
    delete m;
}

long long ucb_mlp_param_count(const ucb_mlp* m) { return m ? m->m->n_params : 0; }

int ucb_mlp_get_params(ucb_mlp* m, float* out, long long n) {
    if (!m || !out || n != m->m->n_params) return UCB_E_INVALID;
    cudaSetDevice(m->e->device);
    return cudaMemcpy(out, m->m->p, n * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess ? UCB_OK : UCB_E_CUDA;
}

int ucb_mlp_set_params(ucb_mlp* m, const float* in, long long n) {
    if (!m || !in || n != m->m->n_params) return UCB_E_INVALID;
    cudaSetDevice(m->e->device);
    std::string err;
    if (cudaMemcpy(m->m->p, in, n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) return UCB_E_CUDA;
    if (!refresh(*m->m, m->e->stream, err) || cudaStreamSynchronize(m->e->stream) != cudaSuccess) {
        m->e->last_error = err;
        return UCB_E_CUDA;
    }
    return UCB_OK;
}

int ucb_mlp_get_fourier(ucb_mlp* m, float* out, long long n) {
    if (!m || !out || n != 2LL * m->m->cfg.fourier) return UCB_E_INVALID;
    cudaSetDevice(m->e->device);
    return cudaMemcpy(out, m->m->Bf, n * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess ? UCB_OK : UCB_E_CUDA;
}

int ucb_mlp_set_target_scale(ucb_mlp* m, float mean, float sd) {
    if (!m || !(sd > 0.f)) return UCB_E_INVALID;
    m->m->y_mean = mean;
    m->m->y_std = sd;
    return UCB_OK;
}

int ucb_mlp_loss_grad(ucb_mlp* h, const float* u, const float* y, long long n, float* loss, float* grad) {
    if (!h || !u || !y || !loss || !grad || n <= 0 || n > (1 << 20)) return UCB_E_INVALID;
    cudaSetDevice(h->e->device);
    Mlp& m = *h->m;
    std::string err;
    const int rows = (int)(((n + 127) / 128) * 128);
    float *du = nullptr, *dy = nullptr;
    int rc = UCB_OK;
    cudaStream_t st = h->e->stream;
    if (!ensure_rows(m, rows, err) || !cu_ok(cudaMalloc(&du, n * 2 * sizeof(float)), err, "alloc u") ||
        !cu_ok(cudaMalloc(&dy, n * sizeof(float)), err, "alloc y") ||
        !cu_ok(cudaMemcpy(du, u, n * 2 * sizeof(float), cudaMemcpyHostToDevice), err, "upload u") ||
        !cu_ok(cudaMemcpy(dy, y, n * sizeof(float), cudaMemcpyHostToDevice), err, "upload y") ||
        !cu_ok(cudaMemsetAsync(m.err, 0, sizeof(int), st), err, "reset err")) {
        rc = UCB_E_CUDA;
    } else {
        MlpInputs in;
        in.u = du;
        in.n = n;
        ucbmlp::FeatureArgs fa = feature_args(m, in, 0, rows, false);
        fa.Xt = m.Xt;
        fa.y = dy;
        fa.yb = m.yb;
        if (!features(m, fa, st, err) || !forward(m, rows, true, st, err, (int)n) || !backward(m, rows, st, err) ||
            !adam(m, rows, false, st, err) || !check_kernel_error(m, st, err) ||
            !cu_ok(cudaMemcpy(grad, m.g, m.n_params * sizeof(float), cudaMemcpyDeviceToHost), err, "read grad") ||
            !cu_ok(cudaMemcpy(loss, m.loss, sizeof(float), cudaMemcpyDeviceToHost), err, "read loss"))
            rc = UCB_E_CUDA;
    }
    if (du) cudaFree(du);
    if (dy) cudaFree(dy);
    if (rc != UCB_OK) h->e->last_error = err;
    return rc;
}

int ucb_mlp_fit(ucb_mlp* h, const float* d_u, const float* d_y, long long n, void* stream, float* loss_out) {
    if (!h || !d_u || !d_y || n <= 0) return UCB_E_INVALID;
    cudaSetDevice(h->e->device);
    std::string err;
    MlpInputs in;
    in.u = d_u;
    in.n = n;
    if (!mlp_fit(h->m, in, d_y, stream ? (cudaStream_t)stream : h->e->stream, loss_out, err)) {
        h->e->last_error = err;
        return UCB_E_CUDA;
    }
    return UCB_OK;
}

int ucb_mlp_predict(ucb_mlp* h, const float* d_u, long long n, float* d_mean, float* d_std, void* stream) {
    if (!h || !d_u || !d_mean || !d_std || n < 0) return UCB_E_INVALID;
    cudaSetDevice(h->e->device);
    std::string err;
    MlpInputs in;
    in.u = d_u;
    in.n = n;
    cudaStream_t st = stream ? (cudaStream_t)stream : h->e->stream;
    if (!mlp_predict(h->m, in, d_mean, d_std, st, err) || !check_kernel_error(*h->m, st, err)) {
        h->e->last_error = err;
        return UCB_E_CUDA;
    }
    return UCB_OK;
}

}  // extern "C"
