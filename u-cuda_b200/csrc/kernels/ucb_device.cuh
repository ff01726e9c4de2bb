// ucb_device.cuh — device library shared by every integrator kernel (NVRTC header).
//
// Compiled together with a generated prelude that defines, at compile time:
//   numb          state type (double: plain FP64 form; float: FP32 state form)
//   UCB_NX        number of state variables (AMOUNTOFX of the reference)
//   UCB_NV        number of entries of a[] (base_values, a[0] reserved)
//   UCB_POV       sweep kind: 1 both axes parameters, 0 both initial conditions,
//                 2 axis 0 an initial condition and axis 1 a parameter (par_or_var)
//   UCB_IDX0/1    swept index of axis 0/1 (a[] index for parameters, X[] for states)
//   UCB_HAXIS     axis that sweeps the step h (-1 none)
//   UCB_DIM       1 or 2 sweep axes
// and one stepper:
//   exact form : calculateDiscreteModel(numb* X, const numb* a, numb h) — the KRS body
//                verbatim, as the reference template splices it (lle2d.template.cu:60-63)
//   native form: ucb_rhs(X1, a, dX) (+ ucb_jvp for tangent vectors) — the right-hand side
//                recognised in the KRS body, integrated by the hand-written RK4 below.
#pragma once

#ifdef __CUDACC_RTC__
typedef signed char int8_t;
typedef unsigned char uint8_t;
typedef short int16_t;
typedef unsigned short uint16_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
#endif

#ifndef UCB_DIM
#define UCB_DIM 2
#endif
// 1: every loop call ends with the reference's extra step (cudaLibrary.cu:863-866),
// 0: nominal step counts.
#ifndef UCB_EXTRA_STEP
#define UCB_EXTRA_STEP 1
#endif
// Launch-shape knobs set by the autotuner (or the caller's options): threads per block
// (the kernels' __launch_bounds__) and the number of steps per unrolled chunk of the step
// loops whose trip count is only known at run time.
#ifndef UCB_BLOCK
#define UCB_BLOCK 128
#endif
#ifndef UCB_UNROLL
#define UCB_UNROLL 1
#endif
// A register cap is a residency request: __launch_bounds__(UCB_BLOCK, UCB_MIN_BLOCKS) asks
// for UCB_MIN_BLOCKS resident blocks per SM, which bounds the registers per thread (a
// --maxrregcount option does not apply to kernels that carry launch bounds).
#ifdef UCB_MIN_BLOCKS
#define UCB_LAUNCH_BOUNDS __launch_bounds__(UCB_BLOCK, UCB_MIN_BLOCKS)
#else
#define UCB_LAUNCH_BOUNDS __launch_bounds__(UCB_BLOCK)
#endif
#define UCB_STR_(x) #x
#define UCB_PRAGMA_(x) _Pragma(UCB_STR_(x))
#define UCB_STEP_LOOP UCB_PRAGMA_(unroll UCB_UNROLL)

namespace ucbdev {

// configCUDA.h constants of the reference (CHECK_INTERVAL, eps_fixed_point, ...).
constexpr int kCheckInterval = 100;
constexpr double kEpsFixedPoint = 1e-8;
constexpr double kEpsPeakDelta = 1e-14;
constexpr double kPeakThreshold = -1e25;
constexpr int kMaxAmountOfPeaks = 2500;

// Sum of |x| and the divergence test of loopCalculateDiscreteModel_int
// (cudaLibrary.cu:829-850): NaN/Inf, or above maxValue when maxValue != 0.
__device__ __forceinline__ bool diverged(const numb* x, numb maxValue) {
    numb checker = 0;
#pragma unroll
    for (int j = 0; j < UCB_NX; ++j) checker = checker + fabs(x[j]);
    if (isnan(checker) || isinf(checker)) return true;
    if (maxValue != 0 && fabs(checker) > maxValue) return true;
    return false;
}

__device__ __forceinline__ int fixed_point_flag(const numb* x, const numb* xPrev) {
    numb tempResult = 0;
#pragma unroll
    for (int j = 0; j < UCB_NX; ++j) tempResult += fabs(x[j] - xPrev[j]);
    return (fabs(tempResult) < (numb)kEpsFixedPoint) ? -1 : 1;
}

// RNG stub of the reference templates (lle2d.template.cu:45-56): splitmix64 mixing of
// (seed, subsequence, offset), then one LCG step per uniform in (0, 1].
struct Rng {
    unsigned long long state;
};
__device__ __forceinline__ void rng_init(unsigned long long seed, unsigned long long seq,
                                         unsigned long long off, Rng* s) {
    unsigned long long z = seed + seq * 0x9E3779B97F4A7C15ULL + off;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    s->state = z ^ (z >> 31);
}
__device__ __forceinline__ float rng_uniform(Rng* s) {
    s->state = s->state * 6364136223846793005ULL + 1442695040888963407ULL;
    return (float)(((s->state >> 40) & 0xFFFFFFULL) + 1ULL) / 16777216.0f;
}

// Random unit probe direction of one cell (LLEKernelCUDA, cudaLibrary.cu:2609-2628).
__device__ __forceinline__ void probe_direction(unsigned long long seq, numb* z) {
    Rng st;
    rng_init(1234567891ULL, seq, 0ULL, &st);
    numb zPower = 0;
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) {
        z[i] = rng_uniform(&st) - 0.5;
        zPower += z[i] * z[i];
    }
    zPower = sqrt(zPower);
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) z[i] /= zPower;
}

// ---------------------------------------------------------------------------
// Steppers
// ---------------------------------------------------------------------------
#ifdef UCB_EXACT
// The KRS body verbatim (the reference's calculateDiscreteModel slot).
struct Stepper {
    __device__ __forceinline__ explicit Stepper(numb) {}
    __device__ __forceinline__ void step(numb* x, const numb* a, numb h) const {
        calculateDiscreteModel(x, a, h);
    }
};
#else
#ifdef UCB_TRIG_PHASE
__device__ __forceinline__ void ucb_sincos(double v, double* s, double* c) { sincos(v, s, c); }
__device__ __forceinline__ void ucb_sincos(float v, float* s, float* c) { sincosf(v, s, c); }
#endif

#ifdef UCB_KAHAN_CLOCK
#define UCB_CLOCK_SAVE(x) const numb clock_prev_ = (x)[UCB_CLOCK_VAR]
#define UCB_CLOCK_ADVANCE(x) (x)[UCB_CLOCK_VAR] = clock_next(clock_prev_)
#else
#define UCB_CLOCK_SAVE(x) (void)0
#define UCB_CLOCK_ADVANCE(x) (void)0
#endif

#if defined(UCB_NUMB_F32) && !defined(UCB_SCALAR_STEP)
// FP32 RK4 updates two components per packed instruction (FFMA2 / FADD2, sm_100): every
// component of a stage point or of the final combination uses the same coefficient, and the
// packed forms round each lane as the scalar ones do, so the results are unchanged.
// out[i] = c k[i] + x[i]
__device__ __forceinline__ void rk4_axpy(float c, const float* k, const float* x, float* out) {
    const float2 cc = make_float2(c, c);
#pragma unroll
    for (int i = 0; i + 1 < UCB_NX; i += 2) {
        const float2 t = __ffma2_rn(cc, make_float2(k[i], k[i + 1]), make_float2(x[i], x[i + 1]));
        out[i] = t.x;
        out[i + 1] = t.y;
    }
    if (UCB_NX & 1) out[UCB_NX - 1] = fmaf(c, k[UCB_NX - 1], x[UCB_NX - 1]);
}
// x[i] = h6 ((k1[i] + k4[i]) + 2 (k2[i] + k3[i])) + x[i]
__device__ __forceinline__ void rk4_combine(float h6, const float* k1, const float* k2, const float* k3,
                                            const float* k4, float* x) {
    const float2 c6 = make_float2(h6, h6), two = make_float2(2.0f, 2.0f);
#pragma unroll
    for (int i = 0; i + 1 < UCB_NX; i += 2) {
        const float2 s14 = __fadd2_rn(make_float2(k1[i], k1[i + 1]), make_float2(k4[i], k4[i + 1]));
        const float2 s23 = __fadd2_rn(make_float2(k2[i], k2[i + 1]), make_float2(k3[i], k3[i + 1]));
        const float2 t = __ffma2_rn(c6, __ffma2_rn(two, s23, s14), make_float2(x[i], x[i + 1]));
        x[i] = t.x;
        x[i + 1] = t.y;
    }
    if (UCB_NX & 1) {
        const int i = UCB_NX - 1;
        x[i] = fmaf(h6, (k1[i] + k4[i]) + 2.0f * (k2[i] + k3[i]), x[i]);
    }
}
#define UCB_RK4_AXPY(c, k, x, out) rk4_axpy((c), (k), (x), (out))
#define UCB_RK4_COMBINE(h6, k1, k2, k3, k4, x) rk4_combine((h6), (k1), (k2), (k3), (k4), (x))
#else
#define UCB_RK4_AXPY(c, k, x, out)                                              \
    do {                                                                        \
        _Pragma("unroll") for (int i_ = 0; i_ < UCB_NX; ++i_)(out)[i_] = fma((c), (k)[i_], (x)[i_]); \
    } while (0)
#define UCB_RK4_COMBINE(h6, k1, k2, k3, k4, x)                                                     \
    do {                                                                                           \
        _Pragma("unroll") for (int i_ = 0; i_ < UCB_NX; ++i_)(x)[i_] =                             \
            fma((h6), ((k1)[i_] + (k4)[i_]) + (numb)2 * ((k2)[i_] + (k3)[i_]), (x)[i_]);          \
    } while (0)
#endif

// Classical RK4 on ucb_rhs, FMA-ordered: the same scheme as codegen.cpp scheme_rk4
// (k1..k4 at t, t+h/2, t+h/2, t+h; x += h/6 (k1 + 2k2 + 2k3 + k4)) with the half/sixth
// step factors hoisted and every update written as a fused multiply-add.
// With a forcing phase p (dX[p]/dt = UCB_TRIG_RATE, sin / cos of X[p] in the system) a step
// takes one sincos of X[p] and rotates it by the constant stage offsets rate h/2 and rate h
// for the other stages, instead of evaluating the forcing at every stage.
struct Stepper {
    numb hh, h6;
#ifdef UCB_TRIG_PHASE
    numb ch, sh, cf, sf;  // cos / sin of rate h/2 and of rate h
#endif
#ifdef UCB_KAHAN_CLOCK
    // Compensated clock (FP32 builds with a variable of constant derivative, one trajectory
    // per Stepper): X[UCB_CLOCK_VAR] gains h * rate per step, and a plain FP32 add loses up
    // to half an ulp of the growing clock every step — at t ~ 1e4 with h = 2 pi / 200 a
    // forcing phase falls about 30 rad behind in 3.5e5 steps, i.e. the forcing runs at the
    // wrong frequency. Kahan summation carries the rounding error in kc (the stored clock
    // exceeds the exact sum by kc), so the clock stays within an ulp of x0 + n h rate.
    numb hr;
    mutable numb kc;
#endif
    __device__ __forceinline__ explicit Stepper(numb h) : hh(h * (numb)0.5), h6(h * (numb)(1.0 / 6.0)) {
#ifdef UCB_TRIG_PHASE
        ucb_sincos((numb)((numb)UCB_TRIG_RATE * hh), &sh, &ch);
        ucb_sincos((numb)((numb)UCB_TRIG_RATE * h), &sf, &cf);
#endif
#ifdef UCB_KAHAN_CLOCK
        hr = h * (numb)UCB_CLOCK_RATE;
        kc = (numb)0;
#endif
    }
#ifdef UCB_KAHAN_CLOCK
    // The clock after one step from xc (Kahan's compensated sum).
    __device__ __forceinline__ numb clock_next(numb xc) const {
        const numb y = hr - kc;
        const numb t = xc + y;
        kc = (t - xc) - y;
        return t;
    }
#endif
    __device__ __forceinline__ void step(numb* x, const numb* a, numb h) const {
#ifdef UCB_TRIG_PHASE
        numb s0, c0;
        ucb_sincos(x[UCB_TRIG_PHASE], &s0, &c0);
#if defined(UCB_KAHAN_CLOCK) && UCB_CLOCK_VAR == UCB_TRIG_PHASE
        {  // the forcing at the compensated phase x - kc (first order in kc <= half an ulp)
            const numb cc = fma(kc, s0, c0);
            s0 = fma(-kc, c0, s0);
            c0 = cc;
        }
#endif
        const numb tc[6] = {c0, s0, fma(c0, ch, -s0 * sh), fma(s0, ch, c0 * sh), fma(c0, cf, -s0 * sf),
                            fma(s0, cf, c0 * sf)};
        step_trig(x, a, h, tc);
#else
        numb k1[UCB_NX], k2[UCB_NX], k3[UCB_NX], k4[UCB_NX], xt[UCB_NX];
        ucb_rhs(x, a, k1);
        UCB_RK4_AXPY(hh, k1, x, xt);
        ucb_rhs(xt, a, k2);
        UCB_RK4_AXPY(hh, k2, x, xt);
        ucb_rhs(xt, a, k3);
        UCB_RK4_AXPY(h, k3, x, xt);
        ucb_rhs(xt, a, k4);
        UCB_CLOCK_SAVE(x);
        UCB_RK4_COMBINE(h6, k1, k2, k3, k4, x);
        UCB_CLOCK_ADVANCE(x);
#endif
    }
#ifdef UCB_TRIG_PHASE
    // The same step with the forcing's (cos, sin) at the three stage phases t, t + h/2 and
    // t + h given by the caller: tc[0..1], tc[2..3], tc[4..5].
    __device__ __forceinline__ void step_trig(numb* x, const numb* a, numb h, const numb* tc) const {
        numb k1[UCB_NX], k2[UCB_NX], k3[UCB_NX], k4[UCB_NX], xt[UCB_NX];
        const numb c0 = tc[0], s0 = tc[1], c1 = tc[2], s1 = tc[3], c2 = tc[4], s2 = tc[5];
        ucb_rhs_trig(x, a, k1, c0, s0);
        UCB_RK4_AXPY(hh, k1, x, xt);
        ucb_rhs_trig(xt, a, k2, c1, s1);
        UCB_RK4_AXPY(hh, k2, x, xt);
        ucb_rhs_trig(xt, a, k3, c1, s1);
        UCB_RK4_AXPY(h, k3, x, xt);
        ucb_rhs_trig(xt, a, k4, c2, s2);
        UCB_CLOCK_SAVE(x);
        UCB_RK4_COMBINE(h6, k1, k2, k3, k4, x);
        UCB_CLOCK_ADVANCE(x);
    }
#endif
#ifdef UCB_HAS_JVP
#if defined(UCB_NUMB_F32) && !defined(UCB_TRIG_PHASE) && !defined(UCB_KAHAN_CLOCK)
    // RK4 of the tangent-linear system (x' = f(x), v' = J(x) v) in one sweep, FP32: the
    // stage points and the final combination of x_i and v_i share their coefficients, so
    // each pair (x_i, v_i) is updated by one packed FFMA2 / FADD2 (sm_100) — the same
    // per-lane roundings as the scalar form, half the issue slots of those updates.
    __device__ __forceinline__ void step_tangent(numb* x, numb* v, const numb* a, numb h) const {
        const float2 c_hh = make_float2(hh, hh), c_h = make_float2(h, h), c_h6 = make_float2(h6, h6);
        const float2 two = make_float2(2.0f, 2.0f);
        numb k[UCB_NX], l[UCB_NX], xt[UCB_NX], vt[UCB_NX];
        float2 p1[UCB_NX], p2[UCB_NX], p3[UCB_NX], p4[UCB_NX], t;
        ucb_rhs(x, a, k);
        ucb_jvp(x, a, v, l);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) {
            p1[i] = make_float2(k[i], l[i]);
            t = __ffma2_rn(c_hh, p1[i], make_float2(x[i], v[i]));
            xt[i] = t.x;
            vt[i] = t.y;
        }
        ucb_rhs(xt, a, k);
        ucb_jvp(xt, a, vt, l);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) {
            p2[i] = make_float2(k[i], l[i]);
            t = __ffma2_rn(c_hh, p2[i], make_float2(x[i], v[i]));
            xt[i] = t.x;
            vt[i] = t.y;
        }
        ucb_rhs(xt, a, k);
        ucb_jvp(xt, a, vt, l);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) {
            p3[i] = make_float2(k[i], l[i]);
            t = __ffma2_rn(c_h, p3[i], make_float2(x[i], v[i]));
            xt[i] = t.x;
            vt[i] = t.y;
        }
        ucb_rhs(xt, a, k);
        ucb_jvp(xt, a, vt, l);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) {
            p4[i] = make_float2(k[i], l[i]);
            // (k1 + k4) + 2 (k2 + k3), then x + h/6 (...)
            t = __ffma2_rn(c_h6, __ffma2_rn(two, __fadd2_rn(p2[i], p3[i]), __fadd2_rn(p1[i], p4[i])),
                           make_float2(x[i], v[i]));
            x[i] = t.x;
            v[i] = t.y;
        }
    }
#else
    // RK4 of the tangent-linear system (x' = f(x), v' = J(x) v) in one sweep.
    __device__ __forceinline__ void step_tangent(numb* x, numb* v, const numb* a, numb h) const {
        numb k1[UCB_NX], k2[UCB_NX], k3[UCB_NX], k4[UCB_NX], xt[UCB_NX];
        numb l1[UCB_NX], l2[UCB_NX], l3[UCB_NX], l4[UCB_NX], vt[UCB_NX];
        ucb_rhs(x, a, k1);
        ucb_jvp(x, a, v, l1);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) { xt[i] = fma(hh, k1[i], x[i]); vt[i] = fma(hh, l1[i], v[i]); }
        ucb_rhs(xt, a, k2);
        ucb_jvp(xt, a, vt, l2);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) { xt[i] = fma(hh, k2[i], x[i]); vt[i] = fma(hh, l2[i], v[i]); }
        ucb_rhs(xt, a, k3);
        ucb_jvp(xt, a, vt, l3);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) { xt[i] = fma(h, k3[i], x[i]); vt[i] = fma(h, l3[i], v[i]); }
        ucb_rhs(xt, a, k4);
        ucb_jvp(xt, a, vt, l4);
        UCB_CLOCK_SAVE(x);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) {
            x[i] = fma(h6, (k1[i] + k4[i]) + (numb)2 * (k2[i] + k3[i]), x[i]);
            v[i] = fma(h6, (l1[i] + l4[i]) + (numb)2 * (l2[i] + l3[i]), v[i]);
        }
        UCB_CLOCK_ADVANCE(x);  // (the tangent's clock component has derivative 0)
    }
#endif
#endif
};

#if defined(UCB_PACKED_CODE)
// Two cells per thread in packed FP32 pairs (.x one cell, .y the other): the same FMA-
// ordered RK4 as Stepper with every add / multiply / fused multiply-add issued as one
// FADD2 / FMUL2 / FFMA2 for both cells (sm_100), half the instructions per cell-step.
struct Stepper2 {
    float2 hh, h6, hf;
    __device__ __forceinline__ explicit Stepper2(float h)
        : hh(ucb_p2(h * 0.5f)), h6(ucb_p2(h * (float)(1.0 / 6.0))), hf(ucb_p2(h)) {}
    __device__ __forceinline__ static float2 comb(float2 k1, float2 k2, float2 k3, float2 k4) {
        // (k1 + k4) + 2 (k2 + k3)
        return __ffma2_rn(ucb_p2(2.0f), __fadd2_rn(k2, k3), __fadd2_rn(k1, k4));
    }
    __device__ __forceinline__ void step(float2* x, const float2* a) const {
        float2 k1[UCB_NX], k2[UCB_NX], k3[UCB_NX], k4[UCB_NX], xt[UCB_NX];
        ucb_rhs2(x, a, k1);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) xt[i] = __ffma2_rn(hh, k1[i], x[i]);
        ucb_rhs2(xt, a, k2);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) xt[i] = __ffma2_rn(hh, k2[i], x[i]);
        ucb_rhs2(xt, a, k3);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) xt[i] = __ffma2_rn(hf, k3[i], x[i]);
        ucb_rhs2(xt, a, k4);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) x[i] = __ffma2_rn(h6, comb(k1[i], k2[i], k3[i], k4[i]), x[i]);
    }
    __device__ __forceinline__ void step_tangent(float2* x, float2* v, const float2* a) const {
        float2 k1[UCB_NX], k2[UCB_NX], k3[UCB_NX], k4[UCB_NX], xt[UCB_NX];
        float2 l1[UCB_NX], l2[UCB_NX], l3[UCB_NX], l4[UCB_NX], vt[UCB_NX];
        ucb_rhs2(x, a, k1);
        ucb_jvp2(x, a, v, l1);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) {
            xt[i] = __ffma2_rn(hh, k1[i], x[i]);
            vt[i] = __ffma2_rn(hh, l1[i], v[i]);
        }
        ucb_rhs2(xt, a, k2);
        ucb_jvp2(xt, a, vt, l2);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) {
            xt[i] = __ffma2_rn(hh, k2[i], x[i]);
            vt[i] = __ffma2_rn(hh, l2[i], v[i]);
        }
        ucb_rhs2(xt, a, k3);
        ucb_jvp2(xt, a, vt, l3);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) {
            xt[i] = __ffma2_rn(hf, k3[i], x[i]);
            vt[i] = __ffma2_rn(hf, l3[i], v[i]);
        }
        ucb_rhs2(xt, a, k4);
        ucb_jvp2(xt, a, vt, l4);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) {
            x[i] = __ffma2_rn(h6, comb(k1[i], k2[i], k3[i], k4[i]), x[i]);
            v[i] = __ffma2_rn(h6, comb(l1[i], l2[i], l3[i], l4[i]), v[i]);
        }
    }
};

// The divergence test of one cell of a pair (diverged(), component c of each entry).
__device__ __forceinline__ bool diverged2(const float2* x, float maxValue, int c) {
    float checker = 0;
#pragma unroll
    for (int j = 0; j < UCB_NX; ++j) checker = checker + fabsf(c ? x[j].y : x[j].x);
    if (isnan(checker) || isinf(checker)) return true;
    if (maxValue != 0 && fabsf(checker) > maxValue) return true;
    return false;
}
#endif
#endif

// ---------------------------------------------------------------------------
// loopCalculateDiscreteModel_int (cudaLibrary.cu:782-895) without recording:
// `iters` steps, the divergence test after iterations 0, 100, 200, ... of this call,
// then one extra step and the fixed-point test. 1 ok / -1 fixed point / 0 diverged.
// ---------------------------------------------------------------------------
template <class S>
__device__ __forceinline__ int loop_single(const S& s, numb* x, const numb* a, numb h, long long iters,
                                           numb maxValue, long long& ns) {
    for (long long i0 = 0; i0 < iters; i0 += kCheckInterval) {
        s.step(x, a, h);
        ns += 1;
        if (diverged(x, maxValue)) return 0;
        const int n = (iters - i0 < kCheckInterval) ? (int)(iters - i0) : kCheckInterval;
        UCB_STEP_LOOP
        for (int i = 1; i < n; ++i) s.step(x, a, h);
        ns += n - 1;
    }
#if UCB_EXTRA_STEP
    numb xPrev[UCB_NX];
#pragma unroll
    for (int j = 0; j < UCB_NX; ++j) xPrev[j] = x[j];
    s.step(x, a, h);
    ns += 1;
    return fixed_point_flag(x, xPrev);
#else
    return 1;
#endif
}

// Two independent trajectories advanced together (the trajectory and its shadow in
// LLEKernelCUDA, :2646-2658). The reference runs them one after the other; advancing
// them in lock step gives the same numbers (they never interact inside a block) and
// two independent dependency chains per thread. Returns 0 if either diverged.
template <class S>
__device__ __forceinline__ int loop_pair(const S& s, numb* x, numb* y, const numb* a, numb h,
                                         long long iters, numb maxValue, long long& ns) {
    for (long long i0 = 0; i0 < iters; i0 += kCheckInterval) {
        s.step(x, a, h);
        s.step(y, a, h);
        ns += 2;
        if (diverged(x, maxValue) || diverged(y, maxValue)) return 0;
        const int n = (iters - i0 < kCheckInterval) ? (int)(iters - i0) : kCheckInterval;
        UCB_STEP_LOOP
        for (int i = 1; i < n; ++i) {
            s.step(x, a, h);
            s.step(y, a, h);
        }
        ns += 2 * (n - 1);
    }
#if UCB_EXTRA_STEP
    s.step(x, a, h);
    s.step(y, a, h);
    ns += 2;
#endif
    return 1;
}

#ifdef UCB_NT
// loop_pair for a block length known at compile time (UCB_NT <= kCheckInterval steps):
// the same sequence — first step of both, divergence test, the remaining UCB_NT - 1
// steps, the extra step — fully unrolled, without loop control.
template <class S>
__device__ __forceinline__ int loop_pair_nt(const S& s, numb* x, numb* y, const numb* a, numb h, numb maxValue,
                                            long long& ns) {
    s.step(x, a, h);
    s.step(y, a, h);
    if (diverged(x, maxValue) || diverged(y, maxValue)) {
        ns += 2;
        return 0;
    }
#pragma unroll
    for (int i = 1; i < UCB_NT; ++i) {
        s.step(x, a, h);
        s.step(y, a, h);
    }
#if UCB_EXTRA_STEP
    s.step(x, a, h);
    s.step(y, a, h);
    ns += 2 * (UCB_NT + 1);
#else
    ns += 2 * UCB_NT;
#endif
    return 1;
}
#endif

// Running product of positive factors as mantissa x 2^exponent (FP64): a sum of logs
// taken with one log at the end instead of one per block.
struct LogProduct {
    double m;
    long long e;
    __device__ __forceinline__ LogProduct() : m(1.0), e(0) {}
    __device__ __forceinline__ void mul(double f) {
        int k;
        m = frexp(m * f, &k);
        e += k;
    }
    __device__ __forceinline__ double log_value() const { return log(m) + (double)e * 0.69314718055994530942; }
};

// ---------------------------------------------------------------------------
// Cell set-up: sweep values of one cell (the par_or_var branches of LLEKernelCUDA
// :2565-2588 / calculateDiscreteModelCUDA :1035-1058). Axis values come from host
// tables computed with the reference's getValueByIdx(_log) formula in numb.
// ---------------------------------------------------------------------------
struct CellAxes {
    int i0, i1;
};

__device__ __forceinline__ CellAxes cell_axes(long long idx, int n) {
    CellAxes c;
    c.i0 = (int)(idx % n);
#if UCB_DIM == 2
    c.i1 = (int)((idx / n) % n);
#else
    c.i1 = 0;
#endif
    return c;
}

__device__ __forceinline__ void apply_sweep(const CellAxes& c, const numb* ax0, const numb* ax1, numb* x,
                                            numb* a) {
#if UCB_POV == 1
#if UCB_HAXIS != 0
    a[UCB_IDX0] = ax0[c.i0];
#endif
#if UCB_DIM == 2 && UCB_HAXIS != 1
    a[UCB_IDX1] = ax1[c.i1];
#endif
#elif UCB_POV == 0
#if UCB_HAXIS != 0
    x[UCB_IDX0] = ax0[c.i0];
#endif
#if UCB_DIM == 2 && UCB_HAXIS != 1
    x[UCB_IDX1] = ax1[c.i1];
#endif
#elif UCB_POV == 2
    x[UCB_IDX0] = ax0[c.i0];
    a[UCB_IDX1] = ax1[c.i1];
#endif
}

// Adds the per-thread work counts of a warp into a global counter (one atomic per warp).
__device__ __forceinline__ void warp_add_steps(unsigned long long* counter, long long ns, int lane) {
    unsigned long long v = (unsigned long long)ns;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0 && counter) atomicAdd(counter, v);
}

// Run control shared with the host: a block of page-locked host memory mapped into the
// device's address space, one per engine, whose address the engine writes into this
// module's `ucb_control` after loading it (null: no control). The host sets `cancel`
// while it waits for a run whose caller cancelled it; `fetched` receives the queue
// position of the latest fetch (the host reads it as progress).
struct UcbControl {
    int cancel;
    int pad;
    unsigned long long fetched;
};

}  // namespace ucbdev

extern "C" __device__ ucbdev::UcbControl* ucb_control = nullptr;

namespace ucbdev {

// True once the host asked the running call to stop (a warp then takes no more work).
__device__ __forceinline__ bool run_cancelled() {
    const UcbControl* c = ucb_control;
    return c && *(const volatile int*)&c->cancel != 0;
}

// Work distribution: one warp takes `batch` consecutive cells per atomic fetch from a
// device counter, so cells of uneven cost (divergence, early exit) balance across a
// persistent grid. The counter is zeroed by the host before each launch. A cancelled
// run hands out no more work (the returned position is past every grid).
__device__ __forceinline__ long long warp_fetch(unsigned long long* counter, int lane,
                                                unsigned long long batch = 32ULL) {
    unsigned long long base = 0;
    if (lane == 0) {
        UcbControl* c = ucb_control;
        if (c && *(volatile int*)&c->cancel) {
            base = 0x7fffffffffffffffULL;
        } else {
            base = atomicAdd(counter, batch);
            if (c) *(volatile unsigned long long*)&c->fetched = base + batch;
        }
    }
    base = __shfl_sync(0xffffffffu, base, 0);
    return (long long)base;
}

}  // namespace ucbdev
