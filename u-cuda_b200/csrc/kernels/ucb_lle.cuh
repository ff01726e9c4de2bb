// ucb_lle.cuh — largest Lyapunov exponent maps (NVRTC header, after ucb_device.cuh).
//
// One thread per cell, state and shadow (or tangent vector) in registers, persistent
// grid fed by a warp-granular atomic work counter. Semantics per cell follow
// LLEKernelCUDA (cudaLibrary.cu:2486-2693):
//   transient (skip steps, 999 on divergence) -> random unit probe z (RNG subsequence
//   = cell index) -> shadow y = x + eps z -> n_blocks x { advance x and y by nt_steps,
//   d = |(1/eps)(x - y)|, floor 1e-14, sum += log d, y = x - (x - y + 1e-14)/d }
//   -> lambda = sum / tMax.
// Output: values[out] (double) and flags[out] = -1 for the 999 sentinel, 1 otherwise,
// where out is the cell index in the user's row-major order (swap_xy transposes, as
// run_lle_2d does on the host, parametric_engine.cpp:2913-2928).
#pragma once

struct UcbLleParams {
    long long total;          // cells in this launch
    long long cell_offset;    // first cell index (kernel order)
    int n_pts;                // grid side
    int swap_xy;              // 1: write transposed (user X = kernel axis 1)
    int n_blocks;             // (int)(tMax / NT), host double arithmetic
    int pad0;
    long long skip;           // (int)(transientTime / h), host double arithmetic
    long long nt_steps;       // (size_t)(NT / h): numb (exact form) or double (native form)
    numb h, NT, tmax, eps, maxv, transient;
    numb ic[UCB_NX];
    numb vals[UCB_NV];
    const numb* axis0;        // n_pts values of kernel axis 0
    const numb* axis1;        // n_pts values of kernel axis 1
    double* out_values;
    int* out_flags;
    unsigned long long* counter;   // work counter, zeroed before launch
    unsigned long long* steps;     // step evaluations performed (accumulated)
    const long long* cell_list;    // optional: kernel cell indices to compute (total entries)
    int list_compact;              // with cell_list: entry i is stored at i instead of its cell
};

namespace ucbdev {

__device__ __forceinline__ void store_cell(const UcbLleParams& p, long long i, long long kidx, double v) {
    long long out = kidx;
    if (p.cell_list && p.list_compact) {
        out = i;
    } else if (p.swap_xy) {
        const long long kix = kidx % p.n_pts, kiy = kidx / p.n_pts;
        out = kix * p.n_pts + kiy;
    }
    p.out_values[out] = v;
    p.out_flags[out] = (v == 999.0 || v == -999.0) ? -1 : 1;
}

// Per-cell step size and step counts (dt-sweep axis: LLEKernelCUDA :2525-2548).
struct CellSteps {
    numb h;
    long long nt, skip;
};

__device__ __forceinline__ CellSteps cell_steps(const UcbLleParams& p, const CellAxes& c) {
    CellSteps s;
    s.h = p.h;
    s.nt = p.nt_steps;
    s.skip = p.skip;
#if UCB_HAXIS == 0
    s.h = p.axis0[c.i0];
#elif UCB_HAXIS == 1
    s.h = p.axis1[c.i1];
#endif
#if UCB_HAXIS != -1
    s.nt = (long long)ceil(p.NT / s.h);
    s.skip = (long long)ceil(p.transient / s.h);
#endif
    return s;
}

__device__ __forceinline__ double lle_cell_shadow(const UcbLleParams& p, long long kidx, long long& ns) {
    const CellAxes c = cell_axes(kidx, p.n_pts);
    const CellSteps cs = cell_steps(p, c);
    if (!(cs.h > 0)) return (double)nan("");
    numb x[UCB_NX], y[UCB_NX], a[UCB_NV];
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) x[i] = p.ic[i];
#pragma unroll
    for (int i = 0; i < UCB_NV; ++i) a[i] = p.vals[i];
    apply_sweep(c, p.axis0, p.axis1, x, a);
    const Stepper st(cs.h);
    if (loop_single(st, x, a, cs.h, cs.skip, p.maxv, ns) == 0) return 999.0;
    numb z[UCB_NX];
    probe_direction((unsigned long long)kidx, z);
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) y[i] = z[i] * p.eps + x[i];
    const numb inv_eps = (numb)1.0 / p.eps;
#ifdef UCB_EXACT
    numb result = 0;  // the reference's numb sum of per-block logs
#else
    LogProduct prod;  // same sum, one log at the end
#endif
    for (int b = 0; b < p.n_blocks; ++b) {
#if defined(UCB_NT) && UCB_HAXIS == -1
        if (loop_pair_nt(st, x, y, a, cs.h, p.maxv, ns) == 0) return 999.0;
#else
        if (loop_pair(st, x, y, a, cs.h, cs.nt, p.maxv, ns) == 0) return 999.0;
#endif
        numb tempData = 0;
#pragma unroll
        for (int l = 0; l < UCB_NX; ++l) {
            const numb t = inv_eps * (x[l] - y[l]);
            tempData += t * t;
        }
        tempData = sqrt(tempData);
        if (tempData <= 1e-14) tempData = (numb)1e-14;
#ifdef UCB_EXACT
        result += log(tempData);
#else
        prod.mul((double)tempData);
#endif
        tempData = (1 / tempData);
#pragma unroll
        for (int j = 0; j < UCB_NX; ++j) y[j] = (numb)(x[j] - ((x[j] - y[j] + 1e-14) * tempData));
    }
#ifdef UCB_EXACT
    return (double)(result / p.tmax);
#else
    return prod.log_value() / (double)p.tmax;
#endif
}

#if defined(UCB_HAS_JVP) && !defined(UCB_EXACT)
// Tangent-vector form: the shadow trajectory is replaced by the tangent-linear
// vector v (v' = J(x) v, same RK4 sweep as x, same step counts including the extra
// step), started from the same random unit direction. Norms and the log sum are
// accumulated in FP64, so the state can be FP32 without the cancellation that an
// FP32 shadow difference x - y of size eps would suffer.
template <class S>
__device__ __forceinline__ int loop_tangent(const S& s, numb* x, numb* v, const numb* a, numb h,
                                            long long iters, numb maxValue, long long& ns) {
#if defined(UCB_NT) && UCB_HAXIS == -1
    (void)iters;
    s.step_tangent(x, v, a, h);
    ns += 2;
    if (diverged(x, maxValue) || diverged(v, (numb)0)) return 0;
#pragma unroll
    for (int i = 1; i < UCB_NT; ++i) s.step_tangent(x, v, a, h);
    ns += 2 * (UCB_NT - 1);
#else
    for (long long i0 = 0; i0 < iters; i0 += kCheckInterval) {
        s.step_tangent(x, v, a, h);
        ns += 2;
        if (diverged(x, maxValue) || diverged(v, (numb)0)) return 0;
        const int n = (iters - i0 < kCheckInterval) ? (int)(iters - i0) : kCheckInterval;
        UCB_STEP_LOOP
        for (int i = 1; i < n; ++i) s.step_tangent(x, v, a, h);
        ns += 2 * (n - 1);
    }
#endif
#if UCB_EXTRA_STEP
    s.step_tangent(x, v, a, h);
    ns += 2;
#endif
    return 1;
}

__device__ __forceinline__ double lle_cell_tangent(const UcbLleParams& p, long long kidx, long long& ns) {
    const CellAxes c = cell_axes(kidx, p.n_pts);
    const CellSteps cs = cell_steps(p, c);
    if (!(cs.h > 0)) return (double)nan("");
    numb x[UCB_NX], v[UCB_NX], a[UCB_NV];
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) x[i] = p.ic[i];
#pragma unroll
    for (int i = 0; i < UCB_NV; ++i) a[i] = p.vals[i];
    apply_sweep(c, p.axis0, p.axis1, x, a);
    const Stepper st(cs.h);
    if (loop_single(st, x, a, cs.h, cs.skip, p.maxv, ns) == 0) return 999.0;
    probe_direction((unsigned long long)kidx, v);
    // lambda = sum_b log(|v_b,end| / |v_b,start|) / tMax. The rescale between blocks is an
    // FP32 reciprocal square root, so |v_b,start| is 1 only to FP32 rounding; both norms
    // are accumulated exactly as FP64 products of squares (one log each at the end).
    LogProduct end2, start2;
    double n2 = 0.0;
#pragma unroll
    for (int j = 0; j < UCB_NX; ++j) n2 = fma((double)v[j], (double)v[j], n2);
    for (int b = 0; b < p.n_blocks; ++b) {
        start2.mul(n2);
        if (loop_tangent(st, x, v, a, cs.h, cs.nt, p.maxv, ns) == 0) return 999.0;
        double d2 = 0.0;
#pragma unroll
        for (int l = 0; l < UCB_NX; ++l) d2 = fma((double)v[l], (double)v[l], d2);
        if (d2 < 1e-28) {  // the reference's floor of the norm at 1e-14
            d2 = 1e-28;
            if (!(fabs((double)v[0]) > 0)) v[0] = (numb)1e-14;
        }
        end2.mul(d2);
        const numb inv = (numb)rsqrt(d2);
        n2 = 0.0;
#pragma unroll
        for (int j = 0; j < UCB_NX; ++j) {
            v[j] *= inv;
            n2 = fma((double)v[j], (double)v[j], n2);
        }
    }
    return 0.5 * (end2.log_value() - start2.log_value()) / (double)p.tmax;
}
#endif

#if defined(UCB_TANGENT) && defined(UCB_PACKED) && defined(UCB_PACKED_CODE) && defined(UCB_NT) && \
    UCB_HAXIS == -1 && !defined(UCB_EXACT)
// lle_cell_tangent for two cells at once (FP32 state and tangent in float2 pairs; per-cell
// divergence tests, norms, FP64 log products and rescaling as in lle_cell_tangent). A cell
// that diverges keeps being stepped with its pair (its lanes of the packed operations are
// independent of the other cell's) but counts no further steps and stores 999.
__device__ __forceinline__ void lle_pair_tangent(const UcbLleParams& p, long long k0, long long k1, bool two,
                                                 double* out, long long& ns) {
    const float h = p.h;
    float2 x[UCB_NX], v[UCB_NX], a[UCB_NV];
    {
        numb xa[UCB_NX], aa[UCB_NV], xb[UCB_NX], ab[UCB_NV];
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) xa[i] = xb[i] = p.ic[i];
#pragma unroll
        for (int i = 0; i < UCB_NV; ++i) aa[i] = ab[i] = p.vals[i];
        apply_sweep(cell_axes(k0, p.n_pts), p.axis0, p.axis1, xa, aa);
        apply_sweep(cell_axes(two ? k1 : k0, p.n_pts), p.axis0, p.axis1, xb, ab);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) x[i] = make_float2(xa[i], xb[i]);
#pragma unroll
        for (int i = 0; i < UCB_NV; ++i) a[i] = make_float2(aa[i], ab[i]);
    }
    out[0] = out[1] = 999.0;
    bool live[2] = {true, two};
    const int n_live = two ? 2 : 1;
    const Stepper2 st(h);
    // transient (loop_single: a divergence test after steps 1, 101, 201, ..., the extra step)
    for (long long i0 = 0; i0 < p.skip; i0 += kCheckInterval) {
        st.step(x, a);
        ns += (live[0] ? 1 : 0) + (live[1] ? 1 : 0);
#pragma unroll
        for (int c = 0; c < 2; ++c)
            if (live[c] && diverged2(x, p.maxv, c)) live[c] = false;
        if (!live[0] && !live[1]) return;
        const int n = (p.skip - i0 < kCheckInterval) ? (int)(p.skip - i0) : kCheckInterval;
        UCB_STEP_LOOP
        for (int i = 1; i < n; ++i) st.step(x, a);
        ns += (long long)(n - 1) * ((live[0] ? 1 : 0) + (live[1] ? 1 : 0));
    }
#if UCB_EXTRA_STEP
    st.step(x, a);
    ns += (live[0] ? 1 : 0) + (live[1] ? 1 : 0);
#endif
    (void)n_live;
    {
        numb za[UCB_NX], zb[UCB_NX];
        probe_direction((unsigned long long)k0, za);
        probe_direction((unsigned long long)(two ? k1 : k0), zb);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) v[i] = make_float2(za[i], zb[i]);
    }
    LogProduct end2[2], start2[2];
    double n2[2] = {0.0, 0.0};
#pragma unroll
    for (int j = 0; j < UCB_NX; ++j) {
        n2[0] = fma((double)v[j].x, (double)v[j].x, n2[0]);
        n2[1] = fma((double)v[j].y, (double)v[j].y, n2[1]);
    }
    for (int b = 0; b < p.n_blocks; ++b) {
#pragma unroll
        for (int c = 0; c < 2; ++c)
            if (live[c]) start2[c].mul(n2[c]);
        // loop_tangent with the compile-time block length: first step, divergence test,
        // the remaining UCB_NT - 1 steps, the extra step
        st.step_tangent(x, v, a);
        int now = (live[0] ? 1 : 0) + (live[1] ? 1 : 0);
        ns += 2 * now;
#pragma unroll
        for (int c = 0; c < 2; ++c)
            if (live[c] && (diverged2(x, p.maxv, c) || diverged2(v, 0.0f, c))) live[c] = false;
        if (!live[0] && !live[1]) return;
        now = (live[0] ? 1 : 0) + (live[1] ? 1 : 0);
#pragma unroll
        for (int i = 1; i < UCB_NT; ++i) st.step_tangent(x, v, a);
        ns += 2 * (UCB_NT - 1) * now;
#if UCB_EXTRA_STEP
        st.step_tangent(x, v, a);
        ns += 2 * now;
#endif
        double d2[2] = {0.0, 0.0};
#pragma unroll
        for (int l = 0; l < UCB_NX; ++l) {
            d2[0] = fma((double)v[l].x, (double)v[l].x, d2[0]);
            d2[1] = fma((double)v[l].y, (double)v[l].y, d2[1]);
        }
        float inv[2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (d2[c] < 1e-28) {  // the reference's floor of the norm at 1e-14
                d2[c] = 1e-28;
                const float v0 = c ? v[0].y : v[0].x;
                if (!(fabsf(v0) > 0)) {
                    if (c) v[0].y = 1e-14f;
                    else v[0].x = 1e-14f;
                }
            }
            if (live[c]) end2[c].mul(d2[c]);
            inv[c] = (float)rsqrt(d2[c]);
        }
        n2[0] = n2[1] = 0.0;
        const float2 iv = make_float2(inv[0], inv[1]);
#pragma unroll
        for (int j = 0; j < UCB_NX; ++j) {
            v[j] = __fmul2_rn(v[j], iv);
            n2[0] = fma((double)v[j].x, (double)v[j].x, n2[0]);
            n2[1] = fma((double)v[j].y, (double)v[j].y, n2[1]);
        }
    }
#pragma unroll
    for (int c = 0; c < 2; ++c)
        if (live[c]) out[c] = 0.5 * (end2[c].log_value() - start2[c].log_value()) / (double)p.tmax;
}
#define UCB_LLE_PAIRED 1
#endif

}  // namespace ucbdev

extern "C" __global__ void UCB_LAUNCH_BOUNDS ucb_lle_kernel(const UcbLleParams p) {
    const int lane = threadIdx.x & 31;
    long long ns = 0;
#if defined(UCB_LLE_PAIRED)
    // 64 cells per warp fetch: lane l takes cells base + l and base + 32 + l (both halves
    // of a warp's stores stay coalesced)
    for (;;) {
        const long long base = ucbdev::warp_fetch(p.counter, lane, 64ULL);
        if (base >= p.total) break;
        const long long i0 = base + lane, i1 = base + 32 + lane;
        if (i0 < p.total) {
            const bool two = i1 < p.total;
            const long long k0 = p.cell_list ? p.cell_list[i0] : p.cell_offset + i0;
            const long long k1 = two ? (p.cell_list ? p.cell_list[i1] : p.cell_offset + i1) : k0;
            double v[2];
            ucbdev::lle_pair_tangent(p, k0, k1, two, v, ns);
            ucbdev::store_cell(p, i0, k0, v[0]);
            if (two) ucbdev::store_cell(p, i1, k1, v[1]);
        }
    }
    ucbdev::warp_add_steps(p.steps, ns, lane);
    return;
#endif
    for (;;) {
        const long long base = ucbdev::warp_fetch(p.counter, lane);
        if (base >= p.total) break;
        const long long i = base + lane;
        if (i < p.total) {
            const long long kidx = p.cell_list ? p.cell_list[i] : p.cell_offset + i;
#if defined(UCB_TANGENT)
            const double v = ucbdev::lle_cell_tangent(p, kidx, ns);
#else
            const double v = ucbdev::lle_cell_shadow(p, kidx, ns);
#endif
            ucbdev::store_cell(p, i, kidx, v);
        }
    }
    ucbdev::warp_add_steps(p.steps, ns, lane);
}

// Final state of every cell after `skip` plain steps from its initial condition (no
// divergence checks, no extra step): a trajectory-parity aid over the same grid.
extern "C" __global__ void UCB_LAUNCH_BOUNDS ucb_state_kernel(const UcbLleParams p) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.total) return;
    const long long kidx = p.cell_offset + i;
    const ucbdev::CellAxes c = ucbdev::cell_axes(kidx, p.n_pts);
    const ucbdev::CellSteps cs = ucbdev::cell_steps(p, c);
    numb x[UCB_NX], a[UCB_NV];
#pragma unroll
    for (int k = 0; k < UCB_NX; ++k) x[k] = p.ic[k];
#pragma unroll
    for (int k = 0; k < UCB_NV; ++k) a[k] = p.vals[k];
    ucbdev::apply_sweep(c, p.axis0, p.axis1, x, a);
    const ucbdev::Stepper st(cs.h);
    for (long long s = 0; s < p.skip; ++s) st.step(x, a, cs.h);
#pragma unroll
    for (int k = 0; k < UCB_NX; ++k) p.out_values[i * UCB_NX + k] = (double)x[k];
}
