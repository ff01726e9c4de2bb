// ucb_ls.cuh — full Lyapunov spectrum maps (NVRTC header, after ucb_device.cuh).
//
// Two methods, one thread per cell, everything in registers, persistent grid:
//
//  * UCB_LS_FIXED (the reference's method, LSKernelCUDA cudaLibrary.cu:2878-3073):
//    fixed-step trajectory + N shadow probes at distance eps, random unit directions
//    (RNG subsequence = cell index) orthonormalised once, then every NT block: advance
//    x and the probes, subtract x, classical Gram-Schmidt (gramSchmidtProcess :2848-2874,
//    projections against the unnormalised b_j), sum log(|b_k| / eps), re-seat the probes.
//
//  * UCB_LS_DP5: tangent-linear spectrum with the adaptive Dormand-Prince 5(4) pair
//    (Dormand & Prince 1980, FSAL) integrating x' = f(x) and V' = J(x) V for N tangent
//    vectors, with the mixed absolute/relative RMS error norm taken over the whole
//    augmented state (x and V: controlling x alone lets the step grow past what the
//    contracting tangent directions need, and the most negative exponents then follow the
//    method's stability function instead of the flow), step factor 0.9 err^-1/5 clamped
//    to [0.2, 5] (2 after a rejection), with
//    modified Gram-Schmidt every `gs_every` accepted steps — or earlier, when the time
//    since the last pass times the running estimate of lambda_1 - lambda_N exceeds the
//    precision's budget (UCB_GS_BUDGET nats: 20 for FP64, 8 for FP32), because beyond it
//    the most contracted direction sinks below the rounding of the stored tangent vectors;
//    the norms, log sums, time and the error norm are FP64 whatever numb is.
#pragma once

struct UcbLsParams {
    long long total;
    long long cell_offset;
    int n_pts;
    int swap_xy;
    int n_blocks;          // (int)(tMax / NT)   [fixed]
    int gs_every;          // accepted steps between MGS   [dp5]
    long long skip;        // (int)(transient / h)        [fixed]
    long long nt_steps;    // (size_t)(NT / h) in numb     [fixed]
    long long max_steps;   // step attempt cap per cell   [dp5]
    numb h, NT, tmax, eps, maxv, transient;
    double rtol, atol, t_end, h0;   // [dp5]
    numb ic[UCB_NX];
    numb vals[UCB_NV];
    const numb* axis0;
    const numb* axis1;
    double* out_values;    // plane-major: values[k * cells + cell] (cells = n^2, or n for one axis)
    int* out_flags;
    unsigned long long* counter;
    unsigned long long* steps;
    long long* out_cell_steps;  // per cell: steps (fixed) / step attempts (DP5); may be null
};

namespace ucbdev {

__device__ __forceinline__ long long ls_out_cell(const UcbLsParams& p, long long kidx) {
    if (!p.swap_xy) return kidx;
    const long long kix = kidx % p.n_pts, kiy = kidx / p.n_pts;
    return kix * p.n_pts + kiy;
}

__device__ __forceinline__ void ls_store(const UcbLsParams& p, long long kidx, const double* v) {
    const long long cell = ls_out_cell(p, kidx);
#if UCB_DIM == 2
    const long long plane = (long long)p.n_pts * p.n_pts;
#else
    const long long plane = p.n_pts;  // one swept axis: n_pts cells per exponent plane
#endif
    bool bad = false;
#pragma unroll
    for (int k = 0; k < UCB_NX; ++k) {
        p.out_values[k * plane + cell] = v[k];
        if (v[k] == 999.0 || v[k] == -999.0) bad = true;
    }
    p.out_flags[cell] = bad ? -1 : 1;
}

#if defined(UCB_LS_FIXED)
// gramSchmidtProcess(a -> b, dens): classical GS, rows are vectors.
__device__ __forceinline__ void gram_schmidt_classical(const numb (*a)[UCB_NX], numb (*b)[UCB_NX], numb* dens) {
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) {
#pragma unroll
        for (int j = 0; j < UCB_NX; ++j) b[i][j] = a[i][j];
#pragma unroll
        for (int j = 0; j < i; ++j) {
            numb num = 0, den = 0;
#pragma unroll
            for (int l = 0; l < UCB_NX; ++l) {
                num += a[i][l] * b[j][l];
                den += b[j][l] * b[j][l];
            }
            const numb frac = den == 0 ? 0 : num / den;
#pragma unroll
            for (int l = 0; l < UCB_NX; ++l) b[i][l] -= frac * b[j][l];
        }
    }
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) {
        numb den = 0;
#pragma unroll
        for (int j = 0; j < UCB_NX; ++j) den += b[i][j] * b[i][j];
        den = sqrt(den);
#pragma unroll
        for (int j = 0; j < UCB_NX; ++j) b[i][j] = den == 0 ? 0 : b[i][j] / den;
        if (dens) dens[i] = den;
    }
}

// x and the N probes advanced in lock step (the reference advances them one after the
// other; they never interact inside a block). 0 if any diverged.
template <class S>
__device__ __forceinline__ int loop_probes(const S& s, numb* x, numb (*y)[UCB_NX], const numb* a, numb h,
                                           long long iters, numb maxValue, long long& ns) {
    for (long long i0 = 0; i0 < iters; i0 += kCheckInterval) {
        s.step(x, a, h);
#pragma unroll
        for (int j = 0; j < UCB_NX; ++j) s.step(y[j], a, h);
        ns += UCB_NX + 1;
        bool bad = diverged(x, maxValue);
#pragma unroll
        for (int j = 0; j < UCB_NX; ++j) bad = bad || diverged(y[j], maxValue);
        if (bad) return 0;
        const long long n = (iters - i0 < kCheckInterval) ? iters - i0 : kCheckInterval;
        for (long long i = 1; i < n; ++i) {
            s.step(x, a, h);
#pragma unroll
            for (int j = 0; j < UCB_NX; ++j) s.step(y[j], a, h);
        }
        ns += (long long)(UCB_NX + 1) * (n - 1);
    }
#if UCB_EXTRA_STEP
    s.step(x, a, h);
#pragma unroll
    for (int j = 0; j < UCB_NX; ++j) s.step(y[j], a, h);
    ns += UCB_NX + 1;
#endif
    return 1;
}

#if defined(UCB_LS_TANGENT) && defined(UCB_HAS_JVP) && !defined(UCB_EXACT)
// Tangent-vector form of the fixed method (native FP32 builds): instead of N shadow
// trajectories x + eps z, whose differences from x fall below FP32 resolution for small eps,
// the N tangent vectors v' = J(x) v are advanced with x in one RK4 sweep (the stage sums
// accumulated stage by stage), and the block's Gram-Schmidt, norms and log sums are FP64.
__device__ __forceinline__ void ls_tangent_step(numb* x, numb (*V)[UCB_NX], const numb* a, numb h) {
    const numb hh = h * (numb)0.5, h6 = h * (numb)(1.0 / 6.0), two = (numb)2;
    numb k[UCB_NX], l[UCB_NX], xt[UCB_NX], sx[UCB_NX];
    numb vt[UCB_NX][UCB_NX], sv[UCB_NX][UCB_NX];
    ucb_rhs(x, a, k);
#pragma unroll
    for (int j = 0; j < UCB_NX; ++j) {
        ucb_jvp(x, a, V[j], l);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) {
            sv[j][i] = l[i];
            vt[j][i] = fma(hh, l[i], V[j][i]);
        }
    }
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) {
        sx[i] = k[i];
        xt[i] = fma(hh, k[i], x[i]);
    }
#pragma unroll
    for (int stage = 2; stage <= 3; ++stage) {
        const numb c = stage == 2 ? hh : h;
        ucb_rhs(xt, a, k);
#pragma unroll
        for (int j = 0; j < UCB_NX; ++j) {
            ucb_jvp(xt, a, vt[j], l);
#pragma unroll
            for (int i = 0; i < UCB_NX; ++i) {
                sv[j][i] = fma(two, l[i], sv[j][i]);
                vt[j][i] = fma(c, l[i], V[j][i]);
            }
        }
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) {
            sx[i] = fma(two, k[i], sx[i]);
            xt[i] = fma(c, k[i], x[i]);
        }
    }
    ucb_rhs(xt, a, k);
#pragma unroll
    for (int j = 0; j < UCB_NX; ++j) {
        ucb_jvp(xt, a, vt[j], l);
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) V[j][i] = fma(h6, sv[j][i] + l[i], V[j][i]);
    }
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) x[i] = fma(h6, sx[i] + k[i], x[i]);
}

// Classical Gram-Schmidt of the rows of V in FP64 (the reference's gramSchmidtProcess
// order): V becomes orthonormal (rounded to numb), dens[i] the norm of row i after
// removing its projections on the earlier rows.
__device__ __forceinline__ void gs_classical_f64(numb (*V)[UCB_NX], double* dens) {
    double b[UCB_NX][UCB_NX];
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) {
#pragma unroll
        for (int l = 0; l < UCB_NX; ++l) b[i][l] = (double)V[i][l];
#pragma unroll
        for (int j = 0; j < i; ++j) {
            double num = 0, den = 0;
#pragma unroll
            for (int l = 0; l < UCB_NX; ++l) {
                num = fma((double)V[i][l], b[j][l], num);
                den = fma(b[j][l], b[j][l], den);
            }
            const double frac = den == 0 ? 0 : num / den;
#pragma unroll
            for (int l = 0; l < UCB_NX; ++l) b[i][l] = fma(-frac, b[j][l], b[i][l]);
        }
    }
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) {
        double den = 0;
#pragma unroll
        for (int l = 0; l < UCB_NX; ++l) den = fma(b[i][l], b[i][l], den);
        den = sqrt(den);
        const double inv = den == 0 ? 0 : 1.0 / den;
#pragma unroll
        for (int l = 0; l < UCB_NX; ++l) V[i][l] = (numb)(b[i][l] * inv);
        dens[i] = den;
    }
}

// NT-step block of x and the tangent vectors with the divergence test of loop_probes
// (tangent vectors: non-finite only). 0 if anything diverged.
__device__ __forceinline__ int loop_tangents(numb* x, numb (*V)[UCB_NX], const numb* a, numb h, long long iters,
                                             numb maxValue, long long& ns) {
    for (long long i0 = 0; i0 < iters; i0 += kCheckInterval) {
        ls_tangent_step(x, V, a, h);
        ns += UCB_NX + 1;
        bool bad = diverged(x, maxValue);
#pragma unroll
        for (int j = 0; j < UCB_NX; ++j) bad = bad || diverged(V[j], (numb)0);
        if (bad) return 0;
        const long long n = (iters - i0 < kCheckInterval) ? iters - i0 : kCheckInterval;
        for (long long i = 1; i < n; ++i) ls_tangent_step(x, V, a, h);
        ns += (long long)(UCB_NX + 1) * (n - 1);
    }
#if UCB_EXTRA_STEP
    ls_tangent_step(x, V, a, h);
    ns += UCB_NX + 1;
#endif
    return 1;
}
#define UCB_LS_FIXED_TANGENT 1
#endif

__device__ __forceinline__ void ls_cell_fixed(const UcbLsParams& p, long long kidx, long long& ns) {
    double outv[UCB_NX];
    const CellAxes c = cell_axes(kidx, p.n_pts);
    numb h = p.h;
    long long nt = p.nt_steps, skip = p.skip;
#if UCB_HAXIS == 0
    h = p.axis0[c.i0];
#elif UCB_HAXIS == 1
    h = p.axis1[c.i1];
#endif
#if UCB_HAXIS != -1
    nt = (long long)ceil(p.NT / h);
    skip = (long long)ceil(p.transient / h);
#endif
    if (!(h > 0)) {
#pragma unroll
        for (int m = 0; m < UCB_NX; ++m) outv[m] = (double)nan("");
        ls_store(p, kidx, outv);
        return;
    }
    numb x[UCB_NX], a[UCB_NV];
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) x[i] = p.ic[i];
#pragma unroll
    for (int i = 0; i < UCB_NV; ++i) a[i] = p.vals[i];
    apply_sweep(c, p.axis0, p.axis1, x, a);
    numb y[UCB_NX][UCB_NX], z[UCB_NX][UCB_NX], dens[UCB_NX];
    double result[UCB_NX];
    {
        Rng st;
        rng_init(1234567891ULL, (unsigned long long)kidx, 0ULL, &st);
#pragma unroll
        for (int j = 0; j < UCB_NX; ++j) {
            numb zPower = 0;
#pragma unroll
            for (int i = 0; i < UCB_NX; ++i) {
                z[j][i] = rng_uniform(&st) - 0.5;
                zPower += z[j][i] * z[j][i];
            }
            zPower = sqrt(zPower);
#pragma unroll
            for (int i = 0; i < UCB_NX; ++i) z[j][i] /= zPower;
        }
    }
    const Stepper st(h);
    if (loop_single(st, x, a, h, skip, p.maxv, ns) == 0) {
#pragma unroll
        for (int m = 0; m < UCB_NX; ++m) outv[m] = 999.0;
        ls_store(p, kidx, outv);
        return;
    }
#if defined(UCB_LS_FIXED_TANGENT)
    {
        double d[UCB_NX], sum[UCB_NX];
        gs_classical_f64(z, d);  // the same random start, orthonormal
#pragma unroll
        for (int k = 0; k < UCB_NX; ++k) sum[k] = 0.0;
        for (int b = 0; b < p.n_blocks; ++b) {
            if (loop_tangents(x, z, a, h, nt, p.maxv, ns) == 0) {
#pragma unroll
                for (int m = 0; m < UCB_NX; ++m) outv[m] = 999.0;
                ls_store(p, kidx, outv);
                return;
            }
            gs_classical_f64(z, d);
#pragma unroll
            for (int k = 0; k < UCB_NX; ++k) sum[k] += log(d[k]);
        }
        (void)y;
        (void)dens;
#pragma unroll
        for (int k = 0; k < UCB_NX; ++k) result[k] = sum[k] / (double)p.tmax;
        ls_store(p, kidx, result);
        return;
    }
#endif
    gram_schmidt_classical(z, y, nullptr);
#pragma unroll
    for (int j = 0; j < UCB_NX; ++j)
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) y[j][i] = y[j][i] * p.eps + x[i];
    numb res_n[UCB_NX];
#pragma unroll
    for (int k = 0; k < UCB_NX; ++k) res_n[k] = 0;
    for (int b = 0; b < p.n_blocks; ++b) {
        if (loop_probes(st, x, y, a, h, nt, p.maxv, ns) == 0) {
#pragma unroll
            for (int m = 0; m < UCB_NX; ++m) outv[m] = 999.0;
            ls_store(p, kidx, outv);
            return;
        }
#pragma unroll
        for (int k = 0; k < UCB_NX; ++k)
#pragma unroll
            for (int l = 0; l < UCB_NX; ++l) y[k][l] = y[k][l] - x[l];
        gram_schmidt_classical(y, z, dens);
#pragma unroll
        for (int k = 0; k < UCB_NX; ++k) {
            res_n[k] += log(dens[k] / p.eps);
#pragma unroll
            for (int j = 0; j < UCB_NX; ++j) y[k][j] = (numb)(x[j] + z[k][j] * p.eps);
        }
    }
#pragma unroll
    for (int k = 0; k < UCB_NX; ++k) result[k] = (double)(res_n[k] / p.tmax);
    ls_store(p, kidx, result);
}
#endif  // UCB_LS_FIXED

#if defined(UCB_LS_DP5)
#ifndef UCB_GS_BUDGET
#define UCB_GS_BUDGET 20.0
#endif
// Dormand-Prince 5(4) coefficients (Dormand & Prince, J. Comp. Appl. Math. 6, 1980).
#define DP_A21 (1.0 / 5.0)
#define DP_A31 (3.0 / 40.0)
#define DP_A32 (9.0 / 40.0)
#define DP_A41 (44.0 / 45.0)
#define DP_A42 (-56.0 / 15.0)
#define DP_A43 (32.0 / 9.0)
#define DP_A51 (19372.0 / 6561.0)
#define DP_A52 (-25360.0 / 2187.0)
#define DP_A53 (64448.0 / 6561.0)
#define DP_A54 (-212.0 / 729.0)
#define DP_A61 (9017.0 / 3168.0)
#define DP_A62 (-355.0 / 33.0)
#define DP_A63 (46732.0 / 5247.0)
#define DP_A64 (49.0 / 176.0)
#define DP_A65 (-5103.0 / 18656.0)
#define DP_B1 (35.0 / 384.0)
#define DP_B3 (500.0 / 1113.0)
#define DP_B4 (125.0 / 192.0)
#define DP_B5 (-2187.0 / 6784.0)
#define DP_B6 (11.0 / 84.0)
#define DP_E1 (71.0 / 57600.0)
#define DP_E3 (-71.0 / 16695.0)
#define DP_E4 (71.0 / 1920.0)
#define DP_E5 (-17253.0 / 339200.0)
#define DP_E6 (22.0 / 525.0)
#define DP_E7 (-1.0 / 40.0)

// Modified Gram-Schmidt on the rows of V; log of the norms added to acc (FP64).
__device__ __forceinline__ bool mgs(numb (*V)[UCB_NX], double* acc) {
#pragma unroll
    for (int k = 0; k < UCB_NX; ++k) {
#pragma unroll
        for (int j = 0; j < k; ++j) {
            double d = 0;
#pragma unroll
            for (int l = 0; l < UCB_NX; ++l) d = fma((double)V[k][l], (double)V[j][l], d);
            const numb dn = (numb)d;
#pragma unroll
            for (int l = 0; l < UCB_NX; ++l) V[k][l] = fma(-dn, V[j][l], V[k][l]);
        }
        double n2 = 0;
#pragma unroll
        for (int l = 0; l < UCB_NX; ++l) n2 = fma((double)V[k][l], (double)V[k][l], n2);
        const double nrm = sqrt(n2);
        if (!(nrm > 0) || !isfinite(nrm)) return false;
        acc[k] += log(nrm);
        const numb inv = (numb)(1.0 / nrm);
#pragma unroll
        for (int l = 0; l < UCB_NX; ++l) V[k][l] *= inv;
    }
    return true;
}

// The Butcher rows scaled by the step once per attempt, so that every stage point is a
// chain of fused multiply-adds from the base point: x + sum_j (h a_ij) k_j.
struct Dp5Coef {
    numb c21, c31, c32, c41, c42, c43, c51, c52, c53, c54, c61, c62, c63, c64, c65, b1, b3, b4, b5, b6;
    double e1, e3, e4, e5, e6, e7;  // h times the error weights (FP64: the error norm is FP64)
};

__device__ __forceinline__ Dp5Coef dp5_coef(numb hn, double h) {
    Dp5Coef c;
    c.c21 = hn * (numb)DP_A21;
    c.c31 = hn * (numb)DP_A31; c.c32 = hn * (numb)DP_A32;
    c.c41 = hn * (numb)DP_A41; c.c42 = hn * (numb)DP_A42; c.c43 = hn * (numb)DP_A43;
    c.c51 = hn * (numb)DP_A51; c.c52 = hn * (numb)DP_A52; c.c53 = hn * (numb)DP_A53; c.c54 = hn * (numb)DP_A54;
    c.c61 = hn * (numb)DP_A61; c.c62 = hn * (numb)DP_A62; c.c63 = hn * (numb)DP_A63; c.c64 = hn * (numb)DP_A64;
    c.c65 = hn * (numb)DP_A65;
    c.b1 = hn * (numb)DP_B1; c.b3 = hn * (numb)DP_B3; c.b4 = hn * (numb)DP_B4; c.b5 = hn * (numb)DP_B5;
    c.b6 = hn * (numb)DP_B6;
    c.e1 = h * DP_E1; c.e3 = h * DP_E3; c.e4 = h * DP_E4; c.e5 = h * DP_E5; c.e6 = h * DP_E6; c.e7 = h * DP_E7;
    return c;
}

// sum_i (e_i / s_i)^2 for s_i > 0, one division per group of four: 1 / (s0 s1 s2 s3) times
// the other three scales gives each 1 / s_i. A group whose product leaves the normal range
// (scales below 1e-75 or above 1e75) divides component by component.
template <int N>
__device__ __forceinline__ double scaled_sum_sq(const double* e, const double* s) {
    double acc = 0.0;
#pragma unroll
    for (int g = 0; g < N; g += 4) {
        const int m = (N - g) < 4 ? (N - g) : 4;
        if (m == 1) {
            const double q = e[g] / s[g];
            acc = fma(q, q, acc);
            continue;
        }
        double pre[4], suf[4];  // products of the scales before / after position i
        pre[0] = 1.0;
#pragma unroll
        for (int i = 1; i < m; ++i) pre[i] = pre[i - 1] * s[g + i - 1];
        suf[m - 1] = 1.0;
#pragma unroll
        for (int i = m - 2; i >= 0; --i) suf[i] = suf[i + 1] * s[g + i + 1];
        const double prod = pre[m - 1] * s[g + m - 1];
        if (prod > 1e-300 && prod < 1e300) {
            const double r = 1.0 / prod;
#pragma unroll
            for (int i = 0; i < m; ++i) {
                const double q = e[g + i] * (r * (pre[i] * suf[i]));
                acc = fma(q, q, acc);
            }
        } else {
#pragma unroll
            for (int i = 0; i < m; ++i) {
                const double q = e[g + i] / s[g + i];
                acc = fma(q, q, acc);
            }
        }
    }
    return acc;
}

// Step-size factor 0.9 err^(-1/5) of the controller, from err^2. A heuristic factor (it is
// clamped to [0.2, facmax] next), so the power is taken in FP32 (relative error ~1e-6),
// off the FP64 pipe; err^2 below the FP32 range gives +inf (clamped to facmax) and above it
// 0 (clamped to 0.2), as the FP64 power would after clamping.
__device__ __forceinline__ double dp5_factor(double err2) {
    return 0.9 * (double)__powf((float)err2, -0.1f);
}

// One DP5 step of the state: stage points X2..X6, the 5th-order solution xn and its
// derivative k7 (FSAL), and the sum of squared scaled errors of the embedded 4th-order
// difference.
struct Dp5State {
    numb X[6][UCB_NX];  // stage points X1 (= x) .. X6
    numb k1[UCB_NX], k7[UCB_NX], xn[UCB_NX];
};

__device__ __forceinline__ double dp5_state_step(Dp5State& S, const numb* a, const Dp5Coef& c, double rtol,
                                                 double atol) {
    numb k2[UCB_NX], k3[UCB_NX], k4[UCB_NX], k5[UCB_NX], k6[UCB_NX];
    const numb* x = S.X[0];
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) S.X[1][i] = fma(c.c21, S.k1[i], x[i]);
    ucb_rhs(S.X[1], a, k2);
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) S.X[2][i] = fma(c.c32, k2[i], fma(c.c31, S.k1[i], x[i]));
    ucb_rhs(S.X[2], a, k3);
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) S.X[3][i] = fma(c.c43, k3[i], fma(c.c42, k2[i], fma(c.c41, S.k1[i], x[i])));
    ucb_rhs(S.X[3], a, k4);
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i)
        S.X[4][i] = fma(c.c54, k4[i], fma(c.c53, k3[i], fma(c.c52, k2[i], fma(c.c51, S.k1[i], x[i]))));
    ucb_rhs(S.X[4], a, k5);
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i)
        S.X[5][i] = fma(c.c65, k5[i], fma(c.c64, k4[i], fma(c.c63, k3[i], fma(c.c62, k2[i], fma(c.c61, S.k1[i], x[i])))));
    ucb_rhs(S.X[5], a, k6);
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i)
        S.xn[i] = fma(c.b6, k6[i], fma(c.b5, k5[i], fma(c.b4, k4[i], fma(c.b3, k3[i], fma(c.b1, S.k1[i], x[i])))));
    ucb_rhs(S.xn, a, S.k7);
    double e[UCB_NX], sc[UCB_NX];
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) {
        e[i] = fma(c.e7, (double)S.k7[i], fma(c.e6, (double)k6[i], fma(c.e5, (double)k5[i],
               fma(c.e4, (double)k4[i], fma(c.e3, (double)k3[i], c.e1 * (double)S.k1[i])))));
        sc[i] = fma(rtol, fmax(fabs((double)x[i]), fabs((double)S.xn[i])), atol);
    }
    return scaled_sum_sq<UCB_NX>(e, sc);
}

// One tangent vector through the same DP5 stages (v' = J(x) v with J at the stored stage
// points): writes the 5th-order vn and returns its sum of squared scaled errors.
__device__ __forceinline__ double dp5_tangent_step(const Dp5State& S, const numb* a, const Dp5Coef& c, double rtol,
                                                   double atol, const numb* v, numb* vn) {
    numb L1[UCB_NX], L2[UCB_NX], L3[UCB_NX], L4[UCB_NX], L5[UCB_NX], L6[UCB_NX], vt[UCB_NX];
    ucb_jvp(S.X[0], a, v, L1);
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) vt[i] = fma(c.c21, L1[i], v[i]);
    ucb_jvp(S.X[1], a, vt, L2);
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) vt[i] = fma(c.c32, L2[i], fma(c.c31, L1[i], v[i]));
    ucb_jvp(S.X[2], a, vt, L3);
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) vt[i] = fma(c.c43, L3[i], fma(c.c42, L2[i], fma(c.c41, L1[i], v[i])));
    ucb_jvp(S.X[3], a, vt, L4);
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i)
        vt[i] = fma(c.c54, L4[i], fma(c.c53, L3[i], fma(c.c52, L2[i], fma(c.c51, L1[i], v[i]))));
    ucb_jvp(S.X[4], a, vt, L5);
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i)
        vt[i] = fma(c.c65, L5[i], fma(c.c64, L4[i], fma(c.c63, L3[i], fma(c.c62, L2[i], fma(c.c61, L1[i], v[i])))));
    ucb_jvp(S.X[5], a, vt, L6);
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i)
        vn[i] = fma(c.b6, L6[i], fma(c.b5, L5[i], fma(c.b4, L4[i], fma(c.b3, L3[i], fma(c.b1, L1[i], v[i])))));
    ucb_jvp(S.xn, a, vn, L2);  // L7, reusing L2's registers
    double e[UCB_NX], sc[UCB_NX];
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) {
        e[i] = fma(c.e7, (double)L2[i], fma(c.e6, (double)L6[i], fma(c.e5, (double)L5[i],
               fma(c.e4, (double)L4[i], fma(c.e3, (double)L3[i], c.e1 * (double)L1[i])))));
        sc[i] = fma(rtol, fmax(fabs((double)v[i]), fabs((double)vn[i])), atol);
    }
    return scaled_sum_sq<UCB_NX>(e, sc);
}

// An adaptive cell whose remaining horizon needs more than this many times its remaining
// step attempts (at the current step size) is given up as escaping.
constexpr double kEscapeFactor = 8.0;

__device__ __forceinline__ void ls_cell_dp5(const UcbLsParams& p, long long kidx, long long& ns) {
    double outv[UCB_NX];
    const CellAxes c = cell_axes(kidx, p.n_pts);
    Dp5State S;
    numb a[UCB_NV];
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) S.X[0][i] = p.ic[i];
#pragma unroll
    for (int i = 0; i < UCB_NV; ++i) a[i] = p.vals[i];
    apply_sweep(c, p.axis0, p.axis1, S.X[0], a);
#ifdef UCB_KAHAN_CLOCK
    // the clock of an FP32 build is set from the FP64 time after every accepted step
    const double clock0 = (double)S.X[0][UCB_CLOCK_VAR];
#endif
    numb V[UCB_NX][UCB_NX];
    {
        Rng st;
        rng_init(1234567891ULL, (unsigned long long)kidx, 0ULL, &st);
#pragma unroll
        for (int j = 0; j < UCB_NX; ++j)
#pragma unroll
            for (int i = 0; i < UCB_NX; ++i) V[j][i] = rng_uniform(&st) - 0.5;
    }
    double acc[UCB_NX], junk[UCB_NX];
#pragma unroll
    for (int k = 0; k < UCB_NX; ++k) acc[k] = junk[k] = 0;
    bool ok = mgs(V, junk);
    // The transient [0, transient) moves the state only; tangents are measured over
    // [transient, transient + t_end] with MGS every gs_every accepted steps and at the end.
    double t = 0.0;
    const double t_stop = (double)p.transient + p.t_end;
    double h = p.h0, facmax = 5.0;
    int since_gs = 0;
    double t_gs = 0.0, t_meas = 0.0, spread = 1e300;  // spread: running lambda_1 - lambda_N
    bool measuring = !((double)p.transient > 0);
    long long attempts = 0, accepted = 0;
    ucb_rhs(S.X[0], a, S.k1);
    while (ok && t < t_stop) {
        if (++attempts > p.max_steps) { ok = false; break; }
        // a cell can take millions of attempts: a cancelled run abandons it
        if ((attempts & 4095) == 0 && run_cancelled()) { ok = false; break; }
        const double t_target = measuring ? t_stop : (double)p.transient;
        bool last = false;
        if (t + h >= t_target) { h = t_target - t; last = true; }
        const Dp5Coef cf = dp5_coef((numb)h, h);
        const double ex2 = dp5_state_step(S, a, cf, p.rtol, p.atol);
        ns += 1;
        // err^2: the mean of the squared scaled errors (the RMS norm, squared)
        double err2 = ex2 * (1.0 / UCB_NX);
        numb Vn[UCB_NX][UCB_NX];
        if (err2 <= 1.0 && measuring) {
            double ev2 = 0;
#pragma unroll
            for (int k = 0; k < UCB_NX; ++k) ev2 += dp5_tangent_step(S, a, cf, p.rtol, p.atol, V[k], Vn[k]);
            err2 = (ex2 + ev2) * (1.0 / (UCB_NX + UCB_NX * UCB_NX));
        }
        if (!isfinite(err2)) { ok = false; break; }
        if (err2 <= 1.0) {
            if (measuring) {
#pragma unroll
                for (int k = 0; k < UCB_NX; ++k)
#pragma unroll
                    for (int i = 0; i < UCB_NX; ++i) V[k][i] = Vn[k][i];
            }
            const double t_new = last ? t_target : t + h;
            if (measuring) t_gs += t_new - t;
            t = t_new;
#pragma unroll
            for (int i = 0; i < UCB_NX; ++i) { S.X[0][i] = S.xn[i]; S.k1[i] = S.k7[i]; }
#ifdef UCB_KAHAN_CLOCK
            S.X[0][UCB_CLOCK_VAR] = (numb)fma((double)UCB_CLOCK_RATE, t, clock0);
#endif
            if (diverged(S.X[0], p.maxv)) { ok = false; break; }
            // Escape test, every 16 accepted steps: at the step size just taken the rest of the
            // horizon would need more than kEscapeFactor times the attempts left. Such a cell
            // (in practice one escaping towards max_value through ever stiffer, ever smaller
            // steps) would end at the attempt cap with the same flag; it ends here instead.
            if ((++accepted & 15) == 0 && t_stop - t > kEscapeFactor * h * (double)(p.max_steps - attempts)) {
                ok = false;
                break;
            }
            if (measuring && (++since_gs >= p.gs_every || last || t_gs * spread > UCB_GS_BUDGET)) {
                ok = mgs(V, acc);
                since_gs = 0;
                t_meas += t_gs;
                t_gs = 0.0;
                spread = fmax(0.0, (acc[0] - acc[UCB_NX - 1]) / t_meas);
            }
            if (last && !measuring) measuring = true;
            const double fac = (err2 > 0) ? dp5_factor(err2) : facmax;
            h *= fmin(facmax, fmax(0.2, fac));
            facmax = 5.0;
        } else {
            h *= fmax(0.2, dp5_factor(err2));
            facmax = 2.0;
            if (!(h > 1e-14)) { ok = false; break; }
        }
    }
#pragma unroll
    for (int k = 0; k < UCB_NX; ++k) outv[k] = ok ? acc[k] / p.t_end : 999.0;
    ls_store(p, kidx, outv);
}
#endif  // UCB_LS_DP5

}  // namespace ucbdev

extern "C" __global__ void UCB_LAUNCH_BOUNDS ucb_ls_kernel(const UcbLsParams p) {
    const int lane = threadIdx.x & 31;
    long long ns = 0;
    for (;;) {
        const long long base = ucbdev::warp_fetch(p.counter, lane);
        if (base >= p.total) break;
        const long long i = base + lane;
        if (i < p.total) {
            const long long ns0 = ns;
#if defined(UCB_LS_DP5)
            ucbdev::ls_cell_dp5(p, p.cell_offset + i, ns);
#else
            ucbdev::ls_cell_fixed(p, p.cell_offset + i, ns);
#endif
            if (p.out_cell_steps) p.out_cell_steps[ucbdev::ls_out_cell(p, p.cell_offset + i)] = ns - ns0;
        }
    }
    ucbdev::warp_add_steps(p.steps, ns, lane);
}
