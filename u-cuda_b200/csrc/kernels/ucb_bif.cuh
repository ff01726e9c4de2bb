// ucb_bif.cuh — bifurcation diagrams with fused peak capture (NVRTC header).
//
// One thread per sweep point. The reference (run_bif1d, parametric_engine.cpp:1940-2084)
// writes the whole recorded series of every point to HBM (calculateDiscreteModelCUDA,
// cudaLibrary.cu:944-1077), re-reads it in a second kernel (peakFinderCUDA, :1641-1674)
// and copies points x record_steps values back. Here the recorded value of every step
// is consumed as it is produced by a streaming form of peakFinder (:1503-1633): a
// three-sample window plus the scan state of its outer/inner loops reproduces the same
// peaks (parabolic interpolation, plateau handling, skip of the sample after a peak,
// first peak dropped, intervals = (t_{k+1} - t_k) * step, count capped at 2500), so only
// the first max_out peaks and intervals per point ever reach memory.
#pragma once

struct UcbBifParams {
    int n_pts;                 // sweep points
    int pre_scaller;
    int writable_var;          // -1: x0 + pi x1 + e x2 combination
    int max_out;               // peaks stored per point
    long long skip;            // (int)(transient / h), host double arithmetic
    long long iters;           // ceil(tMax / worstCaseH / preScaller), host double arithmetic
    numb h, maxv, transient, tmax, time_step;
    numb ic[UCB_NX];
    numb vals[UCB_NV];
    const numb* axis0;         // n_pts sweep values
    int* out_counts;           // per point: peaks (>= 0), -1 fixed point, 0 diverged
    double* out_peaks;         // n_pts x max_out
    double* out_intervals;     // n_pts x max_out
    unsigned long long* counter;
    unsigned long long* steps;
};

namespace ucbdev {

// Streaming peakFinder. Position p is decided when sample p+1 arrives, as in the
// reference loop that looks one sample ahead; positions p >= n-2 are never candidates.
struct PeakScan {
    numb d0, d1, d2;           // samples p-1, p, p+1
    long long next_i;          // first index allowed as a new candidate (outer loop i)
    bool plateau;              // inside the inner loop (j) of a candidate
    int found;                 // peaks found so far (before dropping the first)
    numb prev_t;               // raw time of the previous peak
    __device__ __forceinline__ void init() {
        next_i = 2;
        plateau = false;
        found = 0;
        prev_t = 0;
    }
};

__device__ __forceinline__ numb recorded_value(const numb* x, int wv) {
    if (wv < 0) {
#if UCB_NX >= 3
        return x[0] + pi * x[1] + euler * x[2];
#elif UCB_NX == 2
        return x[0] + pi * x[1];
#else
        return x[0];
#endif
    }
    return x[wv];
}

// Emits a peak at position j with the reference's interpolation.
__device__ __forceinline__ void emit_peak(PeakScan& s, long long j, const UcbBifParams& p, long long cell) {
    numb denom = s.d0 - (numb)2.0 * s.d1 + s.d2;
    numb delta = 0.0;
    if (fabs(denom) > 1e-12) delta = 0.5 * (s.d0 - s.d2) / denom;
    const numb value = s.d1 - 0.25 * (s.d0 - s.d2) * delta;
    const numb t = (numb)(j - 1) + delta;
    if (s.found > 0) {
        const int k = s.found - 1;
        if (k < p.max_out) {
            p.out_peaks[cell * p.max_out + k] = (double)value;
            p.out_intervals[cell * p.max_out + k] = (double)((numb)(t - s.prev_t) * p.time_step);
        }
    }
    s.prev_t = t;
    s.found += 1;
}

// Feeds sample index q (value v). Decides position q-1.
__device__ __forceinline__ void scan_push(PeakScan& s, long long q, numb v, long long n, const UcbBifParams& p,
                                          long long cell) {
    s.d0 = s.d1;
    s.d1 = s.d2;
    s.d2 = v;
    const long long pos = q - 1;  // window is (pos-1, pos, pos+1)
    if (q < 3 || pos > n - 3) return;
    if (s.plateau) {
        if (s.d1 < s.d2) {
            s.plateau = false;
            s.next_i = pos + 2;
        } else if (s.d1 - s.d2 > (numb)kEpsPeakDelta) {
            emit_peak(s, pos, p, cell);
            s.plateau = false;
            s.next_i = pos + 2;
        }
        return;
    }
    if (pos < s.next_i) return;
    if (s.d1 - s.d0 > (numb)kEpsPeakDelta && s.d1 > (numb)kPeakThreshold && s.d1 >= s.d2) {
        // inner loop starts at j = i with the same window
        if (s.d1 - s.d2 > (numb)kEpsPeakDelta) {
            emit_peak(s, pos, p, cell);
            s.next_i = pos + 2;
        } else {
            s.plateau = true;
        }
    }
}

template <class S>
__device__ __forceinline__ int loop_record(const S& st, numb* x, const numb* a, numb h, long long iters, int pre,
                                           int wv, numb maxv, PeakScan& scan, const UcbBifParams& p, long long cell,
                                           long long& ns) {
    for (long long i = 0; i < iters; ++i) {
        scan_push(scan, i, recorded_value(x, wv), iters, p, cell);
        for (int j = 0; j < pre; ++j) st.step(x, a, h);
        ns += pre;
        if (i % kCheckInterval == 0 && diverged(x, maxv)) return 0;
    }
    numb xPrev[UCB_NX];
#pragma unroll
    for (int j = 0; j < UCB_NX; ++j) xPrev[j] = x[j];
    for (int j = 0; j < pre; ++j) st.step(x, a, h);
    ns += pre;
    return fixed_point_flag(x, xPrev);
}

// Transient of calculateDiscreteModelCUDA: one step per iteration, preScaller extra steps.
template <class S>
__device__ __forceinline__ int loop_transient(const S& st, numb* x, const numb* a, numb h, long long iters, int pre,
                                              numb maxv, long long& ns) {
    for (long long i0 = 0; i0 < iters; i0 += kCheckInterval) {
        st.step(x, a, h);
        ns += 1;
        if (diverged(x, maxv)) return 0;
        const long long n = (iters - i0 < kCheckInterval) ? iters - i0 : kCheckInterval;
        for (long long i = 1; i < n; ++i) st.step(x, a, h);
        ns += n - 1;
    }
    numb xPrev[UCB_NX];
#pragma unroll
    for (int j = 0; j < UCB_NX; ++j) xPrev[j] = x[j];
    for (int j = 0; j < pre; ++j) st.step(x, a, h);
    ns += pre;
    return fixed_point_flag(x, xPrev);
}

}  // namespace ucbdev

extern "C" __global__ void __launch_bounds__(128) ucb_bif_kernel(const UcbBifParams p) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    long long ns = 0;
    if (cell < p.n_pts) {
        numb x[UCB_NX], a[UCB_NV];
#pragma unroll
        for (int i = 0; i < UCB_NX; ++i) x[i] = p.ic[i];
#pragma unroll
        for (int i = 0; i < UCB_NV; ++i) a[i] = p.vals[i];
        numb h = p.h;
        long long skip = p.skip, iters = p.iters;
#if UCB_HAXIS == 0
        h = p.axis0[cell];
        skip = (long long)ceil(p.transient / h);
        long long il = (long long)ceil(p.tmax / h / (numb)p.pre_scaller);
        iters = il > p.iters ? p.iters : il;
#elif UCB_POV == 1
        a[UCB_IDX0] = p.axis0[cell];
#else
        x[UCB_IDX0] = p.axis0[cell];
#endif
        int count;
        if (!(h > 0)) {
            count = -1;
        } else {
            const ucbdev::Stepper st(h);
            int flag = ucbdev::loop_transient(st, x, a, h, skip, p.pre_scaller, p.maxv, ns);
            if (flag == 1 || flag == -1) {
                ucbdev::PeakScan scan;
                scan.init();
                scan.d1 = scan.d2 = 0;
                flag = ucbdev::loop_record(st, x, a, h, iters, p.pre_scaller, p.writable_var, p.maxv, scan, p, cell, ns);
                if (flag == 1) {
                    int n = (scan.found > 1) ? scan.found - 1 : 0;
                    if (n >= ucbdev::kMaxAmountOfPeaks) n = ucbdev::kMaxAmountOfPeaks;
                    count = (iters < 5) ? 0 : n;
                } else {
                    count = flag;
                }
            } else {
                count = flag;
            }
        }
        p.out_counts[cell] = count;
    }
    ucbdev::warp_add_steps(p.steps, ns, lane);
}
