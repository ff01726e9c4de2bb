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
    // a select over the components, not x[wv]: a run-time index would move the state out
    // of registers into local memory (wv is validated to [0, N) by the host)
    numb r = x[0];
#pragma unroll
    for (int j = 1; j < UCB_NX; ++j)
        if (wv == j) r = x[j];
    return r;
}

// Where the peaks of one point go: the first max_out peaks and intervals of a 1-D
// diagram (Bif1dSink), or every peak the 2-D period count clusters (Bif2dSink).
struct Bif1dSink {
    double* peaks;
    double* intervals;
    int max_out;
    numb time_step;
    __device__ __forceinline__ void put(int k, numb value, numb dt) const {
        if (k < max_out) {
            peaks[k] = (double)value;
            intervals[k] = (double)((numb)dt * time_step);
        }
    }
};

// Emits a peak at position j with the reference's interpolation.
template <class Sink>
__device__ __forceinline__ void emit_peak(PeakScan& s, long long j, const Sink& sink) {
    numb denom = s.d0 - (numb)2.0 * s.d1 + s.d2;
    numb delta = 0.0;
    if (fabs(denom) > 1e-12) delta = 0.5 * (s.d0 - s.d2) / denom;
    const numb value = s.d1 - 0.25 * (s.d0 - s.d2) * delta;
    const numb t = (numb)(j - 1) + delta;
    if (s.found > 0) sink.put(s.found - 1, value, t - s.prev_t);
    s.prev_t = t;
    s.found += 1;
}

// Feeds sample index q (value v). Decides position q-1.
template <class Sink>
__device__ __forceinline__ void scan_push(PeakScan& s, long long q, numb v, long long n, const Sink& sink) {
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
            emit_peak(s, pos, sink);
            s.plateau = false;
            s.next_i = pos + 2;
        }
        return;
    }
    if (pos < s.next_i) return;
    if (s.d1 - s.d0 > (numb)kEpsPeakDelta && s.d1 > (numb)kPeakThreshold && s.d1 >= s.d2) {
        // inner loop starts at j = i with the same window
        if (s.d1 - s.d2 > (numb)kEpsPeakDelta) {
            emit_peak(s, pos, sink);
            s.next_i = pos + 2;
        } else {
            s.plateau = true;
        }
    }
}

template <class S, class Sink>
__device__ __forceinline__ int loop_record(const S& st, numb* x, const numb* a, numb h, long long iters, int pre,
                                           int wv, numb maxv, PeakScan& scan, const Sink& sink, long long& ns) {
    // Chunks of kCheckInterval samples, the divergence test after the first one's steps
    // (i % kCheckInterval == 0), so the per-sample loop carries no 64-bit modulo: these
    // launches run a warp or so per SM, where every instruction of a sample is latency.
    for (long long i0 = 0; i0 < iters; i0 += kCheckInterval) {
        scan_push(scan, i0, recorded_value(x, wv), iters, sink);
        st.step(x, a, h);
        for (int j = 1; j < pre; ++j) st.step(x, a, h);
        ns += pre;
        if (diverged(x, maxv)) return 0;
        const int n = (iters - i0 < kCheckInterval) ? (int)(iters - i0) : kCheckInterval;
        for (int c = 1; c < n; ++c) {
            scan_push(scan, i0 + c, recorded_value(x, wv), iters, sink);
            st.step(x, a, h);
            for (int j = 1; j < pre; ++j) st.step(x, a, h);
        }
        ns += (long long)pre * (n - 1);
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
        UCB_STEP_LOOP
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

#if !defined(UCB_BIF2D) && !defined(UCB_BIF_NO_KERNELS)
extern "C" __global__ void UCB_LAUNCH_BOUNDS ucb_bif_kernel(const UcbBifParams p) {
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
                const ucbdev::Bif1dSink sink{p.out_peaks + cell * p.max_out, p.out_intervals + cell * p.max_out,
                                             p.max_out, p.time_step};
                flag = ucbdev::loop_record(st, x, a, h, iters, p.pre_scaller, p.writable_var, p.maxv, scan, sink, ns);
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
#endif  // 1-D kernel

#if defined(UCB_BIF2D) && !defined(UCB_BIF_NO_KERNELS)
// ---------------------------------------------------------------------------------------
// 2-D bifurcation (period) maps: run_bif2d (parametric_engine.cpp:5487-5910) = per cell the
// 1-D trajectory + peakFinder above, then dbscan of the peaks (cudaLibrary.cu:2088-2166,
// dbscanCUDA :2321) whose cluster count is the "period". The reference keeps the whole
// recorded series, the peaks, the intervals and a helper array per cell in HBM and runs
// three kernels. Here a warp integrates its 32 cells (one per lane) with the peaks
// streaming into the warp's own scratch slot (one contiguous row of `cap` peaks per
// lane), then runs the dbscan of each of the 32 cells in turn with all 32 lanes: the
// dbscan's control flow (seeds, stack pops) is the same for the whole warp and each scan
// over the peaks is split across the lanes, so no lane waits on another cell's pops.
// Scratch is per resident warp, not per cell.
struct UcbBif2dParams {
    long long total;           // cells
    int n_pts;
    int swap_xy;               // 1: write transposed (user X = kernel axis 1)
    int pre_scaller;
    int writable_var;
    int cap;                   // peaks kept per cell (>= the largest possible count)
    int pad0;
    long long skip;            // (int)(transient / h), host double arithmetic
    long long iters;           // ceil(tMax / worstCaseH / preScaller), host double arithmetic
    numb h, maxv, transient, tmax, eps;
    numb ic[UCB_NX];
    numb vals[UCB_NV];
    const numb* axis0;
    const numb* axis1;
    numb* peaks;               // per warp slot: 32 x cap
    int* work;                 // per warp slot: cap labels + cap stack slots
    double* out_values;        // period (-1 where the dbscan result is negative)
    int* out_flags;            // -1 / 1
    unsigned long long* counter;
    unsigned long long* steps;
};

namespace ucbdev {

struct Bif2dSink {
    numb* peaks;
    int cap;
    __device__ __forceinline__ void put(int k, numb value, numb) const {
        if (k < cap) peaks[k] = value;
    }
};

// The reference's dbscan step for step, one warp per cell: labels (helpful[0, P)) and the
// stack slots (helpful[P, 2P)) as integers — they only ever hold cluster numbers and
// indices below 2,500, exact in numb — with the slots written at P + k and popped at
// P + NumNeibor - 1, inner bound P - 1, result cluster - 1. Peaks enter times mult_peak (1)
// and intervals times mult_interval (0) (configCUDA.h), so the distance is that of the
// peak values. Within one scan each k touches only its own label and slot and NumNeibor
// only counts, so the lanes take k = lane, lane + 32, ... and the hits are summed with a
// ballot.
__device__ __forceinline__ int dbscan_warp(const numb* peaks, int P, int* lab, int* stk, numb eps, int lane) {
    if (P == -1) return -1;
    if (P == 0) return 0;
    if (P == 1) return 1;
    for (int k = lane; k < P; k += 32) {
        lab[k] = 0;
        stk[k] = 0;
    }
    __syncwarp();
    int cluster = 0, nn = 0;
    for (unsigned long long i = 0; i < (unsigned long long)P; i++) {
        if (nn >= 1) {
            const int v = stk[nn - 1];
            __syncwarp();
            if (lane == 0) stk[nn - 1] = 0;
            i = (unsigned long long)v;
            nn = nn - 1;
        } else if (lab[i] == 0) {
            nn = 0;
            ++cluster;
            __syncwarp();
            if (lane == 0) lab[i] = cluster;
        } else {
            continue;
        }
        __syncwarp();
        const numb xi = peaks[i];
        int hits = 0;
        // chunks of 32 are independent (each k touches only its own label and slot): both
        // loads of a lane are issued unconditionally and four chunks are in flight at once
#pragma unroll 4
        for (int k0 = 0; k0 < P - 1; k0 += 32) {
            const int k = k0 + lane;
            const bool in = k < P - 1;
            const int lk = in ? lab[k] : 1;
            const numb pk = in ? peaks[k] : xi;
            // the reference's distance sqrt(dx * dx + 0 * 0) = sqrt(fl(dx * dx)) is exactly
            // |dx| in binary floating point (correctly rounded product and square root; an
            // overflowing or underflowing dx * dx still compares the same against eps)
            const bool hit = in && i != (unsigned long long)k && lk == 0 && fabs(pk - xi) < eps;
            if (hit) {
                lab[k] = cluster;
                stk[k] = k;
            }
            hits += __popc(__ballot_sync(0xFFFFFFFFu, hit));
        }
        nn += hits;
        __syncwarp();
    }
    return cluster - 1;
}

// Trajectory and peaks of one cell of a 2-D period map: the peak count (or the -1 / 0
// trajectory flag), peaks in row[0, min(count, cap)).
__device__ __forceinline__ int bif2d_peaks(const UcbBif2dParams& p, long long kidx, numb* row, long long& ns) {
    const ucbdev::CellAxes c = ucbdev::cell_axes(kidx, p.n_pts);
    numb x[UCB_NX], a[UCB_NV];
#pragma unroll
    for (int k = 0; k < UCB_NX; ++k) x[k] = p.ic[k];
#pragma unroll
    for (int k = 0; k < UCB_NV; ++k) a[k] = p.vals[k];
    ucbdev::apply_sweep(c, p.axis0, p.axis1, x, a);
    numb h = p.h;
    long long skip = p.skip, iters = p.iters;
#if UCB_HAXIS == 0 || UCB_HAXIS == 1
#if UCB_HAXIS == 0
    h = p.axis0[c.i0];
#else
    h = p.axis1[c.i1];
#endif
    skip = (long long)ceil(p.transient / h);
    const long long il = (long long)ceil(p.tmax / h / (numb)p.pre_scaller);
    iters = il > p.iters ? p.iters : il;
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
            const ucbdev::Bif2dSink sink{row, p.cap};
            flag = ucbdev::loop_record(st, x, a, h, iters, p.pre_scaller, p.writable_var, p.maxv, scan, sink, ns);
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
    return count > p.cap ? p.cap : count;  // cannot clip: cap covers the largest count
}

}  // namespace ucbdev

extern "C" __global__ void UCB_LAUNCH_BOUNDS ucb_bif2d_kernel(const UcbBif2dParams p) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    numb* slot = p.peaks + warp * 32 * (long long)p.cap;
    int* lab = p.work + warp * 2 * (long long)p.cap;
    int* stk = lab + p.cap;
    long long ns = 0;
    for (;;) {
        const long long base = ucbdev::warp_fetch(p.counter, lane);
        if (base >= p.total) break;
        const long long i = base + lane;
        const int count = i < p.total ? ucbdev::bif2d_peaks(p, i, slot + (long long)lane * p.cap, ns) : 0;
        __syncwarp();
        int mine = 0;
        for (int c = 0; c < 32; ++c) {
            if (base + c >= p.total) break;
            const int P = __shfl_sync(0xFFFFFFFFu, count, c);
            const int period = ucbdev::dbscan_warp(slot + (long long)c * p.cap, P, lab, stk, p.eps, lane);
            if (lane == c) mine = period;
        }
        if (i < p.total) {
            long long out = i;
            if (p.swap_xy) out = (i % p.n_pts) * p.n_pts + i / p.n_pts;
            p.out_values[out] = mine < 0 ? -1.0 : (double)mine;
            p.out_flags[out] = mine < 0 ? -1 : 1;
        }
        __syncwarp();
    }
    ucbdev::warp_add_steps(p.steps, ns, lane);
}
#endif  // UCB_BIF2D

