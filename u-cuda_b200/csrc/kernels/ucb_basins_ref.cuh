// ucb_basins_ref.cuh — basin features of the reference method (NVRTC header, after
// ucb_device.cuh and ucb_bif.cuh compiled with UCB_BIF_NO_KERNELS).
//
// run_basins (parametric_engine.cpp:6035-6510) integrates every initial-condition cell
// (calculateDiscreteModelCUDA with par_or_var = 0), writes its whole recorded series to
// HBM, and avgPeakFinderCUDA (cudaLibrary.cu:3353-3425) reduces it to a class (1
// oscillating, -1 fixed point, 0 unbound) and two features. Here the recorded samples go
// through the streaming peakFinder of ucb_bif.cuh straight into running sums, so a cell
// costs its integration and 12 bytes of output (class + two features); the clustering of
// the features runs afterwards (basins_ref.cu).
#pragma once

struct UcbBasinsRefParams {
    long long total;           // cells (n_pts^2)
    int n_pts;
    int pre_scaller;
    int writable_var;
    int feature1, feature2;    // BF_* feature kinds (0..11)
    int pad0;
    long long skip;            // (int)(transient / h)
    long long points;          // (int)(tMax / h / preScaller)
    numb h, maxv, mult1, mult2, time_step;
    numb ic[UCB_NX];
    numb vals[UCB_NV];
    const numb* axis0;         // values of the X-axis initial condition
    const numb* axis1;         // values of the Y-axis initial condition
    double* out_f1;            // feature 1 (avg_peaks)
    double* out_f2;            // feature 2 (avg_intervals)
    int* out_class;            // 1 oscillating, -1 fixed point, 0 unbound
    unsigned long long* counter;
    unsigned long long* steps;
};

namespace ucbdev {

// What compute_basin_feature needs of the peaks / intervals (feature_needs).
__device__ __forceinline__ void basin_needs(int f, bool& sp, bool& sp2, bool& si, bool& si2) {
    sp = sp2 = si = si2 = false;
    switch (f) {
        case 0: case 6: sp = true; break;
        case 1: case 7: si = true; break;
        case 2: case 8: sp2 = true; break;
        case 3: case 9: si2 = true; break;
        case 4: case 10: sp = sp2 = true; break;
        case 5: case 11: si = si2 = true; break;
        default: break;
    }
}

__device__ __forceinline__ numb basin_feature(int f, numb mp, numb mi, numb rp, numb ri, numb sp, numb si) {
    switch (f) {
        case 0: return mp;
        case 1: return mi;
        case 2: return rp;
        case 3: return ri;
        case 4: return sp;
        case 5: return si;
        case 6: return mp == (numb)0 ? (numb)0 : (mp > 0 ? log10(mp) : -log10(-mp));
        case 7: return mi == (numb)0 ? (numb)0 : (mi > 0 ? log10(mi) : -log10(-mi));
        case 8: return rp > 0 ? log10(rp) : (numb)-999;
        case 9: return ri > 0 ? log10(ri) : (numb)-999;
        case 10: return sp > 0 ? log10(sp) : (numb)-999;
        case 11: return si > 0 ? log10(si) : (numb)-999;
        default: return (numb)-999;
    }
}

// Running sums of the first max_amount_of_peaks peaks / intervals (the count the
// reference's peakFinder returns).
struct BasinSums {
    bool nsp, nsp2, nsi, nsi2;
    numb time_step;
    mutable numb sp, sp2, si, si2;
    __device__ __forceinline__ void put(int k, numb value, numb dt) const {
        if (k >= kMaxAmountOfPeaks) return;
        if (nsp || nsp2) {
            if (nsp) sp += value;
            if (nsp2) sp2 += value * value;
        }
        if (nsi || nsi2) {
            const numb iv = (numb)dt * time_step;
            if (nsi) si += iv;
            if (nsi2) si2 += iv * iv;
        }
    }
};

__device__ __forceinline__ void basins_ref_cell(const UcbBasinsRefParams& p, long long cell, long long& ns) {
    const CellAxes c = cell_axes(cell, p.n_pts);
    numb x[UCB_NX], a[UCB_NV];
#pragma unroll
    for (int k = 0; k < UCB_NX; ++k) x[k] = p.ic[k];
#pragma unroll
    for (int k = 0; k < UCB_NV; ++k) a[k] = p.vals[k];
    apply_sweep(c, p.axis0, p.axis1, x, a);
    const Stepper st(p.h);
    numb f1, f2;
    int flag = loop_transient(st, x, a, p.h, p.skip, p.pre_scaller, p.maxv, ns);
    BasinSums sums;
    bool a1, a2, a3, a4, b1, b2, b3, b4;
    basin_needs(p.feature1, a1, a2, a3, a4);
    basin_needs(p.feature2, b1, b2, b3, b4);
    sums.nsp = a1 || b1;
    sums.nsp2 = a2 || b2;
    sums.nsi = a3 || b3;
    sums.nsi2 = a4 || b4;
    sums.time_step = p.time_step;
    sums.sp = sums.sp2 = sums.si = sums.si2 = 0;
    PeakScan scan;
    scan.init();
    scan.d1 = scan.d2 = 0;
    if (flag == 1 || flag == -1) flag = loop_record(st, x, a, p.h, p.points, p.pre_scaller, p.writable_var, p.maxv,
                                                     scan, sums, ns);
    if (flag == 0) {
        f1 = 999;
        f2 = 999;
    } else if (flag == -1) {
        f1 = scan.d2;  // the last recorded sample
        f2 = (numb)-1.0;
    } else {
        int n = (scan.found > 1) ? scan.found - 1 : 0;
        if (n >= kMaxAmountOfPeaks) n = kMaxAmountOfPeaks;
        if (p.points < 5) n = 0;
        if (n <= 0) {
            f1 = -999;
            f2 = (numb)-1.0;
        } else {
            const numb inv = (numb)1.0 / (numb)n;
            const numb mp = sums.nsp ? sums.sp * inv : (numb)0;
            const numb mi = sums.nsi ? sums.si * inv : (numb)0;
            const numb rp = sums.nsp2 ? sqrt(sums.sp2 * inv) : (numb)0;
            const numb ri = sums.nsi2 ? sqrt(sums.si2 * inv) : (numb)0;
            numb sdp = 0, sdi = 0;
            if (sums.nsp && sums.nsp2) {
                const numb v = sums.sp2 * inv - mp * mp;
                sdp = sqrt(v < 0 ? (numb)0 : v);
            }
            if (sums.nsi && sums.nsi2) {
                const numb v = sums.si2 * inv - mi * mi;
                sdi = sqrt(v < 0 ? (numb)0 : v);
            }
            f1 = p.mult1 * basin_feature(p.feature1, mp, mi, rp, ri, sdp, sdi);
            f2 = p.mult2 * basin_feature(p.feature2, mp, mi, rp, ri, sdp, sdi);
        }
    }
    p.out_f1[cell] = (double)f1;
    p.out_f2[cell] = (double)f2;
    p.out_class[cell] = flag;
}

}  // namespace ucbdev

extern "C" __global__ void UCB_LAUNCH_BOUNDS ucb_basins_ref_kernel(const UcbBasinsRefParams p) {
    const int lane = threadIdx.x & 31;
    long long ns = 0;
    for (;;) {
        const long long base = ucbdev::warp_fetch(p.counter, lane);
        if (base >= p.total) break;
        const long long i = base + lane;
        if (i < p.total) ucbdev::basins_ref_cell(p, i, ns);
    }
    ucbdev::warp_add_steps(p.steps, ns, lane);
}
