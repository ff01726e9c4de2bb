// ucb_basins.cuh — basins of attraction by stroboscopic classification (NVRTC header).
//
// New semantics (the reference labels basins by DBSCAN over peak features,
// parametric_engine.cpp:6035-6440): every initial-condition cell is integrated one forcing
// period (steps_per_period RK4 steps) at a time; the stroboscopic point P_n (all state
// variables except the phase variable) is compared with P_{n-k}, k = 1..UCB_MAXK. A cell
// converges when, for the smallest k, |P_n - P_{n-k}|_inf < tol holds for `need`
// consecutive periods; it then exits early and its attractor is identified by the period
// k and a canonical point of the cycle (the stroboscopic point with the smallest first
// coordinate). Attractors are registered in a small open-addressing table keyed by the
// quantised canonical point; the host merges table entries closer than the merge radius
// and maps them to labels 1..L ordered by (period, point). Label 0: no convergence within
// max_periods; -1: diverged. The phase variable (if any) is reset to its initial value
// after every period, so its value never grows (exact forcing phase in any precision).
#pragma once

#ifndef UCB_MAXK
#define UCB_MAXK 8
#endif
#ifndef UCB_PHASE
#define UCB_PHASE -1
#endif

struct UcbBasinsParams {
    long long total;
    int n_pts;
    int steps_per_period;
    int max_periods;
    int need;                  // consecutive matches required
    int table_slots;           // power of two
    int pad0;
    numb h, maxv, tol;
    double quantum;            // key quantisation of the canonical point
    numb ic[UCB_NX];
    numb vals[UCB_NV];
    const numb* axis0;         // values of the X-axis state variable (UCB_IDX0)
    const numb* axis1;         // values of the Y-axis state variable (UCB_IDX1)
    int* out_labels;           // provisional: slot + 1, 0 unresolved, -1 diverged
    int* out_periods;          // detected period, 0 / -1 as above
    int* out_iters;            // periods integrated
    unsigned long long* table_keys;   // table_slots, 0 = empty
    double* table_points;      // table_slots x 2 (canonical point of the first registrant)
    int* table_period;         // table_slots
    int* overflow;             // set when the table is full
    unsigned long long* counter;
    unsigned long long* steps;
    // Native form with a forcing phase (UCB_TRIG_PHASE == UCB_PHASE): (cos, sin) of the
    // phase at ic + rate * m * h / 2, m = 0 .. 2 steps_per_period (the phase restarts every
    // period, so a step's three stage phases are the same in every period and cell); null:
    // the step evaluates them itself.
    const numb* trig;
};

namespace ucbdev {

#define UCB_NS (UCB_PHASE >= 0 ? UCB_NX - 1 : UCB_NX)

__device__ __forceinline__ void strobe_point(const numb* x, numb* p) {
    int j = 0;
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) {
        if (i == UCB_PHASE) continue;
        p[j++] = x[i];
    }
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Registers (period, canonical point) and returns slot + 1, or 0 if the table is full.
__device__ __forceinline__ int register_attractor(const UcbBasinsParams& p, int period, double cx, double cy) {
    const long long qx = (long long)llround(cx / p.quantum), qy = (long long)llround(cy / p.quantum);
    unsigned long long key = mix64((unsigned long long)qx * 0x9E3779B97F4A7C15ULL ^ mix64((unsigned long long)qy) ^
                                   ((unsigned long long)period << 56));
    if (key == 0) key = 1;
    const unsigned mask = (unsigned)p.table_slots - 1;
    unsigned slot = (unsigned)(key & mask);
    for (int probe = 0; probe < p.table_slots; ++probe) {
        const unsigned long long prev = atomicCAS(&p.table_keys[slot], 0ULL, key);
        if (prev == 0ULL) {
            p.table_points[2 * slot] = cx;
            p.table_points[2 * slot + 1] = cy;
            p.table_period[slot] = period;
            return (int)slot + 1;
        }
        if (prev == key) return (int)slot + 1;
        slot = (slot + 1) & mask;
    }
    atomicExch(p.overflow, 1);
    return 0;
}

__device__ __forceinline__ void basins_cell(const UcbBasinsParams& p, long long cell, long long& ns) {
    const CellAxes c = cell_axes(cell, p.n_pts);
    numb x[UCB_NX], a[UCB_NV];
#pragma unroll
    for (int i = 0; i < UCB_NX; ++i) x[i] = p.ic[i];
#pragma unroll
    for (int i = 0; i < UCB_NV; ++i) a[i] = p.vals[i];
    x[UCB_IDX0] = p.axis0[c.i0];
    x[UCB_IDX1] = p.axis1[c.i1];
    const Stepper st(p.h);
    numb hist[UCB_MAXK][UCB_NS];  // hist[j] = P_{n-1-j} (shift register, static indices)
    int run[UCB_MAXK];
#pragma unroll
    for (int k = 0; k < UCB_MAXK; ++k) run[k] = 0;
    int label = 0, period = 0, n = 0;
    for (n = 1; n <= p.max_periods; ++n) {
#if defined(UCB_TRIG_PHASE) && !defined(UCB_EXACT) && UCB_PHASE == UCB_TRIG_PHASE
        if (p.trig) {
            UCB_STEP_LOOP
            for (int s = 0; s < p.steps_per_period; ++s) st.step_trig(x, a, p.h, p.trig + 4 * s);
        } else
#endif
        {
            UCB_STEP_LOOP
            for (int s = 0; s < p.steps_per_period; ++s) st.step(x, a, p.h);
        }
        ns += p.steps_per_period;
#if UCB_PHASE >= 0
        x[UCB_PHASE] = p.ic[UCB_PHASE];
#endif
        if (diverged(x, p.maxv)) {
            label = -1;
            period = -1;
            break;
        }
        numb P[UCB_NS];
        strobe_point(x, P);
        int found = 0;
#pragma unroll
        for (int k = 1; k <= UCB_MAXK; ++k) {
            if (n > k) {
                numb d = 0;
#pragma unroll
                for (int i = 0; i < UCB_NS; ++i) d = fmax(d, fabs(P[i] - hist[k - 1][i]));
                run[k - 1] = (d < p.tol) ? run[k - 1] + 1 : 0;
                if (!found && run[k - 1] >= p.need) found = k;
            }
        }
        if (found) {
            // A cycle that repeats after a divisor d of its length to within the merge
            // radius is the period-d orbit (a rounding-level cycle around a fixed point of
            // the stroboscopic map, as FP32 can settle into, counts as that fixed point).
            bool reduced = false;
#pragma unroll
            for (int d = 1; d < UCB_MAXK; ++d) {
                if (!reduced && d < found && found % d == 0) {
                    numb dd = 0;
#pragma unroll
                    for (int i = 0; i < UCB_NS; ++i) dd = fmax(dd, fabs(P[i] - hist[d - 1][i]));
                    if ((double)dd <= p.quantum) {
                        found = d;
                        reduced = true;
                    }
                }
            }
            period = found;
            // canonical point: the smallest first coordinate (then second) of the cycle
            // P_n, P_{n-1}, ..., P_{n-k+1}
            double cx = (double)P[0];
            double cy = UCB_NS > 1 ? (double)P[UCB_NS > 1 ? 1 : 0] : 0.0;
#pragma unroll
            for (int j = 0; j < UCB_MAXK - 1; ++j) {
                if (j + 1 < found) {
                    const double px = (double)hist[j][0];
                    const double py = UCB_NS > 1 ? (double)hist[j][UCB_NS > 1 ? 1 : 0] : 0.0;
                    if (px < cx || (px == cx && py < cy)) {
                        cx = px;
                        cy = py;
                    }
                }
            }
            label = register_attractor(p, period, cx, cy);
            break;
        }
#pragma unroll
        for (int j = UCB_MAXK - 1; j > 0; --j)
#pragma unroll
            for (int i = 0; i < UCB_NS; ++i) hist[j][i] = hist[j - 1][i];
#pragma unroll
        for (int i = 0; i < UCB_NS; ++i) hist[0][i] = P[i];
    }
    p.out_labels[cell] = label;
    p.out_periods[cell] = period;
    p.out_iters[cell] = n > p.max_periods ? p.max_periods : n;
}

}  // namespace ucbdev

extern "C" __global__ void UCB_LAUNCH_BOUNDS ucb_basins_kernel(const UcbBasinsParams p) {
    const int lane = threadIdx.x & 31;
    long long ns = 0;
    for (;;) {
        const long long base = ucbdev::warp_fetch(p.counter, lane);
        if (base >= p.total) break;
        const long long i = base + lane;
        if (i < p.total) ucbdev::basins_cell(p, i, ns);
    }
    ucbdev::warp_add_steps(p.steps, ns, lane);
}

// Provisional slot labels -> final labels (map[slot] for slot + 1 > 0).
extern "C" __global__ void ucb_basins_remap(int* labels, long long total, const int* map) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int l = labels[i];
        if (l > 0) labels[i] = map[l - 1];
    }
}
