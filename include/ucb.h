/*
 * ucb.h — C ABI of the B200 engine for the per-cell integration hot path of U-CUDA.
 *
 * It replaces, for that path, the reference's C++ facade `class ParametricEngine`
 * (parametric_engine.h:844-889) and its request/result structs. Plain C types only:
 * pointers, sizes, doubles; no C++ or torch types cross this boundary.
 *
 * Conventions shared by every run_* entry point (the reference's error behaviour,
 * parametric_engine.cpp:2589-2600 and the *_CHECK macros at :2766-2786):
 *   - nothing throws across the ABI; a failure sets result->ok = 0 and a message in
 *     result->error, and the call returns a non-zero UCB_E* code;
 *   - a set *cancel ends the call with result->cancelled = 1 and UCB_E_CANCELLED. It is
 *     checked before the first launch and, while the map runs, mirrored into the kernels'
 *     run control: warps take no more cells from the work queue (an adaptive DP5 cell also
 *     abandons its steps), so the call returns after the cells in flight;
 *   - *progress (if non-NULL) is written with a value in [0, 1] while the call waits for
 *     the map (the share of cells handed out by the work queue) and 1 at the end;
 *   - output arrays are allocated by the caller with the sizes documented per call;
 *   - one engine may be driven from one host thread at a time (the reference's
 *     session layer enforces the same, analysis_session.cpp:918-966).
 *
 * The C++ header include/ucb_parametric_engine.hpp wraps these calls behind the
 * reference's exact ParametricEngine signatures.
 */
#ifndef UCB_H_
#define UCB_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UCB_ABI_VERSION 1

#if defined(__GNUC__)
#define UCB_API __attribute__((visibility("default")))
#else
#define UCB_API
#endif

/* Return codes */
#define UCB_OK 0
#define UCB_E_INVALID 1   /* request validation failed (message in result->error) */
#define UCB_E_COMPILE 2   /* the step body or a kernel did not compile */
#define UCB_E_CUDA 3      /* CUDA runtime/driver error */
#define UCB_E_CANCELLED 4 /* *cancel was set */
#define UCB_E_NOGPU 5     /* no CUDA device / driver */

/* Arithmetic of the integrator.
 *   UCB_PREC_F64: plain form, FP64 throughout (the oracle precision).
 *   UCB_PREC_F32: FP32 state; tangent-vector norms, log sums and step control in FP64. */
#define UCB_PREC_F64 0
#define UCB_PREC_F32 1

/* How the KRS step body is used.
 *   UCB_MODE_NATIVE: the right-hand side is recognised in the body (codegen RK4 template)
 *     and integrated by the engine's FMA-ordered RK4; bodies that are not a recognised
 *     template fall back to UCB_MODE_EXACT automatically.
 *   UCB_MODE_EXACT: the body is spliced verbatim (as the reference does) and compiled
 *     without FMA contraction: bit-identical trajectories to the krs_cpu CPU path. */
#define UCB_MODE_NATIVE 0
#define UCB_MODE_EXACT 1

/* LLE algorithm: shadow trajectory at distance eps (the reference's Benettin method),
 * or the tangent-linear vector (needs a recognised right-hand side). AUTO picks the
 * shadow for FP64 and the tangent vector for FP32. */
#define UCB_LLE_AUTO 0
#define UCB_LLE_SHADOW 1
#define UCB_LLE_TANGENT 2

typedef struct ucb_options {
    int32_t precision;   /* UCB_PREC_* */
    int32_t mode;        /* UCB_MODE_* */
    int32_t lle_method;  /* UCB_LLE_* */
    int32_t nominal_steps; /* 0: reference step counts (extra step after every loop call,
                              cudaLibrary.cu:863-866); 1: nominal counts */
    /* Launch shape. 0 in a field: the value an earlier ucb_autotune_* call chose for this
     * kernel build on this device (kept by the engine and in the table beside the CUBIN
     * cache), else the default (128 threads, the compiler's register choice, 1 step per
     * chunk). Set explicitly, a field overrides the tuned value. None changes results. */
    int32_t block_threads; /* threads per block, multiple of 32, 32..1024 */
    int32_t max_registers; /* registers per thread cap, 0 = compiler's choice; applied as the
                              resident blocks per SM it allows (__launch_bounds__ minimum
                              blocks), so the build may use fewer registers than the cap */
    int32_t unroll;        /* steps per unrolled chunk of the run-time-length step loops, 1..16 */
    int32_t paired_cells;  /* 1: the FP32 tangent LLE kernel integrates two cells per thread in
                              packed FP32 pairs (FFMA2 / FADD2 / FMUL2; bit-identical results).
                              Off by default: on B200 it measured 12 % slower than one cell per
                              thread (fewer resident warps, FFMA2 pipe rate 94 % of FFMA) */
} ucb_options;

typedef struct ucb_engine ucb_engine;

/* Outcome of an autotuning search (ucb_autotune_*; no reference counterpart): the launch
 * shape chosen for one kernel build and what it measured on the trial workload (the
 * request's own kernel on a coarser grid over the same window with a shortened horizon). */
typedef struct ucb_tune_report {
    int32_t block_threads, max_registers, unroll;
    int32_t candidates;        /* configurations timed */
    int32_t registers;         /* registers per thread of the chosen build */
    int32_t blocks_per_sm;     /* resident blocks per SM of the chosen build */
    double best_ms;            /* trial kernel time, chosen shape */
    double default_ms;         /* trial kernel time, default shape */
    double wall_ms;            /* whole search, compiles included */
    int32_t trial_n_pts;       /* trial grid */
    int32_t from_table;        /* 1: found in the tuned table, nothing timed */
    char key[32];              /* kernel build identity (hash) */
    char error[256];
    /* When the trial's winner is not the default shape, both are timed again on a
     * confirmation workload (the request itself when one run of it takes about a second or
     * less, else its window at the full horizon on a smaller grid); the winner is kept only if
     * it still wins by 2 %. 0 when no confirmation ran. */
    double confirm_default_ms, confirm_best_ms;
    int32_t confirm_n_pts;
    int32_t pad0;
} ucb_tune_report;

/* Creates an engine bound to CUDA device `device` (the reference always uses device 0,
 * parametric_engine.cpp:1490). Creation needs no GPU: the device is initialised by the
 * first run_* call, which reports UCB_E_NOGPU when it cannot be used. */
UCB_API ucb_engine* ucb_create(int device);
UCB_API void ucb_destroy(ucb_engine* e);
UCB_API const char* ucb_last_error(const ucb_engine* e);
UCB_API int ucb_abi_version(void);
/* Number of kernels this engine has launched so far (all entry points). */
UCB_API long long ucb_kernel_launches(const ucb_engine* e);
/* Clears the compiled-module cache (the reference's release_*_module()). */
UCB_API void ucb_clear_cache(ucb_engine* e);
UCB_API void ucb_default_options(ucb_options* o);

/* ------------------------------------------------------------------------------------
 * LLE 2D — replaces ParametricEngine::run_lle_2d(const LLE2DRequest&) -> LLE2DResult
 * (parametric_engine.h:411-482, :871; implementation parametric_engine.cpp:2587-2965).
 * Field meaning is the reference's: param_index* are 1-based indices into base_values
 * (a[0] reserved), var_sweep_index* are 0-based into initial_conditions.
 * ---------------------------------------------------------------------------------- */
typedef struct ucb_lle2d_request {
    const char* krs_body;
    int32_t amount_of_x;
    const double* initial_conditions; /* amount_of_x */
    const double* base_values;        /* n_values (<= 64) */
    int32_t n_values;
    int32_t sweep_over_var, sweep_over_var_2;
    int32_t sweep_over_h, sweep_over_h_2;
    int32_t log_scale, log_scale_2;
    int32_t param_index, var_sweep_index, param_index_2, var_sweep_index_2;
    double param_lo, param_hi, param_lo_2, param_hi_2;
    int32_t n_pts;
    double h, transient_time, t_max, NT, eps, max_value;
    const char* csv_output_path;      /* NULL or "" = no CSV */
    const volatile int32_t* cancel;   /* NULL = no cancellation */
    volatile float* progress;         /* NULL = no progress reporting */
    ucb_options opt;
} ucb_lle2d_request;

typedef struct ucb_lle2d_result {
    /* caller-allocated outputs, n_pts * n_pts each, row-major values[iy*n_pts + ix] */
    double* values;   /* lambda; the reference's sentinel 999 is kept (flag -1) */
    int32_t* flags;   /* 1 ok, -1 diverged */
    /* filled by the call */
    int32_t ok, cancelled, n_pts;
    double param_lo, param_hi, param_lo_2, param_hi_2;
    double min_val, max_val;          /* over cells with flag >= 0 and finite value */
    double kernel_ms;                 /* device time of the integrator kernel(s) */
    long long steps;                  /* step-function evaluations performed (work count) */
    double flops;                     /* algorithmic FLOPs of those steps (0 if unknown) */
    char error[1024];
} ucb_lle2d_result;

UCB_API int ucb_run_lle2d(ucb_engine* e, const ucb_lle2d_request* req, ucb_lle2d_result* res);

/* Device-resident form of ucb_run_lle2d for callers that keep outputs in HBM: enqueues
 * the work on `stream` (a cudaStream_t, NULL = default stream) and returns without
 * synchronising. d_values / d_flags are device pointers of n_pts*n_pts elements. No
 * CSV, no min/max; res->error/ok report validation and launch errors only. */
UCB_API int ucb_lle2d_device(ucb_engine* e, const ucb_lle2d_request* req, double* d_values, int32_t* d_flags,
                     void* stream, ucb_lle2d_result* res);

/* ------------------------------------------------------------------------------------
 * Bifurcation 2D (period maps) — replaces ParametricEngine::run_bifurcation_2d
 * (parametric_engine.h:861, implementation parametric_engine.cpp:5487-5910): per cell of
 * an n_pts x n_pts grid (same sweep fields and axis mapping as the LLE 2D request) the
 * trajectory and peaks of the 1-D diagram, then the reference's per-cell dbscan of the
 * peak values (cudaLibrary.cu:2088-2166, eps_dbscan; intervals weigh 0) whose result is
 * the cell's "period". values[iy*n + ix] = period, -1 with flag -1 where the dbscan result
 * is negative (the fixed-point flag of the trajectory); 0 = no peaks / diverged.
 * ---------------------------------------------------------------------------------- */
typedef struct ucb_bif2d_request {
    const char* krs_body;
    int32_t amount_of_x;
    const double* initial_conditions;
    const double* base_values;
    int32_t n_values;
    int32_t sweep_over_var, sweep_over_var_2;
    int32_t sweep_over_h, sweep_over_h_2;
    int32_t log_scale, log_scale_2;
    int32_t param_index, var_sweep_index, param_index_2, var_sweep_index_2;
    double param_lo, param_hi, param_lo_2, param_hi_2;
    int32_t n_pts;
    int32_t writable_var;     /* recorded variable; -1 = x0 + pi x1 + e x2 */
    double h, transient_time, t_max;
    int32_t pre_scaller;
    double max_value;
    double eps_dbscan;        /* > 0 */
    const char* csv_output_path;
    const volatile int32_t* cancel;
    volatile float* progress;
    ucb_options opt;
} ucb_bif2d_request;

typedef struct ucb_bif2d_result {
    double* values;   /* caller-allocated, n_pts * n_pts */
    int32_t* flags;   /* caller-allocated, n_pts * n_pts: 1 ok, -1 */
    int32_t ok, cancelled, n_pts;
    double param_lo, param_hi, param_lo_2, param_hi_2;
    double min_val, max_val;  /* over cells with flag >= 0 and value >= 0 */
    double kernel_ms;
    long long steps;
    double flops;
    char error[1024];
} ucb_bif2d_result;

UCB_API int ucb_run_bif2d(ucb_engine* e, const ucb_bif2d_request* req, ucb_bif2d_result* res);
UCB_API int ucb_precompile_bif2d(const ucb_bif2d_request* req, char* err_out, int err_len);

/* ------------------------------------------------------------------------------------
 * LLE 1D / LS 1D — replace ParametricEngine::run_lle_1d and run_ls_1d
 * (parametric_engine.h:864-867, implementations parametric_engine.cpp:2196 and :3066):
 * the LLE / spectrum kernels over n_pts values of one swept parameter, initial condition
 * (sweep_over_var) or step h (sweep_over_h). The continuation branch of the reference
 * (sequential by construction) is not part of this path.
 * ---------------------------------------------------------------------------------- */
typedef struct ucb_lle1d_request {
    const char* krs_body;
    int32_t amount_of_x;
    const double* initial_conditions;
    const double* base_values;
    int32_t n_values;
    int32_t sweep_over_var;   /* sweep initial condition var_sweep_index (0-based) */
    int32_t var_sweep_index;
    int32_t sweep_over_h;     /* sweep the step h over [param_lo, param_hi] */
    int32_t log_scale;
    int32_t param_index;      /* 1-based a[] index (parameter sweep) */
    double param_lo, param_hi;
    int32_t n_pts;
    double h, transient_time, t_max, NT, eps, max_value;
    const char* csv_output_path;
    const volatile int32_t* cancel;
    volatile float* progress;
    ucb_options opt;
} ucb_lle1d_request;
typedef ucb_lle1d_request ucb_ls1d_request;

typedef struct ucb_lle1d_result {
    double* values;   /* n_pts: lambda; NaN where the kernel returned 999 / -999 (flag -1),
                         as run_lle_1d does (parametric_engine.cpp:2455-2466) */
    int32_t* flags;   /* 1 ok, -1 diverged */
    int32_t ok, cancelled, n_pts;
    double param_lo, param_hi;
    double kernel_ms;
    long long steps;
    double flops;
    char error[1024];
} ucb_lle1d_result;

typedef struct ucb_ls1d_result {
    double* values;   /* n_pts * amount_of_x, point-major values[i * N + k] (the reference's
                         spectrum[i][k]); the 999 / -999 sentinels are kept */
    int32_t* flags;   /* 1 ok, -1 diverged (from the first exponent, as the reference) */
    int32_t ok, cancelled, n_pts, n_exponents;
    double param_lo, param_hi;
    double kernel_ms;
    long long steps;
    double flops;
    char error[1024];
} ucb_ls1d_result;

UCB_API int ucb_run_lle1d(ucb_engine* e, const ucb_lle1d_request* req, ucb_lle1d_result* res);
UCB_API int ucb_run_ls1d(ucb_engine* e, const ucb_ls1d_request* req, ucb_ls1d_result* res);

/* ------------------------------------------------------------------------------------
 * Bifurcation 1D — replaces ParametricEngine::run_bifurcation_1d (parametric_engine.h:27-126,
 * :853; classical sweep of parametric_engine.cpp:1674-2091; the continuation branch is
 * sequential by construction and not part of this path).
 * ---------------------------------------------------------------------------------- */
typedef struct ucb_bif1d_request {
    const char* krs_body;
    int32_t amount_of_x;
    const double* initial_conditions;
    const double* base_values;
    int32_t n_values;
    int32_t param_index;      /* 1-based a[] index (parameter sweep) */
    int32_t sweep_over_var;   /* sweep initial condition var_sweep_index instead */
    int32_t var_sweep_index;
    int32_t sweep_over_h;     /* sweep the step h over [param_lo, param_hi] */
    int32_t log_scale;
    double param_lo, param_hi;
    int32_t n_pts;
    int32_t writable_var;     /* recorded variable; -1 = x0 + pi x1 + e x2 */
    double h, transient_time, t_max;
    int32_t pre_scaller;
    double max_value;
    int32_t max_peaks;        /* peaks/intervals kept per point (the reference keeps up to 2500) */
    const char* csv_output_path;
    const volatile int32_t* cancel;
    volatile float* progress;
    ucb_options opt;
} ucb_bif1d_request;

typedef struct ucb_bif1d_result {
    /* caller-allocated: counts[n_pts], peaks[n_pts * max_peaks], intervals[n_pts * max_peaks] */
    int32_t* counts;          /* the reference's flags[]: number of peaks (<= 2500), -1 fixed
                                 point, 0 diverged; peaks beyond max_peaks are counted, not stored */
    double* peaks;            /* peak values (first peak of the series dropped) */
    double* intervals;        /* inter-peak intervals (time units) */
    int32_t ok, cancelled, n_pts, record_steps;
    double param_lo, param_hi;
    double kernel_ms;
    long long steps;
    double flops;
    char error[1024];
} ucb_bif1d_result;

UCB_API int ucb_run_bif1d(ucb_engine* e, const ucb_bif1d_request* req, ucb_bif1d_result* res);
/* Compile-only (no GPU) counterpart, like ucb_precompile_lle2d. */
UCB_API int ucb_precompile_bif1d(const ucb_bif1d_request* req, char* err_out, int err_len);

/* ------------------------------------------------------------------------------------
 * Lyapunov spectrum 2D — replaces ParametricEngine::run_ls_2d(const LS2DRequest&)
 * (parametric_engine.h:581-648, :874; implementation parametric_engine.cpp:3430-3786).
 * Two methods:
 *   UCB_LS_FIXED — the reference's: fixed step h, N shadow probes at distance eps,
 *                  classical Gram-Schmidt every NT (LSKernelCUDA, cudaLibrary.cu:2878);
 *   UCB_LS_DP5   — adaptive Dormand-Prince 5(4) with N tangent-linear vectors and
 *                  modified Gram-Schmidt every gs_every accepted steps over the interval
 *                  [transient_time, transient_time + t_end]; needs a recognised RK4 body
 *                  (the right-hand side is taken from it). No reference counterpart.
 * ---------------------------------------------------------------------------------- */
#define UCB_LS_FIXED 0
#define UCB_LS_DP5 1

typedef struct ucb_ls2d_request {
    const char* krs_body;
    int32_t amount_of_x;
    const double* initial_conditions;
    const double* base_values;
    int32_t n_values;
    int32_t sweep_over_var, sweep_over_var_2;
    int32_t sweep_over_h, sweep_over_h_2;
    int32_t log_scale, log_scale_2;
    int32_t param_index, var_sweep_index, param_index_2, var_sweep_index_2;
    double param_lo, param_hi, param_lo_2, param_hi_2;
    int32_t n_pts;
    double h, transient_time, t_max, NT, eps, max_value;
    const char* csv_output_path;
    const volatile int32_t* cancel;
    volatile float* progress;
    ucb_options opt;
    /* method selection and the adaptive method's controls */
    int32_t method;          /* UCB_LS_FIXED / UCB_LS_DP5 */
    int32_t gs_every;        /* accepted steps between modified Gram-Schmidt passes (DP5) */
    double rtol, atol;       /* DP5 error tolerances (0 = 1e-8 / 1e-5 for FP64 / FP32, atol = rtol) */
    double t_end;            /* DP5 measured interval length (0 = t_max) */
    double h0;               /* DP5 initial step (0 = h) */
    long long max_steps;     /* DP5 cap on step attempts per cell (0 = 2 x 10^7); cells that hit
                                it are reported as diverged (999, flag -1) */
} ucb_ls2d_request;

typedef struct ucb_ls2d_result {
    double* values;          /* caller-allocated, amount_of_x * n_pts^2, plane-major
                                values[k * n_pts^2 + iy * n_pts + ix] */
    int32_t* flags;          /* n_pts^2: 1 ok, -1 diverged (sentinel 999 in every plane) */
    double* min_val;         /* amount_of_x (may be NULL) */
    double* max_val;         /* amount_of_x (may be NULL) */
    long long* cell_steps;   /* n_pts^2 (may be NULL): work per cell, as `steps` counts it
                                (no reference counterpart; the cost map of a run) */
    int32_t ok, cancelled, n_pts, n_exponents;
    double kernel_ms;
    long long steps;         /* FIXED: trajectory steps; DP5: step attempts */
    double flops;
    char error[1024];
} ucb_ls2d_result;

UCB_API int ucb_run_ls2d(ucb_engine* e, const ucb_ls2d_request* req, ucb_ls2d_result* res);
/* Compile-only (no GPU) counterpart, like ucb_precompile_lle2d. */
UCB_API int ucb_precompile_ls2d(const ucb_ls2d_request* req, char* err_out, int err_len);

/* ------------------------------------------------------------------------------------
 * Basins of attraction — replaces ParametricEngine::run_basins (parametric_engine.h:659-723,
 * :877) on this path with stroboscopic classification (no reference counterpart for the
 * labelling itself; the reference clusters peak features with DBSCAN, :6035-6440):
 * initial conditions (axis_x_var, axis_y_var) on an n_pts x n_pts grid, other variables
 * from initial_conditions; RK4 with step h = period / steps_per_period; a cell converges
 * when its stroboscopic point repeats with the smallest period k <= 8 to within match_tol
 * for match_count consecutive periods, and exits early; cap max_periods.
 * labels[iy*n + ix]: >= 1 attractor id (ordered by period, then canonical point), 0 not
 * converged within the cap, -1 diverged (max_value / NaN).
 * ---------------------------------------------------------------------------------- */
typedef struct ucb_basins_request {
    const char* krs_body;
    int32_t amount_of_x;
    const double* initial_conditions;
    const double* base_values;
    int32_t n_values;
    int32_t axis_x_var, axis_y_var;   /* 0-based state indices */
    double axis_x_lo, axis_x_hi, axis_y_lo, axis_y_hi;
    int32_t n_pts;
    double period;                    /* forcing period (stroboscope interval), > 0 */
    int32_t steps_per_period;         /* h = period / steps_per_period */
    int32_t max_periods;              /* cap (2000 in the benchmark configuration) */
    int32_t match_count;              /* consecutive period matches to converge (20) */
    double match_tol;                 /* max-norm match tolerance (1e-6); the FP32 form uses at
                                         least 1e-5 (FP32 resolves a stroboscopic point to ~1e-6) */
    int32_t phase_var;                /* state index of the forcing phase (reset every period), -1 none */
    double max_value;
    double merge_radius;              /* canonical points closer than this are one attractor (0 = 1e-4) */
    const char* csv_output_path;
    const volatile int32_t* cancel;
    volatile float* progress;
    ucb_options opt;
} ucb_basins_request;

#define UCB_BASINS_MAX_ATTRACTORS 256
typedef struct ucb_basins_result {
    int32_t* labels;                  /* caller-allocated n_pts^2 */
    int32_t* periods;                 /* caller-allocated n_pts^2 (may be NULL): period, 0, -1 */
    int32_t* iterations;              /* caller-allocated n_pts^2 (may be NULL): periods integrated */
    int32_t ok, cancelled, n_pts;
    int32_t n_attractors;
    int32_t attractor_period[UCB_BASINS_MAX_ATTRACTORS];
    double attractor_point[UCB_BASINS_MAX_ATTRACTORS][2];
    double kernel_ms;
    long long steps;
    double flops;
    char error[1024];
} ucb_basins_result;

UCB_API int ucb_run_basins(ucb_engine* e, const ucb_basins_request* req, ucb_basins_result* res);
UCB_API int ucb_precompile_basins(const ucb_basins_request* req, char* err_out, int err_len);

/* ------------------------------------------------------------------------------------
 * Basins of attraction by the reference's own method — replaces
 * ParametricEngine::run_basins (parametric_engine.h:659-723, BasinsRequest / BasinsResult;
 * parametric_engine.cpp:6035-6510) with the same request fields and results:
 * initial conditions (axis_x_var, axis_y_var) on an n_pts x n_pts grid (numb axis values),
 * the others from initial_conditions; integration of tMax / h / pre_scaller recorded
 * samples after (int)(transient_time / h) transient steps; per cell a class (1 oscillating,
 * -1 fixed point, 0 unbound) and two features of the peaks of writable_var (feature1 /
 * feature2: the BF_* kinds of configCUDA.h, 0 = mean peak, 1 = mean interval, ...; unknown
 * kinds give -999; times mult1 / mult2); then DBSCAN (minPts 1) of the features with
 * eps_dbscan. labels (basin_idx): >= 1 oscillating cluster, <= -1 a cluster that holds a
 * fixed point, 0 unbound; clusters numbered as the reference's seed order does (fixed-point
 * clusters by their lowest fixed-point cell, then the others by their lowest cell).
 * All four arrays row-major iy*n + ix, caller-allocated n_pts^2.
 * ---------------------------------------------------------------------------------- */
typedef struct ucb_basins_dbscan_request {
    const char* krs_body;
    int32_t amount_of_x;
    const double* initial_conditions;
    const double* base_values;
    int32_t n_values;
    int32_t axis_x_var, axis_y_var;   /* 0-based state indices, distinct */
    double axis_x_lo, axis_x_hi, axis_y_lo, axis_y_hi;
    int32_t n_pts;                    /* n_pts^2 <= 2^31 - 1 */
    int32_t writable_var;             /* peak variable, -1..amount_of_x-1 */
    double h, t_max, transient_time;
    int32_t pre_scaller;
    double max_value;
    double eps_dbscan;
    int32_t feature1, feature2;       /* BF_* kinds (reference defaults 0 and 1) */
    double mult1, mult2;              /* reference defaults 1 and 1 */
    const char* csv_output_path;
    const volatile int32_t* cancel;
    volatile float* progress;         /* 0..1 within the current phase */
    volatile int32_t* progress_phase; /* 1 integration, 2 clustering (may be NULL) */
    ucb_options opt;
} ucb_basins_dbscan_request;

typedef struct ucb_basins_dbscan_result {
    int32_t* labels;                  /* caller-allocated n_pts^2: basin_idx */
    double* avg_peaks;                /* caller-allocated n_pts^2: feature 1 (999 unbound) */
    double* avg_intervals;            /* caller-allocated n_pts^2: feature 2 */
    int32_t* classes;                 /* caller-allocated n_pts^2: helpful_array (1, -1, 0) */
    int32_t ok, cancelled, n_pts;
    int32_t n_clusters;               /* max label (oscillating clusters) */
    int32_t min_cluster_idx;          /* min label (-number of fixed-point clusters) */
    double avg_peaks_min, avg_peaks_max;          /* over finite values other than +-999 */
    double avg_intervals_min, avg_intervals_max;
    double kernel_ms;                 /* integration + features */
    double cluster_ms;                /* clustering */
    long long steps;
    char error[1024];
} ucb_basins_dbscan_result;

UCB_API int ucb_run_basins_dbscan(ucb_engine* e, const ucb_basins_dbscan_request* req,
                                  ucb_basins_dbscan_result* res);
UCB_API int ucb_precompile_basins_dbscan(const ucb_basins_dbscan_request* req, char* err_out, int err_len);

/* DBSCAN alone over given features — replaces ParametricEngine::run_basins_recluster
 * (parametric_engine.h:733-753, BasinsReclusterRequest / Result; parametric_engine.cpp:
 * 6523-6600): the clustering of ucb_run_basins_dbscan over caller features (mults already
 * applied) and classes, in the numb of opt.precision. */
typedef struct ucb_basins_recluster_request {
    const char* krs_body;             /* checked non-empty, as the reference does */
    int32_t amount_of_x;
    int32_t n_pts;
    double eps_dbscan;
    const double* avg_peaks;          /* n_pts^2 */
    const double* avg_intervals;      /* n_pts^2 */
    const int32_t* classes;           /* n_pts^2 helpful_array: -1 fixed point, 0 unbound, 1 oscillating */
    const volatile int32_t* cancel;
    volatile float* progress;
    ucb_options opt;
} ucb_basins_recluster_request;

typedef struct ucb_basins_recluster_result {
    int32_t* labels;                  /* caller-allocated n_pts^2: basin_idx */
    int32_t ok, cancelled, n_pts;
    int32_t n_clusters, min_cluster_idx;
    double cluster_ms;
    char error[1024];
} ucb_basins_recluster_result;

UCB_API int ucb_run_basins_recluster(ucb_engine* e, const ucb_basins_recluster_request* req,
                                     ucb_basins_recluster_result* res);

/* ------------------------------------------------------------------------------------
 * Autotuning (no reference counterpart). Searches the launch shape (threads per block,
 * register cap, steps per unrolled chunk; ucb_options) of the kernel build the request
 * would run: each candidate runs the request's own entry point on a trial workload (the
 * same window on a coarser grid, horizon shortened to about 1.2e10 steps; the Bif-2D trial
 * keeps the horizon), timed with CUDA events; coordinate descent, 2 % to win. The chosen
 * shape is used by later calls of any engine on this device whose option fields are 0
 * (it is kept by the engine and appended to the table beside the CUBIN cache). force = 0
 * returns a shape already in the table without timing anything. Results never change:
 * the shape is not part of the arithmetic.
 * ---------------------------------------------------------------------------------- */
UCB_API int ucb_autotune_lle2d(ucb_engine* e, const ucb_lle2d_request* req, int32_t force, ucb_tune_report* rep);
UCB_API int ucb_autotune_ls2d(ucb_engine* e, const ucb_ls2d_request* req, int32_t force, ucb_tune_report* rep);
UCB_API int ucb_autotune_basins(ucb_engine* e, const ucb_basins_request* req, int32_t force, ucb_tune_report* rep);
UCB_API int ucb_autotune_bif2d(ucb_engine* e, const ucb_bif2d_request* req, int32_t force, ucb_tune_report* rep);

/* LLE map without device allocation (no counterpart in the reference).
 *
 * ucb_lle2d_device() keeps its scratch (work-queue counter, step counter, axis value
 * tables) in an engine workspace that it cudaMalloc()s on first use. Callers that cannot
 * allocate device memory — applications that own all of it through their own pool or a
 * fixed pre-reserved budget, and time-critical loops that must not reach cudaMalloc /
 * cudaFree (cudaFree synchronises the device) — use this variant instead: the same
 * kernel, with its scratch in a fixed-size array inside this library that every GPU
 * loading the library holds until the process exits. The caller still provides
 * d_values / d_flags (n_pts * n_pts each).
 *
 * Limits and rules:
 *   - n_pts <= UCB_NOALLOC_MAX_PTS, otherwise UCB_E_INVALID with a message;
 *   - ucb_prepare_lle2d() must have been called on this engine for an equivalent request
 *     (same body, sizes, sweep kinds and options; the swept ranges, step and horizon may
 *     differ): it compiles and loads the kernel (which allocates), pins that kernel and
 *     its launch shape on the engine (a later autotune does not change what the
 *     allocation-free call launches), and looks up the scratch array's device address on
 *     the engine's device. Without it the call returns UCB_E_INVALID ("not prepared").
 *     After a cudaDeviceReset() in the process, call ucb_prepare_lle2d() again: it looks
 *     the address up anew;
 *   - the axis tables are passed to the device as kernel parameters and the counters are
 *     cleared with cudaMemsetAsync, all on `stream`, before the kernel;
 *   - all calls share the one array and it keeps the last call's contents; every call
 *     resets the counters it needs, but calls that overlap on the GPU (other streams,
 *     other engines in the process) race on it and must be serialised by the caller. */
#define UCB_NOALLOC_MAX_PTS 4096
UCB_API int ucb_prepare_lle2d(ucb_engine* e, const ucb_lle2d_request* req);
UCB_API int ucb_lle2d_device_noalloc(ucb_engine* e, const ucb_lle2d_request* req, double* d_values,
                                     int32_t* d_flags, void* stream, ucb_lle2d_result* res);

/* Trajectory parity aid: integrates every cell of the request's grid (same sweep
 * mapping, same step function and precision as ucb_run_lle2d) for n_steps plain steps
 * from its initial condition — no transient, no divergence checks, no extra step — and
 * writes the final states to out_states[cell * amount_of_x + i] (kernel cell order).
 * The reference has no counterpart; it checks its kernels against its CPU twins instead
 * (parametric_engine.cpp:593-616). Error text: ucb_last_error(). */
UCB_API int ucb_lle2d_states(ucb_engine* e, const ucb_lle2d_request* req, long long n_steps, double* out_states);

/* Measures the FMA throughput of the FP64 (precision = UCB_PREC_F64) or FP32 pipe of the
 * current device in TFLOP/s (2 FLOPs per FMA): the roofline denominator of the integrator
 * kernels; UCB_PEAK_F32X2 measures packed FP32 pairs (two FMAs per instruction, sm_100).
 * No reference counterpart (the reference publishes no measurements). */
#define UCB_PEAK_F32X2 2
UCB_API int ucb_measure_fma_peak(int precision, double* tflops);

/* ------------------------------------------------------------------------------------
 * Text front-end: replaces parse_system_from_latex (sysparse.hpp, sysparse.cpp:287) +
 * codegen_scheme (codegen.hpp, codegen.cpp:951). Parses a multi-line LaTeX / plain system
 * with a comma-separated alphabet (parameter order: alphabet, or first appearance when
 * order_as_in_system != 0; func_defs: optional "h(x) = ..." lines) and writes the step
 * body of `scheme` to out; vars_out / params_out (optional) receive comma-separated names
 * (variables map to X[i], parameters to a[1 + j]). On error returns UCB_E_INVALID and the
 * message in out.
 * ---------------------------------------------------------------------------------- */
#define UCB_SCHEME_EULER 0
#define UCB_SCHEME_EULER_CROMER 1
#define UCB_SCHEME_MIDPOINT 2
#define UCB_SCHEME_RK4 3
#define UCB_SCHEME_DOPRI78 4 /* Dormand-Prince 8(7), 13 stages (codegen.cpp:611-675) */
#define UCB_SCHEME_CD 5      /* composition D-method, symmetry coefficient a[0] (codegen.cpp:686-754) */
UCB_API int ucb_codegen(const char* text, const char* alphabet, int order_as_in_system, const char* func_defs,
                        int scheme, char* out, int out_len, char* vars_out, int vars_len, char* params_out,
                        int params_len);

/* Compiles the kernel a ucb_run_lle2d call with this request would use into the on-disk
 * CUBIN cache (<library dir>/_cache or $UCB_CUBIN_CACHE) without touching a GPU. The
 * reference's equivalent is compile_lle_2d_if_needed (parametric_engine.cpp:2487-2572),
 * which only has an in-memory PTX cache. err_out receives a compiler log or a note on
 * the form chosen. */
UCB_API int ucb_precompile_lle2d(const ucb_lle2d_request* req, char* err_out, int err_len);

/* LLE of an explicit list of cells of the request's grid (kernel cell order: cell =
 * iy * n_pts + ix before any swap), written compactly: d_values[i] / d_flags[i] belong to
 * d_cells[i]. Same kernel and semantics as ucb_lle2d_device; used for held-out subsets
 * and re-integration. No reference counterpart. */
UCB_API int ucb_lle2d_cells(ucb_engine* e, const ucb_lle2d_request* req, const long long* d_cells, long long n_cells,
                            double* d_values, int32_t* d_flags, void* stream, ucb_lle2d_result* res);

/* ------------------------------------------------------------------------------------
 * BF16 MLP surrogate (no counterpart in the reference). Input: a point u in [0, 1]^2 (the
 * two sweep coordinates of a map, normalised); Fourier features sin / cos(2 pi u B^T)
 * with a fixed Gaussian B (fourier x 2, std fourier_scale); `layers` hidden layers of
 * width `hidden` with GELU in its tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)));
 * outputs mean and log-variance of the target, trained on the Gaussian negative
 * log-likelihood (beta-NLL weighting: each row's loss is scaled by a constant
 * sigma^(2 beta)) with Adam and a cosine learning-rate decay. Matrix products run on the
 * tensor cores (tcgen05.mma, BF16 operands, FP32 accumulation in tensor memory); masters
 * and Adam moments are FP32. Training adds every partial sum in a fixed order (no
 * floating-point atomics): a fit gives the same parameters bit for bit on every run.
 * Prediction is one fused kernel per call when hidden is 128 or 256 and 2 * fourier <=
 * hidden (features, every layer and the output of 128 rows in one CTA, activations in
 * shared memory); other shapes run layer by layer.
 *
 * Parameter vector layout (ucb_mlp_get_params): for each layer l = 0..layers (the last is
 * the output layer with 2 outputs), W_l[out][in] row-major, then b_l[out].
 * ---------------------------------------------------------------------------------- */
typedef struct ucb_mlp_config {
    int32_t fourier;        /* frequencies; 2 * fourier must be a multiple of 128 (default 64) */
    int32_t hidden;         /* hidden width, a multiple of 128 (default 256) */
    int32_t layers;         /* hidden layers, 1..8 (default 4) */
    float fourier_scale;    /* std of the frequency matrix entries (default 3) */
    uint64_t seed;          /* initialisation, frequency matrix and mini-batch sampling (default 0) */
    int32_t batch;          /* rows per Adam step, a multiple of 128 (default 8192) */
    int32_t train_steps;    /* Adam steps of ucb_mlp_fit (default 1500) */
    float lr;               /* initial learning rate (default 2e-3) */
    float lr_final;         /* learning rate at the last step, cosine decay (default 2e-5) */
    float beta_nll;         /* 0 = plain Gaussian NLL, 1 = mean-squared-error-like (default 0.5) */
    int32_t reserved[5];
} ucb_mlp_config;

typedef struct ucb_mlp ucb_mlp;

UCB_API void ucb_mlp_default_config(ucb_mlp_config* c);
/* Creates the network on the engine's device (parameters initialised from cfg->seed).
 * NULL on failure (message: ucb_last_error(e)). */
UCB_API ucb_mlp* ucb_mlp_create(ucb_engine* e, const ucb_mlp_config* cfg);
UCB_API void ucb_mlp_destroy(ucb_mlp* m);
UCB_API long long ucb_mlp_param_count(const ucb_mlp* m);
/* Host copies of the FP32 parameters (n = ucb_mlp_param_count) and of the frequency
 * matrix B (fourier x 2, row-major). set_params also refreshes the BF16 copies. */
UCB_API int ucb_mlp_get_params(ucb_mlp* m, float* out, long long n);
UCB_API int ucb_mlp_set_params(ucb_mlp* m, const float* in, long long n);
UCB_API int ucb_mlp_get_fourier(ucb_mlp* m, float* out, long long n);
/* Target standardisation (y - mean) / std used by the loss; predictions undo it.
 * ucb_mlp_fit sets it from the training targets. */
UCB_API int ucb_mlp_set_target_scale(ucb_mlp* m, float mean, float std);
/* Mean loss and its gradient with respect to every parameter (host array of
 * ucb_mlp_param_count) for the rows u (n x 2, host) with targets y (host), computed by the
 * training kernels (forward, loss, backward) without an update. */
UCB_API int ucb_mlp_loss_grad(ucb_mlp* m, const float* u, const float* y, long long n, float* loss, float* grad);
/* Trains on n rows (device arrays u: n x 2, y: n); loss_out: loss of the last step. */
UCB_API int ucb_mlp_fit(ucb_mlp* m, const float* d_u, const float* d_y, long long n, void* stream, float* loss_out);
/* Predicted mean and standard deviation for n rows (device arrays). */
UCB_API int ucb_mlp_predict(ucb_mlp* m, const float* d_u, long long n, float* d_mean, float* d_std, void* stream);

/* ------------------------------------------------------------------------------------
 * Surrogate-refined LLE map (no counterpart in the reference). The map of `map` (n =
 * map.n_pts) is computed as:
 *   1. samples: one cell drawn at random in each block of a train_pts x train_pts
 *      partition of the grid, integrated with sample_precision (UCB_PREC_F64: the plain
 *      method). A pilot subset (a 32^2..64^2 subgrid of the blocks) is integrated first;
 *      when a local plane fit through its neighbours predicts less than min_predictable of
 *      it at tol / coverage, no network is trained and every other cell is integrated with
 *      refine_precision (result->gated = 1). Otherwise the rest is integrated and one in
 *      eight samples (by a hash of the block; more, up to half, when that leaves fewer than
 *      1,024) is held out for calibration;
 *   2. the MLP (mlp) is trained on the others on this GPU;
 *   3. it predicts mean and standard deviation for every cell;
 *   4. calibration: the held-out samples, ordered by predicted std, give the largest std
 *      threshold below which the one-sided 90 % Wilson lower bound of the fraction within
 *      `tol` of their integrated value reaches `coverage` (capped by sigma_max when > 0);
 *   5. cells with std above the threshold, |mean| < lle_band, or a 4-neighbour in another
 *      regime (lambda < -lle_band, |lambda| <= lle_band, lambda > lle_band) or differing
 *      by more than jump (when jump > 0) are re-integrated with refine_precision straight
 *      into the map; sample cells keep their integrated value;
 *   6. every other cell takes the predicted mean.
 * flags: 1 integrated, 2 predicted, -1 diverged (as ucb_run_lle2d). Outputs are device
 * arrays of n * n in map order (as ucb_lle2d_device); phase times in the result.
 * ---------------------------------------------------------------------------------- */
typedef struct ucb_surrogate_request {
    ucb_lle2d_request map;
    int32_t train_pts;          /* samples per axis (default 256) */
    int32_t sample_precision;   /* default UCB_PREC_F64 (plain samples) */
    int32_t refine_precision;   /* precision of re-integrated cells (default UCB_PREC_F32) */
    int32_t pad0;
    double tol;                 /* error tolerance of a predicted cell (default 2e-3) */
    double coverage;            /* calibrated fraction within tol (default 0.995) */
    double sigma_max;           /* cap on the std threshold, 0 = none */
    double lle_band;            /* default 0.05; 0 = no band / regime rule */
    double jump;                /* default 0 = off */
    double min_predictable;     /* gate (default 0.05): the network is trained only when this share
                                   of the pilot samples (a 32^2..64^2 subgrid of the sample blocks,
                                   integrated first) is predictable from its neighbours at tol /
                                   coverage; otherwise every other cell is integrated in
                                   refine_precision */
    ucb_mlp_config mlp;
} ucb_surrogate_request;

typedef struct ucb_surrogate_result {
    int32_t ok;
    int32_t n_pts;
    long long n_samples, n_calib, n_refined, n_predicted, n_diverged;
    double sigma_threshold;     /* calibrated std threshold (-1: nothing predicted) */
    double calib_within_tol;    /* fraction of held-out samples under the threshold within tol */
    double pilot_predictable;   /* the gate's share of predictable pilot samples */
    int32_t gated;              /* 1: below min_predictable, no network trained */
    int32_t pad1;
    double sample_ms, train_ms, predict_ms, select_ms, refine_ms, total_ms;
    float final_loss;
    float pad0;
    char error[1024];
} ucb_surrogate_result;

UCB_API void ucb_default_surrogate_request(ucb_surrogate_request* r);
UCB_API int ucb_run_lle2d_surrogate(ucb_engine* e, const ucb_surrogate_request* req, double* d_values,
                                    int32_t* d_flags, void* stream, ucb_surrogate_result* res);

#ifdef __cplusplus
}
#endif

#endif /* UCB_H_ */
