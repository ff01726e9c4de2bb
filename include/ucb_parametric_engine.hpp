// ucb_parametric_engine.hpp — header-only drop-in for the reference's ParametricEngine
// facade (parametric_engine.h:27-889) on the per-cell integration path.
//
// Same class name, same request/result struct names and field names, same result
// conventions (ok / cancelled / error, NaN or sentinel + flags, row-major iy*n+ix, plane-
// major spectra), same shared_ptr<atomic<...>> cancel / progress tokens. Every call goes
// through the C ABI in ucb.h (libucb.so): run_bifurcation_1d, run_bifurcation_2d,
// run_lle_1d, run_ls_1d, run_lle_2d, run_ls_2d, run_basins, run_basins_recluster.
// Entry points of the reference that are not on this path: run_dft_1d and run_fastsync
// are declared and return ok = false with a message; continuation sweeps are rejected by
// validation (continuation = true is an error).
//
// Extension: ParametricEngine::options() selects the arithmetic of the B200 engine
// (UCB_PREC_F64 plain form by default; UCB_PREC_F32 state form; exact or native step).
#pragma once

#include <atomic>
#include <chrono>
#include <cmath>
#include <limits>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "ucb.h"

namespace data_export {
struct Bif1DSnapshot {
    std::vector<double> values, initial_conditions;
    double tMax = 0.0, transientTime = 0.0, h = 0.0;
    int preScaller = 0, writableVar = 0, indexOfMutVar = 0;
    double range_lo = 0.0, range_hi = 0.0;
};
struct LLE2DSnapshot {
    std::vector<double> values, initial_conditions;
    int par_or_var = 1;
    double tMax = 0.0, NT = 0.0, transientTime = 0.0, h = 0.0, eps = 0.0;
    int indexOfMutVar = 0, indexOfMutVar2 = 0;
    double range1_lo = 0.0, range1_hi = 0.0, range2_lo = 0.0, range2_hi = 0.0;
    int n_pts = 0;
};
struct LLE1DSnapshot {
    std::vector<double> values, initial_conditions;
    double tMax = 0.0, NT = 0.0, transientTime = 0.0, h = 0.0, eps = 0.0;
    int indexOfMutVar = 0;
    double range_lo = 0.0, range_hi = 0.0;
};
struct LS1DSnapshot {
    std::vector<double> values, initial_conditions;
    double tMax = 0.0, NT = 0.0, transientTime = 0.0, h = 0.0, eps = 0.0;
    int indexOfMutVar = 0;
    double range_lo = 0.0, range_hi = 0.0;
};
struct Bif2DSnapshot {
    std::vector<double> values, initial_conditions;
    int par_or_var = 1;
    double tMax = 0.0, transientTime = 0.0, h = 0.0;
    int preScaller = 0;
    double eps_dbscan = 0.0;
    int writableVar = 0, indexOfMutVar = 0, indexOfMutVar2 = 0;
    double range1_lo = 0.0, range1_hi = 0.0, range2_lo = 0.0, range2_hi = 0.0;
    int n_pts = 0;
};
struct BasinsSnapshot {
    std::vector<double> values, initial_conditions;
    double tMax = 0.0, transientTime = 0.0, h = 0.0;
    int preScaller = 0;
    double eps_dbscan = 0.0;
    int writableVar = 0, axis_x_var = 0, axis_y_var = 0;
    double axis_x_lo = 0.0, axis_x_hi = 0.0, axis_y_lo = 0.0, axis_y_hi = 0.0;
    int n_pts = 0, feature1 = 0, feature2 = 0;
    double mult1 = 0.0, mult2 = 0.0;
};
struct LS2DSnapshot {
    std::vector<double> values, initial_conditions;
    int par_or_var = 1;
    double tMax = 0.0, NT = 0.0, transientTime = 0.0, h = 0.0, eps = 0.0;
    int indexOfMutVar = 0, indexOfMutVar2 = 0;
    double range1_lo = 0.0, range1_hi = 0.0, range2_lo = 0.0, range2_hi = 0.0;
    int n_pts = 0, n_exponents = 0;
};
// Snapshots of the two analyses this engine does not run (declared for the session layer).
struct Dft1DSnapshot {
    std::vector<double> values, initial_conditions;
    double tMax = 0.0, transientTime = 0.0, h = 0.0;
    int preScaller = 0, writableVar = 0, indexOfMutVar = 0;
    double range_lo = 0.0, range_hi = 0.0;
    int n_freq = 0;
    double freq_lo = 0.0, freq_hi = 0.0;
    int window_type = 1;
};
struct FastSyncSnapshot {
    int mode = 0;
    std::vector<double> values, ic_master, ic_slave, k_forward, k_backward;
    std::vector<std::string> var_names;
    double h = 0.0;
    int iter_of_synchr = 0, preScaller = 0;
    double window = 0.0;
    int type_of_synch = 0, error_estim = 0;
    double fs_error_trs = 0.0;
    double tMax = 0.0, transientTime = 0.0;
    int axis_x_var = 0, axis_y_var = 0;
    double axis_x_lo = 0.0, axis_x_hi = 0.0, axis_y_lo = 0.0, axis_y_hi = 0.0;
    int n_pts = 0;
};
}  // namespace data_export

struct Bifurcation1DRequest {
    std::string krs_body;
    int amountOfX = 0;
    std::vector<double> initial_conditions;
    std::vector<double> base_values;
    int param_index = 0;
    bool sweep_over_var = false;
    int var_sweep_index = 0;
    bool sweep_over_h = false;
    bool log_scale = false;
    bool continuation = false;          // not on this path: rejected with an error
    bool continuation_reverse = false;
    bool use_cpu = false;               // ignored: there is no CPU path in this engine
    double param_lo = 0.0;
    double param_hi = 1.0;
    int n_pts = 1000;
    int writable_var = 0;
    double h = 0.01;
    double transient_time = 0.0;
    double t_max = 0.0;
    int pre_scaller = 1;
    double max_value = 1.0e6;
    std::string csv_output_path;
    std::shared_ptr<std::atomic<bool>> cancel;
    std::shared_ptr<std::atomic<float>> progress;
};

struct Bifurcation1DResult {
    bool ok = false;
    bool cancelled = false;
    std::string error;
    bool continuation_reverse = false;
    double param_lo = 0.0;
    double param_hi = 1.0;
    int n_pts = 0;
    int record_steps = 0;
    std::vector<std::vector<double>> bifurcation_points;
    std::vector<std::vector<double>> peak_times;
    std::vector<int> flags;
    data_export::Bif1DSnapshot snapshot;
};

// LLE 1D / LS 1D (parametric_engine.h:235-387): one swept parameter, initial condition or
// step h. lyapunov[i] is NaN where the kernel flagged the point (flags[i] = -1);
// spectrum[i][k] keeps the 999 / -999 sentinels. Continuation sweeps (sequential, CPU in
// the reference) are answered with ok = false; use_cpu is ignored (no CPU path here).
struct LLE1DRequest {
    std::string krs_body;
    int amountOfX = 0;
    std::vector<double> initial_conditions;
    std::vector<double> base_values;
    bool sweep_over_var = false;
    int var_sweep_index = 0;
    bool sweep_over_h = false;
    bool log_scale = false;
    int param_index = 0;
    bool continuation = false;
    bool continuation_reverse = false;
    bool use_cpu = false;
    double param_lo = 0.0;
    double param_hi = 1.0;
    int n_pts = 500;
    double h = 0.01;
    double transient_time = 0.0;
    double t_max = 100.0;
    double NT = 1.0;
    double eps = 1.0e-4;
    double max_value = 1.0e6;
    std::string csv_output_path;
    std::shared_ptr<std::atomic<bool>> cancel;
    std::shared_ptr<std::atomic<float>> progress;
};

struct LLE1DResult {
    bool ok = false;
    bool cancelled = false;
    std::string error;
    int n_pts = 0;
    double param_lo = 0.0;
    double param_hi = 1.0;
    bool continuation_reverse = false;
    std::vector<double> lyapunov;
    std::vector<int> flags;
    data_export::LLE1DSnapshot snapshot;
};

struct LS1DRequest {
    std::string krs_body;
    int amountOfX = 0;
    std::vector<double> initial_conditions;
    std::vector<double> base_values;
    bool sweep_over_var = false;
    int var_sweep_index = 0;
    bool sweep_over_h = false;
    bool continuation = false;
    bool continuation_reverse = false;
    bool use_cpu = false;
    bool log_scale = false;
    int param_index = 0;
    double param_lo = 0.0;
    double param_hi = 1.0;
    int n_pts = 500;
    double h = 0.01;
    double transient_time = 0.0;
    double t_max = 100.0;
    double NT = 1.0;
    double eps = 1.0e-4;
    double max_value = 1.0e6;
    std::string csv_output_path;
    std::shared_ptr<std::atomic<bool>> cancel;
    std::shared_ptr<std::atomic<float>> progress;
};

struct LS1DResult {
    bool ok = false;
    bool cancelled = false;
    std::string error;
    int n_pts = 0;
    int n_exponents = 0;
    double param_lo = 0.0;
    double param_hi = 1.0;
    bool continuation_reverse = false;
    std::vector<std::vector<double>> spectrum;
    std::vector<int> flags;
    data_export::LS1DSnapshot snapshot;
};

struct LLE2DRequest {
    std::string krs_body;
    int amountOfX = 0;
    std::vector<double> initial_conditions;
    std::vector<double> base_values;
    bool sweep_over_var = false;
    bool sweep_over_var_2 = false;
    bool sweep_over_h = false;
    bool sweep_over_h_2 = false;
    bool log_scale = false;
    bool log_scale_2 = false;
    int param_index = 0;
    int var_sweep_index = 0;
    int param_index_2 = 0;
    int var_sweep_index_2 = 0;
    double param_lo = 0.0;
    double param_hi = 1.0;
    double param_lo_2 = 0.0;
    double param_hi_2 = 1.0;
    int n_pts = 200;
    double h = 0.01;
    double transient_time = 0.0;
    double t_max = 100.0;
    double NT = 1.0;
    double eps = 1.0e-4;
    double max_value = 1.0e6;
    std::string csv_output_path;
    std::shared_ptr<std::atomic<bool>> cancel;
    std::shared_ptr<std::atomic<float>> progress;
};

struct LLE2DResult {
    bool ok = false;
    bool cancelled = false;
    std::string error;
    int n_pts = 0;
    double param_lo = 0.0, param_hi = 1.0, param_lo_2 = 0.0, param_hi_2 = 1.0;
    std::vector<double> values;
    std::vector<int> flags;
    double min_val = 0.0;
    double max_val = 0.0;
    data_export::LLE2DSnapshot snapshot;
};

// Bifurcation 2D (parametric_engine.h: Bifurcation2DRequest / Result): period per cell
// from the reference's dbscan of the peaks; values[iy * n + ix], -1 with flag -1.
struct Bifurcation2DRequest {
    std::string krs_body;
    int amountOfX = 0;
    std::vector<double> initial_conditions;
    std::vector<double> base_values;
    bool sweep_over_var = false;
    bool sweep_over_h = false;
    bool log_scale = false;
    int var_sweep_index = 0;
    int param_index = 0;
    bool sweep_over_var_2 = false;
    bool sweep_over_h_2 = false;
    bool log_scale_2 = false;
    int var_sweep_index_2 = 0;
    int param_index_2 = 0;
    double param_lo = 0.0;
    double param_hi = 1.0;
    double param_lo_2 = 0.0;
    double param_hi_2 = 1.0;
    int n_pts = 200;
    int writable_var = 0;
    double h = 0.01;
    double transient_time = 0.0;
    double t_max = 100.0;
    int pre_scaller = 1;
    double max_value = 1.0e6;
    double eps_dbscan = 0.1;
    std::string csv_output_path;
    std::shared_ptr<std::atomic<bool>> cancel;
    std::shared_ptr<std::atomic<float>> progress;
};

struct Bifurcation2DResult {
    bool ok = false;
    bool cancelled = false;
    std::string error;
    int n_pts = 0;
    double param_lo = 0.0;
    double param_hi = 1.0;
    double param_lo_2 = 0.0;
    double param_hi_2 = 1.0;
    std::vector<double> values;
    std::vector<int> flags;
    double min_val = 0.0;
    double max_val = 0.0;
    data_export::Bif2DSnapshot snapshot;
};

// LS 2D (parametric_engine.h:581-637): full spectrum per cell, the reference's fixed-step
// LSKernelCUDA semantics (classical Gram-Schmidt every NT). values are plane-major:
// values[k * n * n + iy * n + ix]; per-plane min / max over valid cells.
struct LS2DRequest {
    std::string krs_body;
    int amountOfX = 0;
    std::vector<double> initial_conditions;
    std::vector<double> base_values;
    bool sweep_over_var = false;
    bool sweep_over_var_2 = false;
    bool sweep_over_h = false;
    bool sweep_over_h_2 = false;
    bool log_scale = false;
    bool log_scale_2 = false;
    int param_index = 0;
    int var_sweep_index = 0;
    int param_index_2 = 0;
    int var_sweep_index_2 = 0;
    double param_lo = 0.0;
    double param_hi = 1.0;
    double param_lo_2 = 0.0;
    double param_hi_2 = 1.0;
    int n_pts = 200;
    double h = 0.01;
    double transient_time = 0.0;
    double t_max = 100.0;
    double NT = 1.0;
    double eps = 1.0e-4;
    double max_value = 1.0e6;
    std::string csv_output_path;
    std::shared_ptr<std::atomic<bool>> cancel;
    std::shared_ptr<std::atomic<float>> progress;
};

struct LS2DResult {
    bool ok = false;
    bool cancelled = false;
    std::string error;
    int n_pts = 0;
    int n_exponents = 0;
    double param_lo = 0.0;
    double param_hi = 1.0;
    double param_lo_2 = 0.0;
    double param_hi_2 = 1.0;
    std::vector<double> values;
    std::vector<int> flags;
    std::vector<double> min_val;
    std::vector<double> max_val;
    data_export::LS2DSnapshot snapshot;
};

// Basins of attraction (parametric_engine.h:659-723): class and two peak features per
// initial-condition cell, then DBSCAN of the features. basin_idx >= 1 oscillating cluster,
// <= -1 cluster holding a fixed point, 0 unbound; all arrays row-major iy*n + ix.
struct BasinsRequest {
    std::string krs_body;
    int amountOfX = 0;
    std::vector<double> initial_conditions;
    std::vector<double> base_values;
    int axis_x_var = 0;
    int axis_y_var = 1;
    double axis_x_lo = -10.0, axis_x_hi = 10.0;
    double axis_y_lo = -10.0, axis_y_hi = 10.0;
    int n_pts = 200;
    int writable_var = 0;
    double h = 0.01;
    double t_max = 1000.0;
    double transient_time = 10000.0;
    int pre_scaller = 1;
    double max_value = 1.0e6;
    double eps_dbscan = 0.5;
    int feature1 = 0;   // BF_AVG_PEAKS
    int feature2 = 1;   // BF_AVG_INTERVALS
    double mult1 = 1.0;
    double mult2 = 1.0;
    std::string csv_output_path;
    std::shared_ptr<std::atomic<bool>> cancel;
    std::shared_ptr<std::atomic<float>> progress;
    std::shared_ptr<std::atomic<int>> progress_phase;
};

struct BasinsResult {
    bool ok = false;
    bool cancelled = false;
    std::string error;
    int n_pts = 0;
    double axis_x_lo = 0.0, axis_x_hi = 0.0;
    double axis_y_lo = 0.0, axis_y_hi = 0.0;
    int axis_x_var = 0, axis_y_var = 1;
    std::vector<int> basin_idx;
    std::vector<double> avg_peaks;
    std::vector<double> avg_intervals;
    std::vector<int> helpful_array;
    int n_clusters = 0;
    int min_cluster_idx = 0;
    double avg_peaks_min = 0.0, avg_peaks_max = 0.0;
    double avg_intervals_min = 0.0, avg_intervals_max = 0.0;
    data_export::BasinsSnapshot snapshot;
};

// DBSCAN alone over cached features (parametric_engine.h:733-753).
struct BasinsReclusterRequest {
    std::string krs_body;
    int amountOfX = 0;
    int n_pts = 0;
    double eps_dbscan = 0.5;
    std::vector<double> avg_peaks;
    std::vector<double> avg_intervals;
    std::vector<int> helpful_array;
    std::shared_ptr<std::atomic<bool>> cancel;
    std::shared_ptr<std::atomic<float>> progress;
};

struct BasinsReclusterResult {
    bool ok = false;
    bool cancelled = false;
    std::string error;
    int n_pts = 0;
    std::vector<int> basin_idx;
    int n_clusters = 0;
    int min_cluster_idx = 0;
};

// Requests / results of the reference's DFT sweep and Fast Synchro analyses
// (parametric_engine.h:140-227, :767-842). They are not on this engine's path; the
// types and the two entry points exist so that the session layer compiles unchanged,
// and every call returns ok = false with an error message.
struct Dft1DRequest {
    std::string krs_body;
    int amountOfX = 0;
    std::vector<double> initial_conditions, base_values;
    int param_index = 0;
    bool sweep_over_var = false;
    int var_sweep_index = 0;
    bool sweep_over_h = false, log_scale = false, continuation = false, continuation_reverse = false;
    bool use_cpu = false;
    double param_lo = 0.0, param_hi = 1.0;
    int n_pts = 1000;
    int writable_var = 0;
    double h = 0.01, transient_time = 0.0, t_max = 0.0;
    int pre_scaller = 1;
    double max_value = 1.0e6;
    int n_freq = 200;
    double freq_lo = 0.0, freq_hi = 10.0;
    bool freq_log_scale = false;
    int window_type = 1;
    std::string csv_output_path;
    std::shared_ptr<std::atomic<bool>> cancel;
    std::shared_ptr<std::atomic<float>> progress;
};

struct Dft1DResult {
    bool ok = false;
    bool cancelled = false;
    std::string error;
    bool continuation_reverse = false;
    double param_lo = 0.0, param_hi = 1.0;
    int n_pts = 0, n_freq = 0;
    double freq_lo = 0.0, freq_hi = 0.0;
    std::vector<double> ak_cos, bk_sin;
    std::vector<int> flags;
    data_export::Dft1DSnapshot snapshot;
};

struct FastSyncRequest {
    std::string krs_body;
    int amountOfX = 0;
    std::vector<double> values;
    int mode = 0;
    double h = 0.01;
    int iter_of_synchr = 100, pre_scaller = 1;
    double max_value = 1e6;
    std::vector<double> k_forward, k_backward, ic_master, ic_slave;
    double t_max = 100.0, transient_time = 0.0;
    float window = 50.0f;  // the reference's numb (float)
    int axis_x_var = 0, axis_y_var = 1;
    double axis_x_lo = -10.0, axis_x_hi = 10.0, axis_y_lo = -10.0, axis_y_hi = 10.0;
    int n_pts = 200;
    bool grid_swap_master_slave = false;
    int type_of_synch = 0, error_estim = 2;
    double fs_error_trs = 1e-12;
    std::string csv_output_path;
    std::vector<std::string> var_names;
    std::shared_ptr<std::atomic<bool>> cancel;
    std::shared_ptr<std::atomic<float>> progress;
};

struct FastSyncResult {
    bool ok = false;
    bool cancelled = false;
    std::string error;
    int mode = 0;
    int n_pts_traj = 0, amountOfX_traj = 0;
    std::vector<double> traj_full, sync_error;
    int n_pts_grid = 0;
    double axis_x_lo = 0.0, axis_x_hi = 0.0, axis_y_lo = 0.0, axis_y_hi = 0.0;
    int axis_x_var = 0, axis_y_var = 1;
    std::vector<double> heatmap;
    double min_val = 0.0, max_val = 0.0;
    data_export::FastSyncSnapshot snapshot;
};

// The session's cancel / progress tokens (shared_ptr<atomic<...>>, parametric_engine.h)
// mirrored into the C ABI's words for the duration of one call: a watcher thread copies
// a raised cancel token into the word the engine polls while the map runs, and the
// engine's progress into the session's token (the reference updates both between chunks,
// parametric_engine.cpp:2780-2786). Without tokens no thread is started.
class TokenBridge {
public:
    TokenBridge(const std::shared_ptr<std::atomic<bool>>& cancel, const std::shared_ptr<std::atomic<float>>& progress,
                const std::shared_ptr<std::atomic<int>>& phase = nullptr)
        : c_(cancel), p_(progress), ph_(phase) {
        cancel_ = (c_ && c_->load(std::memory_order_relaxed)) ? 1 : 0;
        if (c_ || p_ || ph_) th_ = std::thread([this] { watch(); });
    }
    ~TokenBridge() { finish(); }
    TokenBridge(const TokenBridge&) = delete;
    TokenBridge& operator=(const TokenBridge&) = delete;
    const volatile int32_t* cancel() const { return &cancel_; }
    volatile float* progress() { return &prog_; }
    volatile int32_t* phase() { return &phase_; }
    // Stops the watcher and stores the final progress / phase in the session's tokens.
    void finish() {
        stop_.store(true);
        if (th_.joinable()) th_.join();
        if (p_) p_->store(prog_, std::memory_order_relaxed);
        if (ph_) ph_->store(phase_, std::memory_order_relaxed);
    }

private:
    void watch() {
        while (!stop_.load()) {
            if (c_ && c_->load(std::memory_order_relaxed)) cancel_ = 1;
            if (p_) p_->store(prog_, std::memory_order_relaxed);
            if (ph_) ph_->store(phase_, std::memory_order_relaxed);
            std::this_thread::sleep_for(std::chrono::milliseconds(2));
        }
    }
    std::shared_ptr<std::atomic<bool>> c_;
    std::shared_ptr<std::atomic<float>> p_;
    std::shared_ptr<std::atomic<int>> ph_;
    volatile int32_t cancel_ = 0;
    volatile float prog_ = 0.0f;
    volatile int32_t phase_ = 0;
    std::atomic<bool> stop_{false};
    std::thread th_;
};

class ParametricEngine {
public:
    ParametricEngine() : e_(ucb_create(0)) { ucb_default_options(&opt_); }
    ~ParametricEngine() { ucb_destroy(e_); }
    ParametricEngine(const ParametricEngine&) = delete;
    ParametricEngine& operator=(const ParametricEngine&) = delete;

    ucb_options& options() { return opt_; }

    Bifurcation1DResult run_bifurcation_1d(const Bifurcation1DRequest& r) {
        Bifurcation1DResult res;
        if (r.continuation) {
            res.error = "continuation sweeps are not supported by this engine";
            return res;
        }
        const int mp = 2500;  // max_amount_of_peaks (configCUDA.h)
        ucb_bif1d_request q{};
        q.krs_body = r.krs_body.c_str();
        q.amount_of_x = r.amountOfX;
        q.initial_conditions = r.initial_conditions.data();
        if ((int)r.initial_conditions.size() != r.amountOfX) {
            res.error = "initial_conditions.size() != amountOfX";
            return res;
        }
        q.base_values = r.base_values.data();
        q.n_values = (int)r.base_values.size();
        q.param_index = r.param_index;
        q.sweep_over_var = r.sweep_over_var;
        q.var_sweep_index = r.var_sweep_index;
        q.sweep_over_h = r.sweep_over_h;
        q.log_scale = r.log_scale;
        q.param_lo = r.param_lo;
        q.param_hi = r.param_hi;
        q.n_pts = r.n_pts;
        q.writable_var = r.writable_var;
        q.h = r.h;
        q.transient_time = r.transient_time;
        q.t_max = r.t_max;
        q.pre_scaller = r.pre_scaller;
        q.max_value = r.max_value;
        q.max_peaks = mp;
        q.csv_output_path = r.csv_output_path.c_str();
        q.opt = opt_;
        TokenBridge tokens(r.cancel, r.progress);
        q.cancel = tokens.cancel();
        q.progress = tokens.progress();
        const size_t n = r.n_pts > 0 ? (size_t)r.n_pts : 0;
        std::vector<int32_t> counts(n);
        std::vector<double> peaks(n * mp), intervals(n * mp);
        ucb_bif1d_result o{};
        o.counts = counts.data();
        o.peaks = peaks.data();
        o.intervals = intervals.data();
        ucb_run_bif1d(e_, &q, &o);
        tokens.finish();
        res.ok = o.ok != 0;
        res.cancelled = o.cancelled != 0;
        res.error = o.error;
        if (!res.ok) return res;
        res.n_pts = o.n_pts;
        res.record_steps = o.record_steps;
        res.param_lo = r.param_lo;
        res.param_hi = r.param_hi;
        res.flags.assign(counts.begin(), counts.end());
        res.bifurcation_points.assign(n, {});
        res.peak_times.assign(n, {});
        for (size_t i = 0; i < n; ++i) {
            const int k = counts[i] > 0 ? counts[i] : 0;
            res.bifurcation_points[i].assign(peaks.begin() + i * mp, peaks.begin() + i * mp + k);
            res.peak_times[i].assign(intervals.begin() + i * mp, intervals.begin() + i * mp + k);
        }
        auto& s = res.snapshot;
        s.values = r.base_values;
        s.initial_conditions = r.initial_conditions;
        s.tMax = r.t_max;
        s.transientTime = r.transient_time;
        s.h = r.h;
        s.preScaller = r.pre_scaller;
        s.writableVar = r.writable_var;
        s.indexOfMutVar = r.sweep_over_var ? r.var_sweep_index : r.param_index;
        s.range_lo = r.param_lo;
        s.range_hi = r.param_hi;
        return res;
    }

    LLE1DResult run_lle_1d(const LLE1DRequest& r) {
        LLE1DResult res;
        if (!check_1d(r, res.error)) return res;
        TokenBridge tokens(r.cancel, r.progress);
        ucb_lle1d_request q = request_1d(r, tokens);
        const size_t n = r.n_pts > 0 ? (size_t)r.n_pts : 0;
        res.lyapunov.assign(n, 0.0);
        std::vector<int32_t> f32(n);
        ucb_lle1d_result o{};
        o.values = res.lyapunov.data();
        o.flags = f32.data();
        ucb_run_lle1d(e_, &q, &o);
        tokens.finish();
        res.ok = o.ok != 0;
        res.cancelled = o.cancelled != 0;
        res.error = o.error;
        if (!res.ok) return res;
        res.flags.assign(f32.begin(), f32.end());
        res.n_pts = o.n_pts;
        res.param_lo = o.param_lo;
        res.param_hi = o.param_hi;
        snapshot_1d(r, res.snapshot);
        return res;
    }

    LS1DResult run_ls_1d(const LS1DRequest& r) {
        LS1DResult res;
        if (!check_1d(r, res.error)) return res;
        TokenBridge tokens(r.cancel, r.progress);
        ucb_ls1d_request q = request_1d(r, tokens);
        const size_t n = r.n_pts > 0 ? (size_t)r.n_pts : 0;
        const size_t nx = r.amountOfX > 0 ? (size_t)r.amountOfX : 0;
        std::vector<double> flat(n * nx);
        std::vector<int32_t> f32(n);
        ucb_ls1d_result o{};
        o.values = flat.data();
        o.flags = f32.data();
        ucb_run_ls1d(e_, &q, &o);
        tokens.finish();
        res.ok = o.ok != 0;
        res.cancelled = o.cancelled != 0;
        res.error = o.error;
        if (!res.ok) return res;
        res.flags.assign(f32.begin(), f32.end());
        res.n_pts = o.n_pts;
        res.n_exponents = o.n_exponents;
        res.param_lo = o.param_lo;
        res.param_hi = o.param_hi;
        res.spectrum.resize(n);
        for (size_t i = 0; i < n; ++i)
            res.spectrum[i].assign(flat.begin() + i * nx, flat.begin() + (i + 1) * nx);
        snapshot_1d(r, res.snapshot);
        return res;
    }

    LLE2DResult run_lle_2d(const LLE2DRequest& r) {
        LLE2DResult res;
        if ((int)r.initial_conditions.size() != r.amountOfX) {
            res.error = "initial_conditions.size() != amountOfX";
            return res;
        }
        ucb_lle2d_request q{};
        q.krs_body = r.krs_body.c_str();
        q.amount_of_x = r.amountOfX;
        q.initial_conditions = r.initial_conditions.data();
        q.base_values = r.base_values.data();
        q.n_values = (int)r.base_values.size();
        q.sweep_over_var = r.sweep_over_var;
        q.sweep_over_var_2 = r.sweep_over_var_2;
        q.sweep_over_h = r.sweep_over_h;
        q.sweep_over_h_2 = r.sweep_over_h_2;
        q.log_scale = r.log_scale;
        q.log_scale_2 = r.log_scale_2;
        q.param_index = r.param_index;
        q.var_sweep_index = r.var_sweep_index;
        q.param_index_2 = r.param_index_2;
        q.var_sweep_index_2 = r.var_sweep_index_2;
        q.param_lo = r.param_lo;
        q.param_hi = r.param_hi;
        q.param_lo_2 = r.param_lo_2;
        q.param_hi_2 = r.param_hi_2;
        q.n_pts = r.n_pts;
        q.h = r.h;
        q.transient_time = r.transient_time;
        q.t_max = r.t_max;
        q.NT = r.NT;
        q.eps = r.eps;
        q.max_value = r.max_value;
        q.csv_output_path = r.csv_output_path.c_str();
        TokenBridge tokens(r.cancel, r.progress);
        q.cancel = tokens.cancel();
        q.progress = tokens.progress();
        q.opt = opt_;
        const size_t n = r.n_pts > 0 ? (size_t)r.n_pts * (size_t)r.n_pts : 0;
        res.values.assign(n, 0.0);
        res.flags.assign(n, 0);
        std::vector<int32_t> f32(n);
        ucb_lle2d_result o{};
        o.values = res.values.data();
        o.flags = f32.data();
        ucb_run_lle2d(e_, &q, &o);
        tokens.finish();
        res.ok = o.ok != 0;
        res.cancelled = o.cancelled != 0;
        res.error = o.error;
        if (!res.ok) return res;
        res.flags.assign(f32.begin(), f32.end());
        res.n_pts = o.n_pts;
        res.param_lo = o.param_lo;
        res.param_hi = o.param_hi;
        res.param_lo_2 = o.param_lo_2;
        res.param_hi_2 = o.param_hi_2;
        res.min_val = o.min_val;
        res.max_val = o.max_val;
        auto& s = res.snapshot;
        s.values = r.base_values;
        s.initial_conditions = r.initial_conditions;
        s.par_or_var = (r.sweep_over_var == r.sweep_over_var_2) ? (r.sweep_over_var ? 0 : 1) : 2;
        s.tMax = r.t_max;
        s.NT = r.NT;
        s.transientTime = r.transient_time;
        s.h = r.h;
        s.eps = r.eps;
        s.indexOfMutVar = r.sweep_over_var ? r.var_sweep_index : r.param_index;
        s.indexOfMutVar2 = r.sweep_over_var_2 ? r.var_sweep_index_2 : r.param_index_2;
        s.range1_lo = r.param_lo;
        s.range1_hi = r.param_hi;
        s.range2_lo = r.param_lo_2;
        s.range2_hi = r.param_hi_2;
        s.n_pts = r.n_pts;
        return res;
    }

    Bifurcation2DResult run_bifurcation_2d(const Bifurcation2DRequest& r) {
        Bifurcation2DResult res;
        if ((int)r.initial_conditions.size() != r.amountOfX) {
            res.error = "initial_conditions.size() != amountOfX";
            return res;
        }
        ucb_bif2d_request q{};
        q.krs_body = r.krs_body.c_str();
        q.amount_of_x = r.amountOfX;
        q.initial_conditions = r.initial_conditions.data();
        q.base_values = r.base_values.data();
        q.n_values = (int)r.base_values.size();
        q.sweep_over_var = r.sweep_over_var;
        q.sweep_over_var_2 = r.sweep_over_var_2;
        q.sweep_over_h = r.sweep_over_h;
        q.sweep_over_h_2 = r.sweep_over_h_2;
        q.log_scale = r.log_scale;
        q.log_scale_2 = r.log_scale_2;
        q.param_index = r.param_index;
        q.var_sweep_index = r.var_sweep_index;
        q.param_index_2 = r.param_index_2;
        q.var_sweep_index_2 = r.var_sweep_index_2;
        q.param_lo = r.param_lo;
        q.param_hi = r.param_hi;
        q.param_lo_2 = r.param_lo_2;
        q.param_hi_2 = r.param_hi_2;
        q.n_pts = r.n_pts;
        q.writable_var = r.writable_var;
        q.h = r.h;
        q.transient_time = r.transient_time;
        q.t_max = r.t_max;
        q.pre_scaller = r.pre_scaller;
        q.max_value = r.max_value;
        q.eps_dbscan = r.eps_dbscan;
        q.csv_output_path = r.csv_output_path.c_str();
        TokenBridge tokens(r.cancel, r.progress);
        q.cancel = tokens.cancel();
        q.progress = tokens.progress();
        q.opt = opt_;
        const size_t cells = r.n_pts > 0 ? (size_t)r.n_pts * (size_t)r.n_pts : 0;
        res.values.assign(cells, 0.0);
        std::vector<int32_t> f32(cells);
        ucb_bif2d_result o{};
        o.values = res.values.data();
        o.flags = f32.data();
        ucb_run_bif2d(e_, &q, &o);
        tokens.finish();
        res.ok = o.ok != 0;
        res.cancelled = o.cancelled != 0;
        res.error = o.error;
        if (!res.ok) return res;
        res.flags.assign(f32.begin(), f32.end());
        res.n_pts = o.n_pts;
        res.param_lo = o.param_lo;
        res.param_hi = o.param_hi;
        res.param_lo_2 = o.param_lo_2;
        res.param_hi_2 = o.param_hi_2;
        res.min_val = o.min_val;
        res.max_val = o.max_val;
        auto& s = res.snapshot;
        s.values = r.base_values;
        s.initial_conditions = r.initial_conditions;
        s.par_or_var = (r.sweep_over_var == r.sweep_over_var_2) ? (r.sweep_over_var ? 0 : 1) : 2;
        s.tMax = r.t_max;
        s.transientTime = r.transient_time;
        s.h = r.h;
        s.preScaller = r.pre_scaller;
        s.eps_dbscan = r.eps_dbscan;
        s.writableVar = r.writable_var;
        s.indexOfMutVar = r.sweep_over_var ? r.var_sweep_index : r.param_index;
        s.indexOfMutVar2 = r.sweep_over_var_2 ? r.var_sweep_index_2 : r.param_index_2;
        s.range1_lo = r.param_lo;
        s.range1_hi = r.param_hi;
        s.range2_lo = r.param_lo_2;
        s.range2_hi = r.param_hi_2;
        s.n_pts = r.n_pts;
        return res;
    }

    LS2DResult run_ls_2d(const LS2DRequest& r) {
        LS2DResult res;
        if ((int)r.initial_conditions.size() != r.amountOfX) {
            res.error = "initial_conditions.size() != amountOfX";
            return res;
        }
        ucb_ls2d_request q{};
        q.krs_body = r.krs_body.c_str();
        q.amount_of_x = r.amountOfX;
        q.initial_conditions = r.initial_conditions.data();
        q.base_values = r.base_values.data();
        q.n_values = (int)r.base_values.size();
        q.sweep_over_var = r.sweep_over_var;
        q.sweep_over_var_2 = r.sweep_over_var_2;
        q.sweep_over_h = r.sweep_over_h;
        q.sweep_over_h_2 = r.sweep_over_h_2;
        q.log_scale = r.log_scale;
        q.log_scale_2 = r.log_scale_2;
        q.param_index = r.param_index;
        q.var_sweep_index = r.var_sweep_index;
        q.param_index_2 = r.param_index_2;
        q.var_sweep_index_2 = r.var_sweep_index_2;
        q.param_lo = r.param_lo;
        q.param_hi = r.param_hi;
        q.param_lo_2 = r.param_lo_2;
        q.param_hi_2 = r.param_hi_2;
        q.n_pts = r.n_pts;
        q.h = r.h;
        q.transient_time = r.transient_time;
        q.t_max = r.t_max;
        q.NT = r.NT;
        q.eps = r.eps;
        q.max_value = r.max_value;
        q.csv_output_path = r.csv_output_path.c_str();
        TokenBridge tokens(r.cancel, r.progress);
        q.cancel = tokens.cancel();
        q.progress = tokens.progress();
        q.opt = opt_;
        q.method = UCB_LS_FIXED;
        const size_t cells = r.n_pts > 0 ? (size_t)r.n_pts * (size_t)r.n_pts : 0;
        const size_t nx = r.amountOfX > 0 ? (size_t)r.amountOfX : 0;
        res.values.assign(cells * nx, 0.0);
        res.min_val.assign(nx, 0.0);
        res.max_val.assign(nx, 0.0);
        std::vector<int32_t> f32(cells);
        ucb_ls2d_result o{};
        o.values = res.values.data();
        o.flags = f32.data();
        o.min_val = res.min_val.data();
        o.max_val = res.max_val.data();
        ucb_run_ls2d(e_, &q, &o);
        tokens.finish();
        res.ok = o.ok != 0;
        res.cancelled = o.cancelled != 0;
        res.error = o.error;
        if (!res.ok) return res;
        res.flags.assign(f32.begin(), f32.end());
        res.n_pts = o.n_pts;
        res.n_exponents = o.n_exponents;
        res.param_lo = r.param_lo;
        res.param_hi = r.param_hi;
        res.param_lo_2 = r.param_lo_2;
        res.param_hi_2 = r.param_hi_2;
        auto& s = res.snapshot;
        s.values = r.base_values;
        s.initial_conditions = r.initial_conditions;
        s.par_or_var = (r.sweep_over_var == r.sweep_over_var_2) ? (r.sweep_over_var ? 0 : 1) : 2;
        s.tMax = r.t_max;
        s.NT = r.NT;
        s.transientTime = r.transient_time;
        s.h = r.h;
        s.eps = r.eps;
        s.indexOfMutVar = r.sweep_over_var ? r.var_sweep_index : r.param_index;
        s.indexOfMutVar2 = r.sweep_over_var_2 ? r.var_sweep_index_2 : r.param_index_2;
        s.range1_lo = r.param_lo;
        s.range1_hi = r.param_hi;
        s.range2_lo = r.param_lo_2;
        s.range2_hi = r.param_hi_2;
        s.n_pts = r.n_pts;
        s.n_exponents = res.n_exponents;
        return res;
    }

    BasinsResult run_basins(const BasinsRequest& r) {
        BasinsResult res;
        if ((int)r.initial_conditions.size() != r.amountOfX) {
            res.error = "initial_conditions.size() != amountOfX";
            return res;
        }
        ucb_basins_dbscan_request q{};
        q.krs_body = r.krs_body.c_str();
        q.amount_of_x = r.amountOfX;
        q.initial_conditions = r.initial_conditions.data();
        q.base_values = r.base_values.data();
        q.n_values = (int)r.base_values.size();
        q.axis_x_var = r.axis_x_var;
        q.axis_y_var = r.axis_y_var;
        q.axis_x_lo = r.axis_x_lo;
        q.axis_x_hi = r.axis_x_hi;
        q.axis_y_lo = r.axis_y_lo;
        q.axis_y_hi = r.axis_y_hi;
        q.n_pts = r.n_pts;
        q.writable_var = r.writable_var;
        q.h = r.h;
        q.t_max = r.t_max;
        q.transient_time = r.transient_time;
        q.pre_scaller = r.pre_scaller;
        q.max_value = r.max_value;
        q.eps_dbscan = r.eps_dbscan;
        q.feature1 = r.feature1;
        q.feature2 = r.feature2;
        q.mult1 = r.mult1;
        q.mult2 = r.mult2;
        q.csv_output_path = r.csv_output_path.c_str();
        TokenBridge tokens(r.cancel, r.progress, r.progress_phase);
        q.cancel = tokens.cancel();
        q.progress = tokens.progress();
        q.progress_phase = tokens.phase();
        q.opt = opt_;
        const size_t cells = r.n_pts > 0 ? (size_t)r.n_pts * (size_t)r.n_pts : 0;
        std::vector<int32_t> labels(cells), classes(cells);
        res.avg_peaks.assign(cells, 0.0);
        res.avg_intervals.assign(cells, 0.0);
        ucb_basins_dbscan_result o{};
        o.labels = labels.data();
        o.avg_peaks = res.avg_peaks.data();
        o.avg_intervals = res.avg_intervals.data();
        o.classes = classes.data();
        ucb_run_basins_dbscan(e_, &q, &o);
        tokens.finish();
        res.ok = o.ok != 0;
        res.cancelled = o.cancelled != 0;
        res.error = o.error;
        if (!res.ok) {
            res.avg_peaks.clear();
            res.avg_intervals.clear();
            return res;
        }
        res.n_pts = o.n_pts;
        res.axis_x_lo = r.axis_x_lo;
        res.axis_x_hi = r.axis_x_hi;
        res.axis_y_lo = r.axis_y_lo;
        res.axis_y_hi = r.axis_y_hi;
        res.axis_x_var = r.axis_x_var;
        res.axis_y_var = r.axis_y_var;
        res.basin_idx.assign(labels.begin(), labels.end());
        res.helpful_array.assign(classes.begin(), classes.end());
        res.n_clusters = o.n_clusters;
        res.min_cluster_idx = o.min_cluster_idx;
        res.avg_peaks_min = o.avg_peaks_min;
        res.avg_peaks_max = o.avg_peaks_max;
        res.avg_intervals_min = o.avg_intervals_min;
        res.avg_intervals_max = o.avg_intervals_max;
        auto& s = res.snapshot;
        s.values = r.base_values;
        s.initial_conditions = r.initial_conditions;
        s.tMax = r.t_max;
        s.transientTime = r.transient_time;
        s.h = r.h;
        s.preScaller = r.pre_scaller;
        s.eps_dbscan = r.eps_dbscan;
        s.writableVar = r.writable_var;
        s.axis_x_var = r.axis_x_var;
        s.axis_y_var = r.axis_y_var;
        s.axis_x_lo = r.axis_x_lo;
        s.axis_x_hi = r.axis_x_hi;
        s.axis_y_lo = r.axis_y_lo;
        s.axis_y_hi = r.axis_y_hi;
        s.n_pts = r.n_pts;
        s.feature1 = r.feature1;
        s.feature2 = r.feature2;
        s.mult1 = r.mult1;
        s.mult2 = r.mult2;
        return res;
    }

    // Not on this engine's path (see Dft1DRequest): ok = false with a message.
    Dft1DResult run_dft_1d(const Dft1DRequest&) {
        Dft1DResult res;
        res.error = "run_dft_1d is not supported by this engine (per-cell integration path only)";
        return res;
    }
    FastSyncResult run_fastsync(const FastSyncRequest& r) {
        FastSyncResult res;
        res.mode = r.mode;
        res.error = "run_fastsync is not supported by this engine (per-cell integration path only)";
        return res;
    }

    BasinsReclusterResult run_basins_recluster(const BasinsReclusterRequest& r) {
        BasinsReclusterResult res;
        const size_t cells = r.n_pts > 0 ? (size_t)r.n_pts * (size_t)r.n_pts : 0;
        if (r.n_pts > 0) {
            if (r.avg_peaks.size() != cells) { res.error = "avg_peaks: size does not match n_pts^2"; return res; }
            if (r.avg_intervals.size() != cells) { res.error = "avg_intervals: size does not match n_pts^2"; return res; }
            if (r.helpful_array.size() != cells) { res.error = "helpful_array: size does not match n_pts^2"; return res; }
        }
        std::vector<int32_t> classes(r.helpful_array.begin(), r.helpful_array.end()), labels(cells);
        ucb_basins_recluster_request q{};
        q.krs_body = r.krs_body.c_str();
        q.amount_of_x = r.amountOfX;
        q.n_pts = r.n_pts;
        q.eps_dbscan = r.eps_dbscan;
        q.avg_peaks = r.avg_peaks.data();
        q.avg_intervals = r.avg_intervals.data();
        q.classes = classes.data();
        TokenBridge tokens(r.cancel, r.progress);
        q.cancel = tokens.cancel();
        q.progress = tokens.progress();
        q.opt = opt_;
        ucb_basins_recluster_result o{};
        o.labels = labels.data();
        ucb_run_basins_recluster(e_, &q, &o);
        tokens.finish();
        res.ok = o.ok != 0;
        res.cancelled = o.cancelled != 0;
        res.error = o.error;
        if (!res.ok) return res;
        res.n_pts = o.n_pts;
        res.basin_idx.assign(labels.begin(), labels.end());
        res.n_clusters = o.n_clusters;
        res.min_cluster_idx = o.min_cluster_idx;
        return res;
    }

private:
    // LLE1DRequest and LS1DRequest carry the same fields (parametric_engine.h:235, :332).
    template <class Req>
    static bool check_1d(const Req& r, std::string& error) {
        if (r.continuation) {
            error = "continuation sweeps are not supported by this engine";
            return false;
        }
        if ((int)r.initial_conditions.size() != r.amountOfX) {
            error = "initial_conditions.size() != amountOfX";
            return false;
        }
        return true;
    }

    template <class Req>
    ucb_lle1d_request request_1d(const Req& r, TokenBridge& tokens) const {
        ucb_lle1d_request q{};
        q.krs_body = r.krs_body.c_str();
        q.amount_of_x = r.amountOfX;
        q.initial_conditions = r.initial_conditions.data();
        q.base_values = r.base_values.data();
        q.n_values = (int)r.base_values.size();
        q.sweep_over_var = r.sweep_over_var;
        q.var_sweep_index = r.var_sweep_index;
        q.sweep_over_h = r.sweep_over_h;
        q.log_scale = r.log_scale;
        q.param_index = r.param_index;
        q.param_lo = r.param_lo;
        q.param_hi = r.param_hi;
        q.n_pts = r.n_pts;
        q.h = r.h;
        q.transient_time = r.transient_time;
        q.t_max = r.t_max;
        q.NT = r.NT;
        q.eps = r.eps;
        q.max_value = r.max_value;
        q.csv_output_path = r.csv_output_path.c_str();
        q.cancel = tokens.cancel();
        q.progress = tokens.progress();
        q.opt = opt_;
        return q;
    }

    template <class Req, class Snap>
    static void snapshot_1d(const Req& r, Snap& s) {
        s.values = r.base_values;
        s.initial_conditions = r.initial_conditions;
        s.tMax = r.t_max;
        s.NT = r.NT;
        s.transientTime = r.transient_time;
        s.h = r.h;
        s.eps = r.eps;
        s.indexOfMutVar = r.sweep_over_var ? r.var_sweep_index : r.param_index;
        s.range_lo = r.param_lo;
        s.range_hi = r.param_hi;
    }

    ucb_engine* e_;
    ucb_options opt_;
};
