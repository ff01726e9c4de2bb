// Drives the header-only ParametricEngine shim the way the reference's session layer
// calls ParametricEngine (analysis_session.cpp builds a Request, calls run_*, reads the
// Result). argv[1] = "invalid" / "continuation" / "dft" / "fastsync" (no GPU needed) or "lle1d" /
// "ls1d" / "lle2d" / "ls2d" / "bif1d" / "bif2d" / "basins" / "cancel" (GPU); the RK4 body is
// read from stdin.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <thread>
#include <iostream>
#include <iterator>
#include <string>

#include "ucb_parametric_engine.hpp"

int main(int argc, char** argv) {
    const std::string mode = argc > 1 ? argv[1] : "invalid";
    std::string body((std::istreambuf_iterator<char>(std::cin)), std::istreambuf_iterator<char>());
    ParametricEngine eng;
    if (mode == "dft") {
        Dft1DRequest r;
        r.krs_body = body;
        r.amountOfX = 3;
        Dft1DResult res = eng.run_dft_1d(r);
        std::printf("ok=%d error=%s\n", (int)res.ok, res.error.c_str());
    }
    if (mode == "fastsync") {
        FastSyncRequest r;
        r.krs_body = body;
        r.mode = 1;
        FastSyncResult res = eng.run_fastsync(r);
        std::printf("ok=%d mode=%d error=%s\n", (int)res.ok, res.mode, res.error.c_str());
    }
    if (mode == "cancel") {
        // the session's cancel token raised from another thread 150 ms into a long map
        LLE2DRequest r;
        r.krs_body = body;
        r.amountOfX = 3;
        r.initial_conditions = {1, 1, 1};
        r.base_values = {0, 0.2, 0.2, 5.7};
        r.param_index = 2;
        r.param_index_2 = 3;
        r.param_lo = 0.05; r.param_hi = 2.0; r.param_lo_2 = 2.0; r.param_hi_2 = 20.0;
        r.n_pts = 1024;
        r.h = 0.01; r.transient_time = 100; r.t_max = 2000; r.NT = 0.1;
        r.cancel = std::make_shared<std::atomic<bool>>(false);
        r.progress = std::make_shared<std::atomic<float>>(0.0f);
        {   // the same kernel, compiled and loaded before the timed call
            LLE2DRequest w = r;
            w.n_pts = 8;
            w.t_max = 1;
            w.cancel = nullptr;
            w.progress = nullptr;
            eng.run_lle_2d(w);
        }
        float seen = 0.0f;
        std::thread raiser([&] {
            std::this_thread::sleep_for(std::chrono::milliseconds(150));
            seen = r.progress->load();
            r.cancel->store(true);
        });
        const auto t0 = std::chrono::steady_clock::now();
        LLE2DResult res = eng.run_lle_2d(r);
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        raiser.join();
        std::printf("ok=%d cancelled=%d ms=%.0f progress_at_cancel=%.3f error=%s\n", (int)res.ok, (int)res.cancelled,
                    ms, seen, res.error.c_str());
    }
    if (mode == "invalid" || mode == "lle2d") {
        LLE2DRequest r;
        r.krs_body = body;
        r.amountOfX = 3;
        r.initial_conditions = {1, 1, 1};
        r.base_values = {0, 0.2, 0.2, 5.7};
        r.param_index = 2;
        r.param_index_2 = 3;
        r.param_lo = 0.05; r.param_hi = 2.0; r.param_lo_2 = 2.0; r.param_hi_2 = 20.0;
        r.n_pts = mode == "invalid" ? 0 : 8;
        r.h = 0.01; r.transient_time = 5; r.t_max = 10; r.NT = 0.1;
        r.progress = std::make_shared<std::atomic<float>>(0.0f);
        LLE2DResult res = eng.run_lle_2d(r);
        std::printf("ok=%d error=%s n=%d min=%.6f max=%.6f progress=%.1f\n", (int)res.ok, res.error.c_str(), res.n_pts,
                    res.min_val, res.max_val, r.progress->load());
        if (mode == "lle2d")
            for (size_t i = 0; i < res.values.size(); ++i) std::printf("%.17g %d\n", res.values[i], res.flags[i]);
        return 0;
    }
    if (mode == "lle1d" || mode == "continuation") {
        LLE1DRequest r;
        r.krs_body = body;
        r.amountOfX = 3;
        r.initial_conditions = {0.1, 0.1, 0.1};
        r.base_values = {0, 10.0, 28.0, 8.0 / 3.0};
        r.param_index = 2;
        r.param_lo = 20; r.param_hi = 200; r.n_pts = 16;
        r.h = 0.01; r.transient_time = 5; r.t_max = 20; r.NT = 0.5;
        r.continuation = mode == "continuation";
        r.progress = std::make_shared<std::atomic<float>>(0.0f);
        LLE1DResult res = eng.run_lle_1d(r);
        std::printf("ok=%d error=%s n=%d lo=%g hi=%g idx=%d progress=%.1f\n", (int)res.ok, res.error.c_str(), res.n_pts,
                    res.param_lo, res.param_hi, res.snapshot.indexOfMutVar, r.progress->load());
        for (size_t i = 0; i < res.lyapunov.size(); ++i) std::printf("%.17g %d\n", res.lyapunov[i], res.flags[i]);
        return 0;
    }
    if (mode == "ls1d") {
        LS1DRequest r;
        r.krs_body = body;
        r.amountOfX = 3;
        r.initial_conditions = {0.1, 0.1, 0.1};
        r.base_values = {0, 10.0, 28.0, 8.0 / 3.0};
        r.sweep_over_var = true;
        r.var_sweep_index = 0;
        r.param_lo = -5; r.param_hi = 5; r.n_pts = 10;
        r.h = 0.01; r.transient_time = 5; r.t_max = 20; r.NT = 0.5;
        LS1DResult res = eng.run_ls_1d(r);
        std::printf("ok=%d error=%s n=%d k=%d idx=%d\n", (int)res.ok, res.error.c_str(), res.n_pts, res.n_exponents,
                    res.snapshot.indexOfMutVar);
        for (size_t i = 0; i < res.spectrum.size(); ++i)
            for (double v : res.spectrum[i]) std::printf("%.17g\n", v);
        return 0;
    }
    if (mode == "bif2d") {
        Bifurcation2DRequest r;
        r.krs_body = body;
        r.amountOfX = 3;
        r.initial_conditions = {0.1, 0.1, 0.1};
        r.base_values = {0, 10.0, 28.0, 8.0 / 3.0};
        r.param_index = 2;
        r.param_index_2 = 1;
        r.param_lo = 20; r.param_hi = 200; r.param_lo_2 = 5.0; r.param_hi_2 = 15.0;
        r.n_pts = 6;
        r.h = 0.01; r.transient_time = 20; r.t_max = 60; r.eps_dbscan = 0.1;
        Bifurcation2DResult res = eng.run_bifurcation_2d(r);
        std::printf("ok=%d error=%s n=%d max=%g\n", (int)res.ok, res.error.c_str(), res.n_pts, res.max_val);
        for (size_t i = 0; i < res.values.size(); ++i) std::printf("%.17g %d\n", res.values[i], res.flags[i]);
        return 0;
    }
    if (mode == "basins") {
        BasinsRequest r;
        r.krs_body = body;
        r.amountOfX = 3;
        r.initial_conditions = {0.0, 0.0, 25.0};
        r.base_values = {0, 10.0, 10.0, 8.0 / 3.0};
        r.axis_x_lo = -20; r.axis_x_hi = 20; r.axis_y_lo = -20; r.axis_y_hi = 20;
        r.n_pts = 8;
        r.h = 0.01; r.transient_time = 100; r.t_max = 20; r.eps_dbscan = 0.5;
        r.progress_phase = std::make_shared<std::atomic<int>>(0);
        BasinsResult res = eng.run_basins(r);
        std::printf("ok=%d error=%s n=%d clusters=%d min=%d phase=%d\n", (int)res.ok, res.error.c_str(), res.n_pts,
                    res.n_clusters, res.min_cluster_idx, r.progress_phase->load());
        for (size_t i = 0; i < res.basin_idx.size(); ++i)
            std::printf("%d %.17g %.17g %d\n", res.basin_idx[i], res.avg_peaks[i], res.avg_intervals[i],
                        res.helpful_array[i]);
        // DBSCAN again over the cached features, as the reference's GUI re-clusters
        BasinsReclusterRequest rc;
        rc.krs_body = body;
        rc.amountOfX = 3;
        rc.n_pts = res.n_pts;
        rc.eps_dbscan = 0.5;
        rc.avg_peaks = res.avg_peaks;
        rc.avg_intervals = res.avg_intervals;
        rc.helpful_array = res.helpful_array;
        BasinsReclusterResult rr = eng.run_basins_recluster(rc);
        std::printf("recluster ok=%d same=%d\n", (int)rr.ok, (int)(rr.basin_idx == res.basin_idx));
        return 0;
    }
    if (mode == "ls2d") {
        LS2DRequest r;
        r.krs_body = body;
        r.amountOfX = 3;
        r.initial_conditions = {0.1, 0.1, 0.1};
        r.base_values = {0, 10.0, 28.0, 8.0 / 3.0};
        r.param_index = 2;
        r.param_index_2 = 1;
        r.param_lo = 20; r.param_hi = 40; r.param_lo_2 = 8.0; r.param_hi_2 = 12.0;
        r.n_pts = 6;
        r.h = 0.01; r.transient_time = 5; r.t_max = 20; r.NT = 0.5;
        LS2DResult res = eng.run_ls_2d(r);
        std::printf("ok=%d error=%s n=%d k=%d\n", (int)res.ok, res.error.c_str(), res.n_pts, res.n_exponents);
        for (size_t i = 0; i < res.values.size(); ++i) std::printf("%.17g\n", res.values[i]);
        return 0;
    }
    Bifurcation1DRequest b;
    b.krs_body = body;
    b.amountOfX = 3;
    b.initial_conditions = {0.1, 0.1, 0.1};
    b.base_values = {0, 10.0, 28.0, 8.0 / 3.0};
    b.param_index = 2;
    b.param_lo = 20; b.param_hi = 200; b.n_pts = 8;
    b.h = 0.01; b.transient_time = 10; b.t_max = 30;
    Bifurcation1DResult res = eng.run_bifurcation_1d(b);
    std::printf("ok=%d error=%s n=%d record_steps=%d\n", (int)res.ok, res.error.c_str(), res.n_pts, res.record_steps);
    for (int i = 0; i < res.n_pts; ++i)
        std::printf("%d %zu\n", res.flags[i], res.bifurcation_points[i].size());
    return 0;
}
