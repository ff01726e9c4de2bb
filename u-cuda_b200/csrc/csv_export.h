// CSV output of the run_* entry points: the reference's data_export wire format
// (data_export.cpp — *_config.csv headers and the grid / row layouts), so that results
// drop into existing post-processing unchanged.
#pragma once

#include <string>
#include <vector>

namespace ucb {
namespace csv {

struct Common {
    std::vector<double> values;  // a[]
    std::vector<double> ic;      // X0[]
};

// A value as the kernels used it: narrowed to float when the engine's numb is float
// (precision UCB_PREC_F32), as the reference stages requests to its numb (to_numb,
// parametric_engine.cpp:2256-2265), and unchanged in the FP64 form.
inline double numb_value(double v, bool f32) { return f32 ? (double)(float)v : v; }
// a[] and X0[] for the config files, as the kernels used them (numb_value).
inline Common common(const double* a, int na, const double* x0, int nx, bool f32) {
    Common c;
    for (int i = 0; i < na; ++i) c.values.push_back(numb_value(a[i], f32));
    for (int i = 0; i < nx; ++i) c.ic.push_back(numb_value(x0[i], f32));
    return c;
}

void bif1d(const std::string& path, const Common& c, double tMax, double transient, double h, int pre,
           int writable_var, int index_of_mut_var, double lo, double hi, int n_pts, const int* counts,
           const double* peaks, const double* intervals, int max_peaks);

void lle2d(const std::string& path, const Common& c, int par_or_var, double tMax, double NT, double transient,
           double h, double eps, int idx1, int idx2, double r1lo, double r1hi, double r2lo, double r2hi, int n_pts,
           const double* values);

void ls2d(const std::string& path, const Common& c, int par_or_var, double tMax, double NT, double transient,
          double h, double eps, int idx1, int idx2, double r1lo, double r1hi, double r2lo, double r2hi, int n_pts,
          int n_exp, const double* plane_major_values);

// 2-D bifurcation (data_export.cpp write_bif2d_config / write_bif2d_grid).
void bif2d(const std::string& path, const Common& c, int par_or_var, double tMax, double transient, double h,
           int pre, double eps_dbscan, int writable_var, int idx1, int idx2, double r1lo, double r1hi, double r2lo,
           double r2hi, int n_pts, const double* values);

// Basins of attraction, reference method (data_export.cpp write_basins_config /
// write_basins_ranges / write_basins_grid_*): config, then four files (labels, _1 average
// peaks, _2 average intervals, _3 classes) each with the two-line ranges header and the
// n_pts x n_pts grid; non-finite features are written as 999.
void basins(const std::string& path, const Common& c, double tMax, double transient, double h, int pre,
            double eps_dbscan, int writable_var, int xvar, int yvar, double xlo, double xhi, double ylo, double yhi,
            int n_pts, const int* labels, const double* avg_peaks, const double* avg_intervals, const int* classes);

// 1-D LLE / LS (data_export.cpp write_lle1d_config / write_ls1d_config + rows): config
// title "1D LLE" or "1D LS", rows "param, v0[, v1, ...]" with the parameter value of
// getValueByIdx(_log)_local (parametric_engine.cpp:577-590).
void curve1d(const std::string& path, const char* title, const Common& c, double tMax, double NT, double transient,
             double h, double eps, int index, double lo, double hi, bool log_scale, int n_pts, int n_cols,
             const double* point_major_values);

}  // namespace csv
}  // namespace ucb
