#include "csv_export.h"

#include <cmath>
#include <fstream>
#include <iomanip>

namespace ucb {
namespace csv {

namespace {

constexpr int kPrecision = 15;  // configCUDA.h set_precision

void values_and_ic(std::ofstream& out, const Common& c) {
    out << "a[" << c.values.size() << "] = { ";
    for (size_t k = 0; k < c.values.size(); ++k) out << c.values[k] << (k + 1 < c.values.size() ? ", " : " }\n");
    out << "X0[" << c.ic.size() << "] = { ";
    for (size_t k = 0; k < c.ic.size(); ++k) out << c.ic[k] << (k + 1 < c.ic.size() ? ", " : " }\n");
}

void par_or_var_line(std::ofstream& out, int pov) {
    if (pov == 1) out << "Parameter estimation\n";
    else if (pov == 0) out << "Initial conditions estimation\n";
    else if (pov == 2) out << "Mixed: x=IC, y=parameter\n";
}

void grid(std::ofstream& out, int n, const double* v) {
    for (int iy = 0; iy < n; ++iy) {
        for (int ix = 0; ix < n; ++ix) {
            out << v[(size_t)iy * n + ix];
            if (ix + 1 < n) out << ", ";
        }
        out << '\n';
    }
}

void axes_block(std::ofstream& out, double tMax, double NT, double transient, double h, double eps, int i1, int i2,
                double r1lo, double r1hi, double r2lo, double r2hi, int n) {
    out << "CT = " << tMax << "\nNT = " << NT << "\nTT = " << transient << "\n";
    out << "h = " << h << "\neps = " << eps << "\n";
    out << "indices = " << i1 << ", " << i2 << "\n";
    out << "axis1: " << r1lo << " .. " << r1hi << "\n";
    out << "axis2: " << r2lo << " .. " << r2hi << "\n";
    out << "n_pts = " << n << "x" << n << "\n";
}

}  // namespace

void bif1d(const std::string& path, const Common& c, double tMax, double transient, double h, int pre,
           int writable_var, int index_of_mut_var, double lo, double hi, int n_pts, const int* counts,
           const double* peaks, const double* intervals, int max_peaks) {
    {
        std::ofstream cfg(path + "_config.csv");
        if (!cfg) return;
        cfg << std::setprecision(kPrecision);
        cfg << "1D classical bifurcation\nParameter estimation\n";
        values_and_ic(cfg, c);
        cfg << "CT = " << tMax << "\nTT = " << transient << "\nh = " << h << "\ndecimator = " << pre << "\n";
        cfg << "indexVar for peakfinder = " << writable_var << "\n";
        cfg << "indexPar for estimation = " << index_of_mut_var << "\n";
        cfg << "start value = " << lo << ", stop value = " << hi << "\n";
    }
    std::ofstream out(path);
    if (!out) return;
    out << std::setprecision(kPrecision);
    for (int i = 0; i < n_pts; ++i) {
        const double param = n_pts <= 1 ? lo : lo + (hi - lo) * (double)i / (double)(n_pts - 1);
        const int np = counts[i];
        if (np == 0) {
            out << param << ", " << 0 << ", " << 0 << '\n';
        } else if (np < 0) {
            out << param << ", " << 0 << ", " << -1 << '\n';
        } else {
            const int k = np < max_peaks ? np : max_peaks;
            for (int j = 0; j < k; ++j)
                out << param << ", " << peaks[(size_t)i * max_peaks + j] << ", " << intervals[(size_t)i * max_peaks + j]
                    << '\n';
        }
    }
}

void lle2d(const std::string& path, const Common& c, int par_or_var, double tMax, double NT, double transient,
           double h, double eps, int idx1, int idx2, double r1lo, double r1hi, double r2lo, double r2hi, int n_pts,
           const double* values) {
    {
        std::ofstream cfg(path + "_config.csv");
        if (!cfg) return;
        cfg << std::setprecision(kPrecision);
        cfg << "2D LLE\n";
        par_or_var_line(cfg, par_or_var);
        values_and_ic(cfg, c);
        axes_block(cfg, tMax, NT, transient, h, eps, idx1, idx2, r1lo, r1hi, r2lo, r2hi, n_pts);
    }
    std::ofstream out(path);
    if (!out) return;
    out << std::setprecision(kPrecision);
    grid(out, n_pts, values);
}

void ls2d(const std::string& path, const Common& c, int par_or_var, double tMax, double NT, double transient,
          double h, double eps, int idx1, int idx2, double r1lo, double r1hi, double r2lo, double r2hi, int n_pts,
          int n_exp, const double* values) {
    {
        std::ofstream cfg(path + "_config.csv");
        if (!cfg) return;
        cfg << std::setprecision(kPrecision);
        cfg << "2D LS\n";
        par_or_var_line(cfg, par_or_var);
        values_and_ic(cfg, c);
        axes_block(cfg, tMax, NT, transient, h, eps, idx1, idx2, r1lo, r1hi, r2lo, r2hi, n_pts);
        cfg << "exponents = " << n_exp << "\n";
    }
    std::ofstream out(path);
    if (!out) return;
    out << std::setprecision(kPrecision);
    const size_t total = (size_t)n_pts * n_pts;
    for (size_t cell = 0; cell < total; ++cell) {
        for (int k = 0; k < n_exp; ++k) {
            out << values[(size_t)k * total + cell];
            if (k + 1 < n_exp) out << ", ";
        }
        out << '\n';
    }
}

void bif2d(const std::string& path, const Common& c, int par_or_var, double tMax, double transient, double h,
           int pre, double eps_dbscan, int writable_var, int idx1, int idx2, double r1lo, double r1hi, double r2lo,
           double r2hi, int n_pts, const double* values) {
    {
        std::ofstream cfg(path + "_config.csv");
        if (!cfg) return;
        cfg << std::setprecision(kPrecision);
        cfg << "2D bifurcation (DBSCAN)\n";
        par_or_var_line(cfg, par_or_var);
        values_and_ic(cfg, c);
        cfg << "CT = " << tMax << "\nTT = " << transient << "\nh = " << h << "\ndecimator = " << pre << "\n";
        cfg << "eps_DBSCAN = " << eps_dbscan << "\n";
        cfg << "indexVar for peakfinder = " << writable_var << "\n";
        cfg << "indices = " << idx1 << ", " << idx2 << "\n";
        cfg << "axis1: " << r1lo << " .. " << r1hi << "\n";
        cfg << "axis2: " << r2lo << " .. " << r2hi << "\n";
        cfg << "n_pts = " << n_pts << "x" << n_pts << "\n";
    }
    std::ofstream out(path);
    if (!out) return;
    out << std::setprecision(kPrecision);
    grid(out, n_pts, values);
}

void basins(const std::string& path, const Common& c, double tMax, double transient, double h, int pre,
            double eps_dbscan, int writable_var, int xvar, int yvar, double xlo, double xhi, double ylo, double yhi,
            int n_pts, const int* labels, const double* avg_peaks, const double* avg_intervals, const int* classes) {
    {
        std::ofstream cfg(path + "_config.csv");
        if (cfg) {
            cfg << std::setprecision(kPrecision);
            cfg << "Basins of attraction\n";
            values_and_ic(cfg, c);
            cfg << "CT = " << tMax << "\nTT = " << transient << "\nh = " << h << "\n";
            cfg << "decimator = " << pre << "\neps_DBSCAN = " << eps_dbscan << "\n";
            cfg << "indexVar for peakfinder = " << writable_var << "\n";
            cfg << "indexVar for estimation = " << xvar << ", " << yvar << "\n";
            cfg << "start value_1 = " << xlo << ", stop value_1 = " << xhi << "\n";
            cfg << "start value_2 = " << ylo << ", stop value_2 = " << yhi << "\n";
        }
    }
    auto one = [&](const std::string& p, auto at) {
        std::ofstream o(p);
        if (!o) return;
        o << std::setprecision(kPrecision);
        o << xlo << " " << xhi << "\n" << ylo << " " << yhi << "\n";
        for (int iy = 0; iy < n_pts; ++iy) {
            for (int ix = 0; ix < n_pts; ++ix) {
                o << at((size_t)iy * n_pts + ix);
                if (ix + 1 < n_pts) o << ", ";
            }
            o << '\n';
        }
    };
    auto finite_or_999 = [](double v) { return std::isfinite(v) ? v : 999.0; };
    one(path, [&](size_t k) { return labels[k]; });
    one(path + "_1.csv", [&](size_t k) { return finite_or_999(avg_peaks[k]); });
    one(path + "_2.csv", [&](size_t k) { return finite_or_999(avg_intervals[k]); });
    one(path + "_3.csv", [&](size_t k) { return classes[k]; });
}

void curve1d(const std::string& path, const char* title, const Common& c, double tMax, double NT, double transient,
             double h, double eps, int index, double lo, double hi, bool log_scale, int n_pts, int n_cols,
             const double* v) {
    {
        std::ofstream cfg(path + "_config.csv");
        if (!cfg) return;
        cfg << std::setprecision(kPrecision);
        cfg << title << "\nParameter estimation\n";
        values_and_ic(cfg, c);
        cfg << "CT = " << tMax << "\nNT = " << NT << "\nTT = " << transient << "\n";
        cfg << "h = " << h << "\neps = " << eps << "\n";
        cfg << "indexPar = " << index << "\n";
        cfg << "start value = " << lo << ", stop value = " << hi << "\n";
    }
    std::ofstream out(path);
    if (!out) return;
    out << std::setprecision(kPrecision);
    for (int i = 0; i < n_pts; ++i) {
        double param = lo;
        if (n_pts > 1) {
            if (log_scale) {
                const double l0 = std::log10(lo), l1 = std::log10(hi);
                param = std::pow(10.0, l0 + (l1 - l0) * (double)i / (double)(n_pts - 1));
            } else {
                param = lo + (hi - lo) * (double)i / (double)(n_pts - 1);
            }
        }
        out << param;
        for (int k = 0; k < n_cols; ++k) out << ", " << v[(size_t)i * n_cols + k];
        out << '\n';
    }
}

}  // namespace csv
}  // namespace ucb
