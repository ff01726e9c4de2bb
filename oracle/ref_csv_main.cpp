// TEST INFRASTRUCTURE: writes CSV files with the reference's own writers (data_export.cpp,
// compiled as-is from the reference tree by oracle/build_ref.sh) from given result arrays,
// so that tests can compare the engine's CSV output with the reference's byte for byte.
// It never calls the engine.
//
// The snapshots are filled the way the reference's run_* paths fill them
// (U-CUDA/parametric_engine.cpp): a[] and X0[] narrowed to the device type numb (to_numb,
// :2256-2265 and the same lines of every run_*), the 1-D ranges narrowed to numb
// (`numb ranges[2]`, :2258; run_bif1d :1761), the 2-D ranges and the scalars in double.
// The files are written by the reference's export_* functions, whose layout equals what the
// run_* paths write for linear axes (config, then setprecision(set_precision) rows / grid).
//
// Usage: ref_csv <spec file>. The spec holds "key value..." lines: kind (lle2d, ls2d,
// bif2d, lle1d, ls1d, bif1d, basins), path, values, ic, scalars, and data files of raw
// little-endian arrays (double unless noted).
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "data_export.h"
#include "parametric_engine.h"

namespace {

std::map<std::string, std::vector<std::string>> read_spec(const char* path) {
    std::map<std::string, std::vector<std::string>> m;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream is(line);
        std::string key, tok;
        if (!(is >> key)) continue;
        auto& v = m[key];
        while (is >> tok) v.push_back(tok);
    }
    return m;
}

template <class T>
std::vector<T> read_bin(const std::string& path, size_t count) {
    std::vector<T> v(count);
    std::ifstream f(path, std::ios::binary);
    f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(count * sizeof(T)));
    if ((size_t)f.gcount() != count * sizeof(T)) {
        std::fprintf(stderr, "short read: %s\n", path.c_str());
        std::exit(2);
    }
    return v;
}

struct Spec {
    std::map<std::string, std::vector<std::string>> m;
    std::string s(const char* k) const { return m.at(k).at(0); }
    double d(const char* k) const { return std::stod(s(k)); }
    int i(const char* k) const { return std::stoi(s(k)); }
    std::vector<double> numb_list(const char* k) const {  // narrowed to numb, as to_numb does
        std::vector<double> out;
        for (auto& t : m.at(k)) out.push_back((double)(numb)std::stod(t));
        return out;
    }
};

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: ref_csv <spec>\n");
        return 2;
    }
    const Spec sp{read_spec(argv[1])};
    const std::string kind = sp.s("kind"), path = sp.s("path");
    const int n = sp.i("n_pts");
    const std::vector<double> values = sp.numb_list("values"), ic = sp.numb_list("ic");
    bool ok = false;
    if (kind == "lle2d" || kind == "ls2d" || kind == "bif2d") {
        const size_t cells = (size_t)n * n;
        if (kind == "lle2d") {
            LLE2DResult r;
            auto& s = r.snapshot;
            s.values = values;
            s.initial_conditions = ic;
            s.par_or_var = sp.i("par_or_var");
            s.tMax = sp.d("tMax"); s.NT = sp.d("NT"); s.transientTime = sp.d("transient"); s.h = sp.d("h");
            s.eps = sp.d("eps");
            s.indexOfMutVar = sp.i("idx1"); s.indexOfMutVar2 = sp.i("idx2");
            s.range1_lo = sp.d("r1lo"); s.range1_hi = sp.d("r1hi"); s.range2_lo = sp.d("r2lo"); s.range2_hi = sp.d("r2hi");
            s.n_pts = n;
            r.n_pts = n;
            r.values = read_bin<double>(sp.s("data"), cells);
            ok = data_export::export_lle2d(r, path);
        } else if (kind == "ls2d") {
            LS2DResult r;
            auto& s = r.snapshot;
            s.values = values;
            s.initial_conditions = ic;
            s.par_or_var = sp.i("par_or_var");
            s.tMax = sp.d("tMax"); s.NT = sp.d("NT"); s.transientTime = sp.d("transient"); s.h = sp.d("h");
            s.eps = sp.d("eps");
            s.indexOfMutVar = sp.i("idx1"); s.indexOfMutVar2 = sp.i("idx2");
            s.range1_lo = sp.d("r1lo"); s.range1_hi = sp.d("r1hi"); s.range2_lo = sp.d("r2lo"); s.range2_hi = sp.d("r2hi");
            s.n_pts = n;
            s.n_exponents = sp.i("n_exp");
            r.n_pts = n;
            r.n_exponents = s.n_exponents;
            r.values = read_bin<double>(sp.s("data"), cells * (size_t)s.n_exponents);
            ok = data_export::export_ls2d(r, path);
        } else {
            Bifurcation2DResult r;
            auto& s = r.snapshot;
            s.values = values;
            s.initial_conditions = ic;
            s.par_or_var = sp.i("par_or_var");
            s.tMax = sp.d("tMax"); s.transientTime = sp.d("transient"); s.h = sp.d("h");
            s.preScaller = sp.i("pre");
            s.eps_dbscan = sp.d("eps_dbscan");
            s.writableVar = sp.i("writable_var");
            s.indexOfMutVar = sp.i("idx1"); s.indexOfMutVar2 = sp.i("idx2");
            s.range1_lo = sp.d("r1lo"); s.range1_hi = sp.d("r1hi"); s.range2_lo = sp.d("r2lo"); s.range2_hi = sp.d("r2hi");
            s.n_pts = n;
            r.n_pts = n;
            r.values = read_bin<double>(sp.s("data"), cells);
            ok = data_export::export_bif2d(r, path);
        }
    } else if (kind == "lle1d" || kind == "ls1d") {
        const double lo = (double)(numb)sp.d("lo"), hi = (double)(numb)sp.d("hi");
        if (kind == "lle1d") {
            LLE1DResult r;
            auto& s = r.snapshot;
            s.values = values;
            s.initial_conditions = ic;
            s.tMax = sp.d("tMax"); s.NT = sp.d("NT"); s.transientTime = sp.d("transient"); s.h = sp.d("h");
            s.eps = sp.d("eps");
            s.indexOfMutVar = sp.i("idx1");
            s.range_lo = lo; s.range_hi = hi;
            r.n_pts = n;
            r.lyapunov = read_bin<double>(sp.s("data"), (size_t)n);
            ok = data_export::export_lle1d(r, path);
        } else {
            LS1DResult r;
            auto& s = r.snapshot;
            s.values = values;
            s.initial_conditions = ic;
            s.tMax = sp.d("tMax"); s.NT = sp.d("NT"); s.transientTime = sp.d("transient"); s.h = sp.d("h");
            s.eps = sp.d("eps");
            s.indexOfMutVar = sp.i("idx1");
            s.range_lo = lo; s.range_hi = hi;
            const int ne = sp.i("n_exp");
            r.n_pts = n;
            r.n_exponents = ne;
            const std::vector<double> flat = read_bin<double>(sp.s("data"), (size_t)n * ne);  // point-major
            r.spectrum.assign(n, std::vector<double>(ne));
            for (int p = 0; p < n; ++p)
                for (int k = 0; k < ne; ++k) r.spectrum[p][k] = flat[(size_t)p * ne + k];
            ok = data_export::export_ls1d(r, path);
        }
    } else if (kind == "bif1d") {
        Bifurcation1DResult r;
        auto& s = r.snapshot;
        s.values = values;
        s.initial_conditions = ic;
        s.tMax = sp.d("tMax"); s.transientTime = sp.d("transient"); s.h = sp.d("h");
        s.preScaller = sp.i("pre");
        s.writableVar = sp.i("writable_var");
        s.indexOfMutVar = sp.i("idx1");
        s.range_lo = (double)(numb)sp.d("lo");
        s.range_hi = (double)(numb)sp.d("hi");
        const int cap = sp.i("cap");
        r.n_pts = n;
        const std::vector<int32_t> counts = read_bin<int32_t>(sp.s("counts"), (size_t)n);
        const std::vector<double> pk = read_bin<double>(sp.s("peaks"), (size_t)n * cap);
        const std::vector<double> tm = read_bin<double>(sp.s("intervals"), (size_t)n * cap);
        r.flags.assign(counts.begin(), counts.end());
        r.bifurcation_points.assign(n, {});
        r.peak_times.assign(n, {});
        for (int p = 0; p < n; ++p) {
            const int k = counts[p] > 0 ? (counts[p] < cap ? counts[p] : cap) : 0;
            r.bifurcation_points[p].assign(pk.begin() + (size_t)p * cap, pk.begin() + (size_t)p * cap + k);
            r.peak_times[p].assign(tm.begin() + (size_t)p * cap, tm.begin() + (size_t)p * cap + k);
        }
        ok = data_export::export_bif1d(r, path);
    } else if (kind == "basins") {
        BasinsResult r;
        auto& s = r.snapshot;
        s.values = values;
        s.initial_conditions = ic;
        s.tMax = sp.d("tMax"); s.transientTime = sp.d("transient"); s.h = sp.d("h");
        s.preScaller = sp.i("pre");
        s.eps_dbscan = sp.d("eps_dbscan");
        s.writableVar = sp.i("writable_var");
        s.axis_x_var = sp.i("xvar"); s.axis_y_var = sp.i("yvar");
        s.axis_x_lo = sp.d("xlo"); s.axis_x_hi = sp.d("xhi"); s.axis_y_lo = sp.d("ylo"); s.axis_y_hi = sp.d("yhi");
        s.n_pts = n;
        r.n_pts = n;
        const size_t cells = (size_t)n * n;
        const std::vector<int32_t> lab = read_bin<int32_t>(sp.s("labels"), cells);
        const std::vector<int32_t> cls = read_bin<int32_t>(sp.s("classes"), cells);
        r.basin_idx.assign(lab.begin(), lab.end());
        r.helpful_array.assign(cls.begin(), cls.end());
        r.avg_peaks = read_bin<double>(sp.s("f1"), cells);
        r.avg_intervals = read_bin<double>(sp.s("f2"), cells);
        ok = data_export::export_basins(r, path);
    } else {
        std::fprintf(stderr, "unknown kind %s\n", kind.c_str());
        return 2;
    }
    return ok ? 0 : 1;
}
