// ============================================================================
// ORACLE — test infrastructure, never part of the product.
//
// CPU restatement of the reference's per-cell hot path, used ONLY as the checker
// in tests/, by __graft_entry__.smoke(), and as the timed CPU baseline in bench.py.
// The product (u-cuda_b200/) never links, loads or calls anything in oracle/.
//
// What it restates (reference paths are relative to the U-CUDA project):
//   * krs_cpu.cpp:293-316  make_source  — prelude around the KRS step body; the body is
//     compiled natively (g++ -O2 -ffp-contract=off, dlopen) instead of cl.exe + LoadLibrary
//     (krs_cpu.cpp:405-478).
//   * cudaLibrary.cu:782-895  loopCalculateDiscreteModel_int (CPU twin
//     parametric_engine.cpp:59-101): n steps, optional recording, divergence check
//     every CHECK_INTERVAL=100 iterations, one extra preScaller step, fixed-point test.
//   * cudaLibrary.cu:1344-1361 getValueByIdx, :1381-1396 getValueByIdx_log.
//   * lle2d.template.cu:45-56 RNG stub (splitmix64 init + LCG uniform), identical to
//     the CPU twin at parametric_engine.cpp:196-209.
//   * cudaLibrary.cu:2486-2693 LLEKernelCUDA — per-cell Benettin LLE with a shadow
//     trajectory (GPU semantics: (1/eps)*(x-y), floor 1e-14, result/tMax).
//   * cudaLibrary.cu:2832-2874 projectionOperator / gramSchmidtProcess (classical GS)
//     and :2878-3073 LSKernelCUDA — full spectrum with N shadow probes.
//   * cudaLibrary.cu:944-1077 calculateDiscreteModelCUDA + :1503-1633 peakFinder —
//     bifurcation (transient, recorded series, parabolic peaks, first peak dropped,
//     inter-peak intervals, cap 2500) with the host sizing of parametric_engine.cpp:1816.
//   * parametric_engine.cpp:2587-2965 run_lle_2d host mapping (par_or_var, swap_xy,
//     999 sentinel -> flag -1), :3430-3786 run_ls_2d (plane-major values).
// New-semantics checkers (no reference counterpart, parity unpinned against it):
//   * stroboscopic basin labelling, DP5(4) + modified Gram-Schmidt spectrum and the
//     tangent-linear LLE, restated from their published algorithms (see the functions).
//
// numb is a template parameter: double (the FP64 oracle) or float (the reference's
// shipped configCUDA.h:4 setting).
// ============================================================================
#include <dlfcn.h>
#include <omp.h>
#include <unistd.h>
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

namespace {

constexpr int kCheckInterval = 100;             // configCUDA.h:12
constexpr double kEpsFixedPoint = 1e-8;         // configCUDA.h eps_fixed_point
constexpr double kEpsPeakDelta = 1e-14;         // configCUDA.h eps_peak_delta
constexpr double kPeakThreshold = -1e25;        // configCUDA.h peak_threshold
constexpr int kMaxAmountOfPeaks = 2500;         // configCUDA.h max_amount_of_peaks
constexpr double kPi = 3.1415926535897932384626433832795;
constexpr double kEuler = 2.7182818284590452353602874713527;

std::string g_err;

// ---------------------------------------------------------------------------
// KRS step compilation (krs_cpu.cpp:293-316 prelude, Linux toolchain)
// ---------------------------------------------------------------------------
std::string make_source(const std::string& body, int amountOfX, bool dbl, bool dual, bool rhs = false) {
    std::ostringstream o;
    o << "#include <cmath>\n#include <cstdlib>\nusing std::abs;\n";
    if (dual) {
        // Forward-mode dual numbers: the same step body evaluated on (value, tangent)
        // pairs gives the exact directional derivative of the step map. Used by the
        // tangent-linear checkers; independent of the product's symbolic Jacobian.
        o << "struct D { double v, d; D() : v(0), d(0) {} D(double x) : v(x), d(0) {}\n"
             "  D(double x, double y) : v(x), d(y) {} };\n"
             "static inline D operator+(D a, D b) { return D(a.v + b.v, a.d + b.d); }\n"
             "static inline D operator-(D a, D b) { return D(a.v - b.v, a.d - b.d); }\n"
             "static inline D operator-(D a) { return D(-a.v, -a.d); }\n"
             "static inline D operator*(D a, D b) { return D(a.v * b.v, a.d * b.v + a.v * b.d); }\n"
             "static inline D operator/(D a, D b) { return D(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)); }\n"
             "static inline D& operator+=(D& a, D b) { a = a + b; return a; }\n"
             "static inline D& operator-=(D& a, D b) { a = a - b; return a; }\n"
             "static inline D& operator*=(D& a, D b) { a = a * b; return a; }\n"
             "static inline D& operator/=(D& a, D b) { a = a / b; return a; }\n"
             "static inline bool operator<(D a, D b) { return a.v < b.v; }\n"
             "static inline bool operator>(D a, D b) { return a.v > b.v; }\n"
             "static inline D sin(D a) { return D(std::sin(a.v), std::cos(a.v) * a.d); }\n"
             "static inline D cos(D a) { return D(std::cos(a.v), -std::sin(a.v) * a.d); }\n"
             "static inline D tan(D a) { double t = std::tan(a.v); return D(t, (1 + t * t) * a.d); }\n"
             "static inline D exp(D a) { double e = std::exp(a.v); return D(e, e * a.d); }\n"
             "static inline D log(D a) { return D(std::log(a.v), a.d / a.v); }\n"
             "static inline D sqrt(D a) { double s = std::sqrt(a.v); return D(s, a.d / (2 * s)); }\n"
             "static inline D sinh(D a) { return D(std::sinh(a.v), std::cosh(a.v) * a.d); }\n"
             "static inline D cosh(D a) { return D(std::cosh(a.v), std::sinh(a.v) * a.d); }\n"
             "static inline D tanh(D a) { double t = std::tanh(a.v); return D(t, (1 - t * t) * a.d); }\n"
             "static inline D atan(D a) { return D(std::atan(a.v), a.d / (1 + a.v * a.v)); }\n"
             "static inline D fabs(D a) { return a.v < 0 ? -a : a; }\n"
             "static inline D abs(D a) { return fabs(a); }\n"
             "static inline D pow(D a, D b) { double p = std::pow(a.v, b.v);\n"
             "  double dd = b.d == 0 ? b.v * std::pow(a.v, b.v - 1) * a.d\n"
             "                       : p * (b.d * std::log(a.v) + b.v * a.d / a.v); return D(p, dd); }\n"
             "typedef D numb;\n";
    } else {
        o << "typedef " << (dbl ? "double" : "float") << " numb;\n";
    }
    o << "static inline numb min(numb x, numb y) { return x < y ? x : y; }\n"
         "static inline numb max(numb x, numb y) { return x > y ? x : y; }\n"
         "#define AMOUNTOFX " << amountOfX << "\n"
         "static const numb pi    = (numb)3.1415926535897932384626433832795;\n"
         "static const numb euler = (numb)2.7182818284590452353602874713527;\n"
         "extern \"C\" __attribute__((visibility(\"default\")))\n";
    if (rhs)
        o << "void krs_rhs(const numb* X1, const numb* a, numb* dX) {\n";
    else
        o << "void krs_step(numb* X, const numb* a, numb h) {\n";
    o << "#line 1 \"krs\"\n" << body << "\n}\n";
    return o.str();
}

uint64_t fnv1a(const std::string& s, uint64_t h = 1469598103934665603ULL) {
    for (unsigned char c : s) { h ^= c; h *= 1099511628211ULL; }
    return h;
}

std::string cache_dir() {
    const char* e = std::getenv("UCB_ORACLE_CACHE");
    std::string d = e ? e : "/tmp/ucb_oracle_cache";
    mkdir(d.c_str(), 0755);
    return d;
}

std::mutex g_compile_mu;

struct Krs {
    void* lib = nullptr;
    void* fn = nullptr;
    int nx = 0;
    int numb_bytes = 8;  // 8 double, 4 float, 16 dual
};

Krs* compile_krs(const std::string& body, int nx, int numb_bytes, const char* extra_flags, bool rhs = false) {
    std::lock_guard<std::mutex> lk(g_compile_mu);
    const bool dual = numb_bytes == 16;
    const std::string src = make_source(body, nx, numb_bytes == 8, dual, rhs);
    const std::string flags = std::string("-O2 -ffp-contract=off -fPIC -shared ") + (extra_flags ? extra_flags : "");
    const uint64_t h = fnv1a(flags, fnv1a(src));
    char name[64];
    std::snprintf(name, sizeof name, "krs_%016llx", (unsigned long long)h);
    const std::string dir = cache_dir();
    const std::string so = dir + "/" + name + ".so";
    if (access(so.c_str(), R_OK) != 0) {
        const std::string cpp = dir + "/" + name + ".cpp";
        {
            std::ofstream f(cpp);
            f << src;
        }
        const std::string tmp = so + ".tmp." + std::to_string(getpid());
        const std::string log = dir + "/" + name + ".log";
        const char* cxx_env = std::getenv("UCB_ORACLE_CXX");
        const std::string cxx = cxx_env ? cxx_env : (access("/usr/bin/g++", X_OK) == 0 ? "/usr/bin/g++" : "g++");
        const std::string cmd = cxx + " " + flags + " -o " + tmp + " " + cpp + " > " + log + " 2>&1";
        if (std::system(cmd.c_str()) != 0) {
            std::ifstream lf(log);
            std::stringstream ss;
            ss << lf.rdbuf();
            g_err = "CPU KRS compile failed:\n" + ss.str();
            return nullptr;
        }
        std::rename(tmp.c_str(), so.c_str());
    }
    void* lib = dlopen(so.c_str(), RTLD_NOW | RTLD_LOCAL);
    if (!lib) { g_err = std::string("dlopen: ") + dlerror(); return nullptr; }
    void* fn = dlsym(lib, rhs ? "krs_rhs" : "krs_step");
    if (!fn) { g_err = "step function not exported"; dlclose(lib); return nullptr; }
    Krs* k = new Krs;
    k->lib = lib; k->fn = fn; k->nx = nx; k->numb_bytes = numb_bytes;
    return k;
}

// ---------------------------------------------------------------------------
// loopCalculateDiscreteModel_int (cudaLibrary.cu:782-895)
// ---------------------------------------------------------------------------
template <class T>
using StepFn = void (*)(T*, const T*, T);

template <class T>
int loop_model(StepFn<T> step, T* x, const T* a, T h, int64_t iters, int nx,
               int preScaller, int writableVar, T maxValue, T* data) {
    T xPrev[64];
    for (int64_t i = 0; i < iters; ++i) {
        if (data != nullptr) {
            if (writableVar < 0) {
                if (nx >= 3) data[i] = x[0] + (T)kPi * x[1] + (T)kEuler * x[2];
                else if (nx == 2) data[i] = x[0] + (T)kPi * x[1];
                else data[i] = x[0];
            } else {
                data[i] = x[writableVar];
            }
            for (int j = 0; j < preScaller; ++j) step(x, a, h);
        } else {
            step(x, a, h);
        }
        if (i % kCheckInterval == 0) {
            T checker = 0;
            for (int j = 0; j < nx; ++j) checker = checker + std::fabs(x[j]);
            if (std::isnan(checker) || std::isinf(checker)) return 0;
            if (maxValue != 0)
                if (std::fabs(checker) > maxValue) return 0;
        }
    }
    for (int j = 0; j < nx; ++j) xPrev[j] = x[j];
    for (int j = 0; j < preScaller; ++j) step(x, a, h);
    T tempResult = 0;
    for (int j = 0; j < nx; ++j) tempResult += std::fabs(x[j] - xPrev[j]);
    if (std::fabs(tempResult) < (T)kEpsFixedPoint) return -1;
    return 1;
}

// ---------------------------------------------------------------------------
// getValueByIdx / getValueByIdx_log (cudaLibrary.cu:1344-1396), numb arithmetic
// ---------------------------------------------------------------------------
template <class T>
T value_by_idx(int64_t idx, int nPts, T lo, T hi, int valueNumber) {
    if (nPts <= 0) return lo;
    if (nPts == 1) return hi;
    const int64_t divisor = (valueNumber == 0) ? 1 : nPts;
    const int64_t pointIdx = (idx / divisor) % nPts;
    const T t = static_cast<T>(pointIdx) / static_cast<T>(nPts - 1);
    return (static_cast<T>(1.0) - t) * lo + t * hi;
}

template <class T>
T value_by_idx_log(int64_t idx, int nPts, T lo, T hi, int valueNumber) {
    const T l = std::log10(lo) + (T)(((int64_t)((int64_t)idx / std::pow((T)nPts, (T)valueNumber)) % nPts)
                                   * ((T)(std::log10(hi) - std::log10(lo)) / (T)(nPts - 1)));
    return std::pow((T)10.0, l);
}

// ---------------------------------------------------------------------------
// RNG stub (lle2d.template.cu:45-56 == parametric_engine.cpp:196-209)
// ---------------------------------------------------------------------------
struct Rng { uint64_t state; };
inline void rng_init(uint64_t seed, uint64_t seq, uint64_t off, Rng* s) {
    uint64_t z = seed + seq * 0x9E3779B97F4A7C15ULL + off;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    s->state = z ^ (z >> 31);
}
inline float rng_uniform(Rng* s) {
    s->state = s->state * 6364136223846793005ULL + 1442695040888963407ULL;
    return (float)(((s->state >> 40) & 0xFFFFFFULL) + 1ULL) / 16777216.0f;
}

// ---------------------------------------------------------------------------
// Shared grid description (the kernel arguments of LLEKernelCUDA / LSKernelCUDA /
// calculateDiscreteModelCUDA after run_* host mapping).
// ---------------------------------------------------------------------------
struct Grid {
    int nPts;            // side (1D: number of points)
    int dimension;       // 1 or 2
    int par_or_var;      // 1 param, 0 IC, 2 mixed (axis 0 IC, axis 1 param)
    int idx[2];          // indicesOfMutVars
    double ranges[4];
    int log_mask;
    int h_axis;          // -1 none
};

template <class T>
struct CellInit {
    T x[64];
    T a[64];
    T h;
};

// Applies the sweep of one cell (the par_or_var branches of the kernels).
template <class T>
void init_cell(const Grid& g, int64_t idx, int nx, const double* ic, int nv, const double* vals,
               double h, CellInit<T>* c) {
    for (int i = 0; i < nx; ++i) c->x[i] = (T)ic[i];
    for (int i = 0; i < nv; ++i) c->a[i] = (T)vals[i];
    const T r[4] = {(T)g.ranges[0], (T)g.ranges[1], (T)g.ranges[2], (T)g.ranges[3]};
    auto axis_val = [&](int i) -> T {
        const bool lg = (g.log_mask >> i) & 1;
        return lg ? value_by_idx_log<T>(idx, g.nPts, r[2 * i], r[2 * i + 1], i)
                  : value_by_idx<T>(idx, g.nPts, r[2 * i], r[2 * i + 1], i);
    };
    c->h = (T)h;
    if (g.h_axis == 0) c->h = axis_val(0);
    else if (g.h_axis == 1) c->h = axis_val(1);
    if (g.par_or_var == 1) {
        for (int i = 0; i < g.dimension; ++i) { if (i == g.h_axis) continue; c->a[g.idx[i]] = axis_val(i); }
    } else if (g.par_or_var == 0) {
        for (int i = 0; i < g.dimension; ++i) { if (i == g.h_axis) continue; c->x[g.idx[i]] = axis_val(i); }
    } else if (g.par_or_var == 2) {
        c->x[g.idx[0]] = axis_val(0);
        c->a[g.idx[1]] = axis_val(1);
    }
}

// ---------------------------------------------------------------------------
// LLEKernelCUDA (cudaLibrary.cu:2486-2693), one cell
// ---------------------------------------------------------------------------
template <class T>
T lle_cell(StepFn<T> step, const Grid& g, int64_t idx, int nx, const double* ic, int nv,
           const double* vals, double h_d, double NT_d, double tMax_d, double transient_d,
           double eps_d, double maxv_d, int sizeOfBlock, int skipHost, uint64_t rng_seq) {
    CellInit<T> c;
    init_cell<T>(g, idx, nx, ic, nv, vals, h_d, &c);
    const T h = c.h, NT = (T)NT_d, tMax = (T)tMax_d, eps = (T)eps_d, maxv = (T)maxv_d;
    if (h <= 0) return (T)NAN;
    const int64_t ntp = (g.h_axis != -1) ? (int64_t)std::ceil(NT / h) : (int64_t)(NT / (T)h_d);
    const int64_t skip = (g.h_axis != -1) ? (int64_t)std::ceil((T)transient_d / h) : (int64_t)skipHost;
    T* x = c.x;
    int flag = loop_model<T>(step, x, c.a, h, skip, nx, 1, 0, maxv, nullptr);
    if (flag == 0) return (T)999;
    Rng st;
    rng_init(1234567891ULL, rng_seq, 0ULL, &st);
    T z[64], y[64];
    T zPower = 0;
    for (int i = 0; i < nx; ++i) { z[i] = rng_uniform(&st) - 0.5; zPower += z[i] * z[i]; }
    zPower = std::sqrt(zPower);
    for (int i = 0; i < nx; ++i) z[i] /= zPower;
    for (int i = 0; i < nx; ++i) y[i] = z[i] * eps + x[i];
    T result = 0;
    for (int b = 0; b < sizeOfBlock; ++b) {
        if (loop_model<T>(step, x, c.a, h, ntp, nx, 1, 0, maxv, nullptr) == 0) return (T)999;
        if (loop_model<T>(step, y, c.a, h, ntp, nx, 1, 0, maxv, nullptr) == 0) return (T)999;
        T tempData = 0, tempData2 = 0;
        for (int l = 0; l < nx; ++l) {
            tempData2 = (T)1.0 / eps;
            tempData2 = tempData2 * (x[l] - y[l]);
            tempData += tempData2 * tempData2;
        }
        tempData = std::sqrt(tempData);
        if (tempData <= 1e-14) tempData = (T)1e-14;
        result += std::log(tempData);
        tempData = (1 / tempData);
        for (int j = 0; j < nx; ++j) y[j] = (T)(x[j] - ((x[j] - y[j] + 1e-14) * tempData));
    }
    return result / tMax;
}

// ---------------------------------------------------------------------------
// gramSchmidtProcess (cudaLibrary.cu:2832-2874) — classical GS, row-major N x N
// ---------------------------------------------------------------------------
template <class T>
void projection(const T* a, const T* b, T* minuend, int n) {
    T num = 0, den = 0;
    for (int i = 0; i < n; ++i) { num += a[i] * b[i]; den += b[i] * b[i]; }
    const T frac = den == 0 ? 0 : num / den;
    for (int i = 0; i < n; ++i) minuend[i] -= frac * b[i];
}

template <class T>
void gram_schmidt(const T* a, T* b, int n, T* dens) {
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) b[j + i * n] = a[j + i * n];
        for (int j = 0; j < i; ++j) projection(a + i * n, b + j * n, b + i * n, n);
    }
    for (int i = 0; i < n; ++i) {
        T den = 0;
        for (int j = 0; j < n; ++j) den += b[i * n + j] * b[i * n + j];
        den = std::sqrt(den);
        for (int j = 0; j < n; ++j) b[i * n + j] = den == 0 ? 0 : b[i * n + j] / den;
        if (dens) dens[i] = den;
    }
}

// LSKernelCUDA (cudaLibrary.cu:2878-3073), one cell -> n exponents
template <class T>
void ls_cell(StepFn<T> step, const Grid& g, int64_t idx, int nx, const double* ic, int nv,
             const double* vals, double h_d, double NT_d, double tMax_d, double transient_d,
             double eps_d, double maxv_d, int sizeOfBlock, int skipHost, uint64_t rng_seq, T* out) {
    CellInit<T> c;
    init_cell<T>(g, idx, nx, ic, nv, vals, h_d, &c);
    const T h = c.h, NT = (T)NT_d, tMax = (T)tMax_d, eps = (T)eps_d, maxv = (T)maxv_d;
    if (h <= 0) { for (int m = 0; m < nx; ++m) out[m] = (T)NAN; return; }
    const int64_t ntp = (g.h_axis != -1) ? (int64_t)std::ceil(NT / h) : (int64_t)(NT / (T)h_d);
    const int64_t skip = (g.h_axis != -1) ? (int64_t)std::ceil((T)transient_d / h) : (int64_t)skipHost;
    T* x = c.x;
    std::vector<T> y(nx * nx), z(nx * nx), result(nx, 0), dens(nx, 0);
    Rng st;
    rng_init(1234567891ULL, rng_seq, 0ULL, &st);
    for (int j = 0; j < nx; ++j) {
        T zPower = 0;
        for (int i = 0; i < nx; ++i) {
            z[j * nx + i] = rng_uniform(&st) - 0.5;
            zPower += z[j * nx + i] * z[j * nx + i];
        }
        zPower = std::sqrt(zPower);
        for (int i = 0; i < nx; ++i) z[j * nx + i] /= zPower;
    }
    int flag = loop_model<T>(step, x, c.a, h, skip, nx, 1, 0, maxv, nullptr);
    if (flag == 0) { for (int m = 0; m < nx; ++m) out[m] = (T)999; return; }
    gram_schmidt<T>(z.data(), y.data(), nx, nullptr);
    for (int j = 0; j < nx; ++j)
        for (int i = 0; i < nx; ++i) y[j * nx + i] = y[j * nx + i] * eps + x[i];
    for (int b = 0; b < sizeOfBlock; ++b) {
        if (loop_model<T>(step, x, c.a, h, ntp, nx, 1, 0, maxv, nullptr) == 0) {
            for (int m = 0; m < nx; ++m) out[m] = (T)999;
            return;
        }
        for (int j = 0; j < nx; ++j) {
            if (loop_model<T>(step, y.data() + j * nx, c.a, h, ntp, nx, 1, 0, maxv, nullptr) == 0) {
                for (int m = 0; m < nx; ++m) out[m] = (T)999;
                return;
            }
        }
        for (int k = 0; k < nx; ++k)
            for (int l = 0; l < nx; ++l) y[k * nx + l] = y[k * nx + l] - x[l];
        gram_schmidt<T>(y.data(), z.data(), nx, dens.data());
        for (int k = 0; k < nx; ++k) {
            result[k] += std::log(dens[k] / eps);
            for (int j = 0; j < nx; ++j) y[k * nx + j] = (T)(x[j] + z[k * nx + j] * eps);
        }
    }
    for (int i = 0; i < nx; ++i) out[i] = result[i] / tMax;
}

// ---------------------------------------------------------------------------
// peakFinder (cudaLibrary.cu:1503-1633), block-local indexing
// ---------------------------------------------------------------------------
template <class T>
int peak_finder(const T* data, int64_t n, T* outPeaks, T* timeOfPeaks, T h) {
    int amountOfPeaks = 0;
    if (n < 5) return 0;  // the GPU loop bound n-2 is unsigned; no peaks can exist below 5
    for (int64_t i = 2; i < n - 2; ++i) {
        if (data[i] - data[i - 1] > (T)kEpsPeakDelta && data[i] > (T)kPeakThreshold && data[i] >= data[i + 1]) {
            for (int64_t j = i; j < n - 2; ++j) {
                if (data[j] < data[j + 1]) { i = j + 1; break; }
                if (data[j] - data[j + 1] > (T)kEpsPeakDelta) {
                    T denom = data[j - 1] - (T)2.0 * data[j] + data[j + 1];
                    T delta = 0.0;
                    if (std::fabs(denom) > 1e-12) delta = 0.5 * (data[j - 1] - data[j + 1]) / denom;
                    outPeaks[amountOfPeaks] = data[j] - 0.25 * (data[j - 1] - data[j + 1]) * delta;
                    timeOfPeaks[amountOfPeaks] = (T)(j - 1) + delta;
                    ++amountOfPeaks;
                    i = j + 1;
                    break;
                }
            }
        }
    }
    if (amountOfPeaks > 1) {
        for (int i = 0; i < amountOfPeaks - 1; i++) {
            outPeaks[i] = outPeaks[i + 1];
            timeOfPeaks[i] = (T)(timeOfPeaks[i + 1] - timeOfPeaks[i]) * h;
        }
        amountOfPeaks = amountOfPeaks - 1;
    } else {
        amountOfPeaks = 0;
    }
    if (amountOfPeaks >= kMaxAmountOfPeaks) amountOfPeaks = kMaxAmountOfPeaks;
    return amountOfPeaks;
}

// ---------------------------------------------------------------------------
// Tangent-linear spectrum with adaptive Dormand-Prince 5(4) (new semantics; no reference
// counterpart). Published pair of Dormand & Prince (1980): FSAL, RMS error norm over the
// augmented state (x, V) with sc_i = atol + rtol max(|y_i|, |y_new_i|) (the state alone
// while not measuring), accept if err <= 1, step factor
// 0.9 err^(-1/5) clamped to [0.2, 5] (upper clamp 2 right after a rejection). The N
// tangent vectors follow v' = J(x) v with the same stages (J v from forward-mode dual
// numbers of the right-hand side), modified Gram-Schmidt every gs_every accepted steps
// and at the end; lambda_k = sum log(norm_k) / t_end over [transient, transient + t_end].
// ---------------------------------------------------------------------------
struct Dual { double v, d; };
using RhsFn = void (*)(const double*, const double*, double*);
using RhsDualFn = void (*)(const Dual*, const Dual*, Dual*);

struct Dp5Coef {
    double a[7][6] = {{0}};
    double b[7] = {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84, 0};
    double e[7] = {71.0 / 57600, 0, -71.0 / 16695, 71.0 / 1920, -17253.0 / 339200, 22.0 / 525, -1.0 / 40};
    Dp5Coef() {
        a[1][0] = 1.0 / 5;
        a[2][0] = 3.0 / 40; a[2][1] = 9.0 / 40;
        a[3][0] = 44.0 / 45; a[3][1] = -56.0 / 15; a[3][2] = 32.0 / 9;
        a[4][0] = 19372.0 / 6561; a[4][1] = -25360.0 / 2187; a[4][2] = 64448.0 / 6561; a[4][3] = -212.0 / 729;
        a[5][0] = 9017.0 / 3168; a[5][1] = -355.0 / 33; a[5][2] = 46732.0 / 5247; a[5][3] = 49.0 / 176;
        a[5][4] = -5103.0 / 18656;
    }
};

void jvp(RhsDualFn fd, const double* x, const double* av, int nv, const double* v, double* out, int nx) {
    Dual X[64], A[64], D[64];
    for (int i = 0; i < nx; ++i) X[i] = {x[i], v[i]};
    for (int i = 0; i < nv; ++i) A[i] = {av[i], 0.0};
    fd(X, A, D);
    for (int i = 0; i < nx; ++i) out[i] = D[i].d;
}

bool mgs_cpu(std::vector<double>& V, int n, double* acc) {
    for (int k = 0; k < n; ++k) {
        for (int j = 0; j < k; ++j) {
            double d = 0;
            for (int l = 0; l < n; ++l) d += V[k * n + l] * V[j * n + l];
            for (int l = 0; l < n; ++l) V[k * n + l] -= d * V[j * n + l];
        }
        double n2 = 0;
        for (int l = 0; l < n; ++l) n2 += V[k * n + l] * V[k * n + l];
        const double nrm = std::sqrt(n2);
        if (!(nrm > 0) || !std::isfinite(nrm)) return false;
        if (acc) acc[k] += std::log(nrm);
        for (int l = 0; l < n; ++l) V[k * n + l] /= nrm;
    }
    return true;
}

void ls_cell_dp5_cpu(RhsFn f, RhsDualFn fd, int nx, const double* x0, const double* av, int nv, double transient,
                     double t_end, double rtol, double atol, double h0, int gs_every, long long max_steps,
                     double maxv, uint64_t seq, double* out) {
    static const Dp5Coef C;
    std::vector<double> x(x0, x0 + nx), V((size_t)nx * nx), K(7 * (size_t)nx), xs(nx), xn(nx);
    Rng st;
    rng_init(1234567891ULL, seq, 0ULL, &st);
    for (int j = 0; j < nx; ++j)
        for (int i = 0; i < nx; ++i) V[j * nx + i] = rng_uniform(&st) - 0.5;
    std::vector<double> acc(nx, 0.0);
    bool ok = mgs_cpu(V, nx, nullptr);
    double t = 0.0, h = h0, facmax = 5.0;
    const double t_stop = transient + t_end;
    bool measuring = !(transient > 0);
    int since = 0;
    // Early orthonormalisation when the accumulated spread (time since the last pass x
    // running lambda_1 - lambda_N) exceeds the FP64 budget of 20 nats.
    double t_gs = 0.0, t_meas = 0.0, spread = 1e300;
    long long attempts = 0, accepted = 0;
    std::vector<double> stage((size_t)6 * nx);  // stage points X1..X6
    f(x.data(), av, &K[0]);
    while (ok && t < t_stop) {
        if (++attempts > max_steps) { ok = false; break; }
        const double target = measuring ? t_stop : transient;
        bool last = false;
        if (t + h >= target) { h = target - t; last = true; }
        for (int i = 0; i < nx; ++i) stage[i] = x[i];
        for (int s = 1; s < 6; ++s) {
            for (int i = 0; i < nx; ++i) {
                double acc_s = 0;
                for (int j = 0; j < s; ++j) acc_s += C.a[s][j] * K[j * nx + i];
                stage[s * nx + i] = x[i] + h * acc_s;
            }
            f(&stage[s * nx], av, &K[s * nx]);
        }
        for (int i = 0; i < nx; ++i) {
            double acc_s = 0;
            for (int j = 0; j < 6; ++j) acc_s += C.b[j] * K[j * nx + i];
            xn[i] = x[i] + h * acc_s;
        }
        f(xn.data(), av, &K[6 * nx]);
        double err2 = 0;
        for (int i = 0; i < nx; ++i) {
            double e = 0;
            for (int j = 0; j < 7; ++j) e += C.e[j] * K[j * nx + i];
            e *= h;
            const double sc = atol + rtol * std::max(std::fabs(x[i]), std::fabs(xn[i]));
            err2 += (e / sc) * (e / sc);
        }
        double err = std::sqrt(err2 / nx);
        std::vector<double> Vn(V.size());
        if (err <= 1.0 && measuring) {
            std::vector<double> L((size_t)7 * nx), vt(nx);
            double ev2 = 0;
            for (int k = 0; k < nx; ++k) {
                const double* v = &V[k * nx];
                double* vn = &Vn[k * nx];
                for (int s = 0; s < 6; ++s) {
                    for (int i = 0; i < nx; ++i) {
                        double a_s = 0;
                        for (int j = 0; j < s; ++j) a_s += C.a[s][j] * L[j * nx + i];
                        vt[i] = v[i] + h * a_s;
                    }
                    jvp(fd, &stage[s * nx], av, nv, vt.data(), &L[s * nx], nx);
                }
                for (int i = 0; i < nx; ++i) {
                    double b_s = 0;
                    for (int j = 0; j < 6; ++j) b_s += C.b[j] * L[j * nx + i];
                    vn[i] = v[i] + h * b_s;
                }
                jvp(fd, xn.data(), av, nv, vn, &L[6 * nx], nx);
                for (int i = 0; i < nx; ++i) {
                    double e = 0;
                    for (int j = 0; j < 7; ++j) e += C.e[j] * L[j * nx + i];
                    e *= h;
                    const double sc = atol + rtol * std::max(std::fabs(v[i]), std::fabs(vn[i]));
                    ev2 += (e / sc) * (e / sc);
                }
            }
            err = std::sqrt((err2 + ev2) / (nx + nx * nx));
        }
        if (!std::isfinite(err)) { ok = false; break; }
        if (err <= 1.0) {
            if (measuring) V = Vn;
            const double t_new = last ? target : t + h;
            if (measuring) t_gs += t_new - t;
            t = t_new;
            for (int i = 0; i < nx; ++i) { x[i] = xn[i]; K[i] = K[6 * nx + i]; }
            double checker = 0;
            for (int i = 0; i < nx; ++i) checker += std::fabs(x[i]);
            if (std::isnan(checker) || std::isinf(checker) || (maxv != 0 && checker > maxv)) { ok = false; break; }
            // escape test (the kernel's): every 16 accepted steps, a cell whose remaining
            // horizon needs more than 8x its remaining attempts at the step just taken ends
            if ((++accepted & 15) == 0 && t_stop - t > 8.0 * h * (double)(max_steps - attempts)) { ok = false; break; }
            if (measuring && (++since >= gs_every || last || t_gs * spread > 20.0)) {
                ok = mgs_cpu(V, nx, acc.data());
                since = 0;
                t_meas += t_gs;
                t_gs = 0.0;
                spread = std::max(0.0, (acc[0] - acc[nx - 1]) / t_meas);
            }
            if (last && !measuring) measuring = true;
            const double fac = err > 0 ? 0.9 * std::pow(err, -0.2) : facmax;
            h *= std::min(facmax, std::max(0.2, fac));
            facmax = 5.0;
        } else {
            h *= std::max(0.2, 0.9 * std::pow(err, -0.2));
            facmax = 2.0;
            if (!(h > 1e-14)) { ok = false; break; }
        }
    }
    for (int k = 0; k < nx; ++k) out[k] = ok ? acc[k] / t_end : 999.0;
}

template <class T>
struct Dispatch {
    static StepFn<T> fn(Krs* k) { return reinterpret_cast<StepFn<T>>(k->fn); }
};

int threads_or_default(int nthreads) {
    return nthreads > 0 ? nthreads : omp_get_max_threads();
}

}  // namespace

// ============================================================================
// C ABI of the oracle (used from Python through ctypes in tests/ and bench.py)
// ============================================================================
// dbscan of cudaLibrary.cu:2088-2166 (per-cell peak clustering of run_bif2d): the
// reference's loop as it is, including the stack slots written at amountOfPeaks + k and
// popped at amountOfPeaks + NumNeibor - 1, the inner bound amountOfPeaks - 1, the labels
// and stack held in numb, and the result cluster - 1. mult_peak = 1, mult_interval = 0
// (configCUDA.h), so the intervals enter the distance as zeros.
template <class T>
T dbscan_distance(T x1, T y1, T x2, T y2) {
    if (x1 == x2 && y1 == y2) return 0;
    const T dx = std::fabs(x2 - x1), dy = std::fabs(y2 - y1);
    return std::sqrt(dx * dx + dy * dy);
}

template <class T>
int dbscan_peaks(const T* peaks, int P, T eps, std::vector<T>& helpful) {
    if (P == -1) return -1;
    if (P == 0) return 0;
    if (P == 1) return 1;
    std::vector<T> data(peaks, peaks + P), iv((size_t)P, (T)0);
    for (int i = 0; i < P; ++i) {
        data[i] = data[i] * (T)1.0;
        iv[i] = iv[i] * (T)0.0;
    }
    helpful.assign((size_t)2 * P + 1, (T)0);
    int cluster = 0, NumNeibor = 0;
    for (size_t i = 0; i < (size_t)P; i++) {
        if (NumNeibor >= 1) {
            i = (size_t)helpful[(size_t)P + NumNeibor - 1];
            helpful[(size_t)P + NumNeibor - 1] = 0;
            NumNeibor = NumNeibor - 1;
        } else if (helpful[i] == 0) {
            NumNeibor = 0;
            ++cluster;
            helpful[i] = (T)cluster;
        } else {
            continue;
        }
        for (int k = 0; k < P - 1; k++) {
            if (i != (size_t)k && helpful[k] == 0) {
                if (dbscan_distance<T>(data[i], iv[i], data[k], iv[k]) < eps) {
                    helpful[k] = (T)cluster;
                    helpful[(size_t)P + k] = (T)k;
                    ++NumNeibor;
                }
            }
        }
    }
    return cluster - 1;
}

// Basin features of avgPeakFinderCUDA (cudaLibrary.cu:3310-3425): feature_needs /
// compute_basin_feature for the 12 feature kinds (avg / rms / stdev of the peaks or the
// intervals, and their log10 forms).
template <class T>
T basin_feature(int feat, T mean_p, T mean_i, T rms_p, T rms_i, T std_p, T std_i) {
    switch (feat) {
        case 0: return mean_p;
        case 1: return mean_i;
        case 2: return rms_p;
        case 3: return rms_i;
        case 4: return std_p;
        case 5: return std_i;
        case 6: return mean_p == (T)0 ? (T)0 : (mean_p > 0 ? std::log10(mean_p) : -std::log10(-mean_p));
        case 7: return mean_i == (T)0 ? (T)0 : (mean_i > 0 ? std::log10(mean_i) : -std::log10(-mean_i));
        case 8: return rms_p > 0 ? std::log10(rms_p) : (T)-999;
        case 9: return rms_i > 0 ? std::log10(rms_i) : (T)-999;
        case 10: return std_p > 0 ? std::log10(std_p) : (T)-999;
        case 11: return std_i > 0 ? std::log10(std_i) : (T)-999;
        default: return (T)-999;
    }
}

inline void basin_feature_needs(int feat, bool& sp, bool& sp2, bool& si, bool& si2) {
    sp = sp2 = si = si2 = false;
    switch (feat) {
        case 0: case 6: sp = true; break;
        case 1: case 7: si = true; break;
        case 2: case 8: sp2 = true; break;
        case 3: case 9: si2 = true; break;
        case 4: case 10: sp = sp2 = true; break;
        case 5: case 11: si = si2 = true; break;
        default: break;
    }
}

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

// Right-hand side "dX[i] = ...;" statements over X1[] and a[] (numb_bytes 8 or 16).
void* orc_rhs_compile(const char* body, int nx, int numb_bytes) {
    if (nx <= 0 || nx > 32) { g_err = "amountOfX out of range"; return nullptr; }
    return compile_krs(body, nx, numb_bytes, nullptr, true);
}

// DP5(4) tangent-linear spectrum over a 2-D grid (kernel cell order; values[c*nx + k]).
int orc_ls2d_dp5(void* hrhs, void* hdual, int nPts, int par_or_var, int idx0, int idx1, const double* ranges,
                 int log_mask, const double* ic, int nv, const double* vals, double transient, double t_end,
                 double rtol, double atol, double h0, int gs_every, long long max_steps, double maxv,
                 const long long* cells, long long ncells, double* values, int* flags, int nthreads) {
    Krs* kr = static_cast<Krs*>(hrhs);
    Krs* kd = static_cast<Krs*>(hdual);
    const int nx = kr->nx;
    Grid g{nPts, 2, par_or_var, {idx0, idx1}, {ranges[0], ranges[1], ranges[2], ranges[3]}, log_mask, -1};
    const long long n = cells ? ncells : (long long)nPts * nPts;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads_or_default(nthreads))
    for (long long c = 0; c < n; ++c) {
        const long long kidx = cells ? cells[c] : c;
        CellInit<double> ci;
        init_cell<double>(g, kidx, nx, ic, nv, vals, 0.01, &ci);
        double out[64];
        ls_cell_dp5_cpu(reinterpret_cast<RhsFn>(kr->fn), reinterpret_cast<RhsDualFn>(kd->fn), nx, ci.x, ci.a, nv,
                        transient, t_end, rtol, atol, h0, gs_every, max_steps, maxv, (uint64_t)kidx, out);
        bool bad = false;
        for (int k = 0; k < nx; ++k) {
            values[c * nx + k] = out[k];
            if (out[k] == 999.0) bad = true;
        }
        flags[c] = bad ? -1 : 1;
    }
    return 0;
}

// Stroboscopic basin classification of one grid (new semantics; no reference
// counterpart): per cell, RK4 steps_per_period steps per forcing period, the phase
// variable reset after each period, stroboscopic point P_n = the other state variables;
// converged when for the smallest k <= 8 |P_n - P_{n-k}|_inf < tol for match_count
// consecutive periods, k then reduced to its smallest divisor d with |P_n - P_{n-d}|_inf <=
// merge (the merge radius of the attractor table); canonical point = smallest first (then
// second) coordinate of the k points of the cycle. out_period: k, 0 (not converged by
// max_periods), -1 (diverged).
int orc_basins(void* h, int nPts, int ax, int ay, double lox, double hix, double loy, double hiy, const double* ic,
               int nv, const double* vals, double period, int steps_per_period, int max_periods, int match_count,
               double tol, int phase_var, double maxv, double merge, const long long* cells, long long ncells,
               int* out_period,
               double* out_cx, double* out_cy, int* out_iters, int nthreads) {
    Krs* k = static_cast<Krs*>(h);
    if (k->numb_bytes != 8) { g_err = "basins oracle is FP64"; return -1; }
    const int nx = k->nx;
    StepFn<double> f = Dispatch<double>::fn(k);
    const double hs = period / steps_per_period;
    const long long n = cells ? ncells : (long long)nPts * nPts;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads_or_default(nthreads))
    for (long long c = 0; c < n; ++c) {
        const long long cell = cells ? cells[c] : c;
        double x[64], a[64];
        for (int i = 0; i < nx; ++i) x[i] = ic[i];
        for (int i = 0; i < nv; ++i) a[i] = vals[i];
        x[ax] = value_by_idx<double>(cell % nPts, nPts, lox, hix, 0);
        x[ay] = value_by_idx<double>((cell / nPts) % nPts, nPts, loy, hiy, 0);
        const int K = 8;
        std::vector<std::vector<double>> hist;  // hist[j] = P_{n-1-j}
        int run[8] = {0};
        int per = 0, it = 0;
        double cx = 0, cy = 0;
        for (it = 1; it <= max_periods; ++it) {
            for (int s = 0; s < steps_per_period; ++s) f(x, a, hs);
            if (phase_var >= 0) x[phase_var] = ic[phase_var];
            double checker = 0;
            for (int i = 0; i < nx; ++i) checker += std::fabs(x[i]);
            if (std::isnan(checker) || std::isinf(checker) || (maxv != 0 && checker > maxv)) { per = -1; break; }
            std::vector<double> P;
            for (int i = 0; i < nx; ++i)
                if (i != phase_var) P.push_back(x[i]);
            int found = 0;
            for (int kk = 1; kk <= K; ++kk) {
                if (it > kk) {
                    double d = 0;
                    for (size_t i = 0; i < P.size(); ++i) d = std::max(d, std::fabs(P[i] - hist[kk - 1][i]));
                    run[kk - 1] = d < tol ? run[kk - 1] + 1 : 0;
                    if (!found && run[kk - 1] >= match_count) found = kk;
                }
            }
            if (found) {
                // a cycle repeating after a divisor d of its length to within the merge
                // radius is the period-d orbit
                for (int dd = 1; dd < found; ++dd) {
                    if (found % dd) continue;
                    double d = 0;
                    for (size_t i = 0; i < P.size(); ++i) d = std::max(d, std::fabs(P[i] - hist[dd - 1][i]));
                    if (d <= merge) {
                        found = dd;
                        break;
                    }
                }
                per = found;
                cx = P[0];
                cy = P.size() > 1 ? P[1] : 0.0;
                for (int j = 0; j + 1 < found; ++j) {
                    const double px = hist[j][0], py = P.size() > 1 ? hist[j][1] : 0.0;
                    if (px < cx || (px == cx && py < cy)) { cx = px; cy = py; }
                }
                break;
            }
            hist.insert(hist.begin(), P);
            if ((int)hist.size() > K) hist.pop_back();
        }
        out_period[c] = per;
        out_cx[c] = cx;
        out_cy[c] = cy;
        out_iters[c] = it > max_periods ? max_periods : it;
    }
    return 0;
}

// numb_bytes: 8 (double), 4 (float), 16 (forward-mode dual: value + tangent)
void* orc_krs_compile(const char* body, int nx, int numb_bytes) {
    if (nx <= 0 || nx > 32) { g_err = "amountOfX out of range"; return nullptr; }
    return compile_krs(body, nx, numb_bytes, nullptr);
}

void orc_krs_free(void* h) {
    Krs* k = static_cast<Krs*>(h);
    if (!k) return;
    if (k->lib) dlclose(k->lib);
    delete k;
}

// One call of loopCalculateDiscreteModel_int on a caller-owned state. x, a, data
// are numb arrays matching the compiled precision.
int orc_loop(void* h, void* x, const void* a, double hstep, long long iters, int preScaller,
             int writableVar, double maxValue, void* data) {
    Krs* k = static_cast<Krs*>(h);
    if (k->numb_bytes == 8)
        return loop_model<double>(Dispatch<double>::fn(k), (double*)x, (const double*)a, hstep, iters,
                                  k->nx, preScaller, writableVar, maxValue, (double*)data);
    return loop_model<float>(Dispatch<float>::fn(k), (float*)x, (const float*)a, (float)hstep, iters,
                             k->nx, preScaller, writableVar, (float)maxValue, (float*)data);
}

// Plain repeated stepping (no checks): x <- step^n(x). Used for trajectory parity.
void orc_steps(void* h, void* x, const void* a, double hstep, long long n) {
    Krs* k = static_cast<Krs*>(h);
    if (k->numb_bytes == 8) {
        auto f = Dispatch<double>::fn(k);
        for (long long i = 0; i < n; ++i) f((double*)x, (const double*)a, hstep);
    } else {
        auto f = Dispatch<float>::fn(k);
        for (long long i = 0; i < n; ++i) f((float*)x, (const float*)a, (float)hstep);
    }
}

// Axis value table of one sweep axis: out[i] = getValueByIdx(_log) of point i.
void orc_axis_values(int numb_bytes, int nPts, double lo, double hi, int log_scale, double* out) {
    for (int i = 0; i < nPts; ++i) {
        if (numb_bytes == 8)
            out[i] = log_scale ? value_by_idx_log<double>(i, nPts, lo, hi, 0) : value_by_idx<double>(i, nPts, lo, hi, 0);
        else
            out[i] = log_scale ? (double)value_by_idx_log<float>(i, nPts, (float)lo, (float)hi, 0)
                               : (double)value_by_idx<float>(i, nPts, (float)lo, (float)hi, 0);
    }
}

void orc_rng_uniforms(unsigned long long seq, int n, float* out) {
    Rng st;
    rng_init(1234567891ULL, seq, 0ULL, &st);
    for (int i = 0; i < n; ++i) out[i] = rng_uniform(&st);
}

// LLE 2D (run_lle_2d + LLEKernelCUDA). cells: optional subset of kernel cell indices
// (nullptr = all n^2). values/flags are indexed like the cells array (or n^2 in
// user row-major order when cells == nullptr).
int orc_lle2d(void* h, int nPts, int par_or_var, int idx0, int idx1, const double* ranges,
              int log_mask, int h_axis, int swap_xy, const double* ic, int nv, const double* vals,
              double hstep, double transient, double tMax, double NT, double eps, double maxv,
              const long long* cells, long long ncells, double* values, int* flags, int nthreads) {
    Krs* k = static_cast<Krs*>(h);
    Grid g{nPts, 2, par_or_var, {idx0, idx1}, {ranges[0], ranges[1], ranges[2], ranges[3]}, log_mask, h_axis};
    const int sizeOfBlock = (int)(tMax / NT);
    const int skipHost = (int)(transient / hstep);
    if (sizeOfBlock <= 0) { g_err = "computed amountOfPointsInBlock <= 0"; return -1; }
    const long long total = (long long)nPts * nPts;
    const long long n = cells ? ncells : total;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads_or_default(nthreads))
    for (long long c = 0; c < n; ++c) {
        const long long kidx = cells ? cells[c] : c;
        double v;
        if (k->numb_bytes == 8)
            v = lle_cell<double>(Dispatch<double>::fn(k), g, kidx, k->nx, ic, nv, vals, hstep, NT, tMax,
                                 transient, eps, maxv, sizeOfBlock, skipHost, (uint64_t)kidx);
        else
            v = (double)lle_cell<float>(Dispatch<float>::fn(k), g, kidx, k->nx, ic, nv, vals, hstep, NT, tMax,
                                        transient, eps, maxv, sizeOfBlock, skipHost, (uint64_t)kidx);
        long long out = c;
        if (!cells && swap_xy) {
            const long long kix = kidx % nPts, kiy = kidx / nPts;
            out = kix * nPts + kiy;
        }
        values[out] = v;
        flags[out] = (v == 999.0 || v == -999.0) ? -1 : 1;
    }
    return 0;
}

// LS 2D (run_ls_2d + LSKernelCUDA). values: plane-major [k * n^2 + cell] when cells ==
// nullptr, else [c * nx + k].
int orc_ls2d(void* h, int nPts, int par_or_var, int idx0, int idx1, const double* ranges,
             int log_mask, int h_axis, int swap_xy, const double* ic, int nv, const double* vals,
             double hstep, double transient, double tMax, double NT, double eps, double maxv,
             const long long* cells, long long ncells, double* values, int* flags, int nthreads) {
    Krs* k = static_cast<Krs*>(h);
    Grid g{nPts, 2, par_or_var, {idx0, idx1}, {ranges[0], ranges[1], ranges[2], ranges[3]}, log_mask, h_axis};
    const int sizeOfBlock = (int)(tMax / NT);
    const int skipHost = (int)(transient / hstep);
    if (sizeOfBlock <= 0) { g_err = "computed amountOfPointsInBlock <= 0"; return -1; }
    const int nx = k->nx;
    const long long total = (long long)nPts * nPts;
    const long long n = cells ? ncells : total;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads_or_default(nthreads))
    for (long long c = 0; c < n; ++c) {
        const long long kidx = cells ? cells[c] : c;
        double outv[64];
        if (k->numb_bytes == 8) {
            ls_cell<double>(Dispatch<double>::fn(k), g, kidx, nx, ic, nv, vals, hstep, NT, tMax, transient, eps,
                            maxv, sizeOfBlock, skipHost, (uint64_t)kidx, outv);
        } else {
            float o32[64];
            ls_cell<float>(Dispatch<float>::fn(k), g, kidx, nx, ic, nv, vals, hstep, NT, tMax, transient, eps,
                           maxv, sizeOfBlock, skipHost, (uint64_t)kidx, o32);
            for (int m = 0; m < nx; ++m) outv[m] = o32[m];
        }
        long long cell = c;
        if (!cells && swap_xy) {
            const long long kix = kidx % nPts, kiy = kidx / nPts;
            cell = kix * nPts + kiy;
        }
        bool bad = false;
        for (int m = 0; m < nx; ++m) {
            if (cells) values[c * nx + m] = outv[m];
            else values[(long long)m * total + cell] = outv[m];
            if (outv[m] == 999.0 || outv[m] == -999.0) bad = true;
        }
        flags[cells ? c : cell] = bad ? -1 : 1;
    }
    return 0;
}

// Bifurcation 2D (run_bif2d, parametric_engine.cpp:5487-5910): per cell the bif1d
// trajectory + peakFinder, then dbscan of the peaks; values[out] = period (-1 when the
// dbscan result is negative), flags[out] = -1 / 1; out = cell, transposed with swap_xy
// (with a cell list, out = list position).
int orc_bif2d(void* h, int nPts, int par_or_var, int idx0, int idx1, const double* ranges, int log_mask,
              int h_axis, int swap_xy, const double* ic, int nv, const double* vals, double hstep, double transient,
              double tMax, int preScaller, int writableVar, double maxv, double eps_dbscan, const long long* cells,
              long long ncells, double* values, int* flags, int nthreads) {
    Krs* k = static_cast<Krs*>(h);
    const int nx = k->nx;
    Grid g{nPts, 2, par_or_var, {idx0, idx1}, {ranges[0], ranges[1], ranges[2], ranges[3]}, log_mask, h_axis};
    const double r_h = h_axis == 0 ? ranges[0] : (h_axis == 1 ? ranges[2] : hstep);
    const double worstCaseH = (h_axis != -1) ? (k->numb_bytes == 8 ? r_h : (double)(float)r_h) : hstep;
    const long long amountOfPointsInBlock = (long long)std::ceil(tMax / worstCaseH / preScaller);
    const long long amountOfPointsForSkip = (long long)(transient / hstep);
    if (amountOfPointsInBlock <= 0) { g_err = "computed amountOfPointsInBlock <= 0"; return -1; }
    const long long total = (long long)nPts * nPts;
    const long long n = cells ? ncells : total;
#pragma omp parallel num_threads(threads_or_default(nthreads))
    {
        std::vector<double> d8, p8, t8, h8;
        std::vector<float> d4, p4, t4, h4;
#pragma omp for schedule(dynamic, 1)
        for (long long c = 0; c < n; ++c) {
            const long long idx = cells ? cells[c] : c;
            int period = 0;
            auto run = [&](auto tag, auto& dd, auto& pp, auto& tt, auto& hh) {
                using T = decltype(tag);
                StepFn<T> f = Dispatch<T>::fn(k);
                CellInit<T> ci;
                init_cell<T>(g, idx, nx, ic, nv, vals, hstep, &ci);
                const T hl = ci.h;
                int cnt;
                if (!(hl > 0)) {
                    cnt = -1;
                } else {
                    long long skip_l = amountOfPointsForSkip, iters_l = amountOfPointsInBlock;
                    if (g.h_axis != -1) {
                        skip_l = (long long)std::ceil((T)transient / hl);
                        iters_l = (long long)std::ceil((T)tMax / hl / (T)preScaller);
                    }
                    if (iters_l > amountOfPointsInBlock) iters_l = amountOfPointsInBlock;
                    dd.assign((size_t)iters_l, (T)0);
                    pp.assign((size_t)iters_l, (T)0);
                    tt.assign((size_t)iters_l, (T)0);
                    int flag = loop_model<T>(f, ci.x, ci.a, hl, skip_l, nx, preScaller, writableVar, (T)maxv, nullptr);
                    if (flag == 1 || flag == -1)
                        flag = loop_model<T>(f, ci.x, ci.a, hl, iters_l, nx, preScaller, writableVar, (T)maxv, dd.data());
                    if (flag == -1 || flag == 0) cnt = flag;
                    else cnt = peak_finder<T>(dd.data(), iters_l, pp.data(), tt.data(), (T)(hstep * (double)preScaller));
                }
                period = dbscan_peaks<T>(pp.data(), cnt, (T)eps_dbscan, hh);
            };
            if (k->numb_bytes == 8) run(0.0, d8, p8, t8, h8);
            else run(0.0f, d4, p4, t4, h4);
            long long out = cells ? c : idx;
            if (!cells && swap_xy) out = (idx % nPts) * nPts + idx / nPts;
            values[out] = period < 0 ? -1.0 : (double)period;
            flags[out] = period < 0 ? -1 : 1;
        }
    }
    return 0;
}

// DBSCAN of basin features as run_basins' host loop drives it (parametric_engine.cpp:
// 6330-6420 with CUDA_dbscan_search_fixed_points_kernel / _clear_points_kernel /
// CUDA_dbscan_kernel, cudaLibrary.cu:3501-3563), also the whole of run_basins_recluster
// (:6517-6600): seeds are the lowest-index unlabelled fixed point (helpful -1; cluster ids
// -1, -2, ...), then the lowest-index unlabelled oscillating cell (helpful 1; ids 1, 2,
// ...); a member labels every unlabelled cell within eps (sqrt(dx^2 + dy^2) <= eps in numb)
// and queues it. A queued unbound cell (helpful 0) expands nothing, and its label is reset
// to 0 while an unlabelled cell remains (the kernel's write of 0; its concurrent writes of
// the cluster id are taken to lose).
int orc_dbscan_cells(long long total, const double* f1, const double* f2, const int* helpful, double eps_dbscan,
                     int numb_bytes, int* labels) {
    const bool dbl = numb_bytes == 8;
    for (long long c = 0; c < total; ++c) labels[c] = 0;
    auto within = [&](long long a, long long b) {
        if (dbl) {
            const double dx = f1[a] - f1[b], dy = f2[a] - f2[b];
            return std::sqrt(dx * dx + dy * dy) <= eps_dbscan;
        }
        const float dx = (float)f1[a] - (float)f1[b], dy = (float)f2[a] - (float)f2[b];
        return std::sqrt(dx * dx + dy * dy) <= (float)eps_dbscan;
    };
    int pos = 0, neg = 0;
    std::vector<long long> nb;
    for (;;) {
        long long seed = -1;
        int id = 0;
        for (long long c = 0; c < total && seed < 0; ++c)
            if (helpful[c] == -1 && labels[c] == 0) seed = c;
        if (seed >= 0) {
            id = --neg;
        } else {
            for (long long c = 0; c < total && seed < 0; ++c)
                if (labels[c] == 0 && helpful[c] == 1) seed = c;
            if (seed < 0) break;
            id = ++pos;
        }
        nb.clear();
        auto expand = [&](long long cur) {
            labels[cur] = id;
            bool any = false;
            std::vector<long long> found;
            for (long long c = 0; c < total; ++c) {
                if (labels[c] != 0 || c == cur) continue;
                any = true;
                if (helpful[cur] == 0) continue;
                if (within(cur, c)) found.push_back(c);
            }
            if (helpful[cur] == 0 && any) {
                labels[cur] = 0;
                return;
            }
            for (long long c : found) {
                labels[c] = id;
                nb.push_back(c);
            }
        };
        expand(seed);
        for (size_t ni = 0; ni < nb.size(); ++ni) expand(nb[ni]);
    }
    return 0;
}

// Basins of attraction, reference method (run_basins, parametric_engine.cpp:6035-6510):
// per cell of the initial-condition grid the trajectory class (1 oscillating, -1 fixed
// point, 0 unbound) and two features (avgPeakFinderCUDA), then the host-driven DBSCAN of
// the features (CUDA_dbscan_search_fixed / _clear_points_kernel + CUDA_dbscan_kernel):
// seeds are the lowest-index unlabelled fixed point (cluster ids -1, -2, ...), then the
// lowest-index unlabelled oscillating cell (1, 2, ...); a seed's cluster grows over every
// unlabelled cell within eps (distance <= eps) of a member, through a neighbour list that
// is expanded in order; an unbound cell reached this way is un-labelled again and not
// expanded (the reference's kernel resets it to 0).
int orc_basins_ref(void* h, int nPts, int xvar, int yvar, const double* ranges, const double* ic, int nv,
                   const double* vals, double hstep, double transient, double tMax, int preScaller, int writableVar,
                   double maxv, double eps_dbscan, int feature1, int feature2, double mult1, double mult2,
                   int* labels, double* avg_peaks, double* avg_intervals, int* helpful, int nthreads) {
    Krs* k = static_cast<Krs*>(h);
    const int nx = k->nx;
    Grid g{nPts, 2, 0, {xvar, yvar}, {ranges[0], ranges[1], ranges[2], ranges[3]}, 0, -1};
    const long long points = (long long)(tMax / hstep / preScaller);
    const long long skip = (long long)(transient / hstep);
    if (points <= 0) { g_err = "computed amountOfPointsInBlock <= 0"; return -1; }
    const long long total = (long long)nPts * nPts;
    auto features = [&](auto tag, std::vector<double>& f1, std::vector<double>& f2) {
        using T = decltype(tag);
#pragma omp parallel num_threads(threads_or_default(nthreads))
        {
            std::vector<T> dd, pp, tt;
#pragma omp for schedule(dynamic, 1)
            for (long long c = 0; c < total; ++c) {
                StepFn<T> f = Dispatch<T>::fn(k);
                CellInit<T> ci;
                init_cell<T>(g, c, nx, ic, nv, vals, hstep, &ci);
                const T hl = ci.h;
                dd.assign((size_t)points, (T)0);
                pp.assign((size_t)points, (T)0);
                tt.assign((size_t)points, (T)0);
                int flag = loop_model<T>(f, ci.x, ci.a, hl, skip, nx, preScaller, writableVar, (T)maxv, nullptr);
                if (flag == 1 || flag == -1)
                    flag = loop_model<T>(f, ci.x, ci.a, hl, points, nx, preScaller, writableVar, (T)maxv, dd.data());
                helpful[c] = flag;
                T a_out, b_out;
                if (flag == 0) {
                    a_out = 999;
                    b_out = 999;
                } else if (flag == -1) {
                    a_out = dd[(size_t)points - 1];
                    b_out = (T)-1.0;
                } else {
                    const int np = peak_finder<T>(dd.data(), points, pp.data(), tt.data(), (T)(hstep * preScaller));
                    if (np <= 0) {
                        a_out = -999;
                        b_out = (T)-1.0;
                    } else {
                        bool a1, a2, a3, a4, b1, b2, b3, b4;
                        basin_feature_needs(feature1, a1, a2, a3, a4);
                        basin_feature_needs(feature2, b1, b2, b3, b4);
                        const bool nsp = a1 || b1, nsp2 = a2 || b2, nsi = a3 || b3, nsi2 = a4 || b4;
                        T sp = 0, sp2 = 0, si = 0, si2 = 0;
                        for (int i = 0; i < np; ++i) {
                            if (nsp || nsp2) {
                                const T pv = pp[i];
                                if (nsp) sp += pv;
                                if (nsp2) sp2 += pv * pv;
                            }
                            if (nsi || nsi2) {
                                const T iv = tt[i];
                                if (nsi) si += iv;
                                if (nsi2) si2 += iv * iv;
                            }
                        }
                        const T inv = (T)1.0 / (T)np;
                        const T mp = nsp ? sp * inv : (T)0, mi = nsi ? si * inv : (T)0;
                        const T rp = nsp2 ? std::sqrt(sp2 * inv) : (T)0, ri = nsi2 ? std::sqrt(si2 * inv) : (T)0;
                        T sdp = 0, sdi = 0;
                        if (nsp && nsp2) { const T v = sp2 * inv - mp * mp; sdp = std::sqrt(v < 0 ? (T)0 : v); }
                        if (nsi && nsi2) { const T v = si2 * inv - mi * mi; sdi = std::sqrt(v < 0 ? (T)0 : v); }
                        a_out = (T)mult1 * basin_feature<T>(feature1, mp, mi, rp, ri, sdp, sdi);
                        b_out = (T)mult2 * basin_feature<T>(feature2, mp, mi, rp, ri, sdp, sdi);
                    }
                }
                f1[c] = (double)a_out;
                f2[c] = (double)b_out;
            }
        }
    };
    std::vector<double> f1((size_t)total), f2((size_t)total);
    if (k->numb_bytes == 8) features(0.0, f1, f2);
    else features(0.0f, f1, f2);
    for (long long c = 0; c < total; ++c) {
        avg_peaks[c] = f1[c];
        avg_intervals[c] = f2[c];
        labels[c] = 0;
    }
    return orc_dbscan_cells(total, f1.data(), f2.data(), helpful, eps_dbscan, k->numb_bytes, labels);
}

// Bifurcation 1D (run_bif1d + calculateDiscreteModelCUDA + peakFinderCUDA).
// Outputs per point: count[i] (flag semantics of Bifurcation1DResult::flags),
// peaks[i*max_out + j], intervals[i*max_out + j] for j < min(count, max_out).
int orc_bif1d(void* h, int nPts, int sweep_kind, int sweep_index, double lo, double hi, int log_scale,
              const double* ic, int nv, const double* vals, double hstep, double transient, double tMax,
              int preScaller, int writableVar, double maxv, int max_out, const long long* pts,
              long long npts_subset, int* counts, double* peaks, double* intervals, int nthreads) {
    Krs* k = static_cast<Krs*>(h);
    const int nx = k->nx;
    // sweep_kind: 0 param, 1 IC, 2 h
    Grid g{nPts, 1, sweep_kind == 1 ? 0 : 1, {sweep_index, 0}, {lo, hi, 0, 0}, log_scale ? 1 : 0,
           sweep_kind == 2 ? 0 : -1};
    const double worstCaseH = (sweep_kind == 2) ? (k->numb_bytes == 8 ? lo : (double)(float)lo) : hstep;
    const long long amountOfPointsInBlock = (long long)std::ceil(tMax / worstCaseH / preScaller);
    const long long amountOfPointsForSkip = (long long)(transient / hstep);
    if (amountOfPointsInBlock <= 0) { g_err = "computed amountOfPointsInBlock <= 0"; return -1; }
    const long long n = pts ? npts_subset : nPts;
    int rc = 0;
#pragma omp parallel num_threads(threads_or_default(nthreads))
    {
        std::vector<double> d8, p8, t8;
        std::vector<float> d4, p4, t4;
#pragma omp for schedule(dynamic, 1)
        for (long long c = 0; c < n; ++c) {
            const long long idx = pts ? pts[c] : c;
            int cnt = 0;
            auto run = [&](auto tag, auto& dd, auto& pp, auto& tt) {
                using T = decltype(tag);
                StepFn<T> f = Dispatch<T>::fn(k);
                CellInit<T> ci;
                init_cell<T>(g, idx, nx, ic, nv, vals, hstep, &ci);
                const T hl = ci.h;
                if (hl <= 0) { cnt = -1; return; }
                long long skip_l = amountOfPointsForSkip, iters_l = amountOfPointsInBlock;
                if (g.h_axis != -1) {
                    skip_l = (long long)std::ceil((T)transient / hl);
                    iters_l = (long long)std::ceil((T)tMax / hl / (T)preScaller);
                }
                if (iters_l > amountOfPointsInBlock) iters_l = amountOfPointsInBlock;
                dd.assign((size_t)iters_l, (T)0);
                pp.assign((size_t)iters_l, (T)0);
                tt.assign((size_t)iters_l, (T)0);
                int flag = loop_model<T>(f, ci.x, ci.a, hl, skip_l, nx, preScaller, writableVar, (T)maxv, nullptr);
                if (flag == 1 || flag == -1)
                    flag = loop_model<T>(f, ci.x, ci.a, hl, iters_l, nx, preScaller, writableVar, (T)maxv, dd.data());
                if (flag == -1 || flag == 0) { cnt = flag; return; }
                const T timeStep = (T)(hstep * (double)preScaller);
                cnt = peak_finder<T>(dd.data(), iters_l, pp.data(), tt.data(), timeStep);
                // run_bif1d rescales intervals by param_val / h, param_val from the host
                // copy of getValueByIdx (parametric_engine.cpp:577-590, 1991-2003).
                double time_scale = 1.0;
                if (g.h_axis != -1) {
                    const double rlo = (double)(T)lo, rhi = (double)(T)hi;
                    double pv;
                    if (nPts <= 1) pv = rlo;
                    else if (log_scale)
                        pv = std::pow(10.0, std::log10(rlo) + (std::log10(rhi) - std::log10(rlo)) * (double)idx / (double)(nPts - 1));
                    else
                        pv = rlo + (rhi - rlo) * (double)idx / (double)(nPts - 1);
                    time_scale = pv / hstep;
                }
                const int m = std::min(cnt, max_out);
                for (int j = 0; j < m; ++j) {
                    peaks[c * max_out + j] = (double)pp[j];
                    intervals[c * max_out + j] = (double)tt[j] * time_scale;
                }
            };
            if (k->numb_bytes == 8) run(0.0, d8, p8, t8);
            else run(0.0f, d4, p4, t4);
            counts[c] = cnt;
        }
    }
    return rc;
}

}  // extern "C"
