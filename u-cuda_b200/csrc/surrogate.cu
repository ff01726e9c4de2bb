// Surrogate-refined LLE map (no reference counterpart): plain-method samples -> BF16 MLP
// trained on this GPU -> predicted map -> re-integration of the cells the network cannot
// vouch for. The integrations are the LLE-2D kernel of ucb_engine.cpp run over cell lists;
// the network is mlp.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "engine_internal.h"
#include "mlp.h"

namespace ucbsur {

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// One cell drawn uniformly inside each block of a tp x tp partition of the n x n grid
// (kernel order: cell = iy * n + ix).
__global__ void sample_cells_kernel(int n, int tp, unsigned long long seed, long long* cells) {
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= (long long)tp * tp) return;
    const int si = (int)(s % tp), sj = (int)(s / tp);
    const long long x0 = (long long)si * n / tp, x1 = (long long)(si + 1) * n / tp;
    const long long y0 = (long long)sj * n / tp, y1 = (long long)(sj + 1) * n / tp;
    const unsigned long long h = mix64(seed ^ mix64((unsigned long long)s));
    const long long ix = x0 + (long long)((h & 0xffffffffULL) % (unsigned long long)(x1 - x0));
    const long long iy = y0 + (long long)((h >> 32) % (unsigned long long)(y1 - y0));
    cells[s] = iy * n + ix;
}

__device__ __forceinline__ long long map_pos(long long cell, int n, int swap_xy) {
    if (!swap_xy) return cell;
    return (cell % n) * n + cell / n;
}

// Sample values into the map; mask marks the sample cells.
__global__ void scatter_samples_kernel(const long long* cells, long long ns, const double* sv, const int* sf, int n,
                                       int swap_xy, unsigned char* mask, double* values, int* flags) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    const long long c = cells[i];
    mask[c] = 1;
    const long long o = map_pos(c, n, swap_xy);
    values[o] = sv[i];
    flags[o] = sf[i];
}

__device__ __forceinline__ int regime(float v, float band) { return v > band ? 1 : (v < -band ? -1 : 0); }

// Per non-sample cell: re-integrate (append to list) when the prediction is uncertain
// (std above the calibrated threshold), near zero, or on a regime boundary (a 4-neighbour
// in another class of {lambda < -band, |lambda| <= band, lambda > band}, or differing by
// more than jump); band <= 0 / jump <= 0 switch those rules off. Otherwise the cell takes
// the predicted mean with flag 2.
__global__ void select_kernel(const float* mean, const float* sd, const unsigned char* mask, int n, int swap_xy,
                              float sigma_max, float band, float jump, long long* list, unsigned long long* count,
                              double* values, int* flags) {
    const long long total = (long long)n * n;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool refine = false;
    bool active = c < total && !mask[c];
    if (active) {
        const float m = mean[c];
        refine = !(sd[c] <= sigma_max) || (band > 0.f && fabsf(m) < band) || !isfinite(m);
        if (!refine && (band > 0.f || jump > 0.f)) {
            const int ix = (int)(c % n), iy = (int)(c / n);
            const int rc = regime(m, band);
            const long long nb[4] = {ix > 0 ? c - 1 : -1, ix + 1 < n ? c + 1 : -1, iy > 0 ? c - n : -1,
                                     iy + 1 < n ? c + n : -1};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (nb[k] < 0) continue;
                const float v = mean[nb[k]];
                if ((band > 0.f && regime(v, band) != rc) || (jump > 0.f && fabsf(v - m) > jump)) refine = true;
            }
        }
        if (!refine) {
            const long long o = map_pos(c, n, swap_xy);
            values[o] = (double)m;
            flags[o] = 2;
        }
    }
    // warp-aggregated append
    const unsigned ballot = __ballot_sync(0xffffffffu, active && refine);
    if (ballot) {
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(ballot) - 1;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(count, (unsigned long long)__popc(ballot));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (active && refine) list[base + __popc(ballot & ((1u << lane) - 1u))] = c;
    }
}

__global__ void gather_kernel(const float* mean, const float* sd, const long long* cells, long long n, float* gm,
                              float* gs) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    gm[i] = mean[cells[i]];
    gs[i] = sd[cells[i]];
}

__global__ void count_flag_kernel(const int* flags, long long total, int value, unsigned long long* count) {
    unsigned long long local = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x)
        local += flags[i] == value;
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}

}  // namespace ucbsur

namespace ucb {
namespace {

void set_err(char* dst, const std::string& msg) { std::snprintf(dst, 1024, "%s", msg.c_str()); }

struct DevFree {
    ucb_engine* e;
    cudaStream_t st;
    std::vector<void*> ptrs;
    ~DevFree() {
        for (void* p : ptrs) cudaFreeAsync(p, st);
        cudaStreamSynchronize(st);
    }
    template <class T>
    T* alloc(size_t count, std::string& err, const char* what) {
        void* p = nullptr;
        const cudaError_t ce = dev_alloc(e, &p, std::max<size_t>(count, 1) * sizeof(T), st);
        if (ce != cudaSuccess) {
            err = std::string("cudaMallocAsync(") + what + "): " + cudaGetErrorString(ce);
            return nullptr;
        }
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
};

struct LaunchHandle {
    void* plan = nullptr;
    void* launch = nullptr;
    ~LaunchHandle() {
        if (plan) lle2d_release(plan, launch);
    }
};

// Pilot samples: every pilot_stride(tp)-th block of the tp x tp sample partition along both
// axes: a 32 x 32 .. 64 x 64 pilot grid (all samples when tp <= 32).
int pilot_stride(int tp) { return std::max(1, std::min(4, tp / 32)); }

// The predictability gate, computed from the pilot samples alone before any training.
// v / f: the pilot samples' integrated values and flags on their tq x tq block grid
// (row-major), cells: their map cells (kernel order, iy * n + ix). Each pilot sample with
// a full 5 x 5 pilot neighbourhood is predicted by the least-squares plane through its 24
// neighbours (at their cell positions) evaluated at its own cell: the prediction of a
// smooth predictor that averages out the per-cell probe term, as the network does. It is a
// candidate when all 25 are valid, lie in one regime and the prediction is at least `band`
// from zero (the selection rules select_kernel applies to the network's predictions).
// Ordered by the plane's RMS residual, the longest prefix of candidates of which
// >= coverage lie within tol of the integrated value (and at least 32) is the share of the
// pilot such a predictor could vouch for at the requested coverage. Returns that share of
// all pilot samples.
double pilot_share(const std::vector<double>& v, const std::vector<int>& f, const std::vector<long long>& cells,
                   int n, int tq, double tol, double coverage, double band) {
    struct Cand {
        double spread;
        bool good;
    };
    std::vector<Cand> cand;
    auto regime = [&](double x) { return band > 0 ? (x > band ? 1 : (x < -band ? -1 : 0)) : 0; };
    constexpr int R = 2;
    for (int qy = R; qy + R < tq; ++qy)
        for (int qx = R; qx + R < tq; ++qx) {
            const int c = qy * tq + qx;
            if (f[c] != 1 || !std::isfinite(v[c])) continue;
            const double cx = (double)(cells[c] % n), cy = (double)(cells[c] / n);
            // normal equations of v ~ p0 + p1 (x - cx) + p2 (y - cy) over the neighbours
            double S[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, b[3] = {0, 0, 0};
            bool ok = true;
            for (int dy = -R; dy <= R && ok; ++dy)
                for (int dx = -R; dx <= R && ok; ++dx) {
                    if (!dx && !dy) continue;
                    const int k = (qy + dy) * tq + qx + dx;
                    ok = f[k] == 1 && std::isfinite(v[k]) && regime(v[k]) == regime(v[c]);
                    const double a[3] = {1.0, (double)(cells[k] % n) - cx, (double)(cells[k] / n) - cy};
                    for (int i = 0; i < 3; ++i) {
                        b[i] += a[i] * v[k];
                        for (int j = 0; j < 3; ++j) S[i][j] += a[i] * a[j];
                    }
                }
            if (!ok) continue;
            // 3 x 3 solve by Cramer's rule
            auto det3 = [](const double M[3][3]) {
                return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
                       M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                       M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
            };
            const double d = det3(S);
            if (!(std::fabs(d) > 0)) continue;
            double p[3];
            for (int col = 0; col < 3; ++col) {
                double M[3][3];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) M[i][j] = j == col ? b[i] : S[i][j];
                p[col] = det3(M) / d;
            }
            double rss = 0;
            for (int dy = -R; dy <= R; ++dy)
                for (int dx = -R; dx <= R; ++dx) {
                    if (!dx && !dy) continue;
                    const int k = (qy + dy) * tq + qx + dx;
                    const double r = v[k] - (p[0] + p[1] * ((double)(cells[k] % n) - cx) +
                                             p[2] * ((double)(cells[k] / n) - cy));
                    rss += r * r;
                }
            if (band > 0 && std::fabs(p[0]) < band) continue;
            cand.push_back({std::sqrt(rss / 24.0), std::fabs(p[0] - v[c]) <= tol});
        }
    std::sort(cand.begin(), cand.end(), [](const Cand& a, const Cand& b) { return a.spread < b.spread; });
    long long good = 0, best = 0;
    for (size_t k = 0; k < cand.size(); ++k) {
        good += cand[k].good;
        const long long cnt = (long long)k + 1;
        if (cnt >= 32 && (double)good >= coverage * (double)cnt) best = cnt;
    }
    return v.empty() ? 0.0 : (double)best / (double)v.size();
}

}  // namespace
}  // namespace ucb

using namespace ucb;

extern "C" {

void ucb_default_surrogate_request(ucb_surrogate_request* r) {
    std::memset(r, 0, sizeof *r);
    r->map.opt.precision = UCB_PREC_F32;
    r->map.opt.mode = UCB_MODE_NATIVE;
    r->train_pts = 256;
    r->sample_precision = UCB_PREC_F64;
    r->refine_precision = UCB_PREC_F32;
    r->tol = 2e-3;
    r->coverage = 0.995;
    r->sigma_max = 0.0;
    r->lle_band = 0.05;
    r->jump = 0.0;
    r->min_predictable = 0.05;
    ucb_mlp_default_config(&r->mlp);
}

int ucb_run_lle2d_surrogate(ucb_engine* e, const ucb_surrogate_request* rq, double* d_values, int32_t* d_flags,
                            void* stream, ucb_surrogate_result* res) {
    if (!e || !rq || !res) return UCB_E_INVALID;
    std::memset(res, 0, sizeof *res);
    const auto t_start = std::chrono::steady_clock::now();
    const ucb_surrogate_request& r = *rq;
    const int n = r.map.n_pts;
    auto fail = [&](int code, const std::string& msg) {
        e->last_error = msg;
        set_err(res->error, msg);
        res->ok = 0;
        return code;
    };
    if (!d_values || !d_flags) return fail(UCB_E_INVALID, "output buffers are NULL");
    if (n < 2) return fail(UCB_E_INVALID, "surrogate map needs n_pts >= 2");
    const int tp = std::min(r.train_pts > 0 ? r.train_pts : 256, n);
    auto prec_ok = [](int p) { return p == UCB_PREC_F64 || p == UCB_PREC_F32; };
    if (!prec_ok(r.sample_precision) || !prec_ok(r.refine_precision))
        return fail(UCB_E_INVALID, "sample_precision / refine_precision must be UCB_PREC_F64 or UCB_PREC_F32");
    if (!(r.sigma_max >= 0) || !(r.lle_band >= 0) || !(r.jump >= 0) || !(r.tol > 0) ||
        !(r.coverage > 0 && r.coverage <= 1) || !(r.min_predictable >= 0))
        return fail(UCB_E_INVALID,
                    "need tol > 0, 0 < coverage <= 1, sigma_max / lle_band / jump / min_predictable >= 0");
    std::string err;
    if (!ensure_init(e, err)) return fail(UCB_E_NOGPU, err);
    cudaStream_t st = stream ? (cudaStream_t)stream : e->stream;

    ucb_lle2d_request qs = r.map, qr = r.map;
    qs.opt.precision = r.sample_precision;
    qr.opt.precision = r.refine_precision;
    qs.csv_output_path = qr.csv_output_path = nullptr;
    LaunchHandle hs, hr;
    int rc = lle2d_plan_and_find(e, qs, true, err, &hs.plan, &hs.launch);
    if (rc != UCB_OK) return fail(rc, err);
    rc = lle2d_plan_and_find(e, qr, true, err, &hr.plan, &hr.launch);
    if (rc != UCB_OK) return fail(rc, err);
    SweepMap map;
    int n_blocks = 0, skip = 0;
    long long nt = 0;
    if (!plan_sweep2d(r.map, map, n_blocks, skip, nt, err)) return fail(UCB_E_INVALID, err);

    const long long total = (long long)n * n;
    const long long ns = (long long)tp * tp;
    cudaEvent_t ev[6];
    for (auto& x : ev) cudaEventCreate(&x);
    struct EvFree {
        cudaEvent_t* ev;
        ~EvFree() {
            for (int i = 0; i < 6; ++i) cudaEventDestroy(ev[i]);
        }
    } evf{ev};
    DevFree mem{e, st, {}};
    long long* d_cells = mem.alloc<long long>(ns, err, "sample cells");
    double* d_sv = mem.alloc<double>(ns, err, "sample values");
    int* d_sf = mem.alloc<int>(ns, err, "sample flags");
    unsigned char* d_mask = mem.alloc<unsigned char>(total, err, "mask");
    float* d_mean = mem.alloc<float>(total, err, "mean");
    float* d_sd = mem.alloc<float>(total, err, "std");
    long long* d_list = mem.alloc<long long>(total, err, "refine list");
    unsigned long long* d_count = mem.alloc<unsigned long long>(2, err, "counters");
    if (!d_cells || !d_sv || !d_sf || !d_mask || !d_mean || !d_sd || !d_list || !d_count) return fail(UCB_E_CUDA, err);
    cudaMemsetAsync(d_mask, 0, total, st);
    cudaMemsetAsync(d_count, 0, 2 * sizeof(unsigned long long), st);

    // 1. samples: one random cell per block of the tp x tp partition. The pilot subset
    // (every pilot_stride-th block along both axes) is integrated first and decides whether
    // a network is worth training (pilot_share); the other samples are integrated only then.
    cudaEventRecord(ev[0], st);
    ucbsur::sample_cells_kernel<<<(unsigned)((ns + 255) / 256), 256, 0, st>>>(n, tp, r.mlp.seed ^ 0xC0FFEEULL,
                                                                             d_cells);
    e->launches += 1;
    std::vector<long long> hc(ns);
    if (cudaMemcpyAsync(hc.data(), d_cells, ns * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail(UCB_E_CUDA, std::string("sample cells: ") + cudaGetErrorString(cudaGetLastError()));
    const int ps = pilot_stride(tp);
    const int tq = (tp + ps - 1) / ps;
    std::vector<char> is_pilot(ns, 0);
    std::vector<long long> pilot_idx, rest_idx;
    for (int qy = 0; qy < tq; ++qy)
        for (int qx = 0; qx < tq; ++qx) {
            const long long i = (long long)(qy * ps) * tp + qx * ps;
            pilot_idx.push_back(i);
            is_pilot[i] = 1;
        }
    for (long long i = 0; i < ns; ++i)
        if (!is_pilot[i]) rest_idx.push_back(i);
    const long long np = (long long)pilot_idx.size(), nr = (long long)rest_idx.size();
    auto integrate = [&](const std::vector<long long>& idx, long long*& d_c, double*& d_v, int*& d_f,
                         std::vector<double>& v, std::vector<int>& f) -> int {
        const long long m = (long long)idx.size();
        std::vector<long long> cells(m);
        for (long long k = 0; k < m; ++k) cells[k] = hc[idx[k]];
        d_c = mem.alloc<long long>(m, err, "sample cells");
        d_v = mem.alloc<double>(m, err, "sample values");
        d_f = mem.alloc<int>(m, err, "sample flags");
        if (!d_c || !d_v || !d_f) return UCB_E_CUDA;
        v.resize(m);
        f.resize(m);
        if (m == 0) return UCB_OK;
        cudaMemcpyAsync(d_c, cells.data(), m * 8, cudaMemcpyHostToDevice, st);
        const int q = lle2d_enqueue_cells(e, qs, hs.plan, hs.launch, d_c, m, true, d_v, d_f, st, err);
        if (q != UCB_OK) return q;
        if (cudaMemcpyAsync(v.data(), d_v, m * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(f.data(), d_f, m * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            err = std::string("samples: ") + cudaGetErrorString(cudaGetLastError());
            return UCB_E_CUDA;
        }
        return UCB_OK;
    };
    long long *d_pc = nullptr, *d_rc = nullptr;
    double *d_pv = nullptr, *d_rv = nullptr;
    int *d_pf = nullptr, *d_rf = nullptr;
    std::vector<double> pv, rv;
    std::vector<int> pf, rf;
    rc = integrate(pilot_idx, d_pc, d_pv, d_pf, pv, pf);
    if (rc != UCB_OK) return fail(rc, err);
    {
        std::vector<long long> pcells(np);
        for (long long k = 0; k < np; ++k) pcells[k] = hc[pilot_idx[k]];
        res->pilot_predictable = pilot_share(pv, pf, pcells, n, tq, r.tol, r.coverage, r.lle_band);
    }
    res->gated = res->pilot_predictable < r.min_predictable ? 1 : 0;
    std::vector<double> hv(ns);
    std::vector<int> hf(ns);
    if (!res->gated) {
        rc = integrate(rest_idx, d_rc, d_rv, d_rf, rv, rf);
        if (rc != UCB_OK) return fail(rc, err);
        for (long long k = 0; k < np; ++k) {
            hv[pilot_idx[k]] = pv[k];
            hf[pilot_idx[k]] = pf[k];
        }
        for (long long k = 0; k < nr; ++k) {
            hv[rest_idx[k]] = rv[k];
            hf[rest_idx[k]] = rf[k];
        }
        cudaMemcpyAsync(d_sv, hv.data(), ns * 8, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_sf, hf.data(), ns * 4, cudaMemcpyHostToDevice, st);
    }
    cudaEventRecord(ev[1], st);
    // Samples held out for calibration (by a hash of their block): one in eight, more when
    // that leaves fewer than 1,024 (up to half), so that the calibration's confidence bound
    // can reach the requested coverage at all.
    const long long hold = std::max<long long>(512, std::min<long long>(2048, (1024LL * 4096 + ns - 1) / std::max<long long>(ns, 1)));
    std::vector<float> hu, hy;
    std::vector<long long> cal_cells;
    std::vector<double> cal_y;
    hu.reserve(2 * ns);
    hy.reserve(ns);
    const float inv = 1.0f / (float)(n - 1);
    for (long long i = 0; i < ns && !res->gated; ++i) {
        if (hf[i] != 1 || !std::isfinite(hv[i])) continue;
        unsigned long long z = (unsigned long long)i * 0x9E3779B97F4A7C15ULL + r.mlp.seed;
        z ^= z >> 31;
        if ((long long)(z % 4096) < hold) {
            cal_cells.push_back(hc[i]);
            cal_y.push_back(hv[i]);
            continue;
        }
        hu.push_back((float)(hc[i] % n) * inv);
        hu.push_back((float)(hc[i] / n) * inv);
        hy.push_back((float)hv[i]);
    }
    const long long n_train = (long long)hy.size();
    const long long n_cal = (long long)cal_y.size();
    res->n_samples = res->gated ? np : ns;
    res->n_calib = n_cal;

    // 2. training (the engine keeps the network's buffers between calls with the same
    // configuration; parameters are re-initialised from the seed every call)
    Mlp* net = nullptr;
    float* d_u = mem.alloc<float>(std::max<long long>(2 * n_train, 1), err, "train u");
    float* d_y = mem.alloc<float>(std::max<long long>(n_train, 1), err, "train y");
    if (!d_u || !d_y) return fail(UCB_E_CUDA, err);
    if (n_train > 0) {
        cudaMemcpyAsync(d_u, hu.data(), hu.size() * 4, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_y, hy.data(), hy.size() * 4, cudaMemcpyHostToDevice, st);
        Mlp* cached = static_cast<Mlp*>(e->surrogate_net.get());
        if (cached && std::memcmp(&mlp_config(cached), &r.mlp, sizeof(ucb_mlp_config)) == 0) {
            if (!mlp_reinit(cached, err)) return fail(UCB_E_CUDA, err);
            net = cached;
        } else {
            e->surrogate_net.reset();
            net = mlp_create(e, r.mlp, err);
            if (!net) return fail(UCB_E_INVALID, err);
            e->surrogate_net = std::shared_ptr<void>(net, [](void* q) { mlp_destroy(static_cast<Mlp*>(q)); });
        }
        MlpInputs tin;
        tin.u = d_u;
        tin.n = n_train;
        if (!mlp_fit(net, tin, d_y, st, &res->final_loss, err)) return fail(UCB_E_CUDA, err);
    }
    cudaEventRecord(ev[2], st);

    // 3. prediction over the grid (no training rows: everything is re-integrated)
    if (n_train > 0) {
        MlpInputs pin;
        pin.n = total;
        pin.grid_n = n;
        if (!mlp_predict(net, pin, d_mean, d_sd, st, err)) return fail(UCB_E_CUDA, err);
    } else {
        cudaMemsetAsync(d_mean, 0, total * 4, st);
        cudaMemsetAsync(d_sd, 0, total * 4, st);
    }
    // calibration: the largest std threshold under which >= coverage of the held-out
    // samples lie within tol of their integrated value
    double thr = -1.0, within = 0.0;
    if (n_train > 0 && n_cal > 0) {
        long long* d_cc = mem.alloc<long long>(n_cal, err, "calibration cells");
        float* d_gm = mem.alloc<float>(n_cal, err, "calibration mean");
        float* d_gs = mem.alloc<float>(n_cal, err, "calibration std");
        if (!d_cc || !d_gm || !d_gs) return fail(UCB_E_CUDA, err);
        std::vector<float> gm(n_cal), gs(n_cal);
        cudaMemcpyAsync(d_cc, cal_cells.data(), n_cal * 8, cudaMemcpyHostToDevice, st);
        ucbsur::gather_kernel<<<(unsigned)((n_cal + 255) / 256), 256, 0, st>>>(d_mean, d_sd, d_cc, n_cal, d_gm, d_gs);
        e->launches += 1;
        if (cudaMemcpyAsync(gm.data(), d_gm, n_cal * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(gs.data(), d_gs, n_cal * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return fail(UCB_E_CUDA, std::string("calibration: ") + cudaGetErrorString(cudaGetLastError()));
        std::vector<long long> order(n_cal);
        for (long long i = 0; i < n_cal; ++i) order[i] = i;
        std::sort(order.begin(), order.end(), [&](long long a, long long b) { return gs[a] < gs[b]; });
        // The std threshold is the largest one under which the held-out samples certify the
        // coverage: the one-sided 90 % Wilson lower bound of the fraction within tol must
        // reach it (a point estimate from a few hundred samples would let a per-cell outlier
        // rate of half a percent through).
        long long good = 0;
        const long long min_count = std::min<long long>(n_cal, 32);
        auto wilson_lower = [](double k, double n) {
            const double z = 1.2815515655446004, z2 = z * z, ph = k / n;
            return (ph + z2 / (2 * n) - z * std::sqrt(ph * (1 - ph) / n + z2 / (4 * n * n))) / (1 + z2 / n);
        };
        for (long long k = 0; k < n_cal; ++k) {
            const long long i = order[k];
            good += std::fabs((double)gm[i] - cal_y[i]) <= r.tol;
            const long long cnt = k + 1;
            if (cnt >= min_count && wilson_lower((double)good, (double)cnt) >= r.coverage &&
                (k + 1 == n_cal || gs[order[k + 1]] > gs[i])) {
                thr = gs[i];
                within = (double)good / (double)cnt;
            }
        }
        if (r.sigma_max > 0 && thr > r.sigma_max) thr = r.sigma_max;
    }
    res->sigma_threshold = thr;
    res->calib_within_tol = within;
    cudaEventRecord(ev[3], st);

    // 4. selection
    if (res->gated)  // only the pilot samples were integrated: everything else is
        ucbsur::scatter_samples_kernel<<<(unsigned)((np + 255) / 256), 256, 0, st>>>(
            d_pc, np, d_pv, d_pf, n, map.swap_xy ? 1 : 0, d_mask, d_values, d_flags);
    else
        ucbsur::scatter_samples_kernel<<<(unsigned)((ns + 255) / 256), 256, 0, st>>>(
            d_cells, ns, d_sv, d_sf, n, map.swap_xy ? 1 : 0, d_mask, d_values, d_flags);
    const float sigma = (float)thr;  // < 0 (no network or no calibrated threshold): refine all
    ucbsur::select_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
        d_mean, d_sd, d_mask, n, map.swap_xy ? 1 : 0, sigma, (float)r.lle_band, (float)r.jump, d_list, d_count,
        d_values, d_flags);
    e->launches += 2;
    unsigned long long n_ref = 0;
    if (cudaMemcpyAsync(&n_ref, d_count, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail(UCB_E_CUDA, std::string("select: ") + cudaGetErrorString(cudaGetLastError()));
    cudaEventRecord(ev[4], st);

    // 5. re-integration straight into the map
    rc = lle2d_enqueue_cells(e, qr, hr.plan, hr.launch, d_list, (long long)n_ref, false, d_values, d_flags, st, err);
    if (rc != UCB_OK) return fail(rc, err);
    cudaEventRecord(ev[5], st);
    ucbsur::count_flag_kernel<<<e->sm_count * 4, 256, 0, st>>>(d_flags, total, -1, d_count + 1);
    e->launches += 1;
    unsigned long long n_div = 0;
    if (cudaMemcpyAsync(&n_div, d_count + 1, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail(UCB_E_CUDA, std::string("refine: ") + cudaGetErrorString(cudaGetLastError()));
    float ms[5] = {0, 0, 0, 0, 0};
    for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]);
    res->sample_ms = ms[0];
    res->train_ms = ms[1];
    res->predict_ms = ms[2];
    res->select_ms = ms[3];
    res->refine_ms = ms[4];
    res->n_refined = (long long)n_ref;
    res->n_predicted = total - res->n_samples - (long long)n_ref;  // sample cells are integrated
    res->n_diverged = (long long)n_div;
    res->n_pts = n;
    res->total_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    res->ok = 1;
    return UCB_OK;
}

}  // extern "C"
