// Bifurcation 1D host orchestration.
//
// Validation, sweep mapping and step counts follow run_bif1d (parametric_engine.cpp:
// 1702-1829): amountOfPointsInBlock = ceil(tMax / worstCaseH / preScaller) and
// amountOfPointsForSkip = (int)(transient / h) in double, peak intervals in units of
// h * preScaller, the h-sweep interval rescaling by param_val / h (:1991-2003). The device
// side is one fused kernel (integration + streaming peak capture), see ucb_bif.cuh.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iomanip>

#include "csv_export.h"
#include "engine_internal.h"

using namespace ucb;

namespace {

constexpr int kMaxAmountOfX = 32;
constexpr int kMaxAmountOfValues = 64;

bool validate_bif(const ucb_bif1d_request& q, std::string& err) {
    if (!q.krs_body || !*q.krs_body) { err = "krs_body is empty"; return false; }
    if (q.amount_of_x <= 0 || q.amount_of_x > kMaxAmountOfX) { err = "amountOfX out of [1,32]"; return false; }
    if (!q.initial_conditions) { err = "initial_conditions.size() != amountOfX"; return false; }
    if (q.n_values > kMaxAmountOfValues) { err = "too many base_values"; return false; }
    if (q.sweep_over_h) {
        if (q.param_lo <= 0.0 || q.param_hi <= 0.0) { err = "h lo/hi must be > 0 when sweep_over_h"; return false; }
    } else if (q.sweep_over_var) {
        if (q.var_sweep_index < 0 || q.var_sweep_index >= q.amount_of_x) { err = "var_sweep_index out of range"; return false; }
    } else {
        if (q.param_index <= 0 || q.param_index >= q.n_values) { err = "param_index out of range"; return false; }
    }
    if (q.writable_var < -1 || q.writable_var >= q.amount_of_x) { err = "writable_var out of range"; return false; }
    if (q.n_pts <= 0) { err = "n_pts must be > 0"; return false; }
    if (!(q.h > 0.0)) { err = "h must be > 0"; return false; }
    if (!(q.t_max > 0.0)) { err = "t_max must be > 0"; return false; }
    if (q.transient_time < 0) { err = "transient_time must be >= 0"; return false; }
    if (q.pre_scaller <= 0) { err = "pre_scaller must be > 0"; return false; }
    if (q.log_scale && !(q.param_lo > 0.0 && q.param_hi > 0.0)) { err = "log scale requires param lo/hi > 0"; return false; }
    if (q.max_peaks < 0) { err = "max_peaks must be >= 0"; return false; }
    return true;
}

CompileRequest bif_compile_request(const ucb_bif1d_request& q, SystemCode& sys) {
    SweepMap m;
    m.dim = 1;
    m.par_or_var = q.sweep_over_var ? 0 : 1;
    m.idx[0] = q.sweep_over_h ? 0 : (q.sweep_over_var ? q.var_sweep_index : q.param_index);
    m.h_axis = q.sweep_over_h ? 0 : -1;
    sys = make_system_code(q.krs_body, q.amount_of_x, q.n_values, q.opt.precision, q.opt.mode, false);
    CompileRequest rq;
    rq.name = "ucb_bif1d.cu";
    rq.source = make_prelude(q.opt.precision, q.amount_of_x, q.n_values, m, true, sys, clock_defines(sys)) +
                "#include \"ucb_device.cuh\"\n#include \"ucb_bif.cuh\"\n";
    rq.headers = device_headers();
    rq.options.push_back(sys.exact ? "--fmad=false" : "--fmad=true");
    rq.kernels = {"ucb_bif_kernel"};
    return rq;
}

int fail(ucb_engine* e, ucb_bif1d_result* r, int code, const std::string& msg) {
    e->last_error = msg;
    std::snprintf(r->error, sizeof r->error, "%s", msg.c_str());
    r->ok = 0;
    return code;
}

}  // namespace

extern "C" int ucb_precompile_bif1d(const ucb_bif1d_request* req, char* err_out, int err_len) {
    std::string err;
    if (!req || !validate_bif(*req, err)) {
        if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", err.c_str());
        return UCB_E_INVALID;
    }
    SystemCode sys;
    CompileRequest rq = bif_compile_request(*req, sys);
    TuneConfig shape;
    if (!tune_request(nullptr, req->opt, 32, rq, shape, err)) {
        if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", err.c_str());
        return UCB_E_INVALID;
    }
    if (!precompile_to_disk(rq, err)) {
        if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", err.c_str());
        return UCB_E_COMPILE;
    }
    if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", sys.note.c_str());
    return UCB_OK;
}

extern "C" int ucb_run_bif1d(ucb_engine* e, const ucb_bif1d_request* req, ucb_bif1d_result* res) {
    if (!e || !req || !res) return UCB_E_INVALID;
    const ucb_bif1d_request& q = *req;
    res->ok = res->cancelled = 0;
    res->error[0] = 0;
    res->kernel_ms = 0;
    res->steps = 0;
    res->flops = 0;
    std::string err;
    if (!validate_bif(q, err)) return fail(e, res, UCB_E_INVALID, err);
    if (!res->counts || (q.max_peaks > 0 && (!res->peaks || !res->intervals)))
        return fail(e, res, UCB_E_INVALID, "result buffers are NULL");
    if (q.cancel && *q.cancel) {
        res->cancelled = 1;
        return fail(e, res, UCB_E_CANCELLED, "Cancelled by user");
    }
    const int prec = q.opt.precision;
    // kernel-side numb copies of the range (ranges[] in run_bif1d are numb)
    const double lo_n = prec == UCB_PREC_F64 ? q.param_lo : (double)(float)q.param_lo;
    const double hi_n = prec == UCB_PREC_F64 ? q.param_hi : (double)(float)q.param_hi;
    const double worstCaseH = q.sweep_over_h ? lo_n : q.h;
    const long long pointsInBlock = (long long)std::ceil(q.t_max / worstCaseH / q.pre_scaller);
    const long long pointsForSkip = (long long)(q.transient_time / q.h);
    if (pointsInBlock <= 0) return fail(e, res, UCB_E_INVALID, "computed amountOfPointsInBlock <= 0");
    if (!ensure_init(e, err)) return fail(e, res, UCB_E_NOGPU, err);

    SystemCode sys;
    CompileRequest rq = bif_compile_request(q, sys);
    TuneConfig shape;
    if (!tune_request(e, q.opt, 32, rq, shape, err)) return fail(e, res, UCB_E_INVALID, err);
    auto mod = e->modules.get(rq, err);
    if (!mod) return fail(e, res, UCB_E_COMPILE, err);
    CUfunction fn = mod->functions["ucb_bif_kernel"];

    const int n = q.n_pts;
    const int mo = q.max_peaks;
    std::vector<double> tab_d;
    std::vector<float> tab_f;
    axis_table(prec, n, q.param_lo, q.param_hi, q.log_scale != 0, tab_d, tab_f);
    const size_t esz = prec == UCB_PREC_F64 ? 8 : 4;
    const size_t tab_bytes = (size_t)n * esz;
    if (!ensure_workspace(e, 256 + tab_bytes + 256, err)) return fail(e, res, UCB_E_CUDA, err);
    char* ws = static_cast<char*>(e->ws);
    int32_t* d_counts = nullptr;
    double* d_peaks = nullptr;
    double* d_int = nullptr;
    const size_t pk_elems = (size_t)n * (size_t)std::max(mo, 1);
    cudaError_t ce;
    if ((ce = dev_alloc(e, (void**)&d_counts, (size_t)n * 4, e->stream)) != cudaSuccess ||
        (ce = dev_alloc(e, (void**)&d_peaks, pk_elems * 8, e->stream)) != cudaSuccess ||
        (ce = dev_alloc(e, (void**)&d_int, pk_elems * 8, e->stream)) != cudaSuccess)
        return fail(e, res, UCB_E_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(ce));
    cudaMemcpyAsync(ws + 256, prec == UCB_PREC_F64 ? (const void*)tab_d.data() : (const void*)tab_f.data(), tab_bytes,
                    cudaMemcpyHostToDevice, e->stream);
    cudaMemsetAsync(ws, 0, 16, e->stream);
    ParamPack pk;
    pk.put<int>(n);
    pk.put<int>(q.pre_scaller);
    pk.put<int>(q.writable_var);
    pk.put<int>(std::max(mo, 1));
    pk.put<long long>(pointsForSkip);
    pk.put<long long>(pointsInBlock);
    const double time_step = q.h * (double)q.pre_scaller;
    for (double v : {q.h, q.max_value, q.transient_time, q.t_max, time_step}) pk.put_numb(prec, v);
    for (int i = 0; i < q.amount_of_x; ++i) pk.put_numb(prec, q.initial_conditions[i]);
    for (int i = 0; i < std::max(q.n_values, 1); ++i) pk.put_numb(prec, i < q.n_values ? q.base_values[i] : 0.0);
    pk.put<const void*>(ws + 256);
    pk.put<void*>(d_counts);
    pk.put<void*>(d_peaks);
    pk.put<void*>(d_int);
    pk.put<void*>(ws);
    pk.put<void*>(ws + 8);
    const int block = shape.block;  // default 32: latency-bound, spread the few points over many SMs
    cudaEventRecord(e->ev0, e->stream);
    const bool launched = launch_packed(e, fn, (n + block - 1) / block, block, e->stream, pk, err);
    cudaEventRecord(e->ev1, e->stream);
    int rc = launched ? UCB_OK : UCB_E_CUDA;
    std::vector<double> hp(pk_elems), hi(pk_elems);
    unsigned long long steps = 0;
    if (rc == UCB_OK) {
        if ((ce = cudaMemcpyAsync(res->counts, d_counts, (size_t)n * 4, cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess ||
            (ce = cudaMemcpyAsync(hp.data(), d_peaks, pk_elems * 8, cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess ||
            (ce = cudaMemcpyAsync(hi.data(), d_int, pk_elems * 8, cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess ||
            (ce = cudaMemcpyAsync(&steps, ws + 8, 8, cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess ||
            (ce = cudaStreamSynchronize(e->stream)) != cudaSuccess) {
            rc = UCB_E_CUDA;
            err = std::string("CUDA bif1d: ") + cudaGetErrorString(ce);
        }
    }
    cudaFreeAsync(d_counts, e->stream);
    cudaFreeAsync(d_peaks, e->stream);
    cudaFreeAsync(d_int, e->stream);
    cudaStreamSynchronize(e->stream);
    if (rc != UCB_OK) return fail(e, res, rc, err);
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    res->kernel_ms = ms;
    res->steps = (long long)steps;
    res->flops = (double)steps * sys.flops_step;
    for (int i = 0; i < n; ++i) {
        const int cnt = res->counts[i];
        const int k = std::min(std::max(cnt, 0), mo);
        // h-sweep: intervals are linear in h; rescale by param_val / h as run_bif1d does.
        double ts = 1.0;
        if (q.sweep_over_h) {
            double pv;
            if (n <= 1) pv = lo_n;
            else if (q.log_scale)
                pv = std::pow(10.0, std::log10(lo_n) + (std::log10(hi_n) - std::log10(lo_n)) * (double)i / (double)(n - 1));
            else
                pv = lo_n + (hi_n - lo_n) * (double)i / (double)(n - 1);
            ts = pv / q.h;
        }
        for (int j = 0; j < mo; ++j) {
            res->peaks[(size_t)i * mo + j] = j < k ? hp[(size_t)i * std::max(mo, 1) + j] : NAN;
            res->intervals[(size_t)i * mo + j] = j < k ? hi[(size_t)i * std::max(mo, 1) + j] * ts : NAN;
        }
    }
    res->n_pts = n;
    res->record_steps = (int)pointsInBlock;
    res->param_lo = q.param_lo;
    res->param_hi = q.param_hi;
    if (q.csv_output_path && *q.csv_output_path) {
        const bool f32 = q.opt.precision == UCB_PREC_F32;
        const csv::Common cc = csv::common(q.base_values, q.n_values, q.initial_conditions, q.amount_of_x, f32);
        csv::bif1d(q.csv_output_path, cc, q.t_max, q.transient_time, q.h, q.pre_scaller, q.writable_var,
                   q.sweep_over_var ? q.var_sweep_index : q.param_index, lo_n, hi_n, n, res->counts, res->peaks,
                   res->intervals, mo);
    }
    if (q.progress) *q.progress = 1.0f;
    res->ok = 1;
    return UCB_OK;
}
