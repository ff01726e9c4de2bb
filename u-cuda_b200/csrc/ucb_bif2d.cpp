// Bifurcation 2D (period maps) host orchestration: run_bif2d (parametric_engine.cpp:
// 5487-5910) — its validation, the LLE-2D axis mapping (par_or_var / swap_xy / h axis),
// amountOfPointsInBlock = ceil(tMax / worstCaseH / preScaller) and (int)(transient / h) in
// double, values = period (-1 with flag -1 where the dbscan result is negative), min / max
// over the other cells, CSV. The reference chunks the grid by free memory because it
// keeps the whole recorded series of every cell; here one persistent kernel integrates,
// captures the peaks into a scratch slot per resident warp and clusters them
// (ucb_bif.cuh), so the whole grid is one launch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

#include "csv_export.h"
#include "engine_internal.h"

using namespace ucb;

namespace {

constexpr int kMaxAmountOfX = 32;
constexpr int kMaxAmountOfValues = 64;
constexpr int kMaxAmountOfPeaks = 2500;  // configCUDA.h max_amount_of_peaks

int fail(ucb_engine* e, ucb_bif2d_result* r, int code, const std::string& msg) {
    e->last_error = msg;
    std::snprintf(r->error, sizeof r->error, "%s", msg.c_str());
    r->ok = 0;
    return code;
}

// The LLE-2D request with the same sweep fields (its own NT / eps checks are satisfied by
// placeholders: the period map has no blocks).
ucb_lle2d_request as_lle(const ucb_bif2d_request& q) {
    ucb_lle2d_request l{};
    l.krs_body = q.krs_body;
    l.amount_of_x = q.amount_of_x;
    l.initial_conditions = q.initial_conditions;
    l.base_values = q.base_values;
    l.n_values = q.n_values;
    l.sweep_over_var = q.sweep_over_var;
    l.sweep_over_var_2 = q.sweep_over_var_2;
    l.sweep_over_h = q.sweep_over_h;
    l.sweep_over_h_2 = q.sweep_over_h_2;
    l.log_scale = q.log_scale;
    l.log_scale_2 = q.log_scale_2;
    l.param_index = q.param_index;
    l.var_sweep_index = q.var_sweep_index;
    l.param_index_2 = q.param_index_2;
    l.var_sweep_index_2 = q.var_sweep_index_2;
    l.param_lo = q.param_lo;
    l.param_hi = q.param_hi;
    l.param_lo_2 = q.param_lo_2;
    l.param_hi_2 = q.param_hi_2;
    l.n_pts = q.n_pts;
    l.h = q.h;
    l.transient_time = q.transient_time;
    l.t_max = q.t_max;
    l.NT = q.t_max;
    l.eps = 1.0;
    l.max_value = q.max_value;
    l.opt = q.opt;
    return l;
}

// Validation of run_bif2d (parametric_engine.cpp:5490-5572) and the axis mapping.
bool plan_bif2d(const ucb_bif2d_request& q, SweepMap& m, std::string& err) {
    if (!q.krs_body || !*q.krs_body) { err = "krs_body is empty"; return false; }
    if (q.amount_of_x <= 0 || q.amount_of_x > kMaxAmountOfX) { err = "amountOfX out of [1,32]"; return false; }
    if (!q.initial_conditions) { err = "initial_conditions.size() != amountOfX"; return false; }
    if (q.n_values > kMaxAmountOfValues) { err = "too many base_values"; return false; }
    if (q.n_pts <= 0) { err = "n_pts must be > 0"; return false; }
    if (!(q.h > 0.0)) { err = "h must be > 0"; return false; }
    if (!(q.t_max > 0.0)) { err = "t_max must be > 0"; return false; }
    if (q.transient_time < 0) { err = "transient_time must be >= 0"; return false; }
    if (q.pre_scaller <= 0) { err = "pre_scaller must be > 0"; return false; }
    if (!(q.eps_dbscan > 0.0)) { err = "eps_dbscan must be > 0"; return false; }
    if (q.writable_var < -1 || q.writable_var >= q.amount_of_x) { err = "writable_var out of range"; return false; }
    if ((q.sweep_over_h != 0) != (q.sweep_over_h_2 != 0)) {  // one h axis (both: rejected below)
        if (q.param_lo <= 0.0 || q.param_hi <= 0.0 || q.param_lo_2 <= 0.0 || q.param_hi_2 <= 0.0) {
            err = "h lo/hi must be > 0 with sweep_over_h / sweep_over_h_2";
            return false;
        }
    }
    int n_blocks = 0, skip = 0;
    long long nt = 0;
    return plan_sweep2d(as_lle(q), m, n_blocks, skip, nt, err);
}

CompileRequest bif2d_compile_request(const ucb_bif2d_request& q, const SweepMap& m, SystemCode& sys) {
    sys = make_system_code(q.krs_body, q.amount_of_x, q.n_values, q.opt.precision, q.opt.mode, false);
    CompileRequest rq;
    rq.name = "ucb_bif2d.cu";
    std::vector<std::string> defs = clock_defines(sys);
    defs.push_back("UCB_BIF2D 1");
    rq.source = make_prelude(q.opt.precision, q.amount_of_x, q.n_values, m, true, sys, defs) +
                "#include \"ucb_device.cuh\"\n#include \"ucb_bif.cuh\"\n";
    rq.headers = device_headers();
    rq.options.push_back(sys.exact ? "--fmad=false" : "--fmad=true");
    rq.kernels = {"ucb_bif2d_kernel"};
    return rq;
}

}  // namespace

extern "C" int ucb_precompile_bif2d(const ucb_bif2d_request* req, char* err_out, int err_len) {
    std::string err;
    SweepMap m;
    if (!req || !plan_bif2d(*req, m, err)) {
        if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", err.c_str());
        return UCB_E_INVALID;
    }
    SystemCode sys;
    CompileRequest rq = bif2d_compile_request(*req, m, sys);
    TuneConfig shape;
    if (!tune_request(nullptr, req->opt, 128, rq, shape, err)) {
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

extern "C" int ucb_run_bif2d(ucb_engine* e, const ucb_bif2d_request* req, ucb_bif2d_result* res) {
    if (!e || !req || !res) return UCB_E_INVALID;
    const ucb_bif2d_request& q = *req;
    res->ok = res->cancelled = 0;
    res->error[0] = 0;
    res->kernel_ms = 0;
    res->steps = 0;
    res->flops = 0;
    std::string err;
    SweepMap m;
    if (!plan_bif2d(q, m, err)) return fail(e, res, UCB_E_INVALID, err);
    if (!res->values || !res->flags) return fail(e, res, UCB_E_INVALID, "result buffers are NULL");
    if (q.cancel && *q.cancel) {
        res->cancelled = 1;
        return fail(e, res, UCB_E_CANCELLED, "Cancelled by user");
    }
    const int prec = q.opt.precision;
    const size_t esz = prec == UCB_PREC_F64 ? 8 : 4;
    auto as_numb = [&](double v) { return prec == UCB_PREC_F64 ? v : (double)(float)v; };
    // ranges[] of run_bif2d are numb, in kernel axis order
    const double worstCaseH = m.h_axis == 0 ? as_numb(m.lo[0]) : (m.h_axis == 1 ? as_numb(m.lo[1]) : q.h);
    const long long pointsInBlock = (long long)std::ceil(q.t_max / worstCaseH / q.pre_scaller);
    const long long pointsForSkip = (long long)(q.transient_time / q.h);
    if (pointsInBlock <= 0) return fail(e, res, UCB_E_INVALID, "computed amountOfPointsInBlock <= 0");
    if (!ensure_init(e, err)) return fail(e, res, UCB_E_NOGPU, err);

    SystemCode sys;
    CompileRequest rq = bif2d_compile_request(q, m, sys);
    TuneConfig shape;
    if (!tune_request(e, q.opt, 128, rq, shape, err)) return fail(e, res, UCB_E_INVALID, err);
    auto mod = e->modules.get(rq, err);
    if (!mod) return fail(e, res, UCB_E_COMPILE, err);
    CUfunction fn = mod->functions["ucb_bif2d_kernel"];

    const int n = q.n_pts;
    const long long total = (long long)n * n;
    // A peak needs a rise and a fall: at most one per two recorded samples.
    const int cap = (int)std::min<long long>(kMaxAmountOfPeaks, pointsInBlock / 2 + 2);
    // Scratch per resident warp: 32 rows of peaks + dbscan labels and stack slots. The
    // persistent grid is trimmed if the slots would exceed 40 % of the free memory.
    const int block = shape.block, warps_per_block = block / 32;
    const size_t per_warp = (size_t)cap * (32 * esz + 2 * sizeof(int32_t));
    int grid = persistent_grid(e, fn, block, total);
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const size_t budget = std::max<size_t>((size_t)(0.4 * (double)free_b), (size_t)64 << 20);
    grid = (int)std::max<long long>(1, std::min<long long>(grid, (long long)(budget / (per_warp * warps_per_block))));
    const size_t slot_bytes = (size_t)grid * warps_per_block * 32 * cap * esz;
    const size_t work_bytes = (size_t)grid * warps_per_block * 2 * cap * sizeof(int32_t);

    std::vector<double> t0d, t1d;
    std::vector<float> t0f, t1f;
    axis_table(prec, n, m.lo[0], m.hi[0], m.log_axis[0], t0d, t0f);
    axis_table(prec, n, m.lo[1], m.hi[1], m.log_axis[1], t1d, t1f);
    const size_t tab_bytes = (size_t)n * esz;
    const size_t off0 = 256, off1 = 256 + ((tab_bytes + 255) / 256) * 256;
    if (!ensure_workspace(e, off1 + tab_bytes + 256, err)) return fail(e, res, UCB_E_CUDA, err);
    char* ws = static_cast<char*>(e->ws);
    double* d_values = nullptr;
    int32_t* d_flags = nullptr;
    char* d_slots = nullptr;
    char* d_work = nullptr;
    cudaError_t ce;
    if ((ce = dev_alloc(e, (void**)&d_values, (size_t)total * 8, e->stream)) != cudaSuccess ||
        (ce = dev_alloc(e, (void**)&d_flags, (size_t)total * 4, e->stream)) != cudaSuccess ||
        (ce = dev_alloc(e, (void**)&d_slots, slot_bytes, e->stream)) != cudaSuccess ||
        (ce = dev_alloc(e, (void**)&d_work, work_bytes, e->stream)) != cudaSuccess) {
        for (void* ptr : {(void*)d_values, (void*)d_flags, (void*)d_slots})
            if (ptr) cudaFreeAsync(ptr, e->stream);
        cudaStreamSynchronize(e->stream);
        return fail(e, res, UCB_E_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(ce));
    }
    cudaMemcpyAsync(ws + off0, prec == UCB_PREC_F64 ? (const void*)t0d.data() : (const void*)t0f.data(), tab_bytes,
                    cudaMemcpyHostToDevice, e->stream);
    cudaMemcpyAsync(ws + off1, prec == UCB_PREC_F64 ? (const void*)t1d.data() : (const void*)t1f.data(), tab_bytes,
                    cudaMemcpyHostToDevice, e->stream);
    cudaMemsetAsync(ws, 0, 16, e->stream);
    if (q.progress) *q.progress = 0.0f;
    int rc = UCB_OK;
    // UcbBif2dParams field by field
    ParamPack pk;
    pk.put<long long>(total);
    pk.put<int>(n);
    pk.put<int>(m.swap_xy ? 1 : 0);
    pk.put<int>(q.pre_scaller);
    pk.put<int>(q.writable_var);
    pk.put<int>(cap);
    pk.put<int>(0);
    pk.put<long long>(pointsForSkip);
    pk.put<long long>(pointsInBlock);
    for (double v : {q.h, q.max_value, q.transient_time, q.t_max, q.eps_dbscan}) pk.put_numb(prec, v);
    for (int i = 0; i < q.amount_of_x; ++i) pk.put_numb(prec, q.initial_conditions[i]);
    for (int i = 0; i < std::max(q.n_values, 1); ++i) pk.put_numb(prec, i < q.n_values ? q.base_values[i] : 0.0);
    pk.put<const void*>(ws + off0);
    pk.put<const void*>(ws + off1);
    pk.put<void*>(d_slots);
    pk.put<void*>(d_work);
    pk.put<void*>(d_values);
    pk.put<void*>(d_flags);
    pk.put<void*>(ws);
    pk.put<void*>(ws + 8);
    begin_run(e);
    cudaEventRecord(e->ev0, e->stream);
    if (!launch_packed(e, fn, grid, block, e->stream, pk, err)) rc = UCB_E_CUDA;
    cudaEventRecord(e->ev1, e->stream);
    if (rc == UCB_OK) rc = wait_run(e, e->ev1, q.cancel, q.progress, total, err);
    if (rc == UCB_E_CANCELLED) res->cancelled = 1;
    unsigned long long steps = 0;
    if (rc == UCB_OK) {
        if ((ce = cudaMemcpyAsync(res->values, d_values, (size_t)total * 8, cudaMemcpyDeviceToHost, e->stream)) !=
                cudaSuccess ||
            (ce = cudaMemcpyAsync(res->flags, d_flags, (size_t)total * 4, cudaMemcpyDeviceToHost, e->stream)) !=
                cudaSuccess ||
            (ce = cudaMemcpyAsync(&steps, ws + 8, 8, cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess ||
            (ce = cudaStreamSynchronize(e->stream)) != cudaSuccess) {
            rc = UCB_E_CUDA;
            err = std::string("CUDA bif2d: ") + cudaGetErrorString(ce);
        }
    }
    cudaFreeAsync(d_values, e->stream);
    cudaFreeAsync(d_flags, e->stream);
    cudaFreeAsync(d_slots, e->stream);
    cudaFreeAsync(d_work, e->stream);
    cudaStreamSynchronize(e->stream);
    if (rc != UCB_OK) return fail(e, res, rc, err);
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    res->kernel_ms = ms;
    res->steps = (long long)steps;
    res->flops = (double)steps * sys.flops_step;
    double vmin = std::numeric_limits<double>::infinity(), vmax = -vmin;
    for (long long k = 0; k < total; ++k) {
        if (res->flags[k] < 0) continue;
        const double v = res->values[k];
        if (!std::isfinite(v) || v < 0.0) continue;
        vmin = std::min(vmin, v);
        vmax = std::max(vmax, v);
    }
    res->min_val = std::isfinite(vmin) ? vmin : 0.0;
    res->max_val = std::isfinite(vmax) ? vmax : 0.0;
    res->n_pts = n;
    res->param_lo = q.param_lo;
    res->param_hi = q.param_hi;
    res->param_lo_2 = q.param_lo_2;
    res->param_hi_2 = q.param_hi_2;
    if (q.csv_output_path && *q.csv_output_path) {
        const csv::Common cc = csv::common(q.base_values, q.n_values, q.initial_conditions, q.amount_of_x,
                                           q.opt.precision == UCB_PREC_F32);
        csv::bif2d(q.csv_output_path, cc, m.par_or_var, q.t_max, q.transient_time, q.h, q.pre_scaller, q.eps_dbscan,
                   q.writable_var, q.sweep_over_var ? q.var_sweep_index : q.param_index,
                   q.sweep_over_var_2 ? q.var_sweep_index_2 : q.param_index_2, q.param_lo, q.param_hi, q.param_lo_2,
                   q.param_hi_2, n, res->values);
    }
    if (q.progress) *q.progress = 1.0f;
    res->ok = 1;
    return UCB_OK;
}

extern "C" int ucb_autotune_bif2d(ucb_engine* e, const ucb_bif2d_request* req, int32_t force, ucb_tune_report* rep) {
    if (!e || !req || !rep) return UCB_E_INVALID;
    std::memset(rep, 0, sizeof *rep);
    std::string err;
    auto bad = [&](int code, const std::string& msg) {
        e->last_error = msg;
        std::snprintf(rep->error, sizeof rep->error, "%s", msg.c_str());
        return code;
    };
    SweepMap m;
    if (!plan_bif2d(*req, m, err)) return bad(UCB_E_INVALID, err);
    if (!ensure_init(e, err)) return bad(UCB_E_NOGPU, err);
    ucb_bif2d_request base = *req;
    base.opt.block_threads = base.opt.max_registers = base.opt.unroll = 0;
    base.csv_output_path = nullptr;
    base.cancel = nullptr;
    base.progress = nullptr;
    SystemCode sys;
    const std::string key = tune_key(bif2d_compile_request(base, m, sys));
    // trial: the same window on at most 512^2 cells, the same horizon (the per-cell peak
    // count, and with it the dbscan's share, depends on it)
    ucb_bif2d_request t = base;
    t.n_pts = std::min(base.n_pts, 512);
    std::vector<double> vals((size_t)t.n_pts * t.n_pts);
    std::vector<int32_t> flags(vals.size());
    auto with = [&](const TuneConfig& c) {
        ucb_bif2d_request q = t;
        q.opt.block_threads = c.block;
        q.opt.max_registers = c.maxreg;
        q.opt.unroll = c.unroll;
        return q;
    };
    auto trial = [&](const TuneConfig& c) -> double {
        ucb_bif2d_request q = with(c);
        ucb_bif2d_result r{};
        r.values = vals.data();
        r.flags = flags.data();
        return ucb_run_bif2d(e, &q, &r) == UCB_OK ? r.kernel_ms : -1.0;
    };
    auto build = [&](const TuneConfig& c) {
        ucb_bif2d_request q = with(c);
        SweepMap m2;
        std::string e2;
        plan_bif2d(q, m2, e2);
        SystemCode s2;
        CompileRequest rq = bif2d_compile_request(q, m2, s2);
        TuneConfig shape;
        tune_request(e, q.opt, 128, rq, shape, e2);
        return rq;
    };
    const int rc = autotune_search(e, key, 128, force != 0, trial, build, rep);
    rep->trial_n_pts = t.n_pts;
    return rc;
}
