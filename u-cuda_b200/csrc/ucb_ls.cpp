// Lyapunov spectrum host orchestration: run_ls_2d (parametric_engine.cpp:3430-3786) —
// the LLE-2D validation and axis mapping, plane-major results, per-plane min/max over
// valid cells, CSV — and run_ls_1d (:3066) over one swept axis. Device side: ucb_ls.cuh.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

#include "csv_export.h"
#include "engine_internal.h"

using namespace ucb;

namespace {

int fail(ucb_engine* e, ucb_ls2d_result* r, int code, const std::string& msg) {
    e->last_error = msg;
    std::snprintf(r->error, sizeof r->error, "%s", msg.c_str());
    r->ok = 0;
    return code;
}

ucb_lle2d_request as_lle(const ucb_ls2d_request& q) {
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
    l.NT = q.NT;
    l.eps = q.eps;
    l.max_value = q.max_value;
    l.opt = q.opt;
    return l;
}

CompileRequest ls_compile_request(const ucb_ls2d_request& q, const SweepMap& m, SystemCode& sys) {
    const bool dp5 = q.method == UCB_LS_DP5;
    const int prec = q.opt.precision;
    // the native FP32 form of the fixed method follows tangent vectors (v' = J(x) v) instead
    // of FP32 shadow trajectories, whose differences from x vanish below FP32 resolution
    const bool tangent = !dp5 && prec == UCB_PREC_F32 && q.opt.mode == UCB_MODE_NATIVE;
    sys = make_system_code(q.krs_body, q.amount_of_x, q.n_values, prec, dp5 ? UCB_MODE_NATIVE : q.opt.mode,
                           dp5 || tangent);
    CompileRequest rq;
    rq.name = "ucb_ls2d.cu";
    // DP5 keeps the clock from its FP64 time; the fixed method steps N + 1 trajectories on
    // one Stepper, so it has no compensated clock
    std::vector<std::string> defs = dp5 ? clock_defines(sys) : std::vector<std::string>{};
    defs.push_back(dp5 ? "UCB_LS_DP5 1" : "UCB_LS_FIXED 1");
    if (tangent && sys.has_jvp) defs.push_back("UCB_LS_TANGENT 1");
    defs.push_back(prec == UCB_PREC_F64 ? "UCB_GS_BUDGET 20.0" : "UCB_GS_BUDGET 8.0");
    rq.source = make_prelude(prec, q.amount_of_x, q.n_values, m, q.opt.nominal_steps == 0, sys, defs) +
                "#include \"ucb_device.cuh\"\n#include \"ucb_ls.cuh\"\n";
    rq.headers = device_headers();
    rq.options.push_back(sys.exact ? "--fmad=false" : "--fmad=true");
    rq.kernels = {"ucb_ls_kernel"};
    return rq;
}

}  // namespace

extern "C" int ucb_precompile_ls2d(const ucb_ls2d_request* req, char* err_out, int err_len) {
    std::string err;
    SweepMap m;
    int nb = 0, sk = 0;
    long long nt = 0;
    if (!req || !plan_sweep2d(as_lle(*req), m, nb, sk, nt, err)) {
        if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", err.c_str());
        return UCB_E_INVALID;
    }
    SystemCode sys;
    CompileRequest rq = ls_compile_request(*req, m, sys);
    if (req->method == UCB_LS_DP5 && !sys.has_jvp) {
        if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", sys.note.c_str());
        return UCB_E_INVALID;
    }
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

namespace {

// The spectrum launch over a planned sweep (2-D grid, or one axis when m.dim == 1):
// plane-major values[k * total + cell], flags, per-plane min / max.
int ls_run(ucb_engine* e, const ucb_ls2d_request& q, const SweepMap& m, int n_blocks, int skip, long long nt,
           ucb_ls2d_result* res) {
    std::string err;
    const bool dp5 = q.method == UCB_LS_DP5;
    if (q.method != UCB_LS_FIXED && !dp5) return fail(e, res, UCB_E_INVALID, "unknown LS method");
    if (dp5 && (m.h_axis != -1)) return fail(e, res, UCB_E_INVALID, "the DP5 method does not sweep h");
    if (dp5 && q.gs_every < 0) return fail(e, res, UCB_E_INVALID, "gs_every must be >= 0");
    if (!res->values || !res->flags) return fail(e, res, UCB_E_INVALID, "result buffers are NULL");
    if (q.cancel && *q.cancel) {
        res->cancelled = 1;
        return fail(e, res, UCB_E_CANCELLED, "Cancelled by user");
    }
    if (!ensure_init(e, err)) return fail(e, res, UCB_E_NOGPU, err);
    const int prec = q.opt.precision;
    const int nx = q.amount_of_x;
    SystemCode sys;
    CompileRequest rq = ls_compile_request(q, m, sys);
    if (dp5 && !sys.has_jvp)
        return fail(e, res, UCB_E_INVALID, "the DP5 method needs a recognised RK4 body: " + sys.note);
    TuneConfig shape;
    if (!tune_request(e, q.opt, 128, rq, shape, err)) return fail(e, res, UCB_E_INVALID, err);
    auto mod = e->modules.get(rq, err);
    if (!mod) return fail(e, res, UCB_E_COMPILE, err);
    CUfunction fn = mod->functions["ucb_ls_kernel"];

    const int n = q.n_pts;
    const long long total = m.dim == 2 ? (long long)n * n : (long long)n;
    std::vector<double> t0d, t1d;
    std::vector<float> t0f, t1f;
    axis_table(prec, n, m.lo[0], m.hi[0], m.log_axis[0], t0d, t0f);
    axis_table(prec, n, m.lo[1], m.hi[1], m.log_axis[1], t1d, t1f);
    const size_t esz = prec == UCB_PREC_F64 ? 8 : 4;
    const size_t tab_bytes = (size_t)n * esz;
    const size_t off0 = 256, off1 = 256 + ((tab_bytes + 255) / 256) * 256;
    if (!ensure_workspace(e, off1 + tab_bytes + 256, err)) return fail(e, res, UCB_E_CUDA, err);
    char* ws = static_cast<char*>(e->ws);
    cudaMemcpyAsync(ws + off0, prec == UCB_PREC_F64 ? (const void*)t0d.data() : (const void*)t0f.data(), tab_bytes,
                    cudaMemcpyHostToDevice, e->stream);
    cudaMemcpyAsync(ws + off1, prec == UCB_PREC_F64 ? (const void*)t1d.data() : (const void*)t1f.data(), tab_bytes,
                    cudaMemcpyHostToDevice, e->stream);
    cudaMemsetAsync(ws, 0, 16, e->stream);
    double* d_values = nullptr;
    int32_t* d_flags = nullptr;
    long long* d_cell_steps = nullptr;
    cudaError_t ce;
    if ((ce = dev_alloc(e, (void**)&d_values, (size_t)total * nx * 8, e->stream)) != cudaSuccess ||
        (ce = dev_alloc(e, (void**)&d_flags, (size_t)total * 4, e->stream)) != cudaSuccess ||
        (res->cell_steps &&
         (ce = dev_alloc(e, (void**)&d_cell_steps, (size_t)total * 8, e->stream)) != cudaSuccess)) {
        if (d_values) cudaFreeAsync(d_values, e->stream);
        if (d_flags) cudaFreeAsync(d_flags, e->stream);
        cudaStreamSynchronize(e->stream);
        return fail(e, res, UCB_E_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(ce));
    }

    const double rtol = q.rtol > 0 ? q.rtol : (prec == UCB_PREC_F64 ? 1e-8 : 1e-5);
    const double atol = q.atol > 0 ? q.atol : rtol;
    const double t_end = q.t_end > 0 ? q.t_end : q.t_max;
    ParamPack pk;
    pk.put<long long>(total);
    pk.put<long long>(0);
    pk.put<int>(n);
    pk.put<int>(m.swap_xy ? 1 : 0);
    pk.put<int>(n_blocks);
    pk.put<int>(q.gs_every > 0 ? q.gs_every : 10);
    pk.put<long long>(skip);
    pk.put<long long>(nt);
    pk.put<long long>(q.max_steps > 0 ? q.max_steps : 20000000LL);
    for (double v : {q.h, q.NT, q.t_max, q.eps, q.max_value, q.transient_time}) pk.put_numb(prec, v);
    pk.put<double>(rtol);
    pk.put<double>(atol);
    pk.put<double>(t_end);
    pk.put<double>(q.h0 > 0 ? q.h0 : q.h);
    for (int i = 0; i < nx; ++i) pk.put_numb(prec, q.initial_conditions[i]);
    for (int i = 0; i < std::max(q.n_values, 1); ++i) pk.put_numb(prec, i < q.n_values ? q.base_values[i] : 0.0);
    pk.put<const void*>(ws + off0);
    pk.put<const void*>(ws + off1);
    pk.put<void*>(d_values);
    pk.put<void*>(d_flags);
    pk.put<void*>(ws);
    pk.put<void*>(ws + 8);
    pk.put<void*>(d_cell_steps);
    const int block = shape.block;
    const int grid = persistent_grid(e, fn, block, total);
    begin_run(e);
    cudaEventRecord(e->ev0, e->stream);
    int rc = launch_packed(e, fn, grid, block, e->stream, pk, err) ? UCB_OK : UCB_E_CUDA;
    cudaEventRecord(e->ev1, e->stream);
    if (rc == UCB_OK) rc = wait_run(e, e->ev1, q.cancel, q.progress, total, err);
    if (rc == UCB_E_CANCELLED) res->cancelled = 1;
    unsigned long long steps = 0;
    if (rc == UCB_OK) {
        if ((ce = cudaMemcpyAsync(res->values, d_values, (size_t)total * nx * 8, cudaMemcpyDeviceToHost, e->stream)) !=
                cudaSuccess ||
            (ce = cudaMemcpyAsync(res->flags, d_flags, (size_t)total * 4, cudaMemcpyDeviceToHost, e->stream)) !=
                cudaSuccess ||
            (ce = cudaMemcpyAsync(&steps, ws + 8, 8, cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess ||
            (d_cell_steps && (ce = cudaMemcpyAsync(res->cell_steps, d_cell_steps, (size_t)total * 8,
                                                   cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess) ||
            (ce = cudaStreamSynchronize(e->stream)) != cudaSuccess) {
            rc = UCB_E_CUDA;
            err = std::string("CUDA ls2d: ") + cudaGetErrorString(ce);
        }
    }
    cudaFreeAsync(d_values, e->stream);
    cudaFreeAsync(d_flags, e->stream);
    if (d_cell_steps) cudaFreeAsync(d_cell_steps, e->stream);
    cudaStreamSynchronize(e->stream);
    if (rc != UCB_OK) return fail(e, res, rc, err);
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    res->kernel_ms = ms;
    res->steps = (long long)steps;
    if (dp5) {
        // per step attempt: 6 right-hand sides + stage combinations and error norm of the
        // state (about 56 N), and for the tangent block N x (6 J v products + 40 N)
        const double per = 6.0 * sys.flops_rhs + 56.0 * nx + nx * (6.0 * sys.flops_jvp + 40.0 * nx);
        res->flops = (double)steps * per;
    } else {
        res->flops = (double)steps * (double)sys.flops_step;
    }
    res->n_pts = n;
    res->n_exponents = nx;
    for (int k = 0; k < nx; ++k) {
        double vmin = std::numeric_limits<double>::infinity(), vmax = -vmin;
        for (long long c = 0; c < total; ++c) {
            if (res->flags[c] < 0) continue;
            const double v = res->values[(size_t)k * total + c];
            if (!std::isfinite(v)) continue;
            vmin = std::min(vmin, v);
            vmax = std::max(vmax, v);
        }
        if (!std::isfinite(vmin)) vmin = vmax = 0.0;
        if (res->min_val) res->min_val[k] = vmin;
        if (res->max_val) res->max_val[k] = vmax;
    }
    return UCB_OK;
}

}  // namespace

extern "C" int ucb_run_ls2d(ucb_engine* e, const ucb_ls2d_request* req, ucb_ls2d_result* res) {
    if (!e || !req || !res) return UCB_E_INVALID;
    const ucb_ls2d_request& q = *req;
    res->ok = res->cancelled = 0;
    res->error[0] = 0;
    res->kernel_ms = 0;
    res->steps = 0;
    res->flops = 0;
    std::string err;
    SweepMap m;
    int n_blocks = 0, skip = 0;
    long long nt = 0;
    if (!plan_sweep2d(as_lle(q), m, n_blocks, skip, nt, err)) return fail(e, res, UCB_E_INVALID, err);
    const int rc = ls_run(e, q, m, n_blocks, skip, nt, res);
    if (rc != UCB_OK) return rc;
    const int n = q.n_pts, nx = q.amount_of_x;
    if (q.csv_output_path && *q.csv_output_path) {
        const csv::Common cc = csv::common(q.base_values, q.n_values, q.initial_conditions, nx,
                                           q.opt.precision == UCB_PREC_F32);
        csv::ls2d(q.csv_output_path, cc, m.par_or_var, q.t_max, q.NT, q.transient_time, q.h, q.eps,
                  q.sweep_over_var ? q.var_sweep_index : q.param_index,
                  q.sweep_over_var_2 ? q.var_sweep_index_2 : q.param_index_2, q.param_lo, q.param_hi, q.param_lo_2,
                  q.param_hi_2, n, nx, res->values);
    }
    if (q.progress) *q.progress = 1.0f;
    res->ok = 1;
    return UCB_OK;
}

// run_ls_1d (parametric_engine.cpp:3066): the same kernel over one swept axis; spectrum
// point-major (spectrum[i][k]) with the 999 / -999 sentinels kept, flag from the first
// exponent.
extern "C" int ucb_run_ls1d(ucb_engine* e, const ucb_ls1d_request* req, ucb_ls1d_result* res) {
    if (!e || !req || !res) return UCB_E_INVALID;
    const ucb_ls1d_request& q1 = *req;
    res->ok = res->cancelled = 0;
    res->error[0] = 0;
    res->kernel_ms = 0;
    res->steps = 0;
    res->flops = 0;
    auto fail1 = [&](int code, const std::string& msg) {
        e->last_error = msg;
        std::snprintf(res->error, sizeof res->error, "%s", msg.c_str());
        return code;
    };
    std::string err;
    SweepMap m;
    int n_blocks = 0, skip = 0;
    long long nt = 0;
    if (!plan_sweep1d(q1, m, n_blocks, skip, nt, err)) return fail1(UCB_E_INVALID, err);
    if (!res->values || !res->flags) return fail1(UCB_E_INVALID, "result buffers are NULL");
    const ucb_lle2d_request l = as_lle2d(q1);
    ucb_ls2d_request q{};
    q.krs_body = l.krs_body;
    q.amount_of_x = l.amount_of_x;
    q.initial_conditions = l.initial_conditions;
    q.base_values = l.base_values;
    q.n_values = l.n_values;
    q.sweep_over_var = l.sweep_over_var;
    q.var_sweep_index = l.var_sweep_index;
    q.sweep_over_h = l.sweep_over_h;
    q.log_scale = l.log_scale;
    q.param_index = l.param_index;
    q.param_lo = l.param_lo;
    q.param_hi = l.param_hi;
    q.n_pts = l.n_pts;
    q.h = l.h;
    q.transient_time = l.transient_time;
    q.t_max = l.t_max;
    q.NT = l.NT;
    q.eps = l.eps;
    q.max_value = l.max_value;
    q.opt = l.opt;
    q.method = UCB_LS_FIXED;
    const int n = q1.n_pts, nx = q1.amount_of_x;
    std::vector<double> plane((size_t)n * nx), mn(nx), mx(nx);
    ucb_ls2d_result r2{};
    r2.values = plane.data();
    r2.flags = res->flags;
    r2.min_val = mn.data();
    r2.max_val = mx.data();
    if (q1.cancel && *q1.cancel) {
        res->cancelled = 1;
        return fail1(UCB_E_CANCELLED, "Cancelled by user");
    }
    const int rc = ls_run(e, q, m, n_blocks, skip, nt, &r2);
    if (rc != UCB_OK) {
        std::snprintf(res->error, sizeof res->error, "%s", r2.error);
        return rc;
    }
    for (int i = 0; i < n; ++i) {
        for (int k = 0; k < nx; ++k) res->values[(size_t)i * nx + k] = plane[(size_t)k * n + i];
        const double first = res->values[(size_t)i * nx];
        res->flags[i] = (first == 999.0 || first == -999.0) ? -1 : 1;
    }
    res->n_pts = n;
    res->n_exponents = nx;
    res->param_lo = q1.param_lo;
    res->param_hi = q1.param_hi;
    res->kernel_ms = r2.kernel_ms;
    res->steps = r2.steps;
    res->flops = r2.flops;
    if (q1.csv_output_path && *q1.csv_output_path) {
        const bool f32 = q1.opt.precision == UCB_PREC_F32;
        const csv::Common cc = csv::common(q1.base_values, q1.n_values, q1.initial_conditions, nx, f32);
        csv::curve1d(q1.csv_output_path, "1D LS", cc, q1.t_max, q1.NT, q1.transient_time, q1.h, q1.eps, m.idx[0],
                     csv::numb_value(q1.param_lo, f32), csv::numb_value(q1.param_hi, f32), q1.log_scale != 0, n, nx,
                     res->values);
    }
    if (q1.progress) *q1.progress = 1.0f;
    res->ok = 1;
    return UCB_OK;
}

extern "C" int ucb_autotune_ls2d(ucb_engine* e, const ucb_ls2d_request* req, int32_t force, ucb_tune_report* rep) {
    if (!e || !req || !rep) return UCB_E_INVALID;
    std::memset(rep, 0, sizeof *rep);
    std::string err;
    auto bad = [&](int code, const std::string& msg) {
        e->last_error = msg;
        std::snprintf(rep->error, sizeof rep->error, "%s", msg.c_str());
        return code;
    };
    SweepMap m;
    int n_blocks = 0, skip = 0;
    long long nt = 0;
    if (!plan_sweep2d(as_lle(*req), m, n_blocks, skip, nt, err)) return bad(UCB_E_INVALID, err);
    if (!ensure_init(e, err)) return bad(UCB_E_NOGPU, err);
    ucb_ls2d_request base = *req;
    base.opt.block_threads = base.opt.max_registers = base.opt.unroll = 0;
    base.csv_output_path = nullptr;
    base.cancel = nullptr;
    base.progress = nullptr;
    SystemCode sys;
    const std::string key = tune_key(ls_compile_request(base, m, sys));
    // trial: the same window on at most 384^2 cells, horizon scaled to about 1.2e10 steps
    // (fixed step) or the DP5 interval cut to 50 time units and 20,000 attempts per cell
    // (cells that turn stiff would otherwise run to the full attempt cap in every trial)
    ucb_ls2d_request t = base;
    t.n_pts = std::min(base.n_pts, 384);
    const int nx = base.amount_of_x;
    if (base.method == UCB_LS_DP5) {
        const double t_end = base.t_end > 0 ? base.t_end : base.t_max;
        t.t_end = std::min(t_end, 50.0);
        t.t_max = std::min(base.t_max, t.t_end);
        t.transient_time = std::min(base.transient_time, 50.0);
        t.max_steps = std::min(base.max_steps > 0 ? base.max_steps : 20000LL, 20000LL);
    } else {
        const double steps_cell = skip + (double)n_blocks * (nx + 1) * (double)(nt + 1);
        const double f = trial_scale((double)t.n_pts * t.n_pts, steps_cell);
        if (f < 1.0) {
            t.t_max = std::max(base.NT, std::floor(base.t_max * f / base.NT) * base.NT);
            t.transient_time = base.transient_time * f;
        }
    }
    SweepMap tm;
    if (!plan_sweep2d(as_lle(t), tm, n_blocks, skip, nt, err)) return bad(UCB_E_INVALID, "trial request: " + err);
    std::vector<double> vals((size_t)t.n_pts * t.n_pts * nx);
    std::vector<int32_t> flags((size_t)t.n_pts * t.n_pts);
    std::vector<double> mn(nx), mx(nx);
    auto with = [&](const TuneConfig& c) {
        ucb_ls2d_request q = t;
        q.opt.block_threads = c.block;
        q.opt.max_registers = c.maxreg;
        q.opt.unroll = c.unroll;
        return q;
    };
    auto trial = [&](const TuneConfig& c) -> double {
        ucb_ls2d_request q = with(c);
        ucb_ls2d_result r{};
        r.values = vals.data();
        r.flags = flags.data();
        r.min_val = mn.data();
        r.max_val = mx.data();
        return ucb_run_ls2d(e, &q, &r) == UCB_OK ? r.kernel_ms : -1.0;
    };
    auto build = [&](const TuneConfig& c) {
        ucb_ls2d_request q = with(c);
        SystemCode s2;
        CompileRequest rq = ls_compile_request(q, tm, s2);
        TuneConfig shape;
        std::string e2;
        tune_request(e, q.opt, 128, rq, shape, e2);
        return rq;
    };
    const int rc = autotune_search(e, key, 128, force != 0, trial, build, rep);
    rep->trial_n_pts = t.n_pts;
    return rc;
}
