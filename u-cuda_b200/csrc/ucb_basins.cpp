// Basins of attraction host orchestration: validation, axis tables, the stroboscopic
// kernel (ucb_basins.cuh), attractor table merge and label remap.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iomanip>

#include "engine_internal.h"

using namespace ucb;

namespace {

constexpr int kTableSlots = 4096;

bool validate(const ucb_basins_request& q, std::string& err) {
    if (!q.krs_body || !*q.krs_body) { err = "krs_body is empty"; return false; }
    if (q.amount_of_x <= 1 || q.amount_of_x > 32) { err = "amountOfX out of range"; return false; }
    if (!q.initial_conditions) { err = "initial_conditions.size() != amountOfX"; return false; }
    if (q.n_values > 64) { err = "too many base_values"; return false; }
    if (q.axis_x_var < 0 || q.axis_x_var >= q.amount_of_x) { err = "axis_x_var out of range"; return false; }
    if (q.axis_y_var < 0 || q.axis_y_var >= q.amount_of_x || q.axis_y_var == q.axis_x_var) {
        err = "axis_y_var out of range";
        return false;
    }
    if (q.phase_var >= q.amount_of_x || q.phase_var == q.axis_x_var || q.phase_var == q.axis_y_var) {
        err = "phase_var out of range";
        return false;
    }
    if (q.n_pts <= 0) { err = "n_pts must be > 0"; return false; }
    if (!(q.period > 0)) { err = "period must be > 0"; return false; }
    if (q.steps_per_period <= 0) { err = "steps_per_period must be > 0"; return false; }
    if (q.max_periods <= 0) { err = "max_periods must be > 0"; return false; }
    if (q.match_count <= 0) { err = "match_count must be > 0"; return false; }
    if (!(q.match_tol > 0)) { err = "match_tol must be > 0"; return false; }
    return true;
}

CompileRequest basins_compile_request(const ucb_basins_request& q, SystemCode& sys) {
    SweepMap m;
    m.dim = 2;
    m.par_or_var = 0;
    m.idx[0] = q.axis_x_var;
    m.idx[1] = q.axis_y_var;
    sys = make_system_code(q.krs_body, q.amount_of_x, q.n_values, q.opt.precision, q.opt.mode, false);
    CompileRequest rq;
    rq.name = "ucb_basins.cu";
    rq.source = make_prelude(q.opt.precision, q.amount_of_x, q.n_values, m, true, sys,
                             {"UCB_PHASE " + std::to_string(q.phase_var >= 0 ? q.phase_var : -1)}) +
                "#include \"ucb_device.cuh\"\n#include \"ucb_basins.cuh\"\n";
    rq.headers = device_headers();
    rq.options.push_back(sys.exact ? "--fmad=false" : "--fmad=true");
    rq.kernels = {"ucb_basins_kernel", "ucb_basins_remap"};
    return rq;
}

int fail(ucb_engine* e, ucb_basins_result* r, int code, const std::string& msg) {
    e->last_error = msg;
    std::snprintf(r->error, sizeof r->error, "%s", msg.c_str());
    r->ok = 0;
    return code;
}

}  // namespace

extern "C" int ucb_precompile_basins(const ucb_basins_request* req, char* err_out, int err_len) {
    std::string err;
    if (!req || !validate(*req, err)) {
        if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", err.c_str());
        return UCB_E_INVALID;
    }
    SystemCode sys;
    CompileRequest rq = basins_compile_request(*req, sys);
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

extern "C" int ucb_run_basins(ucb_engine* e, const ucb_basins_request* req, ucb_basins_result* res) {
    if (!e || !req || !res) return UCB_E_INVALID;
    const ucb_basins_request& q = *req;
    res->ok = res->cancelled = 0;
    res->error[0] = 0;
    res->kernel_ms = 0;
    res->steps = 0;
    res->flops = 0;
    res->n_attractors = 0;
    std::string err;
    if (!validate(q, err)) return fail(e, res, UCB_E_INVALID, err);
    if (!res->labels) return fail(e, res, UCB_E_INVALID, "result buffers are NULL");
    if (q.cancel && *q.cancel) {
        res->cancelled = 1;
        return fail(e, res, UCB_E_CANCELLED, "Cancelled by user");
    }
    if (!ensure_init(e, err)) return fail(e, res, UCB_E_NOGPU, err);
    SystemCode sys;
    CompileRequest rq = basins_compile_request(q, sys);
    TuneConfig shape;
    if (!tune_request(e, q.opt, 128, rq, shape, err)) return fail(e, res, UCB_E_INVALID, err);
    auto mod = e->modules.get(rq, err);
    if (!mod) return fail(e, res, UCB_E_COMPILE, err);
    CUfunction fn = mod->functions["ucb_basins_kernel"];
    CUfunction remap = mod->functions["ucb_basins_remap"];

    const int prec = q.opt.precision;
    const int n = q.n_pts;
    const long long total = (long long)n * n;
    std::vector<double> t0d, t1d;
    std::vector<float> t0f, t1f;
    axis_table(prec, n, q.axis_x_lo, q.axis_x_hi, false, t0d, t0f);
    axis_table(prec, n, q.axis_y_lo, q.axis_y_hi, false, t1d, t1f);
    const size_t esz = prec == UCB_PREC_F64 ? 8 : 4;
    const size_t tab_bytes = (size_t)n * esz;
    // workspace: [0] counter [8] steps [16] overflow | tables at 256.. | attractor table
    const size_t off0 = 256, off1 = off0 + ((tab_bytes + 255) / 256) * 256;
    const size_t off_keys = off1 + ((tab_bytes + 255) / 256) * 256;
    const size_t off_pts = off_keys + kTableSlots * 8;
    const size_t off_per = off_pts + kTableSlots * 16;
    const size_t off_map = off_per + kTableSlots * 4;
    // forcing-phase table of the native form: (cos, sin) at the 2 steps_per_period + 1
    // half-step phases of a period (ucb_basins.cuh)
    const bool use_trig = !sys.exact && sys.trig_phase >= 0 && sys.trig_phase == q.phase_var;
    const size_t trig_count = use_trig ? 2 * ((size_t)2 * q.steps_per_period + 1) : 0;
    const size_t off_trig = ((off_map + kTableSlots * 4 + 255) / 256) * 256;
    const size_t ws_need = off_trig + trig_count * esz + 256;
    if (!ensure_workspace(e, ws_need, err)) return fail(e, res, UCB_E_CUDA, err);
    char* ws = static_cast<char*>(e->ws);
    cudaStream_t st = e->stream;
    cudaMemcpyAsync(ws + off0, prec == UCB_PREC_F64 ? (const void*)t0d.data() : (const void*)t0f.data(), tab_bytes,
                    cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(ws + off1, prec == UCB_PREC_F64 ? (const void*)t1d.data() : (const void*)t1f.data(), tab_bytes,
                    cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(ws, 0, 32, st);
    cudaMemsetAsync(ws + off_keys, 0, kTableSlots * 8, st);
    std::vector<double> trig_d;
    std::vector<float> trig_f;
    if (use_trig) {
        const double half = 0.5 * (q.period / q.steps_per_period);
        const double ph0 = q.initial_conditions[q.phase_var];
        for (int m = 0; m <= 2 * q.steps_per_period; ++m) {
            const double ph = ph0 + sys.trig_rate * (m * half);
            trig_d.push_back(std::cos(ph));
            trig_d.push_back(std::sin(ph));
        }
        trig_f.assign(trig_d.begin(), trig_d.end());
        cudaMemcpyAsync(ws + off_trig, prec == UCB_PREC_F64 ? (const void*)trig_d.data() : (const void*)trig_f.data(),
                        trig_count * esz, cudaMemcpyHostToDevice, st);
    }
    int32_t *d_labels = nullptr, *d_periods = nullptr, *d_iters = nullptr;
    cudaError_t ce;
    if ((ce = dev_alloc(e, (void**)&d_labels, (size_t)total * 4, st)) != cudaSuccess ||
        (ce = dev_alloc(e, (void**)&d_periods, (size_t)total * 4, st)) != cudaSuccess ||
        (ce = dev_alloc(e, (void**)&d_iters, (size_t)total * 4, st)) != cudaSuccess)
        return fail(e, res, UCB_E_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(ce));
    const double h = q.period / q.steps_per_period;
    ParamPack pk;
    pk.put<long long>(total);
    pk.put<int>(n);
    pk.put<int>(q.steps_per_period);
    pk.put<int>(q.max_periods);
    pk.put<int>(q.match_count);
    pk.put<int>(kTableSlots);
    pk.put<int>(0);
    pk.put_numb(prec, h);
    pk.put_numb(prec, q.max_value);
    pk.put_numb(prec, prec == UCB_PREC_F32 ? std::max(q.match_tol, 1e-5) : q.match_tol);
    const double merge = q.merge_radius > 0 ? q.merge_radius : 1e-4;
    pk.put<double>(merge);
    for (int i = 0; i < q.amount_of_x; ++i) pk.put_numb(prec, q.initial_conditions[i]);
    for (int i = 0; i < std::max(q.n_values, 1); ++i) pk.put_numb(prec, i < q.n_values ? q.base_values[i] : 0.0);
    pk.put<const void*>(ws + off0);
    pk.put<const void*>(ws + off1);
    pk.put<void*>(d_labels);
    pk.put<void*>(d_periods);
    pk.put<void*>(d_iters);
    pk.put<void*>(ws + off_keys);
    pk.put<void*>(ws + off_pts);
    pk.put<void*>(ws + off_per);
    pk.put<void*>(ws + 16);
    pk.put<void*>(ws);
    pk.put<void*>(ws + 8);
    pk.put<const void*>(use_trig ? (const void*)(ws + off_trig) : nullptr);
    const int block = shape.block;
    begin_run(e);
    cudaEventRecord(e->ev0, st);
    int rc = launch_packed(e, fn, persistent_grid(e, fn, block, total), block, st, pk, err) ? UCB_OK : UCB_E_CUDA;
    if (rc == UCB_OK) {
        cudaEventRecord(e->ev1, st);
        rc = wait_run(e, e->ev1, q.cancel, q.progress, total, err);
        if (rc == UCB_E_CANCELLED) res->cancelled = 1;
    }
    // attractor table -> host: merge, order, map
    std::vector<unsigned long long> keys(kTableSlots);
    std::vector<double> pts(2 * kTableSlots);
    std::vector<int> per(kTableSlots);
    int overflow = 0;
    unsigned long long steps = 0;
    if (rc == UCB_OK) {
        if ((ce = cudaMemcpyAsync(keys.data(), ws + off_keys, kTableSlots * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (ce = cudaMemcpyAsync(pts.data(), ws + off_pts, kTableSlots * 16, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (ce = cudaMemcpyAsync(per.data(), ws + off_per, kTableSlots * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (ce = cudaMemcpyAsync(&overflow, ws + 16, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (ce = cudaMemcpyAsync(&steps, ws + 8, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (ce = cudaStreamSynchronize(st)) != cudaSuccess) {
            rc = UCB_E_CUDA;
            err = std::string("CUDA basins: ") + cudaGetErrorString(ce);
        }
    }
    std::vector<int> map(kTableSlots, 0);
    if (rc == UCB_OK) {
        struct Entry { int slot, period; double x, y; };
        std::vector<Entry> ents;
        for (int s = 0; s < kTableSlots; ++s)
            if (keys[s]) ents.push_back({s, per[s], pts[2 * s], pts[2 * s + 1]});
        std::sort(ents.begin(), ents.end(), [](const Entry& a, const Entry& b) {
            if (a.period != b.period) return a.period < b.period;
            if (a.x != b.x) return a.x < b.x;
            return a.y < b.y;
        });
        // greedy merge: an entry joins the first earlier representative within the radius
        std::vector<int> rep_idx;
        for (size_t i = 0; i < ents.size(); ++i) {
            int joined = -1;
            for (size_t r = 0; r < rep_idx.size(); ++r) {
                const Entry& R = ents[rep_idx[r]];
                if (R.period == ents[i].period && std::fabs(R.x - ents[i].x) <= merge &&
                    std::fabs(R.y - ents[i].y) <= merge) {
                    joined = (int)r;
                    break;
                }
            }
            if (joined < 0) {
                rep_idx.push_back((int)i);
                joined = (int)rep_idx.size() - 1;
            }
            map[ents[i].slot] = joined + 1;
        }
        res->n_attractors = (int)rep_idx.size();
        for (size_t r = 0; r < rep_idx.size() && r < UCB_BASINS_MAX_ATTRACTORS; ++r) {
            res->attractor_period[r] = ents[rep_idx[r]].period;
            res->attractor_point[r][0] = ents[rep_idx[r]].x;
            res->attractor_point[r][1] = ents[rep_idx[r]].y;
        }
        cudaMemcpyAsync(ws + off_map, map.data(), kTableSlots * 4, cudaMemcpyHostToDevice, st);
        void* args[] = {&d_labels, (void*)&total, nullptr};
        int32_t* dmap = reinterpret_cast<int32_t*>(ws + off_map);
        args[2] = &dmap;
        CUresult r = driver().cuLaunchKernel(remap, (unsigned)std::min<long long>((total + 255) / 256, 4096), 1, 1,
                                             256, 1, 1, 0, (CUstream)st, args, nullptr);
        if (r != CUDA_SUCCESS) {
            rc = UCB_E_CUDA;
            err = "cuLaunchKernel(remap): " + cu_error_string(r);
        } else {
            e->launches += 1;
        }
    }
    cudaEventRecord(e->ev1, st);
    if (rc == UCB_OK) {
        if ((ce = cudaMemcpyAsync(res->labels, d_labels, (size_t)total * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (res->periods &&
             (ce = cudaMemcpyAsync(res->periods, d_periods, (size_t)total * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) ||
            (res->iterations &&
             (ce = cudaMemcpyAsync(res->iterations, d_iters, (size_t)total * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) ||
            (ce = cudaStreamSynchronize(st)) != cudaSuccess) {
            rc = UCB_E_CUDA;
            err = std::string("CUDA basins: ") + cudaGetErrorString(ce);
        }
    }
    cudaFreeAsync(d_labels, st);
    cudaFreeAsync(d_periods, st);
    cudaFreeAsync(d_iters, st);
    cudaStreamSynchronize(st);
    if (rc != UCB_OK) return fail(e, res, rc, err);
    if (overflow) return fail(e, res, UCB_E_INVALID, "attractor table overflow (more than 4096 distinct keys)");
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    res->kernel_ms = ms;
    res->steps = (long long)steps;
    res->flops = (double)steps * sys.flops_step;
    res->n_pts = n;
    if (q.csv_output_path && *q.csv_output_path) {
        std::ofstream out(q.csv_output_path);
        for (int iy = 0; iy < n; ++iy) {
            for (int ix = 0; ix < n; ++ix) {
                out << res->labels[(size_t)iy * n + ix];
                if (ix + 1 < n) out << ", ";
            }
            out << '\n';
        }
    }
    if (q.progress) *q.progress = 1.0f;
    res->ok = 1;
    return UCB_OK;
}

extern "C" int ucb_autotune_basins(ucb_engine* e, const ucb_basins_request* req, int32_t force, ucb_tune_report* rep) {
    if (!e || !req || !rep) return UCB_E_INVALID;
    std::memset(rep, 0, sizeof *rep);
    std::string err;
    auto bad = [&](int code, const std::string& msg) {
        e->last_error = msg;
        std::snprintf(rep->error, sizeof rep->error, "%s", msg.c_str());
        return code;
    };
    if (!validate(*req, err)) return bad(UCB_E_INVALID, err);
    if (!ensure_init(e, err)) return bad(UCB_E_NOGPU, err);
    ucb_basins_request base = *req;
    base.opt.block_threads = base.opt.max_registers = base.opt.unroll = 0;
    base.csv_output_path = nullptr;
    base.cancel = nullptr;
    base.progress = nullptr;
    SystemCode sys;
    const std::string key = tune_key(basins_compile_request(base, sys));
    // trial: the same window on at most 768^2 cells; the period cap scaled to about 1.2e10
    // steps in all (at least 3 x match_count periods, so that converging cells still exit)
    ucb_basins_request t = base;
    t.n_pts = std::min(base.n_pts, 768);
    const double f = trial_scale((double)t.n_pts * t.n_pts, (double)base.max_periods * base.steps_per_period);
    if (f < 1.0)
        t.max_periods = std::min(base.max_periods, std::max(3 * base.match_count, (int)(base.max_periods * f)));
    const size_t cells = (size_t)t.n_pts * t.n_pts;
    std::vector<int32_t> labels(cells), periods(cells), iters(cells);
    auto with = [&](const TuneConfig& c) {
        ucb_basins_request q = t;
        q.opt.block_threads = c.block;
        q.opt.max_registers = c.maxreg;
        q.opt.unroll = c.unroll;
        return q;
    };
    auto trial = [&](const TuneConfig& c) -> double {
        ucb_basins_request q = with(c);
        ucb_basins_result r{};
        r.labels = labels.data();
        r.periods = periods.data();
        r.iterations = iters.data();
        return ucb_run_basins(e, &q, &r) == UCB_OK ? r.kernel_ms : -1.0;
    };
    auto build = [&](const TuneConfig& c) {
        ucb_basins_request q = with(c);
        SystemCode s2;
        CompileRequest rq = basins_compile_request(q, s2);
        TuneConfig shape;
        std::string e2;
        tune_request(e, q.opt, 128, rq, shape, e2);
        return rq;
    };
    const int rc = autotune_search(e, key, 128, force != 0, trial, build, rep);
    rep->trial_n_pts = t.n_pts;
    return rc;
}
