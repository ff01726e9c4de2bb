// C-ABI engine: initialisation, system code generation, LLE-2D orchestration.
//
// Host orchestration follows ParametricEngine::Impl::run_lle_2d
// (parametric_engine.cpp:2587-2965): the same validation messages' conditions, the same
// mapping of user sweep axes to the kernel's par_or_var / swap_xy, the same host-side
// step counts ((int)(tMax/NT), (int)(transient/h)) and the same result conventions.
// What differs is the device side: one persistent sm_100a kernel over all cells (the
// reference chunks by free memory and launches 32-thread blocks with state in shared
// memory), per-axis value tables instead of per-thread index arithmetic, and the
// transpose folded into the kernel's store.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <chrono>
#include <thread>
#include <fstream>
#include <iomanip>
#include <limits>
#include <sstream>

#include "csv_export.h"
#include "engine_internal.h"

namespace ucb {

namespace {

constexpr int kMaxAmountOfX = 32;       // parametric_engine.cpp:30
constexpr int kMaxAmountOfValues = 64;  // parametric_engine.cpp:31

void set_error(char* dst, const std::string& msg) {
    std::snprintf(dst, 1024, "%s", msg.c_str());
}

}  // namespace

bool ensure_init(ucb_engine* e, std::string& err) {
    if (e->initialized) {
        cudaSetDevice(e->device);
        return true;
    }
    Driver& d = driver();
    if (!d.loaded) {
        err = d.load_error;
        return false;
    }
    int n = 0;
    cudaError_t ce = cudaGetDeviceCount(&n);
    if (ce != cudaSuccess || n <= e->device) {
        err = std::string("no CUDA device ") + std::to_string(e->device) + ": " +
              (ce != cudaSuccess ? cudaGetErrorString(ce) : "device index out of range");
        return false;
    }
    if ((ce = cudaSetDevice(e->device)) != cudaSuccess || (ce = cudaFree(nullptr)) != cudaSuccess) {
        err = std::string("cudaSetDevice: ") + cudaGetErrorString(ce);
        return false;
    }
    d.cuInit(0);
    cudaDeviceGetAttribute(&e->sm_count, cudaDevAttrMultiProcessorCount, e->device);
    {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = e->device;
        if (cudaMemPoolCreate(&e->pool, &props) == cudaSuccess) {
            unsigned long long keep = ~0ULL;
            cudaMemPoolSetAttribute(e->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        } else {
            e->pool = nullptr;  // the device's default pool then
            cudaGetLastError();
        }
    }
    if ((ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (ce = cudaEventCreate(&e->ev0)) != cudaSuccess || (ce = cudaEventCreate(&e->ev1)) != cudaSuccess) {
        err = std::string("stream/event creation: ") + cudaGetErrorString(ce);
        return false;
    }
    {
        // run control: cancel word and queue position shared with the kernels
        void* h = nullptr;
        void* dptr = nullptr;
        if (cudaHostAlloc(&h, sizeof(ucb_run_control), cudaHostAllocMapped) == cudaSuccess &&
            cudaHostGetDevicePointer(&dptr, h, 0) == cudaSuccess) {
            std::memset(h, 0, sizeof(ucb_run_control));
            e->control = static_cast<ucb_run_control*>(h);
            e->modules.set_control(dptr);
        } else {
            if (h) cudaFreeHost(h);
            cudaGetLastError();
        }
    }
    e->initialized = true;
    return true;
}

void begin_run(ucb_engine* e) {
    if (e->control) e->control->fetched = 0;
}

int wait_run(ucb_engine* e, cudaEvent_t done, const volatile int32_t* cancel, volatile float* progress,
             long long work_items, std::string& err) {
    ucb_run_control* c = e->control;
    cudaError_t ce;
    if (!c || (!cancel && !progress)) {
        if ((ce = cudaEventSynchronize(done)) != cudaSuccess) {
            err = std::string("CUDA: ") + cudaGetErrorString(ce);
            return UCB_E_CUDA;
        }
        return UCB_OK;
    }
    bool cancelled = false;
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        ce = cudaEventQuery(done);
        if (ce == cudaSuccess) break;
        if (ce != cudaErrorNotReady) {
            err = std::string("CUDA: ") + cudaGetErrorString(ce);
            if (cancelled) c->cancel = 0;
            return UCB_E_CUDA;
        }
        if (cancel && *cancel && !cancelled) {
            c->cancel = 1;
            cancelled = true;
        }
        if (progress && work_items > 0) {
            const double f = (double)c->fetched / (double)work_items;
            *progress = (float)std::min(f, 0.999);
        }
        if (std::chrono::steady_clock::now() - t0 < std::chrono::milliseconds(2))
            std::this_thread::yield();
        else
            std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
    if (cancelled) {
        c->cancel = 0;
        err = "Cancelled by user";
        return UCB_E_CANCELLED;
    }
    return UCB_OK;
}

bool ensure_workspace(ucb_engine* e, size_t bytes, std::string& err) {
    if (e->ws_bytes >= bytes) return true;
    if (e->ws) {
        cudaStreamSynchronize(e->stream);
        cudaDeviceSynchronize();
        cudaFree(e->ws);
        e->ws = nullptr;
        e->ws_bytes = 0;
    }
    size_t want = std::max<size_t>(bytes, 1 << 20);
    cudaError_t ce = cudaMalloc(&e->ws, want);
    if (ce != cudaSuccess) {
        err = std::string("cudaMalloc workspace: ") + cudaGetErrorString(ce);
        return false;
    }
    e->ws_bytes = want;
    return true;
}

template <class T>
static T value_by_idx_t(long long idx, int nPts, T lo, T hi) {
    if (nPts <= 0) return lo;
    if (nPts == 1) return hi;
    const long long pointIdx = idx % nPts;
    const T t = static_cast<T>(pointIdx) / static_cast<T>(nPts - 1);
    return (static_cast<T>(1.0) - t) * lo + t * hi;
}

template <class T>
static T value_by_idx_log_t(long long idx, int nPts, T lo, T hi) {
    const T l = std::log10(lo) + (T)(((long long)((long long)idx / std::pow((T)nPts, (T)0)) % nPts) *
                                     ((T)(std::log10(hi) - std::log10(lo)) / (T)(nPts - 1)));
    return std::pow((T)10.0, l);
}

void axis_table(int precision, int n, double lo, double hi, bool log_scale, std::vector<double>& out_d,
                std::vector<float>& out_f) {
    out_d.clear();
    out_f.clear();
    for (int i = 0; i < n; ++i) {
        if (precision == UCB_PREC_F64) {
            out_d.push_back(log_scale ? value_by_idx_log_t<double>(i, n, lo, hi) : value_by_idx_t<double>(i, n, lo, hi));
        } else {
            const float l = (float)lo, h = (float)hi;
            out_f.push_back(log_scale ? value_by_idx_log_t<float>(i, n, l, h) : value_by_idx_t<float>(i, n, l, h));
        }
    }
}

std::string make_prelude(int precision, int nx, int nv, const SweepMap& m, bool extra_step,
                         const SystemCode& sys, const std::vector<std::string>& extra_defines) {
    std::ostringstream o;
    o << "// generated prelude\n";
    o << "#define UCB_NX " << nx << "\n";
    o << "#define UCB_NV " << std::max(nv, 1) << "\n";
    o << "#define UCB_DIM " << m.dim << "\n";
    o << "#define UCB_POV " << m.par_or_var << "\n";
    o << "#define UCB_IDX0 " << m.idx[0] << "\n";
    o << "#define UCB_IDX1 " << m.idx[1] << "\n";
    o << "#define UCB_HAXIS " << m.h_axis << "\n";
    o << "#define UCB_EXTRA_STEP " << (extra_step ? 1 : 0) << "\n";
    o << "#define AMOUNTOFX " << nx << "\n";
    if (sys.exact) o << "#define UCB_EXACT 1\n";
    if (sys.has_jvp) o << "#define UCB_HAS_JVP 1\n";
    for (auto& d : extra_defines) o << "#define " << d << "\n";
    o << "typedef " << (precision == UCB_PREC_F64 ? "double" : "float") << " numb;\n";
    if (precision != UCB_PREC_F64) o << "#define UCB_NUMB_F32 1\n";
    // configCUDA.h pi / euler, visible to step bodies as in the reference template.
    o << "constexpr numb pi = (numb)3.1415926535897932384626433832795;\n";
    o << "constexpr numb euler = (numb)2.7182818284590452353602874713527;\n";
    o << sys.code << "\n";
    return o.str();
}

std::vector<std::string> clock_defines(const SystemCode& sys) {
    if (sys.exact || sys.clock_var < 0) return {};
    return {"UCB_KAHAN_CLOCK 1"};
}

SystemCode make_system_code(const std::string& krs_body, int nx, int nv, int precision, int mode,
                            bool want_jvp) {
    SystemCode s;
    if (mode == UCB_MODE_NATIVE) {
        fe::Rhs r;
        std::string why;
        bool ok = false;
        try {
            ok = fe::recognize_rk4(krs_body, nx, r, why);
        } catch (const std::exception& ex) {
            ok = false;
            why = ex.what();
        }
        if (ok) {
            s.exact = false;
            s.code = fe::emit_rhs_device(r, precision == UCB_PREC_F32);
            s.flops_step = fe::rk4_step_flops(r);
            s.flops_rhs = fe::rhs_flops(r);
            for (auto& f : r.f) s.flops_jvp += fe::flops(fe::directional_derivative(f));
            if (want_jvp) {
                s.code += fe::emit_jvp_device(r, precision == UCB_PREC_F32);
                s.has_jvp = true;
                s.flops_step = fe::rk4_tangent_step_flops(r) / 2;  // per trajectory-step
                if (precision == UCB_PREC_F32) {
                    try {
                        s.code += fe::emit_packed_device(r);
                        s.has_packed = true;
                    } catch (const std::exception&) {
                        s.has_packed = false;  // a call the packed form does not cover
                    }
                }
            }
            int p = -1;
            double rate = 0;
            if (precision == UCB_PREC_F32 && fe::find_clock(r, p, rate)) {
                char rbuf[64];
                std::snprintf(rbuf, sizeof rbuf, "%.17g", rate);
                s.code += "#define UCB_CLOCK_VAR " + std::to_string(p) + "\n#define UCB_CLOCK_RATE " + rbuf + "\n";
                s.clock_var = p;
                s.clock_rate = rate;
            }
            if (fe::find_trig_phase(r, p, rate)) {
                s.flops_step = s.has_jvp ? fe::rk4_tangent_step_flops(r, p) / 2 : fe::rk4_step_flops(r, p);
                s.code += fe::emit_rhs_trig_device(r, p, precision == UCB_PREC_F32);
                char rbuf[64];
                std::snprintf(rbuf, sizeof rbuf, "%.17g", rate);
                s.code += "#define UCB_TRIG_PHASE " + std::to_string(p) + "\n#define UCB_TRIG_RATE " + rbuf + "\n";
                s.trig_phase = p;
                s.trig_rate = rate;
            }
            return s;
        }
        s.note = "native form unavailable (" + why + "); using the exact form";
    }
    (void)nv;
    {
        // Algorithmic FLOPs of the exact form: the same RK4 count when the body is the
        // template, unknown (0) for other bodies.
        fe::Rhs r;
        std::string why;
        try {
            if (fe::recognize_rk4(krs_body, nx, r, why)) s.flops_step = fe::rk4_step_flops(r);
        } catch (...) {
        }
    }
    std::ostringstream o;
    o << "__device__ __forceinline__ void calculateDiscreteModel(numb* X, const numb* a, const numb h) {\n"
      << krs_body << "\n}\n";
    s.exact = true;
    s.code = o.str();
    return s;
}

bool launch_packed(ucb_engine* e, CUfunction f, int grid, int block, cudaStream_t stream, ParamPack& pk,
                   std::string& err) {
    pk.finish();
    size_t psize = pk.buf.size();
    void* cfg[] = {CU_LAUNCH_PARAM_BUFFER_POINTER, pk.buf.data(), CU_LAUNCH_PARAM_BUFFER_SIZE, &psize,
                   CU_LAUNCH_PARAM_END};
    CUresult r = driver().cuLaunchKernel(f, grid, 1, 1, block, 1, 1, 0, (CUstream)stream, nullptr, cfg);
    if (r != CUDA_SUCCESS) {
        err = "cuLaunchKernel: " + cu_error_string(r);
        return false;
    }
    e->launches += 1;
    return true;
}

int persistent_grid(ucb_engine* e, CUfunction f, int block, long long work_items) {
    int per_sm = 1;
    if (driver().cuOccupancyMaxActiveBlocksPerMultiprocessor)
        driver().cuOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, block, 0);
    if (per_sm < 1) per_sm = 1;
    const long long warps = (work_items + 31) / 32;
    const long long blocks_needed = (warps * 32 + block - 1) / block;
    long long g = (long long)e->sm_count * per_sm;
    if (g > blocks_needed) g = blocks_needed;
    if (g < 1) g = 1;
    return (int)g;
}

// ------------------------------------------------------------------------------------
// LLE 2D
// ------------------------------------------------------------------------------------
namespace {

struct LlePlan {
    SweepMap map;
    int amountOfPointsInBlock = 0;
    int amountOfPointsForSkip = 0;
    long long nt_steps = 0;
};

// Validation and axis mapping of run_lle_2d (parametric_engine.cpp:2591-2703).
bool plan_lle2d(const ucb_lle2d_request& q, LlePlan& p, std::string& err) {
    if (!q.krs_body || !*q.krs_body) { err = "krs_body is empty"; return false; }
    if (q.amount_of_x <= 0 || q.amount_of_x > kMaxAmountOfX) { err = "amountOfX out of range"; return false; }
    if (!q.initial_conditions) { err = "initial_conditions.size() != amountOfX"; return false; }
    if (q.n_values > kMaxAmountOfValues) { err = "too many base_values"; return false; }
    if (q.n_values > 0 && !q.base_values) { err = "base_values is NULL"; return false; }
    if (q.n_pts <= 0) { err = "n_pts must be > 0"; return false; }
    if (!(q.h > 0.0)) { err = "h must be > 0"; return false; }
    if (!(q.t_max > 0.0)) { err = "t_max must be > 0"; return false; }
    if (q.transient_time < 0) { err = "transient_time must be >= 0"; return false; }
    if (!(q.NT > 0.0)) { err = "NT must be > 0"; return false; }
    if (!(q.eps > 0.0)) { err = "eps must be > 0"; return false; }
    auto check_param = [&](int p1) { return p1 > 0 && p1 < q.n_values; };
    auto check_var = [&](int v0) { return v0 >= 0 && v0 < q.amount_of_x; };
    SweepMap& m = p.map;
    m.dim = 2;
    bool log_x = q.log_scale, log_y = q.log_scale_2;
    if (q.log_scale && !(q.param_lo > 0.0 && q.param_hi > 0.0)) { err = "log scale requires param lo/hi > 0 (axis X)"; return false; }
    if (q.log_scale_2 && !(q.param_lo_2 > 0.0 && q.param_hi_2 > 0.0)) { err = "log scale requires param lo/hi > 0 (axis Y)"; return false; }
    if (q.sweep_over_h && q.sweep_over_h_2) { err = "sweep_over_h and sweep_over_h_2 cannot both be true"; return false; }
    if (q.sweep_over_h || q.sweep_over_h_2) {
        m.h_axis = q.sweep_over_h ? 0 : 1;
        const bool other_is_var = q.sweep_over_h ? q.sweep_over_var_2 : q.sweep_over_var;
        m.par_or_var = other_is_var ? 0 : 1;
        if (q.sweep_over_h) {
            if (m.par_or_var == 1) {
                if (!check_param(q.param_index_2)) { err = "param_index_2 (axis Y) out of range"; return false; }
                m.idx[1] = q.param_index_2;
            } else {
                if (!check_var(q.var_sweep_index_2)) { err = "var_sweep_index_2 (axis Y) out of range"; return false; }
                m.idx[1] = q.var_sweep_index_2;
            }
            m.idx[0] = 0;
        } else {
            if (m.par_or_var == 1) {
                if (!check_param(q.param_index)) { err = "param_index (axis X) out of range"; return false; }
                m.idx[0] = q.param_index;
            } else {
                if (!check_var(q.var_sweep_index)) { err = "var_sweep_index (axis X) out of range"; return false; }
                m.idx[0] = q.var_sweep_index;
            }
            m.idx[1] = 0;
        }
        m.lo[0] = q.param_lo; m.hi[0] = q.param_hi; m.lo[1] = q.param_lo_2; m.hi[1] = q.param_hi_2;
    } else if ((q.sweep_over_var != 0) == (q.sweep_over_var_2 != 0)) {
        m.par_or_var = q.sweep_over_var ? 0 : 1;
        if (m.par_or_var == 1) {
            if (!check_param(q.param_index)) { err = "param_index (axis X) out of range"; return false; }
            if (!check_param(q.param_index_2)) { err = "param_index_2 (axis Y) out of range"; return false; }
            m.idx[0] = q.param_index; m.idx[1] = q.param_index_2;
        } else {
            if (!check_var(q.var_sweep_index)) { err = "var_sweep_index (axis X) out of range"; return false; }
            if (!check_var(q.var_sweep_index_2)) { err = "var_sweep_index_2 (axis Y) out of range"; return false; }
            m.idx[0] = q.var_sweep_index; m.idx[1] = q.var_sweep_index_2;
        }
        m.lo[0] = q.param_lo; m.hi[0] = q.param_hi; m.lo[1] = q.param_lo_2; m.hi[1] = q.param_hi_2;
    } else if (q.sweep_over_var && !q.sweep_over_var_2) {
        m.par_or_var = 2;
        if (!check_var(q.var_sweep_index)) { err = "var_sweep_index (axis X) out of range"; return false; }
        if (!check_param(q.param_index_2)) { err = "param_index_2 (axis Y) out of range"; return false; }
        m.idx[0] = q.var_sweep_index; m.idx[1] = q.param_index_2;
        m.lo[0] = q.param_lo; m.hi[0] = q.param_hi; m.lo[1] = q.param_lo_2; m.hi[1] = q.param_hi_2;
    } else {
        m.par_or_var = 2;
        if (!check_var(q.var_sweep_index_2)) { err = "var_sweep_index_2 (axis Y) out of range"; return false; }
        if (!check_param(q.param_index)) { err = "param_index (axis X) out of range"; return false; }
        m.idx[0] = q.var_sweep_index_2; m.idx[1] = q.param_index;
        m.lo[0] = q.param_lo_2; m.hi[0] = q.param_hi_2; m.lo[1] = q.param_lo; m.hi[1] = q.param_hi;
        m.swap_xy = true;
        log_x = q.log_scale_2; log_y = q.log_scale;
    }
    m.log_axis[0] = log_x;
    m.log_axis[1] = log_y;
    p.amountOfPointsInBlock = (int)(q.t_max / q.NT);
    p.amountOfPointsForSkip = (int)(q.transient_time / q.h);
    if (p.amountOfPointsInBlock <= 0) { err = "computed amountOfPointsInBlock <= 0 (t_max / NT too small)"; return false; }
    // (size_t)(NT / h) is evaluated in numb inside the reference kernel (cudaLibrary.cu:2547);
    // in float it truncates 0.02f / 0.002f to 9. The exact form keeps that; the native FP32
    // form counts in double so that its blocks span the same time as the FP64 plain form.
    if (q.opt.precision == UCB_PREC_F64 || q.opt.mode == UCB_MODE_NATIVE)
        p.nt_steps = (long long)(q.NT / q.h);
    else
        p.nt_steps = (long long)((float)q.NT / (float)q.h);
    return true;
}

template <class T>
struct LleParamsT {
    long long total;
    long long cell_offset;
    int n_pts;
    int swap_xy;
    int n_blocks;
    int pad0;
    long long skip;
    long long nt_steps;
    T h, NT, tmax, eps, maxv, transient;
};

// Packs UcbLleParams (ucb_lle.cuh) for numb = T and the compile-time NX / NV sizes.
template <class T>
std::vector<char> pack_lle_params(const LleParamsT<T>& head, const double* ic, int nx, const double* vals, int nv,
                                  const void* ax0, const void* ax1, double* out_v, int32_t* out_f, void* counter,
                                  void* steps, const void* cell_list = nullptr, int list_compact = 0) {
    std::vector<char> buf;
    auto put = [&](const void* p, size_t n, size_t align) {
        while (buf.size() % align) buf.push_back(0);
        const char* c = static_cast<const char*>(p);
        buf.insert(buf.end(), c, c + n);
    };
    put(&head.total, 8, 8);
    put(&head.cell_offset, 8, 8);
    put(&head.n_pts, 4, 4);
    put(&head.swap_xy, 4, 4);
    put(&head.n_blocks, 4, 4);
    put(&head.pad0, 4, 4);
    put(&head.skip, 8, 8);
    put(&head.nt_steps, 8, 8);
    const T sc[6] = {head.h, head.NT, head.tmax, head.eps, head.maxv, head.transient};
    for (int i = 0; i < 6; ++i) put(&sc[i], sizeof(T), sizeof(T));
    for (int i = 0; i < nx; ++i) { T v = (T)ic[i]; put(&v, sizeof(T), sizeof(T)); }
    const int nvp = std::max(nv, 1);
    for (int i = 0; i < nvp; ++i) { T v = (i < nv) ? (T)vals[i] : (T)0; put(&v, sizeof(T), sizeof(T)); }
    put(&ax0, 8, 8);
    put(&ax1, 8, 8);
    put(&out_v, 8, 8);
    put(&out_f, 8, 8);
    put(&counter, 8, 8);
    put(&steps, 8, 8);
    put(&cell_list, 8, 8);
    put(&list_compact, 4, 4);
    while (buf.size() % 8) buf.push_back(0);
    return buf;
}

struct LleLaunch {
    std::shared_ptr<Module> mod;
    CUfunction fn = nullptr;
    SystemCode sys;
    bool tangent = false;
    TuneConfig shape;  // launch shape (block size used by the launch)
};

CompileRequest lle_compile_request(const ucb_lle2d_request& q, const LlePlan& plan, LleLaunch& L) {
    const int prec = q.opt.precision;
    bool tangent = false;
    if (q.opt.lle_method == UCB_LLE_TANGENT) tangent = true;
    else if (q.opt.lle_method == UCB_LLE_AUTO) tangent = (prec == UCB_PREC_F32);
    L.sys = make_system_code(q.krs_body, q.amount_of_x, q.n_values, prec, q.opt.mode, tangent);
    if (tangent && !L.sys.has_jvp) tangent = false;  // tangent needs a recognised right-hand side
    L.tangent = tangent;
    std::vector<std::string> defs;
    if (tangent) defs.push_back("UCB_TANGENT 1");
    // The tangent form steps one trajectory per cell (the shadow form two, on one Stepper)
    if (tangent)
        for (auto& d : clock_defines(L.sys)) defs.push_back(d);
    // Two cells per thread in packed FP32 pairs (on request): FP32 tangent form with a
    // uniform step and a compile-time block length, for systems without a clock (the pair
    // step has no compensated clock).
    if (tangent && prec == UCB_PREC_F32 && L.sys.has_packed && plan.map.h_axis == -1 && plan.nt_steps >= 1 &&
        plan.nt_steps <= 100 && q.opt.paired_cells && L.sys.clock_var < 0)
        defs.push_back("UCB_PACKED 1");
    // Block length known at compile time (no h sweep): the block loop unrolls fully.
    if (plan.map.h_axis == -1 && plan.nt_steps >= 1 && plan.nt_steps <= 100)
        defs.push_back("UCB_NT " + std::to_string(plan.nt_steps));
    CompileRequest rq;
    rq.name = "ucb_lle2d.cu";
    rq.source = make_prelude(prec, q.amount_of_x, q.n_values, plan.map, q.opt.nominal_steps == 0, L.sys, defs) +
                "#include \"ucb_device.cuh\"\n#include \"ucb_lle.cuh\"\n";
    rq.headers = device_headers();
    rq.options.push_back(L.sys.exact ? "--fmad=false" : "--fmad=true");
    rq.kernels = {"ucb_lle_kernel", "ucb_state_kernel"};
    return rq;
}

// The compile request with the launch shape of this run applied (e may be null: explicit
// options only).
bool lle_tuned_request(ucb_engine* e, const ucb_lle2d_request& q, const LlePlan& plan, LleLaunch& L,
                       CompileRequest& rq, std::string& err) {
    rq = lle_compile_request(q, plan, L);
    return tune_request(e, q.opt, 128, rq, L.shape, err);
}

bool prepare_lle(ucb_engine* e, const ucb_lle2d_request& q, const LlePlan& plan, LleLaunch& L, std::string& err) {
    CompileRequest rq;
    if (!lle_tuned_request(e, q, plan, L, rq, err)) return false;
    L.mod = e->modules.get(rq, err);
    if (!L.mod) return false;
    L.fn = L.mod->functions["ucb_lle_kernel"];
    return true;
}

// Enqueues the LLE kernel. Workspace layout: [0] work counter, [8] step counter,
// [256..] axis tables.
int enqueue_lle_fn(ucb_engine* e, const ucb_lle2d_request& q, const LlePlan& plan, const LleLaunch& L,
                   double* d_values, int32_t* d_flags, cudaStream_t stream, std::string& err, long long skip_override,
                   bool persistent, char* scratch, const long long* d_cell_list = nullptr, long long n_list = 0,
                   bool list_compact = false, TableUpload upload = nullptr) {
    const int n = q.n_pts;
    const int prec = q.opt.precision;
    const size_t esz = prec == UCB_PREC_F64 ? 8 : 4;
    const size_t tab_bytes = (size_t)n * esz;
    const size_t off_ax0 = 256, off_ax1 = 256 + ((tab_bytes + 255) / 256) * 256;
    char* ws = scratch;
    if (!ws) {
        if (!ensure_workspace(e, off_ax1 + tab_bytes + 256, err)) return UCB_E_CUDA;
        ws = static_cast<char*>(e->ws);
    }
    std::vector<double> t0d, t1d;
    std::vector<float> t0f, t1f;
    axis_table(prec, n, plan.map.lo[0], plan.map.hi[0], plan.map.log_axis[0], t0d, t0f);
    axis_table(prec, n, plan.map.lo[1], plan.map.hi[1], plan.map.log_axis[1], t1d, t1f);
    const void* h0 = prec == UCB_PREC_F64 ? (const void*)t0d.data() : (const void*)t0f.data();
    const void* h1 = prec == UCB_PREC_F64 ? (const void*)t1d.data() : (const void*)t1f.data();
    cudaError_t ce;
    if (upload) {
        if (upload(ws + off_ax0, h0, tab_bytes, stream, err) != UCB_OK ||
            upload(ws + off_ax1, h1, tab_bytes, stream, err) != UCB_OK)
            return UCB_E_CUDA;
        if ((ce = cudaMemsetAsync(ws, 0, 16, stream)) != cudaSuccess) {
            err = std::string("CUDA upload: ") + cudaGetErrorString(ce);
            return UCB_E_CUDA;
        }
    } else if ((ce = cudaMemcpyAsync(ws + off_ax0, h0, tab_bytes, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
               (ce = cudaMemcpyAsync(ws + off_ax1, h1, tab_bytes, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
               (ce = cudaMemsetAsync(ws, 0, 16, stream)) != cudaSuccess) {
        err = std::string("CUDA upload: ") + cudaGetErrorString(ce);
        return UCB_E_CUDA;
    }
    const long long total = d_cell_list ? n_list : (plan.map.dim == 2 ? (long long)n * n : (long long)n);
    std::vector<char> params;
    if (prec == UCB_PREC_F64) {
        LleParamsT<double> hd{total, 0, n, plan.map.swap_xy ? 1 : 0, plan.amountOfPointsInBlock, 0,
                              skip_override >= 0 ? skip_override : plan.amountOfPointsForSkip, plan.nt_steps, q.h,
                              q.NT, q.t_max, q.eps, q.max_value, q.transient_time};
        params = pack_lle_params<double>(hd, q.initial_conditions, q.amount_of_x, q.base_values, q.n_values,
                                         ws + off_ax0, ws + off_ax1, d_values, d_flags, ws, ws + 8, d_cell_list,
                                         list_compact ? 1 : 0);
    } else {
        LleParamsT<float> hd{total, 0, n, plan.map.swap_xy ? 1 : 0, plan.amountOfPointsInBlock, 0,
                             skip_override >= 0 ? skip_override : plan.amountOfPointsForSkip, plan.nt_steps,
                             (float)q.h, (float)q.NT, (float)q.t_max,
                             (float)q.eps, (float)q.max_value, (float)q.transient_time};
        params = pack_lle_params<float>(hd, q.initial_conditions, q.amount_of_x, q.base_values, q.n_values,
                                        ws + off_ax0, ws + off_ax1, d_values, d_flags, ws, ws + 8, d_cell_list,
                                         list_compact ? 1 : 0);
    }
    const int block = L.shape.block;
    const int grid = persistent ? persistent_grid(e, L.fn, block, total) : (int)((total + block - 1) / block);
    size_t psize = params.size();
    void* cfg[] = {CU_LAUNCH_PARAM_BUFFER_POINTER, params.data(), CU_LAUNCH_PARAM_BUFFER_SIZE, &psize,
                   CU_LAUNCH_PARAM_END};
    CUresult r = driver().cuLaunchKernel(L.fn, grid, 1, 1, block, 1, 1, 0, (CUstream)stream, nullptr, cfg);
    if (r != CUDA_SUCCESS) {
        err = "cuLaunchKernel(lle2d): " + cu_error_string(r);
        return UCB_E_CUDA;
    }
    e->launches += 1;
    return UCB_OK;
}

int enqueue_lle(ucb_engine* e, const ucb_lle2d_request& q, const LlePlan& plan, const LleLaunch& L,
                double* d_values, int32_t* d_flags, cudaStream_t stream, std::string& err) {
    return enqueue_lle_fn(e, q, plan, L, d_values, d_flags, stream, err, -1, true, nullptr);
}

}  // namespace

namespace {

// Validation of run_lle_1d (parametric_engine.cpp:2200-2221) and the one-axis mapping of
// its launch: par_or_var 0 (initial condition) / 1 (parameter), h-sweep axis 0.
bool plan_lle1d(const ucb_lle1d_request& q, LlePlan& p, std::string& err) {
    if (!q.krs_body || !*q.krs_body) { err = "krs_body is empty"; return false; }
    if (q.amount_of_x <= 0 || q.amount_of_x > kMaxAmountOfX) { err = "amountOfX out of range"; return false; }
    if (!q.initial_conditions) { err = "initial_conditions.size() != amountOfX"; return false; }
    if (q.n_values > kMaxAmountOfValues) { err = "too many base_values"; return false; }
    if (q.n_values > 0 && !q.base_values) { err = "base_values is NULL"; return false; }
    if (q.sweep_over_h) {
        if (!(q.param_lo > 0.0 && q.param_hi > 0.0)) { err = "h lo/hi must be > 0 with sweep_over_h"; return false; }
    } else if (q.sweep_over_var) {
        if (q.var_sweep_index < 0 || q.var_sweep_index >= q.amount_of_x) { err = "var_sweep_index out of range"; return false; }
    } else {
        if (q.param_index <= 0 || q.param_index >= q.n_values) { err = "param_index out of range"; return false; }
    }
    if (q.n_pts <= 0) { err = "n_pts must be > 0"; return false; }
    if (!(q.h > 0.0)) { err = "h must be > 0"; return false; }
    if (!(q.t_max > 0.0)) { err = "t_max must be > 0"; return false; }
    if (q.transient_time < 0) { err = "transient_time must be >= 0"; return false; }
    if (!(q.NT > 0.0)) { err = "NT must be > 0"; return false; }
    if (!(q.eps > 0.0)) { err = "eps must be > 0"; return false; }
    if (q.log_scale && !(q.param_lo > 0.0 && q.param_hi > 0.0)) { err = "log scale requires param lo/hi > 0"; return false; }
    SweepMap& m = p.map;
    m.dim = 1;
    m.par_or_var = q.sweep_over_var ? 0 : 1;
    m.idx[0] = q.sweep_over_var ? q.var_sweep_index : q.param_index;
    m.idx[1] = 0;
    m.h_axis = q.sweep_over_h ? 0 : -1;
    m.lo[0] = q.param_lo;
    m.hi[0] = q.param_hi;
    m.log_axis[0] = q.log_scale != 0;
    p.amountOfPointsInBlock = (int)(q.t_max / q.NT);
    p.amountOfPointsForSkip = (int)(q.transient_time / q.h);
    if (p.amountOfPointsInBlock <= 0) { err = "computed amountOfPointsInBlock <= 0 (t_max / NT too small)"; return false; }
    if (q.opt.precision == UCB_PREC_F64 || q.opt.mode == UCB_MODE_NATIVE)
        p.nt_steps = (long long)(q.NT / q.h);
    else
        p.nt_steps = (long long)((float)q.NT / (float)q.h);
    return true;
}

}  // namespace

ucb_lle2d_request as_lle2d(const ucb_lle1d_request& q) {
    ucb_lle2d_request r{};
    r.krs_body = q.krs_body;
    r.amount_of_x = q.amount_of_x;
    r.initial_conditions = q.initial_conditions;
    r.base_values = q.base_values;
    r.n_values = q.n_values;
    r.sweep_over_var = q.sweep_over_var;
    r.var_sweep_index = q.var_sweep_index;
    r.sweep_over_h = q.sweep_over_h;
    r.log_scale = q.log_scale;
    r.param_index = q.param_index;
    r.param_lo = q.param_lo;
    r.param_hi = q.param_hi;
    r.n_pts = q.n_pts;
    r.h = q.h;
    r.transient_time = q.transient_time;
    r.t_max = q.t_max;
    r.NT = q.NT;
    r.eps = q.eps;
    r.max_value = q.max_value;
    r.cancel = q.cancel;
    r.progress = q.progress;
    r.opt = q.opt;
    return r;
}

bool plan_sweep1d(const ucb_lle1d_request& q, SweepMap& m, int& n_blocks, int& skip, long long& nt,
                  std::string& err) {
    LlePlan p;
    if (!plan_lle1d(q, p, err)) return false;
    m = p.map;
    n_blocks = p.amountOfPointsInBlock;
    skip = p.amountOfPointsForSkip;
    nt = p.nt_steps;
    return true;
}

bool plan_sweep2d(const ucb_lle2d_request& q, SweepMap& m, int& n_blocks, int& skip, long long& nt_steps,
                  std::string& err) {
    LlePlan p;
    if (!plan_lle2d(q, p, err)) return false;
    m = p.map;
    n_blocks = p.amountOfPointsInBlock;
    skip = p.amountOfPointsForSkip;
    nt_steps = p.nt_steps;
    return true;
}

// Internal hooks used by the scratch-array entry point (noalloc.cu).
int lle2d_plan_and_find(ucb_engine* e, const ucb_lle2d_request& q, bool load_if_missing, std::string& err,
                        void** plan_out, void** launch_out) {
    auto* plan = new LlePlan;
    if (!plan_lle2d(q, *plan, err)) { delete plan; return UCB_E_INVALID; }
    if (!ensure_init(e, err)) { delete plan; return UCB_E_NOGPU; }
    auto* L = new LleLaunch;
    CompileRequest rq;
    if (!lle_tuned_request(e, q, *plan, *L, rq, err)) {
        delete plan;
        delete L;
        return UCB_E_INVALID;
    }
    L->mod = load_if_missing ? e->modules.get(rq, err) : e->modules.find(rq);
    if (!L->mod) {
        if (!load_if_missing)
            err = "kernel not prepared for this request: call ucb_prepare_lle2d first (loading a module allocates "
                  "device memory)";
        delete plan;
        delete L;
        return load_if_missing ? UCB_E_COMPILE : UCB_E_INVALID;
    }
    L->fn = L->mod->functions["ucb_lle_kernel"];
    *plan_out = plan;
    *launch_out = L;
    return UCB_OK;
}

int lle2d_pin(ucb_engine* e, const ucb_lle2d_request& q, std::string& err) {
    LlePlan plan;
    if (!plan_lle2d(q, plan, err)) return UCB_E_INVALID;
    if (!ensure_init(e, err)) return UCB_E_NOGPU;
    auto L = std::make_shared<LleLaunch>();
    CompileRequest rq = lle_compile_request(q, plan, *L);
    const std::string key = tune_key(rq);
    if (!tune_request(e, q.opt, 128, rq, L->shape, err)) return UCB_E_INVALID;
    L->mod = e->modules.get(rq, err);
    if (!L->mod) return UCB_E_COMPILE;
    L->fn = L->mod->functions["ucb_lle_kernel"];
    e->pinned_lle[key] = L;
    return UCB_OK;
}

int lle2d_find_pinned(ucb_engine* e, const ucb_lle2d_request& q, std::string& err, void** plan_out,
                      void** launch_out) {
    auto plan = std::make_unique<LlePlan>();
    if (!plan_lle2d(q, *plan, err)) return UCB_E_INVALID;
    if (!e->initialized) {
        err = "engine not prepared: call ucb_prepare_lle2d first";
        return UCB_E_INVALID;
    }
    cudaSetDevice(e->device);
    LleLaunch probe;
    const std::string key = tune_key(lle_compile_request(q, *plan, probe));
    auto it = e->pinned_lle.find(key);
    if (it == e->pinned_lle.end()) {
        err = "kernel not prepared for this request: call ucb_prepare_lle2d first (loading a module allocates "
              "device memory)";
        return UCB_E_INVALID;
    }
    *launch_out = new LleLaunch(*static_cast<LleLaunch*>(it->second.get()));
    *plan_out = plan.release();
    return UCB_OK;
}

int lle2d_enqueue_with_scratch(ucb_engine* e, const ucb_lle2d_request& q, void* plan, void* launch, double* d_values,
                               int32_t* d_flags, cudaStream_t stream, char* scratch, std::string& err,
                               TableUpload upload) {
    return enqueue_lle_fn(e, q, *static_cast<LlePlan*>(plan), *static_cast<LleLaunch*>(launch), d_values, d_flags,
                          stream, err, -1, true, scratch, nullptr, 0, false, upload);
}

int lle2d_enqueue_cells(ucb_engine* e, const ucb_lle2d_request& q, void* plan, void* launch, const long long* d_cells,
                        long long n_cells, bool compact, double* d_values, int32_t* d_flags, cudaStream_t stream,
                        std::string& err) {
    if (n_cells <= 0) return UCB_OK;
    return enqueue_lle_fn(e, q, *static_cast<LlePlan*>(plan), *static_cast<LleLaunch*>(launch), d_values, d_flags,
                          stream, err, -1, true, nullptr, d_cells, n_cells, compact);
}

long long lle2d_flops_per_step(void* launch) { return static_cast<LleLaunch*>(launch)->sys.flops_step; }

void lle2d_release(void* plan, void* launch) {
    delete static_cast<LlePlan*>(plan);
    delete static_cast<LleLaunch*>(launch);
}

}  // namespace ucb

using namespace ucb;

extern "C" {

int ucb_abi_version(void) { return UCB_ABI_VERSION; }

void ucb_default_options(ucb_options* o) {
    std::memset(o, 0, sizeof *o);
    o->precision = UCB_PREC_F64;
    o->mode = UCB_MODE_NATIVE;
    o->lle_method = UCB_LLE_AUTO;
}

ucb_engine* ucb_create(int device) {
    ucb_engine* e = new ucb_engine;
    e->device = device;
    return e;
}

void ucb_destroy(ucb_engine* e) {
    if (!e) return;
    if (e->initialized) {
        cudaSetDevice(e->device);
        if (e->stream) cudaStreamSynchronize(e->stream);
        e->surrogate_net.reset();
        e->modules.clear();
        if (e->ws) cudaFree(e->ws);
        if (e->ev0) cudaEventDestroy(e->ev0);
        if (e->ev1) cudaEventDestroy(e->ev1);
        if (e->stream) cudaStreamDestroy(e->stream);
        if (e->pool) cudaMemPoolDestroy(e->pool);
        e->pinned_lle.clear();
        if (e->control) cudaFreeHost(e->control);
    }
    delete e;
}

const char* ucb_last_error(const ucb_engine* e) { return e ? e->last_error.c_str() : "null engine"; }

long long ucb_kernel_launches(const ucb_engine* e) { return e ? e->launches : 0; }

void ucb_clear_cache(ucb_engine* e) {
    if (!e) return;
    e->modules.clear();
    if (e->pool) {
        if (e->stream) cudaStreamSynchronize(e->stream);
        cudaMemPoolTrimTo(e->pool, 0);
    }
}

static int fail(ucb_engine* e, char* error, int32_t* ok, int code, const std::string& msg) {
    e->last_error = msg;
    set_error(error, msg);
    *ok = 0;
    return code;
}

int ucb_run_lle2d(ucb_engine* e, const ucb_lle2d_request* req, ucb_lle2d_result* res) {
    if (!e || !req || !res) return UCB_E_INVALID;
    res->ok = 0;
    res->cancelled = 0;
    res->error[0] = 0;
    res->kernel_ms = 0;
    res->steps = 0;
    res->flops = 0;
    const ucb_lle2d_request& q = *req;
    LlePlan plan;
    std::string err;
    if (!plan_lle2d(q, plan, err)) return fail(e, res->error, &res->ok, UCB_E_INVALID, err);
    if (!res->values || !res->flags) return fail(e, res->error, &res->ok, UCB_E_INVALID, "result buffers are NULL");
    if (q.cancel && *q.cancel) {
        res->cancelled = 1;
        return fail(e, res->error, &res->ok, UCB_E_CANCELLED, "Cancelled by user");
    }
    if (!ensure_init(e, err)) return fail(e, res->error, &res->ok, UCB_E_NOGPU, err);
    LleLaunch L;
    if (!prepare_lle(e, q, plan, L, err)) return fail(e, res->error, &res->ok, UCB_E_COMPILE, err);
    if (q.progress) *q.progress = 0.0f;
    const int n = q.n_pts;
    const size_t total = (size_t)n * n;
    double* d_values = nullptr;
    int32_t* d_flags = nullptr;
    cudaError_t ce;
    if ((ce = dev_alloc(e, (void**)&d_values, total * sizeof(double), e->stream)) != cudaSuccess ||
        (ce = dev_alloc(e, (void**)&d_flags, total * sizeof(int32_t), e->stream)) != cudaSuccess)
        return fail(e, res->error, &res->ok, UCB_E_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(ce));
    begin_run(e);
    cudaEventRecord(e->ev0, e->stream);
    int rc = enqueue_lle(e, q, plan, L, d_values, d_flags, e->stream, err);
    cudaEventRecord(e->ev1, e->stream);
    if (rc == UCB_OK) rc = wait_run(e, e->ev1, q.cancel, q.progress, (long long)total, err);
    if (rc == UCB_E_CANCELLED) res->cancelled = 1;
    if (rc == UCB_OK) {
        unsigned long long steps = 0;
        if ((ce = cudaMemcpyAsync(res->values, d_values, total * sizeof(double), cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess ||
            (ce = cudaMemcpyAsync(res->flags, d_flags, total * sizeof(int32_t), cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess ||
            (ce = cudaMemcpyAsync(&steps, static_cast<char*>(e->ws) + 8, 8, cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess ||
            (ce = cudaStreamSynchronize(e->stream)) != cudaSuccess) {
            rc = UCB_E_CUDA;
            err = std::string("CUDA lle2d: ") + cudaGetErrorString(ce);
        } else {
            float ms = 0;
            cudaEventElapsedTime(&ms, e->ev0, e->ev1);
            res->kernel_ms = ms;
            res->steps = (long long)steps;
            res->flops = (double)steps * (double)L.sys.flops_step;
        }
    }
    cudaFreeAsync(d_values, e->stream);
    cudaFreeAsync(d_flags, e->stream);
    cudaStreamSynchronize(e->stream);
    if (rc != UCB_OK) return fail(e, res->error, &res->ok, rc, err);
    if (q.progress) *q.progress = 1.0f;
    res->n_pts = n;
    res->param_lo = q.param_lo;
    res->param_hi = q.param_hi;
    res->param_lo_2 = q.param_lo_2;
    res->param_hi_2 = q.param_hi_2;
    double vmin = std::numeric_limits<double>::infinity(), vmax = -std::numeric_limits<double>::infinity();
    for (size_t k = 0; k < total; ++k) {
        if (res->flags[k] < 0) continue;
        const double v = res->values[k];
        if (!std::isfinite(v)) continue;
        vmin = std::min(vmin, v);
        vmax = std::max(vmax, v);
    }
    if (std::isfinite(vmin) && std::isfinite(vmax)) {
        res->min_val = vmin;
        res->max_val = vmax;
    } else {
        res->min_val = res->max_val = 0.0;
    }
    if (q.csv_output_path && *q.csv_output_path) {
        const csv::Common cc = csv::common(q.base_values, q.n_values, q.initial_conditions, q.amount_of_x,
                                           q.opt.precision == UCB_PREC_F32);
        csv::lle2d(q.csv_output_path, cc, plan.map.par_or_var, q.t_max, q.NT, q.transient_time, q.h, q.eps,
                   q.sweep_over_var ? q.var_sweep_index : q.param_index,
                   q.sweep_over_var_2 ? q.var_sweep_index_2 : q.param_index_2, q.param_lo, q.param_hi, q.param_lo_2,
                   q.param_hi_2, n, res->values);
    }
    if (!L.sys.note.empty()) e->last_error = L.sys.note;
    res->ok = 1;
    return UCB_OK;
}

int ucb_run_lle1d(ucb_engine* e, const ucb_lle1d_request* req, ucb_lle1d_result* res) {
    if (!e || !req || !res) return UCB_E_INVALID;
    res->ok = 0;
    res->cancelled = 0;
    res->error[0] = 0;
    res->kernel_ms = 0;
    res->steps = 0;
    res->flops = 0;
    const ucb_lle1d_request& q1 = *req;
    LlePlan plan;
    std::string err;
    if (!plan_lle1d(q1, plan, err)) return fail(e, res->error, &res->ok, UCB_E_INVALID, err);
    if (!res->values || !res->flags) return fail(e, res->error, &res->ok, UCB_E_INVALID, "result buffers are NULL");
    if (q1.cancel && *q1.cancel) {
        res->cancelled = 1;
        return fail(e, res->error, &res->ok, UCB_E_CANCELLED, "Cancelled by user");
    }
    if (!ensure_init(e, err)) return fail(e, res->error, &res->ok, UCB_E_NOGPU, err);
    const ucb_lle2d_request q = as_lle2d(q1);
    LleLaunch L;
    if (!prepare_lle(e, q, plan, L, err)) return fail(e, res->error, &res->ok, UCB_E_COMPILE, err);
    if (q1.progress) *q1.progress = 0.0f;
    const int n = q1.n_pts;
    double* d_values = nullptr;
    int32_t* d_flags = nullptr;
    cudaError_t ce;
    if ((ce = dev_alloc(e, (void**)&d_values, (size_t)n * sizeof(double), e->stream)) != cudaSuccess ||
        (ce = dev_alloc(e, (void**)&d_flags, (size_t)n * sizeof(int32_t), e->stream)) != cudaSuccess)
        return fail(e, res->error, &res->ok, UCB_E_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(ce));
    begin_run(e);
    cudaEventRecord(e->ev0, e->stream);
    int rc = enqueue_lle(e, q, plan, L, d_values, d_flags, e->stream, err);
    cudaEventRecord(e->ev1, e->stream);
    if (rc == UCB_OK) rc = wait_run(e, e->ev1, q1.cancel, q1.progress, (long long)n, err);
    if (rc == UCB_E_CANCELLED) res->cancelled = 1;
    unsigned long long steps = 0;
    if (rc == UCB_OK) {
        if ((ce = cudaMemcpyAsync(res->values, d_values, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost,
                                  e->stream)) != cudaSuccess ||
            (ce = cudaMemcpyAsync(res->flags, d_flags, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                  e->stream)) != cudaSuccess ||
            (ce = cudaMemcpyAsync(&steps, static_cast<char*>(e->ws) + 8, 8, cudaMemcpyDeviceToHost, e->stream)) !=
                cudaSuccess ||
            (ce = cudaStreamSynchronize(e->stream)) != cudaSuccess) {
            rc = UCB_E_CUDA;
            err = std::string("CUDA lle1d: ") + cudaGetErrorString(ce);
        }
    }
    cudaFreeAsync(d_values, e->stream);
    cudaFreeAsync(d_flags, e->stream);
    cudaStreamSynchronize(e->stream);
    if (rc != UCB_OK) return fail(e, res->error, &res->ok, rc, err);
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    res->kernel_ms = ms;
    res->steps = (long long)steps;
    res->flops = (double)steps * (double)L.sys.flops_step;
    // sentinel -> NaN, as run_lle_1d does (parametric_engine.cpp:2455-2466)
    for (int i = 0; i < n; ++i)
        if (res->flags[i] < 0) res->values[i] = std::numeric_limits<double>::quiet_NaN();
    res->n_pts = n;
    res->param_lo = q1.param_lo;
    res->param_hi = q1.param_hi;
    if (q1.csv_output_path && *q1.csv_output_path) {
        const bool f32 = q1.opt.precision == UCB_PREC_F32;
        const csv::Common cc = csv::common(q1.base_values, q1.n_values, q1.initial_conditions, q1.amount_of_x, f32);
        csv::curve1d(q1.csv_output_path, "1D LLE", cc, q1.t_max, q1.NT, q1.transient_time, q1.h, q1.eps,
                     plan.map.idx[0], csv::numb_value(q1.param_lo, f32), csv::numb_value(q1.param_hi, f32),
                     q1.log_scale != 0, n, 1, res->values);
    }
    if (q1.progress) *q1.progress = 1.0f;
    if (!L.sys.note.empty()) e->last_error = L.sys.note;
    res->ok = 1;
    return UCB_OK;
}

int ucb_lle2d_states(ucb_engine* e, const ucb_lle2d_request* req, long long n_steps, double* out_states) {
    if (!e || !req || !out_states) return UCB_E_INVALID;
    LlePlan plan;
    std::string err;
    if (!plan_lle2d(*req, plan, err)) { e->last_error = err; return UCB_E_INVALID; }
    if (n_steps < 0) { e->last_error = "n_steps must be >= 0"; return UCB_E_INVALID; }
    if (!ensure_init(e, err)) { e->last_error = err; return UCB_E_NOGPU; }
    LleLaunch L;
    if (!prepare_lle(e, *req, plan, L, err)) { e->last_error = err; return UCB_E_COMPILE; }
    const long long total = (long long)req->n_pts * req->n_pts;
    const size_t bytes = (size_t)total * req->amount_of_x * sizeof(double);
    double* d_out = nullptr;
    cudaError_t ce = dev_alloc(e, (void**)&d_out, bytes, e->stream);
    if (ce != cudaSuccess) { e->last_error = cudaGetErrorString(ce); return UCB_E_CUDA; }
    LlePlan p2 = plan;
    p2.amountOfPointsForSkip = (int)n_steps;
    ucb_lle2d_request q = *req;
    LleLaunch L2 = L;
    L2.fn = L.mod->functions["ucb_state_kernel"];
    int rc = enqueue_lle_fn(e, q, p2, L2, d_out, nullptr, e->stream, err, n_steps, /*persistent=*/false, nullptr);
    if (rc == UCB_OK) {
        if ((ce = cudaMemcpyAsync(out_states, d_out, bytes, cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess ||
            (ce = cudaStreamSynchronize(e->stream)) != cudaSuccess) {
            rc = UCB_E_CUDA;
            err = cudaGetErrorString(ce);
        }
    }
    cudaFreeAsync(d_out, e->stream);
    cudaStreamSynchronize(e->stream);
    if (rc != UCB_OK) e->last_error = err;
    return rc;
}

int ucb_precompile_lle2d(const ucb_lle2d_request* req, char* err_out, int err_len) {
    LlePlan plan;
    std::string err;
    if (!req || !plan_lle2d(*req, plan, err)) {
        if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", err.c_str());
        return UCB_E_INVALID;
    }
    LleLaunch L;
    CompileRequest rq;
    if (!lle_tuned_request(nullptr, *req, plan, L, rq, err)) {
        if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", err.c_str());
        return UCB_E_INVALID;
    }
    if (!precompile_to_disk(rq, err)) {
        if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", err.c_str());
        return UCB_E_COMPILE;
    }
    if (err_out && err_len > 0) std::snprintf(err_out, (size_t)err_len, "%s", L.sys.note.c_str());
    return UCB_OK;
}

int ucb_lle2d_device(ucb_engine* e, const ucb_lle2d_request* req, double* d_values, int32_t* d_flags, void* stream,
                     ucb_lle2d_result* res) {
    if (!e || !req || !res) return UCB_E_INVALID;
    res->ok = 0;
    res->error[0] = 0;
    LlePlan plan;
    std::string err;
    if (!plan_lle2d(*req, plan, err)) return fail(e, res->error, &res->ok, UCB_E_INVALID, err);
    if (!ensure_init(e, err)) return fail(e, res->error, &res->ok, UCB_E_NOGPU, err);
    LleLaunch L;
    if (!prepare_lle(e, *req, plan, L, err)) return fail(e, res->error, &res->ok, UCB_E_COMPILE, err);
    int rc = enqueue_lle(e, *req, plan, L, d_values, d_flags, (cudaStream_t)stream, err);
    if (rc != UCB_OK) return fail(e, res->error, &res->ok, rc, err);
    res->n_pts = req->n_pts;
    res->ok = 1;
    return UCB_OK;
}

int ucb_lle2d_cells(ucb_engine* e, const ucb_lle2d_request* req, const long long* d_cells, long long n_cells,
                    double* d_values, int32_t* d_flags, void* stream, ucb_lle2d_result* res) {
    if (!e || !req || !res) return UCB_E_INVALID;
    res->ok = 0;
    res->error[0] = 0;
    LlePlan plan;
    std::string err;
    if (!plan_lle2d(*req, plan, err)) return fail(e, res->error, &res->ok, UCB_E_INVALID, err);
    if (n_cells < 0 || (n_cells > 0 && (!d_cells || !d_values || !d_flags)))
        return fail(e, res->error, &res->ok, UCB_E_INVALID, "cell list or output buffers missing");
    if (!ensure_init(e, err)) return fail(e, res->error, &res->ok, UCB_E_NOGPU, err);
    LleLaunch L;
    if (!prepare_lle(e, *req, plan, L, err)) return fail(e, res->error, &res->ok, UCB_E_COMPILE, err);
    if (n_cells > 0) {
        const int rc = enqueue_lle_fn(e, *req, plan, L, d_values, d_flags, (cudaStream_t)stream, err, -1, true,
                                      nullptr, d_cells, n_cells, true);
        if (rc != UCB_OK) return fail(e, res->error, &res->ok, rc, err);
    }
    res->n_pts = req->n_pts;
    res->ok = 1;
    return UCB_OK;
}

int ucb_autotune_lle2d(ucb_engine* e, const ucb_lle2d_request* req, int32_t force, ucb_tune_report* rep) {
    if (!e || !req || !rep) return UCB_E_INVALID;
    std::memset(rep, 0, sizeof *rep);
    LlePlan plan;
    std::string err;
    auto bad = [&](int code, const std::string& m) {
        e->last_error = m;
        std::snprintf(rep->error, sizeof rep->error, "%s", m.c_str());
        return code;
    };
    if (!plan_lle2d(*req, plan, err)) return bad(UCB_E_INVALID, err);
    if (!ensure_init(e, err)) return bad(UCB_E_NOGPU, err);
    // the kernel build of the request itself (its key), shape fields cleared
    ucb_lle2d_request base = *req;
    base.opt.block_threads = base.opt.max_registers = base.opt.unroll = 0;
    base.csv_output_path = nullptr;
    base.cancel = nullptr;
    base.progress = nullptr;
    LleLaunch L0;
    const std::string key = tune_key(lle_compile_request(base, plan, L0));
    // trial workload: the same window on a grid of at most 768^2 cells (a few resident
    // waves), horizon scaled to about 1.2e10 steps in all
    ucb_lle2d_request t = base;
    t.n_pts = std::min(base.n_pts, 768);
    const double steps_cell =
        plan.amountOfPointsForSkip + (double)plan.amountOfPointsInBlock * 2.0 * (double)(plan.nt_steps + 1);
    const double f = trial_scale((double)t.n_pts * t.n_pts, steps_cell);
    if (f < 1.0) {
        t.t_max = std::max(base.NT, std::floor(base.t_max * f / base.NT) * base.NT);
        t.transient_time = base.transient_time * f;
    }
    LlePlan tp;
    if (!plan_lle2d(t, tp, err)) return bad(UCB_E_INVALID, "trial request: " + err);
    std::vector<double> vals((size_t)t.n_pts * t.n_pts);
    std::vector<int32_t> flags(vals.size());
    auto with = [&](const TuneConfig& c) {
        ucb_lle2d_request q = t;
        q.opt.block_threads = c.block;
        q.opt.max_registers = c.maxreg;
        q.opt.unroll = c.unroll;
        return q;
    };
    auto trial = [&](const TuneConfig& c) -> double {
        ucb_lle2d_request q = with(c);
        ucb_lle2d_result r{};
        r.values = vals.data();
        r.flags = flags.data();
        return ucb_run_lle2d(e, &q, &r) == UCB_OK ? r.kernel_ms : -1.0;
    };
    auto build = [&](const TuneConfig& c) {
        ucb_lle2d_request q = with(c);
        LleLaunch L;
        CompileRequest rq;
        std::string e2;
        lle_tuned_request(e, q, tp, L, rq, e2);
        return rq;
    };
    // confirmation: the request's own window and horizon, on its grid when one run is
    // estimated at <= 1.5 s from the trial's default time, else on the largest grid that is
    std::vector<double> cvals;
    std::vector<int32_t> cflags;
    ucb_lle2d_request cq = base;
    auto confirm = [&](const TuneConfig& c) -> double {
        if (cvals.empty()) {
            const double trial_steps = (double)t.n_pts * t.n_pts *
                                       (tp.amountOfPointsForSkip +
                                        (double)tp.amountOfPointsInBlock * 2.0 * (double)(tp.nt_steps + 1));
            const double ms_per_cell = rep->default_ms / trial_steps * steps_cell;
            const double cells = std::min((double)base.n_pts * base.n_pts, 1500.0 / std::max(ms_per_cell, 1e-12));
            cq.n_pts = std::max(64, std::min(base.n_pts, (int)std::floor(std::sqrt(cells))));
            rep->confirm_n_pts = cq.n_pts;
            cvals.resize((size_t)cq.n_pts * cq.n_pts);
            cflags.resize(cvals.size());
        }
        ucb_lle2d_request q = cq;
        q.opt.block_threads = c.block;
        q.opt.max_registers = c.maxreg;
        q.opt.unroll = c.unroll;
        ucb_lle2d_result r{};
        r.values = cvals.data();
        r.flags = cflags.data();
        return ucb_run_lle2d(e, &q, &r) == UCB_OK ? r.kernel_ms : -1.0;
    };
    const int rc = autotune_search(e, key, 128, force != 0, trial, build, rep, confirm);
    rep->trial_n_pts = t.n_pts;
    return rc;
}

}  // extern "C"
