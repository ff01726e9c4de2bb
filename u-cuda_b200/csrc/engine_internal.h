// Internal pieces shared by the C-ABI entry points (not part of the ABI).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/ucb.h"
#include "frontend.h"
#include "jit.h"

namespace ucb {
// Launch shape of a kernel build (see ucb_options): threads per block, registers per
// thread cap (0 = compiler's choice), steps per unrolled chunk of the step loops.
struct TuneConfig {
    int block = 128;
    int maxreg = 0;
    int unroll = 1;
    bool operator==(const TuneConfig& o) const { return block == o.block && maxreg == o.maxreg && unroll == o.unroll; }
};
}  // namespace ucb

// Host view of the run-control block the kernels poll (kernels/ucb_device.cuh UcbControl):
// page-locked host memory mapped into the device's address space.
struct ucb_run_control {
    volatile int32_t cancel;
    int32_t pad;
    volatile unsigned long long fetched;
};

struct ucb_engine {
    int device = 0;
    bool initialized = false;
    int sm_count = 0;
    std::string last_error;
    ucb::ModuleCache modules;
    cudaStream_t stream = nullptr;   // engine stream for the host-buffer entry points
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // Device workspace: work counters, step counters, axis tables. Grown on demand.
    void* ws = nullptr;
    size_t ws_bytes = 0;
    // Stream-ordered allocations of the run_* calls come from this pool, which keeps what
    // is freed for the next call (no release threshold) until ucb_clear_cache / destroy.
    cudaMemPool_t pool = nullptr;
    long long launches = 0;
    // Launch shapes chosen by the autotuner, by kernel-build key (plus the entries of the
    // on-disk table for this device, read on first use).
    std::map<std::string, ucb::TuneConfig> tuned;
    bool tuned_loaded = false;
    // Network of the last surrogate-refined map, kept for reuse by the next call with the
    // same configuration (owned; released with the engine).
    std::shared_ptr<void> surrogate_net;
    // LLE kernels pinned by ucb_prepare_lle2d for ucb_lle2d_device_noalloc: module, kernel
    // and launch shape as resolved at prepare time, by kernel-build key (an autotune after
    // the prepare does not change what the allocation-free call launches).
    std::map<std::string, std::shared_ptr<void>> pinned_lle;
    // Run control of the host-buffer entry points (null when mapped memory is unavailable).
    ucb_run_control* control = nullptr;
};

namespace ucb {

// Kernel-order sweep description after the reference's host mapping
// (run_lle_2d parametric_engine.cpp:2602-2703).
struct SweepMap {
    int dim = 2;
    int par_or_var = 1;
    int idx[2] = {0, 0};
    double lo[2] = {0, 0}, hi[2] = {0, 0};
    bool log_axis[2] = {false, false};
    int h_axis = -1;
    bool swap_xy = false;
};

// The step function of a run: either the verbatim KRS body (exact form) or the
// right-hand side recognised in it (native form).
struct SystemCode {
    bool exact = true;
    bool has_jvp = false;
    bool has_packed = false; // ucb_rhs2 / ucb_jvp2 (packed FP32 pairs) emitted too
    std::string code;     // device source defining calculateDiscreteModel or ucb_rhs/ucb_jvp
    int flops_step = 0;   // algorithmic FLOPs of one step (native form; 0 if unknown)
    int flops_rhs = 0;    // FLOPs of one right-hand-side evaluation (recognised bodies)
    int flops_jvp = 0;    // FLOPs of one J(x) v product (recognised bodies)
    std::string note;     // why the exact form was chosen, when native was requested
    int trig_phase = -1;  // native form: forcing phase variable (ucb_rhs_trig), -1 none
    double trig_rate = 0; // its constant rate (dX[p]/dt)
    int clock_var = -1;   // native FP32 form: a variable with a constant derivative (-1 none)
    double clock_rate = 0;
};
// The define that turns on the compensated clock of the native FP32 step
// (UCB_KAHAN_CLOCK), for kernels where each Stepper serves one trajectory; empty if the
// build has no clock.
std::vector<std::string> clock_defines(const SystemCode& sys);

bool ensure_init(ucb_engine* e, std::string& err);
bool ensure_workspace(ucb_engine* e, size_t bytes, std::string& err);

// Stream-ordered device allocation from the engine's pool (released with cudaFreeAsync).
inline cudaError_t dev_alloc(ucb_engine* e, void** p, size_t bytes, cudaStream_t st) {
    return e->pool ? cudaMallocFromPoolAsync(p, bytes, e->pool, st) : cudaMallocAsync(p, bytes, st);
}

// ---- autotuning (autotune.cpp) ----
// Identity of a kernel build without its launch-shape knobs (hex of a 64-bit hash).
std::string tune_key(const CompileRequest& rq);
// The launch shape a run uses: explicit option fields first, then the shape tuned for
// this key (engine memory or the on-disk table; e may be null), else the defaults (with
// `default_block` threads). False with a message for invalid option fields.
bool resolve_tuning(ucb_engine* e, const ucb_options& o, const std::string& key, int default_block, TuneConfig& out,
                    std::string& err);
// Adds the knobs of a non-default shape to a compile request (defines, --maxrregcount).
void apply_tuning(CompileRequest& rq, const TuneConfig& c);
// Resolves and applies in one go; returns the launch shape.
bool tune_request(ucb_engine* e, const ucb_options& o, int default_block, CompileRequest& rq, TuneConfig& out,
                  std::string& err);
// Coordinate search over block size, unroll and register cap. `trial` runs the request's
// kernel on the trial workload with the given shape (as explicit options) and returns its
// kernel milliseconds (< 0: the shape failed); `build` gives the compile request of a
// shape (for the register count and occupancy of the chosen build). The best shape is
// stored for `key` (engine + on-disk table). force = false returns a stored shape as is.
// `confirm` (optional) times a shape on a workload closer to the real run; when the trial's
// winner is not the default shape, it must also win there by 2 % to be kept (a short trial
// can rank shapes differently from a full-horizon run).
int autotune_search(ucb_engine* e, const std::string& key, int default_block, bool force,
                    const std::function<double(const TuneConfig&)>& trial,
                    const std::function<CompileRequest(const TuneConfig&)>& build, ucb_tune_report* rep,
                    const std::function<double(const TuneConfig&)>& confirm = nullptr);

// Horizon factor of an autotuning trial: about `target_steps` steps over `cells` cells of
// `steps_per_cell` steps each (1 when the request is already that small).
inline double trial_scale(double cells, double steps_per_cell, double target_steps = 1.2e10) {
    const double full = cells * std::max(steps_per_cell, 1.0);
    return full <= target_steps ? 1.0 : target_steps / full;
}

// Builds the step-function source for a run.
SystemCode make_system_code(const std::string& krs_body, int nx, int nv, int precision, int mode,
                            bool want_jvp);

// Common prelude: numb typedef, configCUDA.h constants pi/euler, sizes, sweep macros.
std::string make_prelude(int precision, int nx, int nv, const SweepMap& m, bool extra_step,
                         const SystemCode& sys, const std::vector<std::string>& extra_defines);

// Embedded device headers (generated at build time from csrc/kernels/*.cuh).
const std::vector<std::pair<std::string, std::string>>& device_headers();

// Axis value table of one sweep axis in numb arithmetic (getValueByIdx,
// cudaLibrary.cu:1344-1361, and getValueByIdx_log, :1381-1396; valueNumber 0).
void axis_table(int precision, int n, double lo, double hi, bool log_scale, std::vector<double>& out_d,
                std::vector<float>& out_f);

// Packs a kernel parameter struct field by field with natural alignment (the layout a
// single by-value struct parameter has on the device).
struct ParamPack {
    std::vector<char> buf;
    template <class T>
    void put(const T& v) {
        while (buf.size() % alignof(T)) buf.push_back(0);
        const char* c = reinterpret_cast<const char*>(&v);
        buf.insert(buf.end(), c, c + sizeof(T));
    }
    // numb-typed value (double or float by precision)
    void put_numb(int precision, double v) {
        if (precision == UCB_PREC_F64) put<double>(v);
        else put<float>((float)v);
    }
    void finish() {
        while (buf.size() % 8) buf.push_back(0);
    }
};

// Launches a kernel with one by-value struct parameter.
bool launch_packed(ucb_engine* e, CUfunction f, int grid, int block, cudaStream_t stream, ParamPack& pk,
                   std::string& err);

// Validation and axis mapping of run_lle_2d (shared by the 2-D maps): kernel-order sweep,
// (int)(t_max/NT), (int)(transient/h) and (size_t)(NT/h) in numb.
bool plan_sweep2d(const ucb_lle2d_request& q, SweepMap& m, int& n_blocks, int& skip, long long& nt_steps,
                  std::string& err);

// Validation and axis mapping of run_lle_1d / run_ls_1d (parametric_engine.cpp:2200-2221,
// :3070-3100): a one-axis sweep (dim 1) with the same step counts.
bool plan_sweep1d(const ucb_lle1d_request& q, SweepMap& m, int& n_blocks, int& skip, long long& nt,
                  std::string& err);
// The 2-D request with the fields a 1-D run shares (for the common launch code).
ucb_lle2d_request as_lle2d(const ucb_lle1d_request& q);

// Launch helper: persistent grid size for a kernel.
int persistent_grid(ucb_engine* e, CUfunction f, int block, long long work_items);

// Run control of the host-buffer entry points (ucb_run_*). begin_run resets the queue
// position before a launch. wait_run waits for `done` (an event recorded after the run's
// main kernel); while it waits it mirrors the caller's *cancel into the control block (the
// kernels' warps then take no more cells and an adaptive cell abandons its steps) and
// writes the queue position / work_items to *progress. Without cancel and progress words
// it simply synchronises. Returns UCB_OK, UCB_E_CANCELLED (the control block is clear
// again once the kernel has ended) or UCB_E_CUDA.
void begin_run(ucb_engine* e);
int wait_run(ucb_engine* e, cudaEvent_t done, const volatile int32_t* cancel, volatile float* progress,
             long long work_items, std::string& err);

// LLE-2D launch pieces for entry points outside ucb_engine.cpp. plan / launch are opaque
// (released with lle2d_release); load_if_missing = false only looks up an already loaded
// module (no allocation).
int lle2d_plan_and_find(ucb_engine* e, const ucb_lle2d_request& q, bool load_if_missing, std::string& err,
                        void** plan_out, void** launch_out);
// Allocation-free launch pieces (noalloc.cu). lle2d_pin compiles / loads the kernel of a
// request and pins it on the engine (allocates); lle2d_find_pinned looks the pinned kernel
// up again (no allocation; UCB_E_INVALID "not prepared" when absent).
int lle2d_pin(ucb_engine* e, const ucb_lle2d_request& q, std::string& err);
int lle2d_find_pinned(ucb_engine* e, const ucb_lle2d_request& q, std::string& err, void** plan_out,
                      void** launch_out);
// Copies `bytes` (a multiple of 4) from host memory to device memory in stream order.
typedef int (*TableUpload)(void* dst, const void* src, size_t bytes, cudaStream_t stream, std::string& err);
int lle2d_enqueue_with_scratch(ucb_engine* e, const ucb_lle2d_request& q, void* plan, void* launch, double* d_values,
                               int32_t* d_flags, cudaStream_t stream, char* scratch, std::string& err,
                               TableUpload upload = nullptr);
// Cells d_cells[0..n_cells) of the grid; compact: entry i is stored at d_values[i],
// otherwise at the cell's map position.
int lle2d_enqueue_cells(ucb_engine* e, const ucb_lle2d_request& q, void* plan, void* launch, const long long* d_cells,
                        long long n_cells, bool compact, double* d_values, int32_t* d_flags, cudaStream_t stream,
                        std::string& err);
long long lle2d_flops_per_step(void* launch);
void lle2d_release(void* plan, void* launch);

}  // namespace ucb
