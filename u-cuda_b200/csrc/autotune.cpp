// Launch-shape autotuning of the integrator kernels.
//
// Per-cell work is uneven (divergence, early exit, adaptive steps) and the best launch
// shape depends on the system's step body (registers, latency chains), the precision and
// the form, so the shape is searched per kernel build on the device itself: threads per
// block (the kernels' __launch_bounds__ and the launch), a register cap (--maxrregcount,
// trading registers for resident warps) and the number of steps per unrolled chunk of the
// step loops whose trip count is only known at run time. A trial runs the request's own
// entry point on a reduced copy of the request (the caller builds it: coarser grid over the
// same window, shortened horizon), with the shape as explicit options, and reads back the
// kernel time the entry measures with CUDA events. The search is coordinate descent
// (block, then unroll, then register caps at the occupancy steps below the build's own
// register count); a shape must beat the incumbent by 2 % to replace it. Results live in
// the engine and in a table beside the CUBIN cache, keyed by device and kernel build.
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "engine_internal.h"

namespace ucb {
namespace {

std::string device_tag(ucb_engine* e) {
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, e->device) != cudaSuccess) return "unknown";
    std::string name = prop.name;
    for (char& c : name)
        if (c == '\t' || c == '\n' || c == ' ') c = '_';
    return name + "|sm" + std::to_string(prop.major) + std::to_string(prop.minor) + "|" +
           std::to_string(prop.multiProcessorCount);
}

// $UCB_TUNE_TABLE, else tuned.tsv in the CUBIN cache directory.
std::string table_path() {
    const char* env = std::getenv("UCB_TUNE_TABLE");
    if (env && *env) return env;
    const std::string dir = cubin_cache_dir();
    return dir.empty() ? "" : dir + "/tuned.tsv";
}

// Lines: device tag, key, block, register cap, unroll, trial ms (tab-separated). Later
// lines override earlier ones.
void load_table(ucb_engine* e) {
    if (e->tuned_loaded) return;
    e->tuned_loaded = true;
    const std::string path = table_path();
    if (path.empty()) return;
    std::ifstream f(path);
    if (!f) return;
    const std::string tag = device_tag(e);
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream ss(line);
        std::string t, key;
        TuneConfig c;
        double ms = 0;
        if (!std::getline(ss, t, '\t') || !std::getline(ss, key, '\t')) continue;
        if (!(ss >> c.block >> c.maxreg >> c.unroll >> ms)) continue;
        if (t != tag || c.block < 32 || c.block > 1024 || c.block % 32 || c.unroll < 1 || c.unroll > 16 ||
            (c.maxreg != 0 && (c.maxreg < 16 || c.maxreg > 255)))
            continue;
        e->tuned[key] = c;
    }
}

void store(ucb_engine* e, const std::string& key, const TuneConfig& c, double ms) {
    e->tuned[key] = c;
    const std::string path = table_path();
    if (path.empty()) return;
    const auto slash = path.find_last_of('/');
    if (slash != std::string::npos && slash > 0) mkdir(path.substr(0, slash).c_str(), 0755);
    std::ofstream f(path, std::ios::app);
    if (!f) return;
    char buf[256];
    std::snprintf(buf, sizeof buf, "%s\t%s\t%d\t%d\t%d\t%.4f\n", device_tag(e).c_str(), key.c_str(), c.block, c.maxreg,
                  c.unroll, ms);
    f << buf;
}

// Resident blocks per SM at `regs` registers per thread (register file only).
int blocks_by_registers(int regs, int block) {
    const int r = ((std::max(regs, 1) + 7) / 8) * 8;
    const int by_regs = 65536 / (r * block);
    const int by_threads = 2048 / block;
    return std::max(0, std::min({by_regs, by_threads, 32}));
}

// Resident blocks per SM to request so that the compiler keeps to `maxreg` registers per
// thread or fewer: the occupancy level that cap allows (at least one block).
int min_blocks_for(int maxreg, int block) { return std::max(1, blocks_by_registers(maxreg, block)); }

// Main kernel of a loaded build (the first one the request names) and its registers.
CUfunction main_kernel(const Module& m, const CompileRequest& rq) {
    auto it = rq.kernels.empty() ? m.functions.end() : m.functions.find(rq.kernels[0]);
    return it == m.functions.end() ? nullptr : it->second;
}

int kernel_registers(CUfunction f) {
    int r = 0;
    if (f && driver().cuFuncGetAttribute) driver().cuFuncGetAttribute(&r, CU_FUNC_ATTRIBUTE_NUM_REGS, f);
    return r;
}

}  // namespace

std::string tune_key(const CompileRequest& rq) {
    uint64_t h = fnv1a64(rq.name);
    h = fnv1a64(rq.source, h);
    for (const auto& o : rq.options) h = fnv1a64("\x01" + o, h);
    for (const auto& k : rq.kernels) h = fnv1a64("\x02" + k, h);
    char buf[32];
    std::snprintf(buf, sizeof buf, "%016llx", (unsigned long long)h);
    return buf;
}

bool resolve_tuning(ucb_engine* e, const ucb_options& o, const std::string& key, int default_block, TuneConfig& out,
                    std::string& err) {
    if (o.block_threads != 0 && (o.block_threads < 32 || o.block_threads > 1024 || o.block_threads % 32 != 0)) {
        err = "block_threads must be 0 or a multiple of 32 in [32, 1024]";
        return false;
    }
    if (o.max_registers != 0 && (o.max_registers < 16 || o.max_registers > 255)) {
        err = "max_registers must be 0 or in [16, 255]";
        return false;
    }
    if (o.unroll != 0 && (o.unroll < 1 || o.unroll > 16)) {
        err = "unroll must be 0 or in [1, 16]";
        return false;
    }
    TuneConfig t;
    t.block = default_block;
    if (e && e->initialized) {
        load_table(e);
        auto it = e->tuned.find(key);
        if (it != e->tuned.end()) t = it->second;
    }
    out.block = o.block_threads ? o.block_threads : t.block;
    out.maxreg = o.max_registers ? o.max_registers : t.maxreg;
    out.unroll = o.unroll ? o.unroll : t.unroll;
    return true;
}

void apply_tuning(CompileRequest& rq, const TuneConfig& c) {
    std::string defs;
    if (c.block != 128) defs += "#define UCB_BLOCK " + std::to_string(c.block) + "\n";
    if (c.unroll != 1) defs += "#define UCB_UNROLL " + std::to_string(c.unroll) + "\n";
    // the cap as the number of resident blocks it allows (see UCB_LAUNCH_BOUNDS)
    if (c.maxreg > 0) defs += "#define UCB_MIN_BLOCKS " + std::to_string(min_blocks_for(c.maxreg, c.block)) + "\n";
    rq.source = defs + rq.source;
}

bool tune_request(ucb_engine* e, const ucb_options& o, int default_block, CompileRequest& rq, TuneConfig& out,
                  std::string& err) {
    if (!resolve_tuning(e, o, tune_key(rq), default_block, out, err)) return false;
    apply_tuning(rq, out);
    return true;
}

int autotune_search(ucb_engine* e, const std::string& key, int default_block, bool force,
                    const std::function<double(const TuneConfig&)>& trial,
                    const std::function<CompileRequest(const TuneConfig&)>& build, ucb_tune_report* rep,
                    const std::function<double(const TuneConfig&)>& confirm) {
    const auto t0 = std::chrono::steady_clock::now();
    std::memset(rep, 0, sizeof *rep);
    std::snprintf(rep->key, sizeof rep->key, "%s", key.c_str());
    load_table(e);
    auto describe = [&](const TuneConfig& c) {
        rep->block_threads = c.block;
        rep->max_registers = c.maxreg;
        rep->unroll = c.unroll;
        std::string err;
        const CompileRequest rq = build(c);
        auto m = e->modules.get(rq, err);
        CUfunction f = m ? main_kernel(*m, rq) : nullptr;
        if (f) {
            rep->registers = kernel_registers(f);
            int n = 0;
            if (driver().cuOccupancyMaxActiveBlocksPerMultiprocessor &&
                driver().cuOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, c.block, 0) == CUDA_SUCCESS)
                rep->blocks_per_sm = n;
        }
    };
    auto it = e->tuned.find(key);
    if (!force && it != e->tuned.end()) {
        describe(it->second);
        rep->from_table = 1;
        rep->wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return UCB_OK;
    }
    // trials pass every knob explicitly, but a register cap of 0 ("compiler's choice")
    // would pick a stored cap up again: forget the stored shape while searching
    e->tuned.erase(key);
    // one run to compile / load, then the better of two
    auto measure = [&](const TuneConfig& c) -> double {
        if (trial(c) < 0) return -1;
        const double a = trial(c), b = trial(c);
        rep->candidates += 1;
        return (a < 0 || b < 0) ? -1 : std::min(a, b);
    };
    TuneConfig best;
    best.block = default_block;
    double best_ms = measure(best);
    if (!(best_ms > 0)) {
        std::snprintf(rep->error, sizeof rep->error, "trial of the default launch shape failed: %s",
                      e->last_error.c_str());
        return UCB_E_CUDA;
    }
    rep->default_ms = best_ms;
    auto consider = [&](const TuneConfig& c) {
        if (c == best) return;
        const double ms = measure(c);
        if (ms > 0 && ms < 0.98 * best_ms) {
            best = c;
            best_ms = ms;
        }
    };
    for (int b : {64, 128, 256, 512}) {
        TuneConfig c = best;
        c.block = b;
        consider(c);
    }
    for (int u : {2, 4}) {
        TuneConfig c = best;
        c.unroll = u;
        consider(c);
    }
    // register caps at the next two occupancy steps below the build's own count
    {
        std::string err;
        const CompileRequest rq = build(best);
        auto m = e->modules.get(rq, err);
        const int regs = m ? kernel_registers(main_kernel(*m, rq)) : 0;
        if (regs > 32) {
            const TuneConfig base = best;
            int level = blocks_by_registers(regs, base.block), found = 0;
            for (int r = ((regs + 7) / 8) * 8 - 8; r >= 32 && found < 2; r -= 8) {
                const int b = blocks_by_registers(r, base.block);
                if (b > level) {
                    TuneConfig c = base;
                    c.maxreg = r;
                    consider(c);
                    level = b;
                    ++found;
                }
            }
        }
    }
    TuneConfig dflt;
    dflt.block = default_block;
    if (confirm && !(best == dflt)) {
        auto twice = [&](const TuneConfig& c) {
            const double a = confirm(c), b = confirm(c);
            return (a < 0 || b < 0) ? -1.0 : std::min(a, b);
        };
        const double dm = twice(dflt), bm = twice(best);
        rep->confirm_default_ms = dm;
        rep->confirm_best_ms = bm;
        if (!(dm > 0 && bm > 0 && bm < 0.98 * dm)) {
            best = dflt;
            best_ms = rep->default_ms;
        }
    }
    store(e, key, best, best_ms);
    rep->best_ms = best_ms;
    describe(best);
    rep->wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return UCB_OK;
}

}  // namespace ucb
