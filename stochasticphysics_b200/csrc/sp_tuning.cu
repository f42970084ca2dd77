// sp_tuning.cu — launch configuration per kernel key: defaults, the autotuner
// and its cache, and environment overrides (SP_BLOCK, SP_CHUNK, SP_PERSISTENT, SP_PPT).
//
// The autotuner times candidate launch shapes on a probe ensemble (a prefix of
// the caller's particles) with CUDA events and keeps the fastest per kernel key
// (problem, anisotropy, solver, precision, noise).  Shapes: tile size 64/128/256
// particles (the step kernel is register-bound, so tile size moves occupancy and
// tail effects), one or two particles per thread (FP32: two independent step
// chains per thread), persistent grid or one CTA per tile, and the
// chunk length of the captured graph (per-chunk kernels: field table, window
// reduction, commit).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "sp_runtime.h"

namespace sp {

namespace {
std::mutex g_tune_mu;
std::unordered_map<std::string, LaunchConfig> g_tuned;
std::unordered_map<std::string, double> g_tuned_rate;

std::string key_of(const sp_ensemble_desc& d) {
    return std::to_string(d.problem) + "/" + std::to_string(d.anisotropy) + "/" +
           std::to_string(solver_slot(d.solver, d.jacobian)) + "/" + std::to_string(d.precision) + "/" +
           std::to_string(d.noise);
}

unsigned long long round_chunk(unsigned long long chunk, unsigned long long W) {
    return W >= chunk ? W : (chunk / W) * W;
}
}  // namespace

void store_tuned(const sp_ensemble_desc& d, const LaunchConfig& c) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[key_of(d)] = c;
}

bool lookup_tuned(const sp_ensemble_desc& d, LaunchConfig& c) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(key_of(d));
    if (it == g_tuned.end()) return false;
    c = it->second;
    return true;
}

double tuned_rate(const sp_ensemble_desc& d) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned_rate.find(key_of(d));
    return it == g_tuned_rate.end() ? 0.0 : it->second;
}

LaunchConfig launch_config_for(const sp_context* ctx, const sp_ensemble_desc& d) {
    LaunchConfig c = default_launch(ctx, d);
    LaunchConfig t;
    if (lookup_tuned(d, t)) {
        c.block = t.block;
        c.persistent = t.persistent;
        c.ppt = t.ppt;
        if (t.chunk) c.chunk = round_chunk(t.chunk, d.oversampling);
        // small ensembles keep enough CTAs to cover the SMs
        const int sms = ctx ? ctx->sms : 148;
        while (c.block > 32 && (d.n_particles + c.block - 1) / c.block < static_cast<unsigned long long>(sms)) c.block >>= 1;
    }
    if (const char* s = std::getenv("SP_BLOCK")) {
        const int b = std::atoi(s);
        if (b == 32 || b == 64 || b == 128 || b == 256) c.block = b;
    }
    if (const char* s = std::getenv("SP_CHUNK")) {
        const long long v = std::atoll(s);
        if (v > 0) c.chunk = static_cast<unsigned long long>(v);
    }
    if (const char* s = std::getenv("SP_PERSISTENT")) c.persistent = std::atoi(s) != 0;
    if (const char* s = std::getenv("SP_PPT")) c.ppt = std::atoi(s) == 2 ? 2 : 1;
    const KernelSet& ks = kernel_set(d.problem, d.anisotropy, solver_slot(d.solver, d.jacobian), d.precision,
                                     d.noise == SP_NOISE_INJECTED ? 1 : 0);
    c.ppt = usable_ppt(ks, c.ppt, c.block);
    return c;
}

namespace {
// particle-steps/s of one shape on the probe: one warm-up chunk (first graph
// launch, caches), then `timed` steps between CUDA events on the probe's stream
double time_shape(sp_context* ctx, const sp_ensemble_desc& probe, const LaunchConfig& lc, unsigned long long timed) {
    Ensemble e(ctx, probe, lc, true, false);  // the in-kernel noise path the shape is tuned for
    e.advance(e.L.chunk, nullptr);
    e.synchronize();
    e.device_ms = 0.0;
    const unsigned long long before = e.particle_steps;
    e.advance(timed, nullptr);
    e.synchronize();
    const double ps = static_cast<double>(e.particle_steps - before);
    return e.device_ms > 0.0 ? ps / (e.device_ms * 1e-3) : 0.0;
}

void to_c(const LaunchConfig& c, double rate, sp_launch_config* o) {
    o->block = c.block;
    o->persistent = c.persistent;
    o->chunk_steps = c.chunk;
    o->particle_steps_per_s = rate;
    o->particles_per_thread = c.ppt;
    o->reserved0 = 0;
}
}  // namespace

}  // namespace sp

using namespace sp;

sp_status sp_autotune(sp_context* ctx, const sp_ensemble_desc* desc, uint64_t probe_particles, sp_launch_config* best,
                      sp_launch_config* candidates, int32_t max_candidates, int32_t* n_candidates) {
    SP_GUARD_BEGIN
    if (!ctx) return fail(SP_ERR_INVALID_ARG, "ctx is NULL");
    std::string why;
    const sp_status s = validate_desc(desc, why);
    if (s != SP_OK) return fail(s, why);
    if (desc->noise == SP_NOISE_INJECTED) return fail(SP_ERR_INVALID_ARG, "autotune needs in-kernel (Philox) noise");
    check_cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
    const unsigned long long W = desc->oversampling;
    const unsigned long long c0 = default_launch(ctx, *desc).chunk;
    const unsigned long long c_long = round_chunk(4 * c0, W);
    sp_ensemble_desc probe = *desc;
    probe.n_particles = std::min<unsigned long long>(desc->n_particles, probe_particles ? probe_particles : 65536ull);
    probe.record_trajectories = 0;
    // room for a warm-up chunk and a timed stretch of the longest candidate chunk
    const unsigned long long need = 2 * std::max(c0, c_long);
    probe.number_of_steps = (need / W + 2) * W;

    std::vector<std::pair<LaunchConfig, double>> timed;
    auto run = [&](const LaunchConfig& lc) {
        const double r = time_shape(ctx, probe, lc, std::max(c0, lc.chunk));
        timed.emplace_back(lc, r);
        return r;
    };
    // CTA size x grid form at the default chunk, then the chunk length for the winner
    LaunchConfig win;
    double win_rate = -1.0;
    const KernelSet& ks = kernel_set(desc->problem, desc->anisotropy, solver_slot(desc->solver, desc->jacobian),
                                     desc->precision, 0);
    const int max_ppt = ks.step[1] ? 2 : 1;
    for (int ppt = 1; ppt <= max_ppt; ++ppt)
        for (int persistent = 0; persistent <= 1; ++persistent)
            for (int block : {64, 128, 256}) {
                if ((probe.n_particles + block - 1) / block < static_cast<unsigned long long>(ctx->sms) && block > 64) continue;
                LaunchConfig lc;
                lc.block = block;
                lc.persistent = persistent;
                lc.chunk = c0;
                lc.ppt = ppt;
                const double r = run(lc);
                if (r > win_rate) { win = lc; win_rate = r; }
            }
    // Chunk length for the winning shape: a tenth and a fifth of the default, the default
    // and four times it.  Each chunk launch ends with its CTAs draining; ensembles advanced
    // on other streams (and the server's other groups) fill the SMs so freed only between
    // chunks, so a short chunk costs little alone and lets concurrent launches interleave
    // (two 65536-particle Brown+Neel ensembles side by side run 15 % faster with 1000-step
    // chunks than with 10000).  The shortest chunk within kChunkSlack of the best rate on
    // the probe is kept.
    constexpr double kChunkSlack = 0.98;
    std::vector<std::pair<unsigned long long, double>> by_chunk{{c0, win_rate}};
    for (const unsigned long long c : {round_chunk(c0 / 10, W), round_chunk(c0 / 5, W), c_long}) {
        bool seen = false;
        for (const auto& bc : by_chunk) seen = seen || bc.first == c;
        if (seen) continue;
        LaunchConfig lc = win;
        lc.chunk = c;
        by_chunk.emplace_back(c, run(lc));
    }
    double best_rate = 0.0;
    for (const auto& bc : by_chunk) best_rate = std::max(best_rate, bc.second);
    unsigned long long pick = 0;
    for (const auto& bc : by_chunk)
        if (bc.second >= kChunkSlack * best_rate && (pick == 0 || bc.first < pick)) {
            pick = bc.first;
            win_rate = bc.second;
        }
    win.chunk = pick;
    store_tuned(*desc, win);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned_rate[key_of(*desc)] = win_rate;
    }
    if (best) to_c(win, win_rate, best);
    const int nt = static_cast<int>(timed.size());
    if (candidates)
        for (int i = 0; i < std::min(nt, static_cast<int>(max_candidates)); ++i) to_c(timed[i].first, timed[i].second, &candidates[i]);
    if (n_candidates) *n_candidates = nt;
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_launch_config_for(sp_context* ctx, const sp_ensemble_desc* desc, sp_launch_config* out) {
    SP_GUARD_BEGIN
    if (!out) return fail(SP_ERR_INVALID_ARG, "out is NULL");
    std::string why;
    const sp_status s = validate_desc(desc, why);
    if (s != SP_OK) return fail(s, why);
    const LaunchConfig c = launch_config_for(ctx, *desc);
    double rate = 0.0;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned_rate.find(key_of(*desc));
        if (it != g_tuned_rate.end()) rate = it->second;
    }
    to_c(c, rate, out);
    return SP_OK;
    SP_GUARD_END
}

// "problem/anisotropy/solver/precision/noise block persistent chunk rate ppt" per line
// (a line without ppt reads as one particle per thread)
sp_status sp_tuning_save(const char* path) {
    SP_GUARD_BEGIN
    if (!path) return fail(SP_ERR_INVALID_ARG, "path is NULL");
    std::ofstream f(path);
    if (!f) return fail(SP_ERR_INVALID_ARG, std::string("cannot write ") + path);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const auto& kv : g_tuned) {
        auto r = g_tuned_rate.find(kv.first);
        f << kv.first << ' ' << kv.second.block << ' ' << kv.second.persistent << ' ' << kv.second.chunk << ' '
          << (r == g_tuned_rate.end() ? 0.0 : r->second) << ' ' << kv.second.ppt << '\n';
    }
    return f.good() ? SP_OK : fail(SP_ERR_INVALID_ARG, std::string("write failed: ") + path);
    SP_GUARD_END
}

sp_status sp_tuning_load(const char* path) {
    SP_GUARD_BEGIN
    if (!path) return fail(SP_ERR_INVALID_ARG, "path is NULL");
    std::ifstream f(path);
    if (!f) return fail(SP_ERR_INVALID_ARG, std::string("cannot read ") + path);
    std::string line;
    std::vector<std::pair<std::string, std::pair<LaunchConfig, double>>> rows;
    while (std::getline(f, line)) {
        if (line.empty()) continue;
        std::istringstream is(line);
        std::string key;
        LaunchConfig c;
        double rate = 0.0;
        if (!(is >> key >> c.block >> c.persistent >> c.chunk)) return fail(SP_ERR_INVALID_ARG, "malformed line: " + line);
        is >> rate;
        if (!(is >> c.ppt)) c.ppt = 1;
        int parts[5];
        if (std::sscanf(key.c_str(), "%d/%d/%d/%d/%d", &parts[0], &parts[1], &parts[2], &parts[3], &parts[4]) != 5)
            return fail(SP_ERR_INVALID_ARG, "malformed key: " + key);
        if (!(c.block == 32 || c.block == 64 || c.block == 128 || c.block == 256) || c.chunk == 0 ||
            !(c.ppt == 1 || c.ppt == 2))
            return fail(SP_ERR_INVALID_ARG, "invalid launch shape: " + line);
        rows.push_back({key, {c, rate}});
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const auto& r : rows) {
        g_tuned[r.first] = r.second.first;
        g_tuned_rate[r.first] = r.second.second;
    }
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_tuning_reset(void) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned.clear();
    g_tuned_rate.clear();
    return SP_OK;
}
