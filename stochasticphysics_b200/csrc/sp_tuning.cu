// sp_tuning.cu — launch configuration per kernel key: defaults, the autotuner
// cache and environment overrides (SP_BLOCK, SP_CHUNK, SP_PERSISTENT).
#include <cstdlib>
#include <mutex>
#include <string>
#include <unordered_map>

#include "sp_runtime.h"

namespace sp {

namespace {
std::mutex g_tune_mu;
std::unordered_map<std::string, LaunchConfig> g_tuned;

std::string key_of(const sp_ensemble_desc& d) {
    return std::to_string(d.problem) + "/" + std::to_string(d.anisotropy) + "/" + std::to_string(d.solver) + "/" +
           std::to_string(d.precision) + "/" + std::to_string(d.noise);
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

LaunchConfig launch_config_for(const sp_context* ctx, const sp_ensemble_desc& d) {
    LaunchConfig c = default_launch(ctx, d);
    LaunchConfig t;
    if (lookup_tuned(d, t)) {
        c.block = t.block;
        c.persistent = t.persistent;
        if (t.chunk) c.chunk = (d.oversampling >= t.chunk) ? d.oversampling : (t.chunk / d.oversampling) * d.oversampling;
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
    return c;
}

}  // namespace sp
