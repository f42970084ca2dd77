// sp_runtime.h — internal host-side declarations shared by the runtime units.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/stophys_b200.h"
#include "sp_dispatch.h"
#include "sp_types.h"

struct sp_context {
    int device = 0;
    int sms = 148;
    int cc_major = 0, cc_minor = 0;
    size_t total_mem = 0;
    cudaStream_t stream = nullptr;
    // every ensemble's device buffers come from this pool; freed memory stays in it
    // (release threshold = max), so repeated runs and server requests reuse it
    // instead of paying for cudaMalloc / cudaFree each time
    cudaMemPool_t pool = nullptr;
    // pinned host staging for particle uploads, grown on demand and reused across calls
    // (pageable copies go through the driver's own bounce buffers at a fraction of the
    // bandwidth); callers uploading at the same time take turns on the mutex
    std::mutex stage_mu;
    double* stage = nullptr;
    size_t stage_doubles = 0;
};

namespace sp {

struct Error : std::runtime_error {
    sp_status status;
    Error(sp_status s, const std::string& m);
};

extern thread_local std::string g_last_error;
extern std::atomic<unsigned long long> g_launch_count;

void check_cuda(cudaError_t e, const char* what);
inline void launches_add(unsigned long long n) { g_launch_count += n; }
sp_status fail(sp_status s, const std::string& msg);
sp_status validate_desc(const sp_ensemble_desc* d, std::string& why);
int state_dim(int p);
int noise_dim(int p);
int out_dim(int p);
int param_count(int p, int aniso);
double double_noise_rho(int p);
FieldParams field_params(const sp_field_desc& f);
void reference_times(unsigned long long K, unsigned long long W, double dt, double* times);

// launch shape of one kernel key: CTA size, persistent grid, steps per chunk
struct LaunchConfig {
    int block = 128;       // particles per tile
    int persistent = 0;
    unsigned long long chunk = 10000;
    int ppt = 1;           // particles per thread: the CTA has block / ppt threads
};
// the particles per thread a kernel set and tile size allow (2 needs the FP32 kernel and
// at least one warp per CTA)
inline int usable_ppt(const KernelSet& ks, int ppt, int block) {
    return (ppt == 2 && ks.step[1] && block >= 64) ? 2 : 1;
}
LaunchConfig default_launch(const sp_context* ctx, const sp_ensemble_desc& d);
// default_launch refined by the autotuner cache and SP_BLOCK / SP_CHUNK / SP_PERSISTENT
LaunchConfig launch_config_for(const sp_context* ctx, const sp_ensemble_desc& d);
// particle-steps/s the autotuner measured for d's kernel key (0 when untuned)
double tuned_rate(const sp_ensemble_desc& d);

struct EnsembleLayout {
    int D = 0, Mn = 0, OUT = 0, P = 0, real = 8, slots = 2;
    unsigned long long n = 0, Np = 0, W = 1, K = 0, S = 0, chunk = 1;
    unsigned long long bytes = 0;
};
EnsembleLayout layout_of(const sp_ensemble_desc& d, const LaunchConfig& lc);

// device-side provider (sp_provider.cu): draws the particles of d into a pooled
// [18][n] buffer on stream s (the caller frees it); provided_raw views it
double* provide_particles(sp_context* ctx, const sp_ensemble_desc& d, cudaStream_t s);
RawParticles provided_raw(const double* dev, unsigned long long n);

// One device-resident ensemble (one reference "simulation" of n particles).
struct Ensemble {
    sp_context* ctx;
    sp_ensemble_desc desc;  // host pointers are not used after construction
    LaunchConfig launch;
    const KernelSet* ks = nullptr;
    EnsembleLayout L;
    cudaStream_t stream = nullptr, last_stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    bool pending_timing = false;
    double device_ms = 0.0;
    unsigned long long launches = 0, particle_steps = 0, steps_done = 0;
    unsigned long long h2d_bytes = 0, d2h_bytes = 0;
    int block = 128, grid = 1, ntiles = 0, ppt = 1;
    bool pregen = false;  // pregenerated noise: a noise kernel per chunk, the injected step kernel
    int noise_grid = 1;
    unsigned long long traj_stride = 0, traj_n = 0;  // recorded particles: every traj_stride-th, traj_n of them
    EnsDev hdev;
    void *d_state = nullptr, *d_ksum = nullptr, *d_kcomp = nullptr, *d_slo = nullptr, *d_params = nullptr, *d_dw = nullptr,
         *d_ftab = nullptr;
    double *d_moment = nullptr, *d_partial = nullptr, *d_msum = nullptr, *d_wsum = nullptr, *d_traj = nullptr,
           *d_field = nullptr;
    unsigned char* d_status = nullptr;
    EnsCtl* d_ctl = nullptr;
    EnsDev* d_ens = nullptr;
    TileDesc* d_tiles = nullptr;
    std::vector<void*> allocs;

    // chunk_graph: capture the ensemble's own chunk graph now (the server launches its
    // groups' graphs instead and passes false; advance() then captures it on first use).
    // pregen_ok: a small FP64 ensemble with in-kernel noise may pregenerate each chunk's
    // increments (pregen_wanted); the server's groups and the autotuner's probes pass false.
    Ensemble(sp_context* c, const sp_ensemble_desc& d, const LaunchConfig& lc, bool chunk_graph = true,
             bool pregen_ok = true);
    ~Ensemble();
    Ensemble(const Ensemble&) = delete;
    Ensemble& operator=(const Ensemble&) = delete;

    void* dalloc(size_t bytes);
    void upload_and_init(const sp_ensemble_desc& d);
    void enqueue_chunk(cudaStream_t s);
    void build_graph();
    void advance(unsigned long long nsteps, cudaStream_t s);
    void synchronize();
    void read(sp_result* out, sp_stats* st);
};

}  // namespace sp

// every C entry point: no exception crosses the ABI
#define SP_GUARD_BEGIN try {
#define SP_GUARD_END                                                                                   \
    }                                                                                                  \
    catch (const sp::Error& e) { return sp::fail(e.status, e.what()); }                                \
    catch (const std::bad_alloc&) { return sp::fail(SP_ERR_OUT_OF_MEMORY, "host allocation failed"); } \
    catch (const std::exception& e) { return sp::fail(SP_ERR_CUDA, e.what()); }
