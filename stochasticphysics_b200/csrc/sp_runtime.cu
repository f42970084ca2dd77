// sp_runtime.cu — host runtime behind include/stophys_b200.h (ensembles, context, C ABI).
//
// Host code only; the kernels live in sp_k_*.cu / sp_misc.cu.  Every C entry
// point catches all C++ exceptions and turns them into an sp_status plus the
// thread-local text returned by sp_last_error().
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <limits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/stophys_b200.h"
#include "sp_dispatch.h"
#include "sp_runtime.h"

namespace sp {

thread_local std::string g_last_error;
std::atomic<unsigned long long> g_launch_count{0};

Error::Error(sp_status s, const std::string& m) : std::runtime_error(m), status(s) {}

void check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    const sp_status s = (e == cudaErrorMemoryAllocation) ? SP_ERR_OUT_OF_MEMORY : SP_ERR_CUDA;
    throw Error(s, std::string(what) + ": " + cudaGetErrorString(e));
}

sp_status fail(sp_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}

int state_dim(int p) { return p == 0 ? 3 : p == 1 ? 2 : p == 2 ? 5 : 6; }
int noise_dim(int p) { return (p == 0 || p == 1) ? 3 : 6; }
int out_dim(int p) { return p == 0 ? 3 : p == 1 ? 3 : p == 2 ? 9 : 6; }
int param_count(int p, int aniso) { return param_count_of(p, aniso); }

// sqrt(rho_p) of the double Stratonovich integral approximation (Kloeden & Platen
// 1992, sec. 5.8): rho_p = 1/12 - 1/(2 pi^2) sum_{r=1}^{p} 1/r^2; p < 1 keeps 1/12
// (DoubleNoiseMatrix.h sqrtpp<prec, p>)
double double_noise_rho(int p) {
    const double kPi = 3.14159265358979323846;
    double s = 0.0;
    for (int r = 1; r <= p; ++r) s += 1.0 / (static_cast<double>(r) * r);
    return std::sqrt(1.0 / 12.0 - s / (2.0 * kPi * kPi));
}

// ------------------------------------------------------------------ validation
sp_status validate_desc(const sp_ensemble_desc* d, std::string& why) {
    auto bad = [&](const std::string& m) { why = m; return SP_ERR_INVALID_ARG; };
    if (!d) return bad("description is NULL");
    if (d->abi_version != SP_ABI_VERSION) return bad("abi_version mismatch");
    if (d->problem < 0 || d->problem > 3) return bad("unknown problem");
    if (d->anisotropy < 0 || d->anisotropy > 2) return bad("unknown anisotropy");
    if (d->solver < 0 || d->solver > 7) return bad("unknown solver");
    if (d->precision < 0 || d->precision > 1) return bad("unknown precision");
    if (d->noise < 0 || d->noise > 1) return bad("unknown noise mode");
    if (d->field.type < 0 || d->field.type > 6) return bad("unknown field type");
    if (d->field.type >= SP_FIELD_TRIANGULAR && !(d->field.periode > 0.0 && std::isfinite(d->field.periode)))
        return bad("triangular, rectangular and sinc fields need a finite periode > 0");
    if (d->n_particles == 0) return bad("n_particles must be > 0");
    if (d->n_particles > (1ull << 31)) return bad("n_particles exceeds 2^31");
    if (d->oversampling == 0) return bad("oversampling must be > 0");
    if (d->record_trajectories < 0) return bad("record_trajectories must be >= 0 (0 = none, s = every s-th particle)");
    if (d->oversampling >= (1ull << 31)) return bad("oversampling must be < 2^31");
    if (d->number_of_steps < d->oversampling) return bad("number_of_steps must be >= oversampling");
    if (!(d->timestep > 0.0) || !std::isfinite(d->timestep)) return bad("timestep must be finite and > 0");
    if (!(d->temperature >= 0.0) || !std::isfinite(d->temperature)) return bad("temperature must be finite and >= 0");
    const sp_particles& q = d->particles;
    if (d->provider) {
        const sp_provider_desc& pv = *d->provider;
        if (pv.n_templates < 1 || pv.n_templates > 64 || !pv.templates) return bad("provider needs 1..64 templates");
        double total = 0.0;
        for (int k = 0; k < pv.n_templates; ++k) {
            const sp_particle_template& t = pv.templates[k];
            if (!(t.weight >= 0.0) || !std::isfinite(t.weight)) return bad("provider template weights must be finite and >= 0");
            total += t.weight;
            if (!(t.magnetic_radius > 0.0) || !(t.saturation_magnetisation > 0.0)) return bad("provider template needs radius and Ms > 0");
            for (const sp_dist* ds : {&t.magnetic_radius_dist, &t.hydrodynamic_shell_dist, &t.anisotropy_dist, &t.cubic_dist})
                if (ds->type < SP_DIST_DELTA || ds->type > SP_DIST_LOGNORMAL || !(ds->width >= 0.0))
                    return bad("provider template distribution: unknown type or negative width");
        }
        if (!pv.sequential && !(total > 0.0)) return bad("provider template weights must not all be zero");
    } else {
        if (!q.magnetic_radius || !q.saturation_magnetisation || !q.damping_constant || !q.gyromagnetic_ratio ||
            !q.anisotropy_constant || !q.orientation || !q.magnetisation)
            return bad("a required per-particle array is NULL");
        if ((d->problem == SP_PROBLEM_BROWN_AND_NEEL || d->problem == SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL) &&
            (!q.hydrodynamic_radius || !q.viscosity))
            return bad("Brown problems need hydrodynamic_radius and viscosity");
    }
    if (d->noise == SP_NOISE_INJECTED && !d->injected_dw) return bad("injected noise mode needs injected_dw");
    if (d->anisotropy == SP_ANISOTROPY_UNIAXIAL_CUBIC) {
        if (!d->provider && (!q.cubic_constant || !q.uniaxial_rotation))
            return bad("uniaxial+cubic anisotropy needs cubic_constant and uniaxial_rotation");
        if (d->problem == SP_PROBLEM_BROWN_AND_NEEL) {
            why = "uniaxial+cubic anisotropy is not defined for the coupled Cartesian problem (the reference's cubic "
                  "torque divides by the sine of zero Euler angles there)";
            return SP_ERR_UNSUPPORTED_COMBO;
        }
    }
    if (d->solver == SP_SOLVER_IMPLICIT_MIDPOINT) {
        if (d->problem == SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL) {
            why = "ImplicitMidpoint needs Jacobians, which BrownAndNeelEulerSpherical does not provide";
            return SP_ERR_UNSUPPORTED_COMBO;
        }
        if (d->max_iteration < 1 || d->max_iteration > 1000) return bad("ImplicitMidpoint needs 1 <= max_iteration <= 1000");
        if (!(d->accuracy_goal > 0.0)) return bad("ImplicitMidpoint needs accuracy_goal > 0");
        if (d->jacobian == SP_JACOBIAN_EXACT && d->problem != SP_PROBLEM_NEEL) {
            why = "the exact Newton Jacobian is implemented for the Neel (Cartesian) problem only";
            return SP_ERR_UNSUPPORTED_COMBO;
        }
    }
    if (d->jacobian != SP_JACOBIAN_REFERENCE && d->jacobian != SP_JACOBIAN_EXACT) return bad("unknown jacobian mode");
    if (d->solver >= SP_SOLVER_HEUN_NOT_CONSISTENT && d->noise == SP_NOISE_INJECTED) {
        why = "Heun_NotConsistent, WeakTest and ExplicitStrong_1.0 draw extra normals per step and take in-kernel "
              "(Philox) noise only";
        return SP_ERR_UNSUPPORTED_COMBO;
    }
    // RuntimeDoubleNoiseMatrixSelection accepts -1..10 (SimulationManager.h:503-525)
    if ((d->solver == SP_SOLVER_WEAK_TEST || d->solver == SP_SOLVER_EXPLICIT_STRONG_1) &&
        (d->double_noise_approx < -1 || d->double_noise_approx > 10))
        return bad("double_noise_approx must be in -1..10");
    const unsigned long long K = d->number_of_steps / d->oversampling;
    if (K > (1ull << 31)) return bad("too many samples");
    return SP_OK;
}

// ------------------------------------------------------------------ launch heuristics
LaunchConfig default_launch(const sp_context* ctx, const sp_ensemble_desc& d) {
    LaunchConfig c;
    const int sms = ctx ? ctx->sms : 148;
    int block = 256;
    const unsigned long long n = d.n_particles;
    while (block > 32 && (n + block - 1) / block < static_cast<unsigned long long>(2 * sms)) block >>= 1;
    c.block = block;
    c.persistent = 0;
    const unsigned long long W = d.oversampling;
    const unsigned long long target = 10000;
    c.chunk = W >= target ? W : (target / W) * W;
    return c;
}

// ------------------------------------------------------------------ ensemble
static unsigned long long round_up(unsigned long long x, unsigned long long m) { return (x + m - 1) / m * m; }

EnsembleLayout layout_of(const sp_ensemble_desc& d, const LaunchConfig& lc) {
    EnsembleLayout L;
    L.D = state_dim(d.problem);
    L.Mn = noise_dim(d.problem);
    L.OUT = out_dim(d.problem);
    L.P = param_count(d.problem, d.anisotropy);
    L.real = d.precision == SP_PRECISION_FP32 ? 4 : 8;
    L.n = d.n_particles;
    L.Np = round_up(L.n, kPad);
    L.W = d.oversampling;
    L.K = d.number_of_steps / d.oversampling;
    L.S = (L.K - 1) * L.W;
    L.chunk = std::max<unsigned long long>(1, std::min<unsigned long long>(lc.chunk, std::max<unsigned long long>(L.S, 1)));
    L.slots = static_cast<int>(L.chunk / L.W + 2);
    const unsigned long long nw = L.Np / 32;
    L.bytes = L.Np * ((L.real == 4 ? 2ull : 1ull) * L.D + 2ull * L.OUT + L.P) * L.real + L.Np * 8 + L.Np +
              nw * L.slots * L.OUT * 8 +
              L.K * L.OUT * 8 + L.OUT * 8 + L.K * 3 * 8 + L.chunk * 3 * L.real + sizeof(EnsCtl) + sizeof(EnsDev) +
              ((L.Np + 31) / 32 + 1) * sizeof(TileDesc);
    if (d.record_trajectories > 0) L.bytes += L.K * L.OUT * (L.n / d.record_trajectories) * 8;
    if (d.noise == SP_NOISE_INJECTED) L.bytes += L.S * L.Mn * L.Np * L.real;
    return L;
}

void* Ensemble::dalloc(size_t bytes) {
    void* p = nullptr;
    // 256-byte granularity keeps every buffer aligned for vector and TMA access
    const size_t b = (std::max<size_t>(bytes, 16) + 255) / 256 * 256;
    check_cuda(cudaMallocFromPoolAsync(&p, b, ctx->pool, stream), "cudaMallocFromPoolAsync");
    allocs.push_back(p);
    return p;
}

// Pregenerated noise.  A small ensemble leaves most SMs idle and each step's time is the
// latency of one thread's step chain, of which the FP64 Philox draw and Box-Muller (double
// log, sqrt and sincospi) are about half (Neel Heun, 1024 particles: 0.94 us per step with
// in-kernel noise, 0.43 with the increments read from memory).  With at most two warps per
// SM scheduler, an FP64 ensemble with in-kernel noise therefore draws each chunk's
// increments in a separate, fully parallel kernel (the same Philox counters and
// arithmetic, so the results are bit-identical) into a chunk-sized buffer that the
// injected step kernel stages like caller-supplied increments.
constexpr unsigned long long kPregenWarpsPerSM = 8;  // measured crossover: between 7 and 10
constexpr unsigned long long kPregenBytes = 256ull << 20;  // cap on the chunk's increments buffer

static bool pregen_wanted(const sp_context* ctx, const sp_ensemble_desc& d) {
    if (d.noise != SP_NOISE_PHILOX || d.precision != SP_PRECISION_FP64) return false;
    if (d.n_particles > kPregenWarpsPerSM * 32ull * static_cast<unsigned long long>(ctx->sms)) return false;
    const KernelSet& inj = kernel_set(d.problem, d.anisotropy, solver_slot(d.solver, d.jacobian), d.precision, 1);
    return inj.valid && inj.noise;
}

Ensemble::Ensemble(sp_context* c, const sp_ensemble_desc& d, const LaunchConfig& lc, bool chunk_graph, bool pregen_ok)
    : ctx(c), desc(d), launch(lc) {
    pregen = pregen_ok && pregen_wanted(c, d);
    ks = &kernel_set(d.problem, d.anisotropy, solver_slot(d.solver, d.jacobian), d.precision,
                     (d.noise == SP_NOISE_INJECTED || pregen) ? 1 : 0);
    if (!ks->valid) throw Error(SP_ERR_UNSUPPORTED_COMBO, "no kernel for this problem/solver combination");
    if (pregen) {  // the chunk's increments buffer stays within kPregenBytes
        const unsigned long long row = static_cast<unsigned long long>(noise_dim(d.problem)) *
                                       round_up(d.n_particles, kPad) * 8ull;
        launch.chunk = std::max<unsigned long long>(1, std::min(launch.chunk, kPregenBytes / row));
    }
    L = layout_of(d, launch);
    if (pregen) L.bytes += L.chunk * L.Mn * L.Np * L.real;
    check_cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
    check_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    check_cuda(cudaEventCreate(&ev0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&ev1), "cudaEventCreate");

    const size_t R = L.real;
    d_state = dalloc(L.Np * L.D * R);
    d_ksum = dalloc(L.Np * L.OUT * R);
    d_kcomp = dalloc(L.Np * L.OUT * R);
    if (L.real == 4) d_slo = dalloc(L.Np * L.D * R);
    d_params = dalloc(L.Np * L.P * R);
    d_moment = static_cast<double*>(dalloc(L.Np * 8));
    d_status = static_cast<unsigned char*>(dalloc(L.Np));
    d_partial = static_cast<double*>(dalloc((L.Np / 32) * L.slots * L.OUT * 8));
    d_msum = static_cast<double*>(dalloc(L.K * L.OUT * 8));
    d_wsum = static_cast<double*>(dalloc(L.OUT * 8));
    d_field = static_cast<double*>(dalloc(L.K * 3 * 8));
    d_ftab = dalloc(L.chunk * 3 * R);
    d_ctl = static_cast<EnsCtl*>(dalloc(sizeof(EnsCtl)));
    d_ens = static_cast<EnsDev*>(dalloc(sizeof(EnsDev)));
    traj_stride = d.record_trajectories > 0 ? static_cast<unsigned long long>(d.record_trajectories) : 0;
    traj_n = traj_stride ? L.n / traj_stride : 0;
    if (traj_n) d_traj = static_cast<double*>(dalloc(L.K * L.OUT * traj_n * 8));
    check_cuda(cudaMemsetAsync(d_msum, 0, L.K * L.OUT * 8, stream), "memset");
    check_cuda(cudaMemsetAsync(d_ctl, 0, sizeof(EnsCtl), stream), "memset");

    if (pregen) d_dw = dalloc(L.chunk * L.Mn * L.Np * R);  // [chunk][M][Np], written per chunk
    // injected increments: [S][M][n] FP64 host -> [S][M][Np] Real device
    if (d.noise == SP_NOISE_INJECTED && L.S > 0) {
        d_dw = dalloc(L.S * L.Mn * L.Np * R);
        const size_t rows = L.S * L.Mn;
        std::vector<unsigned char> host(rows * L.Np * R, 0);
        for (size_t r = 0; r < rows; ++r) {
            const double* src = d.injected_dw + r * L.n;
            if (R == 8) {
                std::memcpy(host.data() + r * L.Np * 8, src, L.n * 8);
            } else {
                float* dst = reinterpret_cast<float*>(host.data() + r * L.Np * 4);
                for (size_t i = 0; i < L.n; ++i) dst[i] = static_cast<float>(src[i]);
            }
        }
        check_cuda(cudaMemcpyAsync(d_dw, host.data(), host.size(), cudaMemcpyHostToDevice, stream), "upload dW");
        check_cuda(cudaStreamSynchronize(stream), "sync");
    }

    // device descriptor
    EnsDev& e = hdev;
    std::memset(&e, 0, sizeof(e));
    e.n = L.n; e.Np = L.Np; e.K = L.K; e.W = L.W; e.S = L.S; e.chunk = L.chunk;
    e.seed = d.seed; e.pid_offset = d.particle_id_offset;
    e.dt = d.timestep; e.sqrt_dt = std::sqrt(d.timestep);
    e.field = field_params(d.field);
    e.max_iter = d.max_iteration; e.tol = d.accuracy_goal;
    e.dna = d.double_noise_approx; e.rho = double_noise_rho(d.double_noise_approx);
    const double kPi = 3.14159265358979323846;
    if (d.problem == SP_PROBLEM_NEEL_SPHERICAL) {
        e.rot_brown = d.problem_settings.use_coordinate_transformation;
        e.min1 = d.problem_settings.min_angle_before_transformation;
        e.max1 = kPi - e.min1;
    } else if (d.problem == SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL) {
        e.rot_brown = d.problem_settings.use_euler_coordinate_transformation;
        e.rot_neel = d.problem_settings.use_spherical_coordinate_transformation;
        e.min1 = d.problem_settings.brown_min_angle_before_transformation;
        e.max1 = kPi - e.min1;
        e.min2 = d.problem_settings.neel_min_angle_before_transformation;
        e.max2 = kPi - e.min2;
    }
    e.slots = L.slots;
    e.state = d_state; e.ksum = d_ksum; e.kcomp = d_kcomp; e.slo = d_slo; e.params = d_params; e.moment = d_moment;
    e.dw = d_dw; e.dw_chunk = pregen ? 1 : 0; e.partial = d_partial; e.msum = d_msum; e.wsum = d_wsum; e.traj = d_traj; e.ftab = d_ftab;
    e.traj_stride = traj_stride ? traj_stride : 1; e.traj_n = traj_n;
    e.status = d_status; e.ctl = d_ctl;
    check_cuda(cudaMemcpyAsync(d_ens, &e, sizeof(EnsDev), cudaMemcpyHostToDevice, stream), "upload EnsDev");

    // tiles
    block = launch.block;
    ntiles = static_cast<int>((L.n + block - 1) / block);
    std::vector<TileDesc> tiles(ntiles);
    for (int t = 0; t < ntiles; ++t) tiles[t] = TileDesc{0u, static_cast<unsigned>(t * block)};
    d_tiles = static_cast<TileDesc*>(dalloc(tiles.size() * sizeof(TileDesc)));
    check_cuda(cudaMemcpyAsync(d_tiles, tiles.data(), tiles.size() * sizeof(TileDesc), cudaMemcpyHostToDevice, stream),
               "upload tiles");
    ppt = usable_ppt(*ks, launch.ppt, block);
    grid = ntiles;
    if (pregen)
        noise_grid = static_cast<int>(std::min<unsigned long long>((L.chunk * L.n + 255) / 256,
                                                                   8ull * static_cast<unsigned long long>(ctx->sms)));
    if (ks->prepare) ks->prepare();
    if (launch.persistent) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ks->step_fn[ppt - 1], block / ppt,
                                                      ks->dyn_smem ? ks->dyn_smem(block / ppt) : 0);
        grid = std::min(ntiles, std::max(1, per_sm) * ctx->sms);
    }

    // raw particle properties -> init kernel
    upload_and_init(d);
    if (chunk_graph) build_graph();
    check_cuda(cudaStreamSynchronize(stream), "ensemble init");
}

FieldParams field_params(const sp_field_desc& f) {
    FieldParams p;
    std::memset(&p, 0, sizeof(p));
    p.type = f.type;
    const double two_pi = 6.28318530717958647692;  // math::constants::two_pi (SinusoidalField.h:39)
    for (int i = 0; i < 3; ++i) {
        p.offset[i] = f.offset[i];
        p.amplitude[i] = f.amplitude[i];
        p.omega[i] = two_pi * (f.type == SP_FIELD_SINUSOIDAL ? f.frequency[0] : f.frequency[i]);
        p.phase[i] = f.type == SP_FIELD_SINUSOIDAL ? f.phase[0] : f.phase[i];
    }
    p.periode = f.periode;
    p.half_periode = f.periode / 2.0;
    p.time_offset = f.time_offset;
    p.sinc_a = 11.0 / (f.periode * 0.5);  // SincField.h:35
    if (f.type == SP_FIELD_RECTANGULAR) {
        // RectangularField.h:30-38: derived constants of the (alternating) waveform
        p.inv_tau = std::abs(f.tau) <= std::numeric_limits<double>::min() ? std::numeric_limits<double>::max() : 1.0 / f.tau;
        double amp[3], maxf[3], na = 0.0, nm = 0.0;
        for (int i = 0; i < 3; ++i) {
            amp[i] = f.alternating ? 2.0 * f.amplitude[i] : f.amplitude[i];
            maxf[i] = amp[i] * (-std::expm1(-p.half_periode * p.inv_tau));
            na += amp[i] * amp[i];
            nm += maxf[i] * maxf[i];
        }
        const double toff = f.alternating ? f.time_offset - std::log(1.0 - std::sqrt(nm) / (2.0 * std::sqrt(na))) * f.tau
                                          : f.time_offset;
        p.time_offset = toff;
        for (int i = 0; i < 3; ++i) {
            p.amplitude[i] = amp[i];
            p.max_field[i] = maxf[i];
            p.offset[i] = f.alternating ? amp[i] * std::expm1(-toff * p.inv_tau) + f.offset[i] : f.offset[i];
        }
    }
    return p;
}

void Ensemble::upload_and_init(const sp_ensemble_desc& d) {
    const size_t n = L.n;
    if (d.provider) {  // particles drawn on the device: nothing to upload
        double* dev = provide_particles(ctx, d, stream);
        RawParticles rp = provided_raw(dev, n);
        rp.temperature = d.temperature;
        rp.simple_model = d.problem_settings.use_simple_model;
        ks->init(d_ens, rp, L.Np, stream);
        ks->reduce(d_ens, 1, 2, 1, stream);
        launch_field_window(hdev.field, d.timestep, L.W, L.K, d_field, stream);
        check_cuda(cudaGetLastError(), "init kernels");
        launches += 4;
        g_launch_count += 3;
        check_cuda(cudaFreeAsync(dev, stream), "cudaFreeAsync");
        return;
    }
    const sp_particles& q = d.particles;
    const bool brown = d.problem == SP_PROBLEM_BROWN_AND_NEEL || d.problem == SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL;
    // one staging buffer: 7 scalars + 6 vector components per particle (+ K_cubic and the
    // uniaxial rotation for the uniaxial+cubic anisotropy), in the context's pinned buffer
    // (a pageable vector if pinned memory cannot be had)
    const bool uc = d.anisotropy == SP_ANISOTROPY_UNIAXIAL_CUBIC;
    const size_t need = n * (uc ? 17 : 13);
    std::lock_guard<std::mutex> lk(ctx->stage_mu);
    if (ctx->stage_doubles < need) {
        if (ctx->stage) cudaFreeHost(ctx->stage);
        ctx->stage = nullptr;
        ctx->stage_doubles = 0;
        if (cudaMallocHost(reinterpret_cast<void**>(&ctx->stage), need * 8) == cudaSuccess) ctx->stage_doubles = need;
        else { ctx->stage = nullptr; cudaGetLastError(); }
    }
    std::vector<double> pageable;
    double* host = ctx->stage;
    if (!host) {
        pageable.resize(need);
        host = pageable.data();
    }
    const double* src[7] = {q.magnetic_radius, q.saturation_magnetisation, q.damping_constant, q.gyromagnetic_ratio,
                            q.anisotropy_constant, brown ? q.hydrodynamic_radius : nullptr, brown ? q.viscosity : nullptr};
    for (int k = 0; k < 7; ++k) {
        if (src[k]) std::memcpy(host + k * n, src[k], n * 8);
        else std::memset(host + k * n, 0, n * 8);
    }
    std::memcpy(host + 7 * n, q.orientation, n * 24);
    std::memcpy(host + 10 * n, q.magnetisation, n * 24);
    if (uc) {
        std::memcpy(host + 13 * n, q.cubic_constant, n * 8);
        std::memcpy(host + 14 * n, q.uniaxial_rotation, n * 24);
    }
    double* dev = nullptr;
    check_cuda(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&dev), need * 8, ctx->pool, stream),
               "cudaMallocFromPoolAsync");
    check_cuda(cudaMemcpyAsync(dev, host, need * 8, cudaMemcpyHostToDevice, stream), "upload particles");
    h2d_bytes += need * 8;
    RawParticles rp;
    rp.radius = dev; rp.Ms = dev + n; rp.alpha = dev + 2 * n; rp.gamma = dev + 3 * n; rp.K = dev + 4 * n;
    rp.rh = dev + 5 * n; rp.viscosity = dev + 6 * n; rp.euler = dev + 7 * n; rp.mag = dev + 10 * n;
    rp.K2 = uc ? dev + 13 * n : nullptr;
    rp.urot = uc ? dev + 14 * n : nullptr;
    rp.temperature = d.temperature;
    rp.simple_model = d.problem_settings.use_simple_model;
    ks->init(d_ens, rp, L.Np, stream);
    ks->reduce(d_ens, 1, 2, 1, stream);
    launch_field_window(hdev.field, d.timestep, L.W, L.K, d_field, stream);
    check_cuda(cudaGetLastError(), "init kernels");
    launches += 3;
    g_launch_count += 3;
    check_cuda(cudaFreeAsync(dev, stream), "cudaFreeAsync");
    // the staging buffer must outlive the asynchronous copy (and stays locked until then)
    check_cuda(cudaStreamSynchronize(stream), "init");
}

void Ensemble::enqueue_chunk(cudaStream_t s) {
    const int midpoint = desc.solver == SP_SOLVER_IMPLICIT_MIDPOINT ? 1 : 0;
    ks->field(d_ens, 1, L.chunk, midpoint, s);
    if (pregen) ks->noise(d_ens, 1, noise_grid, s);
    ks->step[ppt - 1](d_ens, d_tiles, ntiles, grid, block, s);
    ks->reduce(d_ens, 1, L.slots, 0, s);
    launch_commit(d_ens, 1, s);
}

void Ensemble::build_graph() {
    cudaStream_t cs;
    check_cuda(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "capture stream");
    check_cuda(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture");
    enqueue_chunk(cs);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    check_cuda(ce, "end capture");
    graph = g;
    check_cuda(cudaGraphInstantiate(&gexec, graph, 0), "graph instantiate");
}

void Ensemble::advance(unsigned long long nsteps, cudaStream_t s) {
    if (!s) s = stream;
    const unsigned long long target = std::min(steps_done + nsteps, L.S);
    if (target <= steps_done) return;
    if (!gexec) build_graph();
    launch_set_target(d_ctl, target, s);
    const unsigned long long nchunks = (target - steps_done + L.chunk - 1) / L.chunk;
    check_cuda(cudaEventRecord(ev0, s), "event");
    for (unsigned long long i = 0; i < nchunks; ++i) check_cuda(cudaGraphLaunch(gexec, s), "graph launch");
    check_cuda(cudaEventRecord(ev1, s), "event");
    pending_timing = true;
    const unsigned long long per_chunk = pregen ? 5 : 4;
    launches += 1 + per_chunk * nchunks;
    g_launch_count += 1 + per_chunk * nchunks;
    particle_steps += (target - steps_done) * L.n;
    steps_done = target;
    last_stream = s;
}

void Ensemble::synchronize() {
    if (last_stream) check_cuda(cudaStreamSynchronize(last_stream), "synchronize");
    check_cuda(cudaStreamSynchronize(stream), "synchronize");
    if (pending_timing) {
        float ms = 0.f;
        check_cuda(cudaEventElapsedTime(&ms, ev0, ev1), "event time");
        device_ms += ms;
        pending_timing = false;
    }
}

// Simulator/SingleParticleSimulator.h:236-273 (times of the samples)
void reference_times(unsigned long long K, unsigned long long W, double dt, double* times) {
    if (K == 0) return;
    double start = 0.0, end = 0.0;
    const double timeshift = dt * static_cast<double>(W) * 0.5;
    times[0] = start;
    unsigned long long counter = 0;
    for (unsigned long long k = 1; k < K; ++k) {
        start = end + dt;
        counter += W;
        end = dt * static_cast<double>(counter) + start;
        times[k] = (end - start) - timeshift;
    }
}

void Ensemble::read(sp_result* out, sp_stats* st) {
    synchronize();
    EnsCtl ctl;
    check_cuda(cudaMemcpy(&ctl, d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost), "read ctl");
    if (ctl.fault) throw Error(SP_ERR_DEVICE_TIMEOUT, "a staged copy of injected increments did not arrive in time");
    const int OUT = L.OUT;
    std::vector<double> msum(L.K * OUT), wsum(OUT);
    check_cuda(cudaMemcpy(msum.data(), d_msum, msum.size() * 8, cudaMemcpyDeviceToHost), "read msum");
    check_cuda(cudaMemcpy(wsum.data(), d_wsum, OUT * 8, cudaMemcpyDeviceToHost), "read wsum");
    d2h_bytes += (msum.size() + OUT) * 8;
    if (out) {
        if (out->mean) {
            // MeanSimulationResult::normalize (Results/MeanSimulationResult.h:63-75)
            bool allzero = true;
            for (int c = 0; c < OUT; ++c) allzero = allzero && wsum[c] == 0.0;
            for (size_t k = 0; k < L.K; ++k)
                for (int c = 0; c < OUT; ++c) out->mean[k * OUT + c] = allzero ? msum[k * OUT + c] : msum[k * OUT + c] / wsum[c];
        }
        if (out->weight) std::memcpy(out->weight, wsum.data(), OUT * 8);
        if (out->weighted_sum) std::memcpy(out->weighted_sum, msum.data(), msum.size() * 8);
        if (out->time) reference_times(L.K, L.W, desc.timestep, out->time);
        if (out->field) {
            check_cuda(cudaMemcpy(out->field, d_field, L.K * 3 * 8, cudaMemcpyDeviceToHost), "read field");
            d2h_bytes += L.K * 3 * 8;
        }
        if (out->trajectories) {
            if (!traj_stride)
                throw Error(SP_ERR_INVALID_ARG, "trajectories were not recorded (record_trajectories = 0)");
            std::vector<double> t(L.K * OUT * traj_n);
            if (traj_n) check_cuda(cudaMemcpy(t.data(), d_traj, t.size() * 8, cudaMemcpyDeviceToHost), "read traj");
            d2h_bytes += t.size() * 8;
            for (size_t p = 0; p < traj_n; ++p)
                for (size_t k = 0; k < L.K; ++k)
                    for (int c = 0; c < OUT; ++c) out->trajectories[(p * L.K + k) * OUT + c] = t[(k * OUT + c) * traj_n + p];
        }
        if (out->final_state) {
            std::vector<unsigned char> s(L.D * L.Np * L.real);
            check_cuda(cudaMemcpy(s.data(), d_state, s.size(), cudaMemcpyDeviceToHost), "read state");
            d2h_bytes += s.size();
            for (size_t p = 0; p < L.n; ++p)
                for (int i = 0; i < L.D; ++i)
                    out->final_state[p * L.D + i] =
                        L.real == 8 ? reinterpret_cast<double*>(s.data())[i * L.Np + p]
                                    : static_cast<double>(reinterpret_cast<float*>(s.data())[i * L.Np + p]);
        }
    }
    if (st) {
        std::vector<unsigned char> status(L.Np);
        check_cuda(cudaMemcpy(status.data(), d_status, L.Np, cudaMemcpyDeviceToHost), "read status");
        std::memset(st, 0, sizeof(*st));
        st->particle_steps = particle_steps;
        for (size_t p = 0; p < L.n; ++p) st->nonfinite_particles += status[p] != 0;
        st->newton_iterations = ctl.newton_iterations;
        st->newton_unconverged = ctl.newton_unconverged;
        st->kernel_launches = launches;
        st->device_ms = device_ms;
    }
}

Ensemble::~Ensemble() {
    if (last_stream) cudaStreamSynchronize(last_stream);
    if (stream) cudaStreamSynchronize(stream);
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    for (void* p : allocs) cudaFreeAsync(p, stream);  // back to the context's pool
    if (stream) cudaStreamSynchronize(stream);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
}

}  // namespace sp

using namespace sp;

// ====================================================================== C ABI

extern "C" {

const char* sp_last_error(void) { return g_last_error.c_str(); }
uint32_t sp_abi_version(void) { return SP_ABI_VERSION; }
uint64_t sp_kernel_launch_count(void) { return g_launch_count.load(); }

sp_status sp_query_dims(int32_t problem, int32_t* sd, int32_t* nd, int32_t* od) {
    if (problem < 0 || problem > 3) return fail(SP_ERR_INVALID_ARG, "unknown problem");
    if (sd) *sd = state_dim(problem);
    if (nd) *nd = noise_dim(problem);
    if (od) *od = out_dim(problem);
    return SP_OK;
}

sp_status sp_validate(const sp_ensemble_desc* desc) {
    std::string why;
    const sp_status s = validate_desc(desc, why);
    return s == SP_OK ? SP_OK : fail(s, why);
}

// MeanSimulationResult::operator+= over shards (Results/MeanSimulationResult.h:87-119):
// sums and weights added in shard order, then normalize() (:63-75), which leaves the
// sums as they are when every weight is zero.
sp_status sp_merge_shards(int32_t n_shards, uint64_t n_samples, int32_t out_dim, const double* const* weighted_sums,
                          const double* const* weights, double* mean_out, double* weighted_sum_out,
                          double* weight_out) {
    SP_GUARD_BEGIN
    if (n_shards < 1) return fail(SP_ERR_INVALID_ARG, "n_shards must be at least 1");
    if (out_dim < 1 || out_dim > 9) return fail(SP_ERR_INVALID_ARG, "out_dim must be 1..9");
    if (!weighted_sums || !weights) return fail(SP_ERR_INVALID_ARG, "weighted_sums and weights are required");
    for (int32_t s = 0; s < n_shards; ++s)
        if (!weighted_sums[s] || !weights[s])
            return fail(SP_ERR_INVALID_ARG, "shard " + std::to_string(s) + " has a NULL weighted_sum or weight");
    const size_t cells = static_cast<size_t>(n_samples) * static_cast<size_t>(out_dim);
    std::vector<double> sum(cells, 0.0), w(out_dim, 0.0);
    for (int32_t s = 0; s < n_shards; ++s) {
        for (int32_t c = 0; c < out_dim; ++c) w[c] += weights[s][c];
        const double* src = weighted_sums[s];
        for (size_t i = 0; i < cells; ++i) sum[i] += src[i];
    }
    bool allzero = true;
    for (int32_t c = 0; c < out_dim; ++c) allzero = allzero && w[c] == 0.0;
    if (mean_out)
        for (size_t i = 0; i < cells; ++i) mean_out[i] = allzero ? sum[i] : sum[i] / w[i % out_dim];
    if (weighted_sum_out) std::memcpy(weighted_sum_out, sum.data(), cells * 8);
    if (weight_out) std::memcpy(weight_out, w.data(), static_cast<size_t>(out_dim) * 8);
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_create(sp_context** out, int32_t device) {
    SP_GUARD_BEGIN
    if (!out) return fail(SP_ERR_INVALID_ARG, "ctx pointer is NULL");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return fail(SP_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= count) return fail(SP_ERR_INVALID_ARG, "device index out of range");
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    auto* c = new sp_context();
    c->device = device;
    cudaDeviceProp prop;
    check_cuda(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    c->sms = prop.multiProcessorCount;
    c->total_mem = prop.totalGlobalMem;
    c->cc_major = prop.major;
    c->cc_minor = prop.minor;
    check_cuda(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    check_cuda(cudaMemPoolCreate(&c->pool, &props), "cudaMemPoolCreate");
    uint64_t keep = UINT64_MAX;
    check_cuda(cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
    *out = c;
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_destroy(sp_context* ctx) {
    SP_GUARD_BEGIN
    if (!ctx) return SP_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
    if (ctx->pool) {
        cudaDeviceSynchronize();  // frees issued on ensemble streams have reached the pool
        cudaMemPoolDestroy(ctx->pool);
    }
    if (ctx->stage) cudaFreeHost(ctx->stage);
    delete ctx;
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_ensemble_footprint(const sp_ensemble_desc* desc, uint64_t* bytes) {
    SP_GUARD_BEGIN
    std::string why;
    const sp_status s = validate_desc(desc, why);
    if (s != SP_OK) return fail(s, why);
    if (bytes) *bytes = layout_of(*desc, default_launch(nullptr, *desc)).bytes;
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_ensemble_create(sp_context* ctx, const sp_ensemble_desc* desc, sp_ensemble** ens) {
    SP_GUARD_BEGIN
    if (!ctx || !ens) return fail(SP_ERR_INVALID_ARG, "NULL argument");
    std::string why;
    const sp_status s = validate_desc(desc, why);
    if (s != SP_OK) return fail(s, why);
    auto* e = new Ensemble(ctx, *desc, launch_config_for(ctx, *desc));
    *ens = reinterpret_cast<sp_ensemble*>(e);
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_ensemble_create_shaped(sp_context* ctx, const sp_ensemble_desc* desc, const sp_launch_config* shape,
                                    sp_ensemble** ens) {
    SP_GUARD_BEGIN
    if (!shape) return sp_ensemble_create(ctx, desc, ens);
    if (!ens) return fail(SP_ERR_INVALID_ARG, "ens is NULL");
    std::string why;
    const sp_status s = validate_desc(desc, why);
    if (s != SP_OK) return fail(s, why);
    // the shape is checked before the context, so hosts can check it without a device
    const int b = shape->block;
    if (b != 32 && b != 64 && b != 128 && b != 256) return fail(SP_ERR_INVALID_ARG, "shape.block must be 32, 64, 128 or 256");
    if (shape->persistent != 0 && shape->persistent != 1) return fail(SP_ERR_INVALID_ARG, "shape.persistent must be 0 or 1");
    if (shape->chunk_steps < 1) return fail(SP_ERR_INVALID_ARG, "shape.chunk_steps must be at least 1");
    if (shape->particles_per_thread != 1 && shape->particles_per_thread != 2)
        return fail(SP_ERR_INVALID_ARG, "shape.particles_per_thread must be 1 or 2");
    if (!ctx) return fail(SP_ERR_INVALID_ARG, "ctx is NULL");
    LaunchConfig lc;
    lc.block = b;
    lc.persistent = shape->persistent;
    const unsigned long long W = desc->oversampling;
    lc.chunk = shape->chunk_steps <= W ? W : shape->chunk_steps / W * W;
    lc.ppt = shape->particles_per_thread;
    auto* e = new Ensemble(ctx, *desc, lc);
    *ens = reinterpret_cast<sp_ensemble*>(e);
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_ensemble_advance(sp_ensemble* ens, uint64_t n_steps, void* cuda_stream) {
    SP_GUARD_BEGIN
    if (!ens) return fail(SP_ERR_INVALID_ARG, "NULL ensemble");
    auto* e = reinterpret_cast<Ensemble*>(ens);
    check_cuda(cudaSetDevice(e->ctx->device), "cudaSetDevice");
    e->advance(n_steps, static_cast<cudaStream_t>(cuda_stream));
    check_cuda(cudaGetLastError(), "advance");
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_ensemble_steps_done(const sp_ensemble* ens, uint64_t* done, uint64_t* total) {
    if (!ens) return fail(SP_ERR_INVALID_ARG, "NULL ensemble");
    auto* e = reinterpret_cast<const Ensemble*>(ens);
    if (done) *done = e->steps_done;
    if (total) *total = e->L.S;
    return SP_OK;
}

sp_status sp_ensemble_read(sp_ensemble* ens, sp_result* out, sp_stats* stats) {
    SP_GUARD_BEGIN
    if (!ens) return fail(SP_ERR_INVALID_ARG, "NULL ensemble");
    auto* e = reinterpret_cast<Ensemble*>(ens);
    check_cuda(cudaSetDevice(e->ctx->device), "cudaSetDevice");
    e->read(out, stats);
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_ensemble_destroy(sp_ensemble* ens) {
    SP_GUARD_BEGIN
    if (!ens) return SP_OK;
    auto* e = reinterpret_cast<Ensemble*>(ens);
    cudaSetDevice(e->ctx->device);
    delete e;
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_simulate(sp_context* ctx, const sp_ensemble_desc* desc, sp_result* out, sp_stats* stats) {
    SP_GUARD_BEGIN
    if (!ctx) return fail(SP_ERR_INVALID_ARG, "NULL context");
    std::string why;
    const sp_status s = validate_desc(desc, why);
    if (s != SP_OK) return fail(s, why);
    sp_ensemble_desc d = *desc;
    if (out && out->trajectories && d.record_trajectories == 0) d.record_trajectories = 1;
    using Clock = std::chrono::steady_clock;
    const auto ms = [](Clock::time_point a, Clock::time_point b) {
        return std::chrono::duration<double, std::milli>(b - a).count();
    };
    const Clock::time_point t0 = Clock::now();
    Ensemble e(ctx, d, launch_config_for(ctx, d));
    const Clock::time_point t1 = Clock::now();
    e.advance(e.L.S, nullptr);
    e.synchronize();
    const Clock::time_point t2 = Clock::now();
    e.read(out, stats);
    if (stats) {
        stats->setup_ms = ms(t0, t1);
        stats->run_ms = ms(t1, t2);
        stats->readback_ms = ms(t2, Clock::now());
    }
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_debug_philox_normals(sp_context* ctx, uint64_t seed, uint64_t pid, uint64_t n, uint64_t step0,
                                  uint64_t nsteps, int32_t noise_dim, int32_t precision, double* out) {
    SP_GUARD_BEGIN
    if (!ctx || !out) return fail(SP_ERR_INVALID_ARG, "NULL argument");
    if (noise_dim != 3 && noise_dim != 6) return fail(SP_ERR_INVALID_ARG, "noise_dim must be 3 or 6");
    if (precision != 0 && precision != 1) return fail(SP_ERR_INVALID_ARG, "unknown precision");
    if (n == 0 || nsteps == 0) return SP_OK;
    check_cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
    const size_t bytes = n * nsteps * noise_dim * 8;
    double* d = nullptr;
    check_cuda(cudaMalloc(&d, bytes), "cudaMalloc");
    launch_debug_normals(seed, pid, n, step0, nsteps, noise_dim, precision, d, ctx->stream);
    g_launch_count += 1;
    cudaError_t e1 = cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    check_cuda(e1, "copy normals");
    check_cuda(e2, "normals kernel");
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_measure_fma_peak(sp_context* ctx, int32_t precision, double* tflops) {
    SP_GUARD_BEGIN
    if (!ctx || !tflops) return fail(SP_ERR_INVALID_ARG, "NULL argument");
    if (precision != 0 && precision != 1) return fail(SP_ERR_INVALID_ARG, "unknown precision");
    check_cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
    *tflops = measure_fma_peak(precision, ctx->sms, ctx->stream);
    g_launch_count += 4;
    return SP_OK;
    SP_GUARD_END
}

}  // extern "C"
