// sp_noalloc.cu — sp_simulate_noalloc: an ensemble run that allocates no device memory.
//
// Some hosts cannot let a plug-in allocate GPU memory while they run: they hand
// it device buffers from their own pre-reserved pool (real-time or embedded
// control loops, hosts that account every byte of device memory, sandboxes that
// forbid cudaMalloc after start-up).  This entry point serves them.  The caller
// passes the per-particle inputs and the result buffers in device memory; every
// internal buffer (state, Kahan sums, prefactors, per-warp window partials, the
// field table, the control block, the work list) is carved out of one
// file-scope array, kNoAllocScratchBytes = 32 MiB, that every GPU which loads
// the library holds until the process exits.  Requests that need more scratch
// are refused with SP_ERR_INVALID_ARG and the byte counts.
//
// Set-up: the first call on each device resolves the array's device address
// with cudaGetSymbolAddress (with that device current) and caches it; make that
// first call before any stream capture begins.  The cached address belongs to the
// device's current context: after cudaDeviceReset (or any teardown of the primary
// context) the library must be reloaded before this entry point is used again.
// All calls share the array and each call re-initialises what it uses, so calls
// whose work overlaps on the GPU (different streams or threads at once) race;
// serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "sp_runtime.h"

namespace sp {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {};

// the ensemble descriptor and the tile list: the descriptor travels as a kernel
// argument (copied when the launch is issued), so nothing is read from host memory
// after the call returns
__global__ void noalloc_setup_kernel(EnsDev* dst, EnsDev e, TileDesc* tiles, int ntiles, int block) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *dst = e;
    if (i < ntiles) tiles[i] = TileDesc{0u, static_cast<unsigned>(i * block)};
}

// MeanSimulationResult::normalize (Results/MeanSimulationResult.h:63-75), in place
__global__ void noalloc_normalize_kernel(double* mean, const double* weight, unsigned long long K, int OUT) {
    const unsigned long long i = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= K * OUT) return;
    bool allzero = true;
    for (int c = 0; c < OUT; ++c) allzero = allzero && weight[c] == 0.0;
    if (!allzero) mean[i] = mean[i] / weight[i % OUT];
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

void* scratch_base(int device) {
    if (device < 0 || device >= 64) throw Error(SP_ERR_INVALID_ARG, "device index out of range for the scratch table");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw Error(SP_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_noalloc_addr[device] = p;
    }
    return g_noalloc_addr[device];
}

}  // namespace
}  // namespace sp

using namespace sp;

extern "C" SP_API sp_status sp_simulate_noalloc(const sp_ensemble_desc* desc, const sp_particles* device_particles,
                                                double* device_mean, double* device_weight, void* cuda_stream) {
    try {
        std::string why;
        const sp_status vs = validate_desc(desc, why);
        if (vs != SP_OK) return fail(vs, why);
        if (!device_particles || !device_mean || !device_weight)
            return fail(SP_ERR_INVALID_ARG, "device_particles, device_mean and device_weight are required");
        if (desc->noise == SP_NOISE_INJECTED)
            return fail(SP_ERR_INVALID_ARG, "sp_simulate_noalloc draws its noise in-kernel (SP_NOISE_PHILOX only)");
        if (desc->record_trajectories) return fail(SP_ERR_INVALID_ARG, "sp_simulate_noalloc keeps no trajectories");
        if (desc->provider) return fail(SP_ERR_INVALID_ARG, "sp_simulate_noalloc takes its particles from device_particles");
        const sp_particles& dp = *device_particles;
        const bool brown = desc->problem == SP_PROBLEM_BROWN_AND_NEEL || desc->problem == SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL;
        if (!dp.magnetic_radius || !dp.saturation_magnetisation || !dp.damping_constant || !dp.gyromagnetic_ratio ||
            !dp.anisotropy_constant || !dp.orientation || !dp.magnetisation || (brown && (!dp.hydrodynamic_radius || !dp.viscosity)) ||
            (desc->anisotropy == SP_ANISOTROPY_UNIAXIAL_CUBIC && (!dp.cubic_constant || !dp.uniaxial_rotation)))
            return fail(SP_ERR_INVALID_ARG, "a required device per-particle array is NULL");

        int device = 0;
        check_cuda(cudaGetDevice(&device), "cudaGetDevice");
        sp_context c;
        c.device = device;
        check_cuda(cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
        const LaunchConfig lc = default_launch(&c, *desc);
        const EnsembleLayout L = layout_of(*desc, lc);
        const KernelSet& ks = kernel_set(desc->problem, desc->anisotropy, solver_slot(desc->solver, desc->jacobian),
                                         desc->precision, 0);
        if (!ks.valid) return fail(SP_ERR_UNSUPPORTED_COMBO, "no kernel for this problem/solver combination");

        // carve the scratch
        const size_t R = L.real;
        const int ntiles = static_cast<int>((L.n + lc.block - 1) / lc.block);
        size_t off = 0;
        auto take = [&](size_t bytes) { const size_t at = off; off += align256(bytes); return at; };
        const size_t o_ens = take(sizeof(EnsDev)), o_ctl = take(sizeof(EnsCtl)), o_tiles = take(ntiles * sizeof(TileDesc));
        const size_t o_state = take(L.Np * L.D * R), o_ksum = take(L.Np * L.OUT * R), o_kcomp = take(L.Np * L.OUT * R);
        const size_t o_slo = R == 4 ? take(L.Np * L.D * R) : 0;
        const size_t o_params = take(L.Np * L.P * R), o_moment = take(L.Np * 8), o_status = take(L.Np);
        const size_t o_partial = take((L.Np / 32) * L.slots * L.OUT * 8), o_ftab = take(L.chunk * 3 * R);
        if (off > kNoAllocScratchBytes)
            return fail(SP_ERR_INVALID_ARG, "ensemble needs " + std::to_string(off) + " bytes of scratch; the static scratch of "
                                                "sp_simulate_noalloc holds " + std::to_string(kNoAllocScratchBytes) + " bytes");

        unsigned char* base = static_cast<unsigned char*>(scratch_base(device));
        cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);

        EnsDev e;
        std::memset(&e, 0, sizeof(e));
        e.n = L.n; e.Np = L.Np; e.K = L.K; e.W = L.W; e.S = L.S; e.chunk = L.chunk;
        e.seed = desc->seed; e.pid_offset = desc->particle_id_offset;
        e.dt = desc->timestep; e.sqrt_dt = std::sqrt(desc->timestep);
        e.field = field_params(desc->field);
        e.max_iter = desc->max_iteration; e.tol = desc->accuracy_goal;
        e.dna = desc->double_noise_approx; e.rho = double_noise_rho(desc->double_noise_approx);
        const double kPi = 3.14159265358979323846;
        if (desc->problem == SP_PROBLEM_NEEL_SPHERICAL) {
            e.rot_brown = desc->problem_settings.use_coordinate_transformation;
            e.min1 = desc->problem_settings.min_angle_before_transformation;
            e.max1 = kPi - e.min1;
        } else if (desc->problem == SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL) {
            e.rot_brown = desc->problem_settings.use_euler_coordinate_transformation;
            e.rot_neel = desc->problem_settings.use_spherical_coordinate_transformation;
            e.min1 = desc->problem_settings.brown_min_angle_before_transformation;
            e.max1 = kPi - e.min1;
            e.min2 = desc->problem_settings.neel_min_angle_before_transformation;
            e.max2 = kPi - e.min2;
        }
        e.slots = L.slots;
        e.state = base + o_state; e.ksum = base + o_ksum; e.kcomp = base + o_kcomp; e.params = base + o_params;
        e.slo = R == 4 ? base + o_slo : nullptr;
        e.moment = reinterpret_cast<double*>(base + o_moment); e.status = base + o_status;
        e.partial = reinterpret_cast<double*>(base + o_partial); e.ftab = base + o_ftab;
        e.msum = device_mean; e.wsum = device_weight; e.traj = nullptr; e.dw = nullptr;
        e.traj_stride = 1; e.traj_n = 0;
        e.ctl = reinterpret_cast<EnsCtl*>(base + o_ctl);
        EnsDev* d_ens = reinterpret_cast<EnsDev*>(base + o_ens);
        TileDesc* d_tiles = reinterpret_cast<TileDesc*>(base + o_tiles);

        // the array keeps the previous call's contents: clear the control block and the outputs
        check_cuda(cudaMemsetAsync(e.ctl, 0, sizeof(EnsCtl), s), "clear control block");
        check_cuda(cudaMemsetAsync(device_mean, 0, L.K * L.OUT * 8, s), "clear mean");
        noalloc_setup_kernel<<<(std::max(ntiles, 1) + 127) / 128, 128, 0, s>>>(d_ens, e, d_tiles, ntiles, lc.block);

        RawParticles rp;
        rp.radius = dp.magnetic_radius; rp.Ms = dp.saturation_magnetisation; rp.alpha = dp.damping_constant;
        rp.gamma = dp.gyromagnetic_ratio; rp.K = dp.anisotropy_constant;
        rp.rh = brown ? dp.hydrodynamic_radius : dp.magnetic_radius;  // unread by the Neel problems
        rp.viscosity = brown ? dp.viscosity : dp.magnetic_radius;
        rp.euler = dp.orientation; rp.mag = dp.magnetisation;
        rp.K2 = dp.cubic_constant; rp.urot = dp.uniaxial_rotation;
        rp.temperature = desc->temperature;
        rp.simple_model = desc->problem_settings.use_simple_model;
        ks.init(d_ens, rp, L.Np, s);
        ks.reduce(d_ens, 1, 2, 1, s);
        launches_add(3);  // descriptor and tiles, init, reduce
        if (L.S > 0) {
            launch_set_target(e.ctl, L.S, s);
            const int midpoint = desc->solver == SP_SOLVER_IMPLICIT_MIDPOINT ? 1 : 0;
            const unsigned long long nchunks = (L.S + L.chunk - 1) / L.chunk;
            for (unsigned long long i = 0; i < nchunks; ++i) {
                ks.field(d_ens, 1, L.chunk, midpoint, s);
                ks.step[0](d_ens, d_tiles, ntiles, ntiles, lc.block, s);
                ks.reduce(d_ens, 1, L.slots, 0, s);
                launch_commit(d_ens, 1, s);
            }
            launches_add(1 + 4 * nchunks);
        }
        noalloc_normalize_kernel<<<static_cast<unsigned>((L.K * L.OUT + 255) / 256), 256, 0, s>>>(device_mean, device_weight, L.K, L.OUT);
        launches_add(1);
        check_cuda(cudaGetLastError(), "sp_simulate_noalloc launches");
        return SP_OK;
    } catch (const Error& e) {
        return fail(e.status, e.what());
    } catch (const std::exception& e) {
        return fail(SP_ERR_CUDA, e.what());
    }
}
