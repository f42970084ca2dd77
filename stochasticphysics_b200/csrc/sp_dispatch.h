// sp_dispatch.h — host-side table of the instantiated kernels.
#pragma once

#include <cuda_runtime.h>

#include "sp_types.h"

namespace sp {

struct KernelSet {
    bool valid = false;
    int D = 0, Mn = 0, OUT = 0, P = 0, real_bytes = 0;
    void (*init)(const EnsDev* e, const RawParticles& rp, unsigned long long Np, cudaStream_t s) = nullptr;
    // step[ppt - 1]: the step kernel with 1 or 2 particles per thread (2: FP32 only);
    // `block` is the tile's particle count, the CTA has block / ppt threads
    void (*step[2])(const EnsDev* e, const TileDesc* t, int ntiles, int grid, int block, cudaStream_t s) = {nullptr, nullptr};
    void (*reduce)(const EnsDev* e, int n_ens, int max_slots, int mode, cudaStream_t s) = nullptr;
    void (*field)(const EnsDev* e, int n_ens, unsigned long long chunk, int midpoint, cudaStream_t s) = nullptr;
    const void* step_fn[2] = {nullptr, nullptr};  // for cudaFuncGetAttributes / occupancy queries
    // dynamic shared memory of a step launch of `threads` threads (injected increments'
    // staging; 0 for in-kernel noise), and the once-per-device opt-in it needs above the
    // default limit: call prepare() with the device current before the first launch
    size_t (*dyn_smem)(int threads) = nullptr;
    void (*prepare)() = nullptr;
    // injected-noise sets of solvers with one draw per step: the pregenerated-noise kernel
    // (the chunk's increments as the in-kernel path draws them) over `grid` x n_ens CTAs
    void (*noise)(const EnsDev* e, int n_ens, int grid, cudaStream_t s) = nullptr;
};

// index: problem, anisotropy, solver slot (see solver_slot),
// precision (0 FP64, 1 FP32), injected noise
const KernelSet& kernel_set(int problem, int aniso, int solver, int precision, int inject);
constexpr int kSolverSlots = 9;
inline int kernel_index(int aniso, int solver, int precision, int inject) {
    return ((aniso * kSolverSlots + solver) * 2 + precision) * 2 + inject;
}
constexpr int kAnisoSlots = 3;
constexpr int kKernelsPerProblem = kAnisoSlots * kSolverSlots * 2 * 2;
// solver slot of a description: sp_solver 0-4 as is, ImplicitMidpoint with
// SP_JACOBIAN_EXACT in kImplicitMidpointExact, sp_solver 5-7 in slots 6-8
inline int solver_slot(int solver, int jacobian) {
    if (solver == kImplicitMidpoint && jacobian == 1) return kImplicitMidpointExact;
    return solver >= 5 ? solver + 1 : solver;
}

void fill_neel(KernelSet* tab);
void fill_neel_spherical(KernelSet* tab);
void fill_brown_neel_euler(KernelSet* tab);
void fill_brown_neel(KernelSet* tab);

void launch_commit(const EnsDev* e, int n_ens, cudaStream_t s);
void launch_set_target(EnsCtl* ctl, unsigned long long target, cudaStream_t s);
void launch_field_window(const FieldParams& f, double dt, unsigned long long W, unsigned long long K, double* out,
                         cudaStream_t s);
double measure_fma_peak(int precision, int sms, cudaStream_t s);
void launch_debug_normals(unsigned long long seed, unsigned long long pid0, unsigned long long n,
                          unsigned long long step0, unsigned long long nsteps, int noise_dim, int precision, double* out,
                          cudaStream_t s);

}  // namespace sp
