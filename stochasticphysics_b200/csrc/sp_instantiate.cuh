// sp_instantiate.cuh — builds the KernelSet entries of one problem.
#pragma once

#include <mutex>

#include "sp_dispatch.h"
#include "sp_kernels.cuh"

namespace sp {

template <int PROB, class R, int A>
size_t inj_smem_t(int threads) {
    return DwStream<R, ProblemOf<PROB, R, A>::type::Mn>::smem_bytes(threads);
}
template <int PROB, class R, int A, int SOLVER, bool INJ, int PPT>
void launch_step_t(const EnsDev* e, const TileDesc* t, int ntiles, int grid, int block, cudaStream_t s) {
    const size_t dyn = INJ ? inj_smem_t<PROB, R, A>(block / PPT) : 0;
    step_kernel<PROB, R, A, SOLVER, INJ, PPT><<<grid, block / PPT, dyn, s>>>(e, t, ntiles);
}
// the injected kernels' staging exceeds the default dynamic shared memory limit: raise it
// once per device for the largest CTA
template <int PROB, class R, int A, int SOLVER>
void prepare_inj_t() {
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lk(mu);
    if (done[dev]) return;
    if (cudaFuncSetAttribute(reinterpret_cast<const void*>(&step_kernel<PROB, R, A, SOLVER, true, 1>),
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(inj_smem_t<PROB, R, A>(kMaxBlock))) == cudaSuccess)
        done[dev] = true;
}
template <int PROB, class R, int A>
void launch_noise_t(const EnsDev* e, int n_ens, int grid, cudaStream_t s) {
    noise_chunk_kernel<PROB, R, A><<<dim3(static_cast<unsigned>(grid), static_cast<unsigned>(n_ens)), 256, 0, s>>>(e);
}
template <int PROB, class R, int A>
void launch_init_t(const EnsDev* e, const RawParticles& rp, unsigned long long Np, cudaStream_t s) {
    init_kernel<PROB, R, A><<<static_cast<unsigned>(Np / kPad), kPad, 0, s>>>(e, rp);
}
template <class R>
void launch_field_chunk_t(const EnsDev* e, int n_ens, unsigned long long chunk, int midpoint, cudaStream_t s) {
    field_chunk_kernel<R><<<dim3(static_cast<unsigned>((chunk + 255) / 256), static_cast<unsigned>(n_ens)), 256, 0, s>>>(e, midpoint);
}
template <int OUT>
void launch_reduce_t(const EnsDev* e, int n_ens, int max_slots, int mode, cudaStream_t s) {
    reduce_kernel<OUT><<<dim3(static_cast<unsigned>(max_slots * OUT), static_cast<unsigned>(n_ens)), kReduceThreads, 0, s>>>(e, mode);
}

template <int PROB, class R, int A, int SOLVER, bool INJ>
KernelSet make_set() {
    using Prob = typename ProblemOf<PROB, R, A>::type;
    KernelSet k;
    if constexpr (SOLVER == kImplicitMidpoint && !Prob::kHasJacobian) {
        return k;  // not supported by the reference either
    } else if constexpr (SOLVER == kImplicitMidpointExact && !Prob::kHasExactJacobian) {
        return k;  // no analytic Newton matrix for this problem
    } else if constexpr (SOLVER >= kHeunNotConsistent && INJ) {
        return k;  // these take in-kernel noise only (their extra draws have no injection layout)
    } else {
        k.valid = true;
        k.D = Prob::D; k.Mn = Prob::Mn; k.OUT = Prob::OUT; k.P = ProblemOf<PROB, R, A>::P;
        k.real_bytes = static_cast<int>(sizeof(R));
        k.init = &launch_init_t<PROB, R, A>;
        k.step[0] = &launch_step_t<PROB, R, A, SOLVER, INJ, 1>;
        k.step_fn[0] = reinterpret_cast<const void*>(&step_kernel<PROB, R, A, SOLVER, INJ, 1>);
        if constexpr (sizeof(R) == 4 && !INJ) {  // two particles per thread: FP32, in-kernel noise
            k.step[1] = &launch_step_t<PROB, R, A, SOLVER, INJ, 2>;
            k.step_fn[1] = reinterpret_cast<const void*>(&step_kernel<PROB, R, A, SOLVER, INJ, 2>);
        }
        if constexpr (INJ) {
            k.dyn_smem = &inj_smem_t<PROB, R, A>;
            k.prepare = &prepare_inj_t<PROB, R, A, SOLVER>;
            k.noise = &launch_noise_t<PROB, R, A>;
        }
        k.reduce = &launch_reduce_t<Prob::OUT>;
        k.field = &launch_field_chunk_t<R>;
        return k;
    }
}

template <int PROB, int A, int SOLVER>
void fill_solver(KernelSet* tab) {
    tab[kernel_index(A, SOLVER, 0, 0)] = make_set<PROB, double, A, SOLVER, false>();
    tab[kernel_index(A, SOLVER, 0, 1)] = make_set<PROB, double, A, SOLVER, true>();
    tab[kernel_index(A, SOLVER, 1, 0)] = make_set<PROB, float, A, SOLVER, false>();
    tab[kernel_index(A, SOLVER, 1, 1)] = make_set<PROB, float, A, SOLVER, true>();
}
template <int PROB, int A>
void fill_aniso(KernelSet* tab) {
    fill_solver<PROB, A, kEulerMaruyama>(tab);
    fill_solver<PROB, A, kHeun>(tab);
    fill_solver<PROB, A, kMillstein>(tab);
    fill_solver<PROB, A, kImplicitMidpoint>(tab);
    fill_solver<PROB, A, kEulerMaruyamaNormalized>(tab);
    fill_solver<PROB, A, kImplicitMidpointExact>(tab);
    fill_solver<PROB, A, kHeunNotConsistent>(tab);
    fill_solver<PROB, A, kWeakTest>(tab);
    fill_solver<PROB, A, kExplicitStrong1>(tab);
}
template <int PROB>
void fill_problem(KernelSet* tab) {
    fill_aniso<PROB, kUniaxial>(tab);
    fill_aniso<PROB, kCubic>(tab);
    if constexpr (PROB != kBrownNeel) fill_aniso<PROB, kUniaxialCubic>(tab);  // see SP_ANISOTROPY_UNIAXIAL_CUBIC
}

}  // namespace sp
