// Small kernels of the runtime and the kernel table.
#include <mutex>

#include "sp_dispatch.h"
#include "sp_kernels.cuh"
#include "sp_runtime.h"

namespace sp {

__global__ void commit_kernel(const EnsDev* __restrict__ ensembles, int n_ens) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_ens) return;
    const EnsDev& e = ensembles[i];
    const unsigned long long s0 = e.ctl->step_done, tgt = e.ctl->step_target;
    const unsigned long long nsteps = tgt > s0 ? min(e.chunk, tgt - s0) : 0ull;
    e.ctl->step_done = s0 + nsteps;
}

// one thread per window k >= 1; plain summation in reference order
__global__ void field_window_kernel(FieldParams f, double dt, unsigned long long W, unsigned long long K, double* out) {
    const unsigned long long k = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= K) return;
    double B[3];
    if (k == 0) {
        field_eval(f, 0.0, B);
        for (int i = 0; i < 3; ++i) out[i] = B[i];
        return;
    }
    double acc[3] = {0.0, 0.0, 0.0};
    for (unsigned long long l = 0; l < W; ++l) {
        const unsigned long long counter = (k - 1) * W + l + 1;
        field_eval(f, dt * static_cast<double>(counter), B);
        for (int i = 0; i < 3; ++i) acc[i] += B[i];
    }
    for (int i = 0; i < 3; ++i) out[3 * k + i] = acc[i] / static_cast<double>(W);
}

__global__ void set_target_kernel(EnsCtl* ctl, unsigned long long target) { ctl->step_target = target; }

__global__ void bump_target_kernel(const EnsDev* __restrict__ ensembles, int n_ens) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_ens) return;
    const EnsDev& e = ensembles[i];
    const unsigned long long done = e.ctl->step_done;
    e.ctl->step_target = min(done + e.chunk, e.S);
}

void launch_bump_targets(const EnsDev* e, int n_ens, cudaStream_t s) {
    bump_target_kernel<<<(n_ens + 127) / 128, 128, 0, s>>>(e, n_ens);
}

void launch_commit(const EnsDev* e, int n_ens, cudaStream_t s) {
    commit_kernel<<<(n_ens + 127) / 128, 128, 0, s>>>(e, n_ens);
}
void launch_set_target(EnsCtl* ctl, unsigned long long target, cudaStream_t s) {
    set_target_kernel<<<1, 1, 0, s>>>(ctl, target);
}
void launch_field_window(const FieldParams& f, double dt, unsigned long long W, unsigned long long K, double* out,
                         cudaStream_t s) {
    const unsigned blocks = static_cast<unsigned>((K + 127) / 128);
    field_window_kernel<<<blocks, 128, 0, s>>>(f, dt, W, K, out);
}
void launch_debug_normals(unsigned long long seed, unsigned long long pid0, unsigned long long n,
                          unsigned long long step0, unsigned long long nsteps, int noise_dim, int precision, double* out,
                          cudaStream_t s) {
    const unsigned long long total = n * nsteps;
    const unsigned blocks = static_cast<unsigned>((total + 255) / 256);
    if (noise_dim == 3) {
        if (precision == 0) debug_normals_kernel<double, 3><<<blocks, 256, 0, s>>>(seed, pid0, n, step0, nsteps, out);
        else debug_normals_kernel<float, 3><<<blocks, 256, 0, s>>>(seed, pid0, n, step0, nsteps, out);
    } else {
        if (precision == 0) debug_normals_kernel<double, 6><<<blocks, 256, 0, s>>>(seed, pid0, n, step0, nsteps, out);
        else debug_normals_kernel<float, 6><<<blocks, 256, 0, s>>>(seed, pid0, n, step0, nsteps, out);
    }
}

// FMA-chain throughput: 8 independent dependency chains per thread, so the FMA
// pipe (not latency) limits the rate.  2 flops per FMA.
template <class R>
__global__ void __launch_bounds__(256) fma_peak_kernel(R* out, int iters, R b, R c) {
    R a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = static_cast<R>(threadIdx.x + j) * R(1e-7);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = fma(a[j], b, c);
    }
    R s = a[0] + a[1] + a[2] + a[3] + a[4] + a[5] + a[6] + a[7];
    if (s == R(12345.678)) out[blockIdx.x] = s;  // never true; keeps the chains live
}

double measure_fma_peak(int precision, int sms, cudaStream_t s) {
    const int blocks = sms * 8, threads = 256, iters = 4096;
    void* out = nullptr;
    check_cuda(cudaMalloc(&out, blocks * 8), "cudaMalloc");
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(a, s);
        if (precision == 0)
            fma_peak_kernel<double><<<blocks, threads, 0, s>>>(static_cast<double*>(out), iters, 0.9999999, 1e-9);
        else
            fma_peak_kernel<float><<<blocks, threads, 0, s>>>(static_cast<float*>(out), iters, 0.9999999f, 1e-9f);
        cudaEventRecord(b, s);
        check_cuda(cudaEventSynchronize(b), "fma peak");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (rep > 0) best = ms < best ? ms : best;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    const double flops = 2.0 * 8.0 * iters * static_cast<double>(blocks) * threads;
    return flops / (best * 1e-3) / 1e12;
}

const KernelSet& kernel_set(int problem, int aniso, int solver, int precision, int inject) {
    static KernelSet table[4][kKernelsPerProblem];
    static std::once_flag once;
    std::call_once(once, [] {
        fill_neel(table[kNeel]);
        fill_neel_spherical(table[kNeelSpherical]);
        fill_brown_neel_euler(table[kBrownNeelEuler]);
        fill_brown_neel(table[kBrownNeel]);
    });
    static const KernelSet invalid{};
    if (problem < 0 || problem > 3 || aniso < 0 || aniso >= kAnisoSlots || solver < 0 || solver >= kSolverSlots || precision < 0 ||
        precision > 1 || inject < 0 || inject > 1)
        return invalid;
    return table[problem][kernel_index(aniso, solver, precision, inject)];
}

}  // namespace sp
