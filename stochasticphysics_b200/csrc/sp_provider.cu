// sp_provider.cu — particles drawn on the device (sp_provider_desc).
//
// The reference's provider picks a template per particle
// (Provider/ParticleProvider.h:194-217), applies the template's distributions in
// the order anisotropy, magnetic radius, hydrodynamic shell around the drawn radius
// (Settings/ParticleSimulationSettings.h:62-101,138-144; Anisotropy/Uniaxial.hpp:41-85;
// UniaxialCubic.hpp:52-75) and the problem draws random initial states
// (NeelRelaxation.h:226-283, BrownAndNeelRelaxation.inl:288-315,
// ParticleStateInitializer.h:50-123).  Here every draw of particle i comes from its
// own Philox4x32-10 block: counter {draw, 0x50524F56, i_lo, i_hi}, key = provider
// seed; uniform u = (x + 1/2) 2^-32 of word x, normal = sqrt(-2 ln u(x)) cos(2 pi u(y)).
// Draw numbers: 0 template, 1 K, 2 K_cubic, 3-5 uniaxial rotation, 6 radius,
// 7 shell, 8-10 orientation, 11-13 magnetisation.
#include <cmath>
#include <cstring>
#include <vector>

#include "sp_math.cuh"
#include "sp_runtime.h"

namespace sp {

namespace {

constexpr uint32_t kProviderTag = 0x50524F56u;
constexpr double kTwoPiD = 6.28318530717958647692;
constexpr double kPiD = 3.14159265358979323846;

struct DrawStream {
    unsigned long long seed, i;
    __device__ uint4 block(uint32_t draw) const {
        return philox4x32_10(make_uint4(draw, kProviderTag, static_cast<uint32_t>(i), static_cast<uint32_t>(i >> 32)),
                             static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
    }
    __device__ static double u01(uint32_t w) { return fma(static_cast<double>(w), 2.3283064365386963e-10, 1.1641532182693481e-10); }
    __device__ double uniform(uint32_t draw) const { return u01(block(draw).x); }
    __device__ double normal(uint32_t draw) const {
        const uint4 b = block(draw);
        return ::sqrt(-2.0 * ::log(u01(b.x))) * ::cos(kTwoPiD * u01(b.y));
    }
};

__device__ double dist_sample(int type, double mean, double sigma, double z) {
    if (type == SP_DIST_DELTA || !(sigma > 0.0)) return mean;
    if (type == SP_DIST_NORMAL) return mean + sigma * z;
    const double s2 = ::log1p((sigma * sigma) / (mean * mean));
    return ::exp((::log(mean) - 0.5 * s2) + ::sqrt(s2) * z);
}
// relative: value * X, X from (1, width); absolute: drawn around the value with sigma
// value * width (radius, shell) or width (anisotropy constants)
__device__ double dist_apply(const sp_dist& d, double value, double z, bool sigma_times_mean) {
    if (d.relative) return value * dist_sample(d.type, 1.0, d.width, z);
    return dist_sample(d.type, value, sigma_times_mean ? value * d.width : d.width, z);
}

// out: [18][n] columns r, Ms, alpha, gamma, K, rh, eta, K2, template, then the
// [n][3] blocks euler, mag, urot (the RawParticles layout)
__global__ void provide_kernel(const sp_particle_template* __restrict__ tpl, int nt, int sequential,
                               unsigned long long seed, unsigned long long id0, unsigned long long n, int problem,
                               int aniso, double* __restrict__ out) {
    const unsigned long long p = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const DrawStream ds{seed, id0 + p};
    // template (ParticleProvider.h:196-215)
    int t = 0;
    if (sequential) {
        double cum = 0.0;
        const double i = static_cast<double>(id0 + p);
        for (int k = 0; k < nt; ++k) {
            cum += tpl[k].weight;
            if (i < cum) { t = k; break; }
        }
    } else {
        double total = 0.0;
        for (int k = 0; k < nt; ++k) total += tpl[k].weight;
        const double u = ds.uniform(0) * total;
        double cum = 0.0;
        t = nt - 1;
        for (int k = 0; k < nt; ++k) {
            cum += tpl[k].weight;
            if (u < cum) { t = k; break; }
        }
    }
    const sp_particle_template& T = tpl[t];
    const bool uc = aniso == SP_ANISOTROPY_UNIAXIAL_CUBIC;
    const double K = dist_apply(T.anisotropy_dist, T.anisotropy_constant, ds.normal(1), false);
    const double K2 = uc ? dist_apply(T.cubic_dist, T.cubic_constant, ds.normal(2), false) : 0.0;
    double ur[3] = {0.0, 0.0, 0.0};
    if (uc) {
        if (T.random_uniaxial_rotation) {
            ur[0] = ds.uniform(3) * kTwoPiD; ur[1] = ds.uniform(4) * kPiD; ur[2] = ds.uniform(5) * kTwoPiD;
        } else {
            ur[0] = T.uniaxial_rotation[0]; ur[1] = T.uniaxial_rotation[1]; ur[2] = T.uniaxial_rotation[2];
        }
    }
    const double r = dist_apply(T.magnetic_radius_dist, T.magnetic_radius, ds.normal(6), true);
    const double rh = dist_apply(T.hydrodynamic_shell_dist, T.hydrodynamic_radius - r, ds.normal(7), true) + r;
    double e[3] = {T.orientation[0], T.orientation[1], T.orientation[2]};
    if (T.random_orientation) {
        if (problem == SP_PROBLEM_NEEL) {
            e[0] = ds.uniform(8) * kTwoPiD; e[1] = ds.uniform(9) * kTwoPiD; e[2] = ds.uniform(10) * kTwoPiD;
        } else if (problem == SP_PROBLEM_BROWN_AND_NEEL) {
            // a uniformly drawn axis, handed over as ZXZ angles whose rotated x axis it is
            double d[3] = {ds.normal(8), ds.normal(9), ds.normal(10)};
            const double nd = ::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            for (double& c : d) c /= nd;
            e[0] = ::acos(fmin(1.0, fmax(-1.0, d[0]))); e[1] = ::atan2(d[2], -d[1]); e[2] = 0.0;
        } else {
            e[0] = ds.uniform(8) * kTwoPiD; e[1] = ds.uniform(9) * kPiD; e[2] = ds.uniform(10) * kTwoPiD;
        }
    }
    double m[3] = {T.magnetisation[0], T.magnetisation[1], T.magnetisation[2]};
    if (T.random_magnetisation) {
        if (problem == SP_PROBLEM_NEEL || problem == SP_PROBLEM_BROWN_AND_NEEL) {
            m[0] = ds.normal(11); m[1] = ds.normal(12); m[2] = ds.normal(13);
        } else {
            const double ph = ds.uniform(11) * kTwoPiD, th = ds.uniform(12) * kPiD;
            m[0] = ::cos(ph) * ::sin(th); m[1] = ::sin(ph) * ::sin(th); m[2] = ::cos(th);
        }
    }
    const double nm = ::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    if (nm > 0.0) for (double& c : m) c /= nm;
    const double col[9] = {r, T.saturation_magnetisation, T.damping_constant, T.gyromagnetic_ratio, K, rh, T.viscosity, K2,
                           static_cast<double>(t)};
    for (int c = 0; c < 9; ++c) out[c * n + p] = col[c];
    for (int c = 0; c < 3; ++c) {
        out[9 * n + 3 * p + c] = e[c];
        out[12 * n + 3 * p + c] = m[c];
        out[15 * n + 3 * p + c] = ur[c];
    }
}

}  // namespace

double* provide_particles(sp_context* ctx, const sp_ensemble_desc& d, cudaStream_t s) {
    const sp_provider_desc& pv = *d.provider;
    const unsigned long long n = d.n_particles;
    sp_particle_template* dt = nullptr;
    double* out = nullptr;
    check_cuda(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&dt), pv.n_templates * sizeof(sp_particle_template), ctx->pool, s),
               "cudaMallocFromPoolAsync");
    check_cuda(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&out), 18 * n * sizeof(double), ctx->pool, s),
               "cudaMallocFromPoolAsync");
    check_cuda(cudaMemcpyAsync(dt, pv.templates, pv.n_templates * sizeof(sp_particle_template), cudaMemcpyHostToDevice, s),
               "upload templates");
    provide_kernel<<<static_cast<unsigned>((n + 127) / 128), 128, 0, s>>>(dt, pv.n_templates, pv.sequential, pv.seed,
                                                                          d.particle_id_offset, n, d.problem, d.anisotropy, out);
    check_cuda(cudaGetLastError(), "provide_kernel");
    g_launch_count += 1;
    check_cuda(cudaFreeAsync(dt, s), "cudaFreeAsync");
    return out;
}

RawParticles provided_raw(const double* dev, unsigned long long n) {
    RawParticles rp;
    rp.radius = dev; rp.Ms = dev + n; rp.alpha = dev + 2 * n; rp.gamma = dev + 3 * n; rp.K = dev + 4 * n;
    rp.rh = dev + 5 * n; rp.viscosity = dev + 6 * n; rp.K2 = dev + 7 * n;
    rp.euler = dev + 9 * n; rp.mag = dev + 12 * n; rp.urot = dev + 15 * n;
    rp.temperature = 0.0;
    rp.simple_model = 0;
    return rp;
}

}  // namespace sp

using namespace sp;

sp_status sp_provide_particles(sp_context* ctx, const sp_ensemble_desc* desc, double* out) {
    SP_GUARD_BEGIN
    if (!ctx || !out) return fail(SP_ERR_INVALID_ARG, "NULL argument");
    std::string why;
    const sp_status s = validate_desc(desc, why);
    if (s != SP_OK) return fail(s, why);
    if (!desc->provider) return fail(SP_ERR_INVALID_ARG, "the description has no provider");
    check_cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
    const unsigned long long n = desc->n_particles;
    double* dev = provide_particles(ctx, *desc, ctx->stream);
    std::vector<double> host(18 * n);
    check_cuda(cudaMemcpyAsync(host.data(), dev, host.size() * 8, cudaMemcpyDeviceToHost, ctx->stream), "read particles");
    check_cuda(cudaFreeAsync(dev, ctx->stream), "cudaFreeAsync");
    check_cuda(cudaStreamSynchronize(ctx->stream), "provide");
    // [n][20]: r Ms alpha gamma K rh eta euler[3] mag[3] K2 urot[3] template reserved
    for (unsigned long long p = 0; p < n; ++p) {
        double* o = out + 20 * p;
        for (int c = 0; c < 7; ++c) o[c] = host[c * n + p];
        for (int c = 0; c < 3; ++c) {
            o[7 + c] = host[9 * n + 3 * p + c];
            o[10 + c] = host[12 * n + 3 * p + c];
            o[14 + c] = host[15 * n + 3 * p + c];
        }
        o[13] = host[7 * n + p];
        o[17] = host[8 * n + p];
        o[18] = 0.0;
        o[19] = 0.0;
    }
    return SP_OK;
    SP_GUARD_END
}
