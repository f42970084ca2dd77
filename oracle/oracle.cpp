// oracle.cpp — CPU restatement of the reference's per-particle simulation loop,
// solvers and ensemble mean, exported through a small C ABI for ctypes.
//
// TEST INFRASTRUCTURE ONLY (the checker): loaded by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline leg; never by the
// product library.  See oracle_core.hpp for what is and is not pinned by the
// reference's golden vectors.
#include <algorithm>
#include <cmath>
#include <limits>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include <atomic>
#include <thread>

#include "../include/stophys_b200.h"
#include "oracle_problems.hpp"

namespace orc {

// ====================================================================== counting scalar
// Counts adds/subs/muls (an FMA counts as 2), divisions and transcendental calls
// of the restated formulas; used to derive the algorithmic work per step.
struct OpCounts {
    uint64_t flops = 0, divs = 0, transc = 0, sqrts = 0;
};
static thread_local OpCounts g_ops;

struct Cnt {
    double v;
    Cnt() : v(0.0) {}
    Cnt(double x) : v(x) {}  // NOLINT (implicit on purpose)
    explicit operator double() const { return v; }
};
inline Cnt operator+(Cnt a, Cnt b) { ++g_ops.flops; return Cnt(a.v + b.v); }
inline Cnt operator-(Cnt a, Cnt b) { ++g_ops.flops; return Cnt(a.v - b.v); }
inline Cnt operator*(Cnt a, Cnt b) { ++g_ops.flops; return Cnt(a.v * b.v); }
inline Cnt operator/(Cnt a, Cnt b) { ++g_ops.divs; return Cnt(a.v / b.v); }
inline Cnt operator-(Cnt a) { return Cnt(-a.v); }
inline Cnt operator+(Cnt a) { return a; }
inline bool operator<(Cnt a, Cnt b) { return a.v < b.v; }
inline bool operator>(Cnt a, Cnt b) { return a.v > b.v; }
inline bool operator<=(Cnt a, Cnt b) { return a.v <= b.v; }
inline bool operator==(Cnt a, Cnt b) { return a.v == b.v; }
inline Cnt sin(Cnt a) { ++g_ops.transc; return Cnt(std::sin(a.v)); }
inline Cnt cos(Cnt a) { ++g_ops.transc; return Cnt(std::cos(a.v)); }
inline Cnt acos(Cnt a) { ++g_ops.transc; return Cnt(std::acos(a.v)); }
inline Cnt atan2(Cnt a, Cnt b) { ++g_ops.transc; return Cnt(std::atan2(a.v, b.v)); }
inline Cnt fmod(Cnt a, Cnt b) { ++g_ops.transc; return Cnt(std::fmod(a.v, b.v)); }
inline Cnt sqrt(Cnt a) { ++g_ops.sqrts; return Cnt(std::sqrt(a.v)); }
inline Cnt abs(Cnt a) { return Cnt(std::fabs(a.v)); }
inline bool isinf(Cnt a) { return std::isinf(a.v); }
inline double to_double(Cnt a) { return a.v; }
inline double to_double(double a) { return a; }
inline double to_double(long double a) { return static_cast<double>(a); }

// ====================================================================== Philox4x32-10 noise
// Counter-based generator (Salmon et al., SC'11).  The device kernels use the
// same counter layout, so particle p at step n draws the same 32-bit words on
// the CPU and on the GPU:
//   counter = {n_lo, n_hi, pid_lo, (pid_hi & 0xFFFFFF) | call << 24}, key = seed.
inline void philox4x32_10(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * ctr[0];
        const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * ctr[2];
        const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
        const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
        const uint32_t n0 = hi1 ^ ctr[1] ^ k0, n2 = hi0 ^ ctr[3] ^ k1;
        ctr[0] = n0; ctr[1] = lo1; ctr[2] = n2; ctr[3] = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}
// The four unit normals of Philox call `call` for (seed, particle id, step):
// Box-Muller on uniforms u = (w + 1/2) 2^-32.
inline void philox_call_normals(uint64_t seed, uint64_t pid, uint64_t step, uint32_t call, double* v) {
    uint32_t c[4] = {static_cast<uint32_t>(step), static_cast<uint32_t>(step >> 32), static_cast<uint32_t>(pid),
                     (static_cast<uint32_t>(pid >> 32) & 0xFFFFFFu) | (call << 24)};
    philox4x32_10(c, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
    const double inv = 2.3283064365386963e-10;  // 2^-32
    const double u0 = (c[0] + 0.5) * inv, u1 = (c[1] + 0.5) * inv;
    const double u2 = (c[2] + 0.5) * inv, u3 = (c[3] + 0.5) * inv;
    const double r0 = std::sqrt(-2.0 * std::log(u0));
    const double r1 = std::sqrt(-2.0 * std::log(u2));
    const double t0 = kTwoPi * u1, t1 = kTwoPi * u3;
    v[0] = r0 * std::cos(t0); v[1] = r0 * std::sin(t0); v[2] = r1 * std::cos(t1); v[3] = r1 * std::sin(t1);
}
// m unit normals for (seed, particle id, step) from calls call0, call0 + 1:
// call call0 + j yields z[4j..4j+3].  Calls 0-1 carry dW, calls 2-3
// Heun_NotConsistent's second increment, calls 2.. the double-noise draws.
inline void philox_normals(uint64_t seed, uint64_t pid, uint64_t step, int m, double* z, uint32_t call0 = 0) {
    const int calls = (m + 3) / 4;
    for (int j = 0; j < calls; ++j) {
        double v[4];
        philox_call_normals(seed, pid, step, call0 + static_cast<uint32_t>(j), v);
        for (int i = 0; i < 4 && 4 * j + i < m; ++i) z[4 * j + i] = v[i];
    }
}

// ====================================================================== provider
// Particles drawn by an sp_provider_desc, restated from the reference's provider and
// initialisers (ParticleProvider.h:196-215, ParticleSimulationSettings.h:62-101,138-144,
// Uniaxial.hpp:41-85, UniaxialCubic.hpp:52-75, NeelRelaxation.h:226-283,
// BrownAndNeelRelaxation.inl:288-315, ParticleStateInitializer.h:50-123).  Draw k of
// particle i is the Philox block with counter {k, 0x50524F56, i_lo, i_hi} and the
// provider's seed as key: uniform (x + 1/2) 2^-32, normal sqrt(-2 ln u(x)) cos(2 pi u(y)).
// Draws: 0 template, 1 K, 2 K_cubic, 3-5 rotation, 6 radius, 7 shell, 8-10 orientation,
// 11-13 magnetisation.
struct ProviderDraws {
    uint64_t seed, i;
    void block(uint32_t k, uint32_t* c) const {
        c[0] = k; c[1] = 0x50524F56u; c[2] = static_cast<uint32_t>(i); c[3] = static_cast<uint32_t>(i >> 32);
        philox4x32_10(c, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
    }
    static double u01(uint32_t w) { return (w + 0.5) * 2.3283064365386963e-10; }
    double uniform(uint32_t k) const { uint32_t c[4]; block(k, c); return u01(c[0]); }
    double normal(uint32_t k) const {
        uint32_t c[4];
        block(k, c);
        return std::sqrt(-2.0 * std::log(u01(c[0]))) * std::cos(kTwoPi * u01(c[1]));
    }
};
inline double provider_sample(int type, double mean, double sigma, double z) {
    if (type == SP_DIST_DELTA || !(sigma > 0.0)) return mean;
    if (type == SP_DIST_NORMAL) return mean + sigma * z;
    const double s2 = std::log1p((sigma * sigma) / (mean * mean));  // lognormal with this mean and sigma
    return std::exp((std::log(mean) - 0.5 * s2) + std::sqrt(s2) * z);
}
inline double provider_apply(const sp_dist& d, double value, double z, bool sigma_times_mean) {
    if (d.relative) return value * provider_sample(d.type, 1.0, d.width, z);
    return provider_sample(d.type, value, sigma_times_mean ? value * d.width : d.width, z);
}
// o[20]: r Ms alpha gamma K rh eta euler[3] mag[3] K2 urot[3] template reserved[2]
void provide_particle(const sp_provider_desc& pv, uint64_t i, int problem, int aniso, double* o) {
    const ProviderDraws ds{pv.seed, i};
    int t = 0;
    if (pv.sequential) {
        double cum = 0.0;
        for (int k = 0; k < pv.n_templates; ++k) {
            cum += pv.templates[k].weight;
            if (static_cast<double>(i) < cum) { t = k; break; }
        }
    } else {
        double total = 0.0;
        for (int k = 0; k < pv.n_templates; ++k) total += pv.templates[k].weight;
        const double u = ds.uniform(0) * total;
        double cum = 0.0;
        t = pv.n_templates - 1;
        for (int k = 0; k < pv.n_templates; ++k) {
            cum += pv.templates[k].weight;
            if (u < cum) { t = k; break; }
        }
    }
    const sp_particle_template& T = pv.templates[t];
    const bool uc = aniso == SP_ANISOTROPY_UNIAXIAL_CUBIC;
    o[4] = provider_apply(T.anisotropy_dist, T.anisotropy_constant, ds.normal(1), false);
    o[13] = uc ? provider_apply(T.cubic_dist, T.cubic_constant, ds.normal(2), false) : 0.0;
    for (int c = 0; c < 3; ++c) o[14 + c] = uc ? T.uniaxial_rotation[c] : 0.0;
    if (uc && T.random_uniaxial_rotation) {
        o[14] = ds.uniform(3) * kTwoPi; o[15] = ds.uniform(4) * kPi; o[16] = ds.uniform(5) * kTwoPi;
    }
    const double r = provider_apply(T.magnetic_radius_dist, T.magnetic_radius, ds.normal(6), true);
    o[0] = r;
    o[5] = provider_apply(T.hydrodynamic_shell_dist, T.hydrodynamic_radius - r, ds.normal(7), true) + r;
    o[1] = T.saturation_magnetisation; o[2] = T.damping_constant; o[3] = T.gyromagnetic_ratio; o[6] = T.viscosity;
    double* e = o + 7;
    for (int c = 0; c < 3; ++c) e[c] = T.orientation[c];
    if (T.random_orientation) {
        if (problem == SP_PROBLEM_NEEL) {
            for (int c = 0; c < 3; ++c) e[c] = ds.uniform(8 + c) * kTwoPi;
        } else if (problem == SP_PROBLEM_BROWN_AND_NEEL) {
            double d[3] = {ds.normal(8), ds.normal(9), ds.normal(10)};
            const double nd = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            for (double& c : d) c /= nd;
            e[0] = std::acos(std::min(1.0, std::max(-1.0, d[0]))); e[1] = std::atan2(d[2], -d[1]); e[2] = 0.0;
        } else {
            e[0] = ds.uniform(8) * kTwoPi; e[1] = ds.uniform(9) * kPi; e[2] = ds.uniform(10) * kTwoPi;
        }
    }
    double* m = o + 10;
    for (int c = 0; c < 3; ++c) m[c] = T.magnetisation[c];
    if (T.random_magnetisation) {
        if (problem == SP_PROBLEM_NEEL || problem == SP_PROBLEM_BROWN_AND_NEEL) {
            for (int c = 0; c < 3; ++c) m[c] = ds.normal(11 + c);
        } else {
            const double ph = ds.uniform(11) * kTwoPi, th = ds.uniform(12) * kPi;
            m[0] = std::cos(ph) * std::sin(th); m[1] = std::sin(ph) * std::sin(th); m[2] = std::cos(th);
        }
    }
    const double nm = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    if (nm > 0.0) for (int c = 0; c < 3; ++c) m[c] /= nm;
    o[17] = t; o[18] = 0.0; o[19] = 0.0;
}

// Host arrays of a provided ensemble, kept alive beside a description that points at them
struct ProvidedArrays {
    std::vector<double> r, Ms, alpha, gamma, K, rh, eta, euler, mag, K2, urot;
    sp_ensemble_desc desc;
    explicit ProvidedArrays(const sp_ensemble_desc& d) : desc(d) {
        const uint64_t n = d.n_particles;
        for (auto* v : {&r, &Ms, &alpha, &gamma, &K, &rh, &eta, &K2}) v->resize(n);
        euler.resize(3 * n); mag.resize(3 * n); urot.resize(3 * n);
        double o[20];
        for (uint64_t p = 0; p < n; ++p) {
            provide_particle(*d.provider, d.particle_id_offset + p, d.problem, d.anisotropy, o);
            r[p] = o[0]; Ms[p] = o[1]; alpha[p] = o[2]; gamma[p] = o[3]; K[p] = o[4]; rh[p] = o[5]; eta[p] = o[6];
            K2[p] = o[13];
            for (int c = 0; c < 3; ++c) { euler[3 * p + c] = o[7 + c]; mag[3 * p + c] = o[10 + c]; urot[3 * p + c] = o[14 + c]; }
        }
        desc.particles = sp_particles{r.data(), Ms.data(), alpha.data(), gamma.data(), K.data(), rh.data(), eta.data(),
                                      euler.data(), mag.data(), K2.data(), urot.data()};
        desc.provider = nullptr;
    }
};

// ====================================================================== fields
// Fields/SinusoidalField.h:47-51, Fields/LissajousField.h:98-101, ConstantField.h:43, ZeroField.h:39
// Fields/TriangularField.h:52-70, Fields/RectangularField.h:30-63, Fields/SincField.h:32-48
struct FieldEval {
    int type = SP_FIELD_ZERO;
    double offset[3] = {0, 0, 0}, amplitude[3] = {0, 0, 0}, angfreq[3] = {0, 0, 0}, phase[3] = {0, 0, 0};
    double P = 0, halfP = 0, toff = 0;
    // rectangular waveform: amplitude and offset after the alternating transform
    double invTau = 0, rAmp[3] = {0, 0, 0}, rMax[3] = {0, 0, 0}, rOff[3] = {0, 0, 0}, rToff = 0;
    double sincA = 0;
    void init(const sp_field_desc& f) {
        type = f.type;
        for (int i = 0; i < 3; ++i) {
            offset[i] = f.offset[i]; amplitude[i] = f.amplitude[i];
            angfreq[i] = kTwoPi * (type == SP_FIELD_SINUSOIDAL ? f.frequency[0] : f.frequency[i]);
            phase[i] = (type == SP_FIELD_SINUSOIDAL ? f.phase[0] : f.phase[i]);
        }
        P = f.periode; halfP = f.periode / 2.0; toff = f.time_offset;
        sincA = 11.0 / (f.periode * 0.5);
        if (type == SP_FIELD_RECTANGULAR) {
            invTau = std::abs(f.tau) <= std::numeric_limits<double>::min() ? std::numeric_limits<double>::max() : 1.0 / f.tau;
            double na2 = 0.0, nm2 = 0.0;
            for (int i = 0; i < 3; ++i) {
                rAmp[i] = f.alternating ? 2.0 * f.amplitude[i] : f.amplitude[i];
                rMax[i] = rAmp[i] * (-std::expm1(-halfP * invTau));
                na2 += rAmp[i] * rAmp[i];
                nm2 += rMax[i] * rMax[i];
            }
            rToff = f.alternating ? f.time_offset - std::log(1.0 - std::sqrt(nm2) / (2.0 * std::sqrt(na2))) * f.tau
                                  : f.time_offset;
            for (int i = 0; i < 3; ++i)
                rOff[i] = f.alternating ? rAmp[i] * std::expm1(-rToff * invTau) + f.offset[i] : f.offset[i];
        }
    }
    static double sinc(double x) { return std::fabs(x) < 1e-4 ? 1.0 + x * x * (-1.0 / 6.0 + x * x * (1.0 / 120.0)) : std::sin(x) / x; }
    void eval(double time, double* B) const {
        switch (type) {
            case SP_FIELD_ZERO: B[0] = B[1] = B[2] = 0.0; break;
            case SP_FIELD_CONSTANT: for (int i = 0; i < 3; ++i) B[i] = offset[i]; break;
            case SP_FIELD_SINUSOIDAL: {
                const double sinwt = std::sin(angfreq[0] * time + phase[0]);
                for (int i = 0; i < 3; ++i) B[i] = amplitude[i] * sinwt + offset[i];
                break;
            }
            case SP_FIELD_LISSAJOUS:
                for (int i = 0; i < 3; ++i) B[i] = offset[i] + amplitude[i] * std::sin(angfreq[i] * time + phase[i]);
                break;
            case SP_FIELD_TRIANGULAR: {
                const double t = time + toff;
                const double pos = t < 0 ? P + std::fmod(t, P) : std::fmod(t, P);
                const double w = pos > halfP ? 2.0 * pos / halfP - 1.0 : -2.0 * pos / halfP + 3.0;
                for (int i = 0; i < 3; ++i) B[i] = w * amplitude[i] + offset[i];
                break;
            }
            case SP_FIELD_RECTANGULAR: {
                const double t = time + rToff;
                const double pos = t < 0 ? std::fmod(t + P, P) : std::fmod(t, P);
                if (pos <= halfP) {
                    const double g = -std::expm1(-pos * invTau);
                    for (int i = 0; i < 3; ++i) B[i] = rAmp[i] * g + rOff[i];
                } else {
                    const double g = std::exp(-(pos - halfP) * invTau);
                    for (int i = 0; i < 3; ++i) B[i] = rAmp[i] * g + rOff[i] - (rAmp[i] - rMax[i]);
                }
                break;
            }
            default: {  // SP_FIELD_SINC
                const double pos = (time < 0 ? std::fmod(time + P, P) : std::fmod(time, P)) - halfP;
                const double sc = sinc(kPi * sincA * pos);
                for (int i = 0; i < 3; ++i) B[i] = amplitude[i] * (sc * sc) + offset[i];
            }
        }
    }
};

// ====================================================================== linear solve (Newton step)
template <class T, int N>
bool solve_dense(Mat<T, N, N> A, Vec<T, N> b, Vec<T, N>& x) {
    using std::fabs;
    for (int k = 0; k < N; ++k) {
        int piv = k;
        for (int i = k + 1; i < N; ++i)
            if (std::fabs(to_double(A(i, k))) > std::fabs(to_double(A(piv, k)))) piv = i;
        if (to_double(A(piv, k)) == 0.0) return false;
        if (piv != k) { for (int j = 0; j < N; ++j) std::swap(A(k, j), A(piv, j)); std::swap(b[k], b[piv]); }
        for (int i = k + 1; i < N; ++i) {
            const T f = A(i, k) / A(k, k);
            for (int j = k; j < N; ++j) A(i, j) = A(i, j) - f * A(k, j);
            b[i] = b[i] - f * b[k];
        }
    }
    for (int i = N - 1; i >= 0; --i) {
        T s = b[i];
        for (int j = i + 1; j < N; ++j) s = s - A(i, j) * x[j];
        x[i] = s / A(i, i);
    }
    return true;
}

// ====================================================================== solvers
// One fixed step, Stratonovich interpretation (all four problems are
// Stratonovich, e.g. Problems/Definitions/NeelRelaxation_Definitions.h:104-106,
// so FixedTimestepSelector<false> is taken: SDEFramework/Solver/GeneralSDESolver.h:48-56).
struct NewtonStats { uint64_t iterations = 0, unconverged = 0; };

template <class P, class T>
struct Stepper {
    using Dep = typename P::Dep;
    static constexpr int D = P::D, M = P::M;

    // SDEFramework/Solver/EulerMaruyama.inl:42-72
    static Dep euler_maruyama(P& pr, const Dep& yi, const V3<T>& xi, const Vec<T, M>& dW, const T& dt) {
        Dep res = yi;
        pr.prepareCalculations(res);
        const Dep a = pr.getDeterministicVector(res, xi);
        const Dep D_ = pr.getDrift(res);
        const auto b = pr.getStochasticMatrix(res);
        res = res + ((a + D_) * dt + b * dW);
        pr.finishCalculations(res);
        return res;
    }
    // SDEFramework/Solver/EulerMaruyama_Normalized.inl:40-56: EulerMaruyama, then normalize
    static Dep euler_maruyama_normalized(P& pr, const Dep& yi, const V3<T>& xi, const Vec<T, M>& dW, const T& dt) {
        Dep res = euler_maruyama(pr, yi, xi, dW, dt);
        pr.normalize(res);
        return res;
    }
    // SDEFramework/Solver/Heun_Strong.inl:37-47.  The reference's Heun is not
    // wired into its simulator (SimulationManager.h:322-328) and never calls
    // prepare/finish; this restatement evaluates both stages in the chart that
    // prepareCalculations chose for y_n (no-op for the Cartesian problems, where
    // it is exactly the reference formula) and finishes once.
    static Dep heun(P& pr, const Dep& yi_in, const V3<T>& xi, const Vec<T, M>& dW, const T& dt) {
        Dep yi = yi_in;
        pr.prepareCalculations(yi);
        const Dep ayi = pr.getDeterministicVector(yi, xi) + pr.getDrift(yi);
        const auto byi = pr.getStochasticMatrix(yi);
        const Dep bdW = byi * dW;
        const Dep Support = yi + ayi * dt + bdW;
        pr.recomputeCache(Support);
        const Dep a2 = pr.getDeterministicVector(Support, xi) + pr.getDrift(Support);
        Dep res = yi + (T(0.5) * (a2 + ayi)) * dt + bdW;
        pr.finishCalculations(res);
        return res;
    }
    // SDEFramework/Solver/Millstein.inl:35-44 (Stratonovich form), with
    // prepare/finish around the single evaluation point like EulerMaruyama.
    static Dep millstein(P& pr, const Dep& yi_in, const V3<T>& xi, const Vec<T, M>& dW, const T& dt) {
        Dep yi = yi_in;
        pr.prepareCalculations(yi);
        const Dep a_ = pr.getDeterministicVector(yi, xi);
        const Dep bb = pr.getDrift(yi);
        const auto b = pr.getStochasticMatrix(yi);
        Dep res = ((yi + a_ * dt) + b * dW) + bb * dot(dW, dW);
        pr.finishCalculations(res);
        return res;
    }
    // SDEFramework/Solver/Heun_NotConsistent.inl:35-47 (Stratonovich): support point
    // with dW, corrector with the mean of b at both points times an independent dW2;
    // both points in the chart prepareCalculations chose for y_n, finished once.
    static Dep heun_not_consistent(P& pr, const Dep& yi_in, const V3<T>& xi, const Vec<T, M>& dW,
                                   const Vec<T, M>& dW2, const T& dt) {
        Dep yi = yi_in;
        pr.prepareCalculations(yi);
        const Dep ayi = pr.getDeterministicVector(yi, xi) + pr.getDrift(yi);
        const auto byi = pr.getStochasticMatrix(yi);
        const Dep bdW = byi * dW;
        const Dep Support = yi + ayi * dt + bdW;
        pr.recomputeCache(Support);
        const Dep a2 = pr.getDeterministicVector(Support, xi) + pr.getDrift(Support);
        const auto bS = pr.getStochasticMatrix(Support);
        Dep res = yi + (T(0.5) * (a2 + ayi)) * dt + T(0.5) * ((bS + byi) * dW2);
        pr.finishCalculations(res);
        return res;
    }
    // SDEFramework/Solver/Explicit_Strong_1.inl:20-78 (no drift correction): support
    // points tmp +- b.col(j1) sqrt(dt) for j1 < D around tmp = y + a dt,
    //   y' = sum_j1 (b(S+) - b(S-)) J.col(j1) / sqrt(dt) + (tmp + b dW).
    static Dep explicit_strong_1(P& pr, const Dep& yi_in, const V3<T>& xi, const Vec<T, M>& dW,
                                 const Mat<T, M, M>& J, const T& dt, const T& sqrtdt) {
        Dep yi = yi_in;
        pr.prepareCalculations(yi);
        const Dep a = pr.getDeterministicVector(yi, xi);
        const auto b = pr.getStochasticMatrix(yi);
        const Dep tmpvec = yi + a * dt;
        Dep tmpvec2 = Dep::zero();
        for (int j1 = D; j1--;) {
            Dep col;
            for (int i = 0; i < D; ++i) col[i] = b(i, j1);
            Vec<T, M> Jc;
            for (int r = 0; r < M; ++r) Jc[r] = J(r, j1);
            const Dep Sp = tmpvec + col * sqrtdt, Sm = tmpvec - col * sqrtdt;
            pr.recomputeCache(Sp);
            const auto bSp = pr.getStochasticMatrix(Sp);
            pr.recomputeCache(Sm);
            const auto bSm = pr.getStochasticMatrix(Sm);
            tmpvec2 = tmpvec2 + (bSp - bSm) * Jc;
        }
        for (int i = 0; i < D; ++i) tmpvec2[i] = tmpvec2[i] / sqrtdt;
        Dep res = tmpvec2 + (tmpvec + b * dW);
        pr.finishCalculations(res);
        return res;
    }
    // SDEFramework/Solver/WeakTest.inl:18-63
    static Dep weak_test(P& pr, const Dep& yi_in, const V3<T>& xi, const Vec<T, M>& dW, const Mat<T, M, M>& J,
                         const T& dt, const T& sqrtdt) {
        Dep yi = yi_in;
        pr.prepareCalculations(yi);
        const Dep a = pr.getDeterministicVector(yi, xi);
        const auto b = pr.getStochasticMatrix(yi);
        const Dep adt = a * dt;
        const Dep tmpvec = yi + adt;
        const Dep bdW = b * dW;
        const Dep ys = tmpvec + bdW;
        pr.recomputeCache(ys);
        const Dep as = pr.getDeterministicVector(ys, xi);
        Dep tmpvec2 = Dep::zero();
        for (int j1 = D; j1--;) {
            Dep col;
            for (int i = 0; i < D; ++i) col[i] = b(i, j1);
            Vec<T, M> Jc;
            for (int r = 0; r < M; ++r) Jc[r] = J(r, j1);
            const Dep Sp = tmpvec + col * sqrtdt, Sm = tmpvec - col * sqrtdt;
            pr.recomputeCache(Sp);
            const auto bSp = pr.getStochasticMatrix(Sp);
            pr.recomputeCache(Sm);
            const auto bSm = pr.getStochasticMatrix(Sm);
            Dep diff = (bSp - bSm) * Jc;
            for (int i = 0; i < D; ++i) diff[i] = diff[i] / sqrtdt;
            tmpvec2 = tmpvec2 + diff;
            tmpvec2 = tmpvec2 + (bSp + bSm) * dW;
        }
        for (int i = 0; i < D; ++i) tmpvec2[i] = tmpvec2[i] / T(4.0);
        tmpvec2 = tmpvec2 + T(0.5) * bdW;
        const Dep ys2 = ((yi + (T(0.5) * as) * dt) + T(0.5) * adt) + tmpvec2;
        pr.recomputeCache(ys2);
        const Dep as2 = pr.getDeterministicVector(ys2, xi);
        Dep res = ((yi + (T(0.5) * as2) * dt) + T(0.5) * adt) + tmpvec2;
        pr.finishCalculations(res);
        return res;
    }
    // SDEFramework/Solver/Implicit_Midpoint.inl:40-188: Newton on
    //   f(y) = finish(prepare((y+y_n)/2) + a dt + b dW) + y_n/2 - 3y/2
    // with S = -I + dt/2 J_a + 1/2 J_b (:83-98), initial guess y_n (:56),
    // accept when |dy| <= AccuracyGoal (legacy loop :175), at most MaxIteration.
    static Dep implicit_midpoint(P& pr, const Dep& yi, const V3<T>& xj, const Vec<T, M>& dW, const T& dt,
                                 int maxIter, double tol, bool exact, NewtonStats& st) {
        Dep yj = yi;
        bool converged = false;
        for (int it = 0; it < maxIter; ++it) {
            Dep res = (yj + yi) * T(0.5);
            pr.prepareCalculations(res);
            pr.prepareJacobiCalculations(res);
            const Dep a = pr.getDeterministicVector(res, xj);
            const auto b = pr.getStochasticMatrix(res);
            auto Ja = pr.getJacobiDeterministic(res, xj, dt);
            auto Jb = pr.getJacobiStochastic(dW);
            if constexpr (P::HasExactJacobian) {
                if (exact) {  // analytic Newton matrix (not in the reference)
                    Ja = pr.getJacobiDeterministicExact(res, xj);
                    Jb = pr.getJacobiStochasticExact(res, dW);
                }
            }
            auto S = (Mat<T, D, D>::identity() * T(-1.0) + (T(0.5) * dt) * Ja) + T(0.5) * Jb;
            res = res + (a * dt + b * dW);
            pr.finishCalculations(res);
            res = res + (yi * T(0.5) - yj * T(1.5));
            pr.finishJacobiCalculations(S);
            Dep dx;
            Dep rhs = res * T(-1.0);
            ++st.iterations;
            if (!solve_dense<T, D>(S, rhs, dx)) break;
            yj = yj + dx;
            double n2 = 0.0;
            for (int i = 0; i < D; ++i) n2 += to_double(dx[i]) * to_double(dx[i]);
            if (std::sqrt(n2) <= tol) { converged = true; break; }
        }
        if (!converged) ++st.unconverged;
        return yj;
    }
};

// ====================================================================== double noise matrix
// SDEFramework/DoubleNoiseMatrix.h getNoiseMatrix (orders p >= 1, p = 0, p = -1),
// after Kloeden & Platen 1992, sec. 5.8: J(j1, j2) = dW_j1 dW_j2 / 2 +- A for j1 > j2,
// J(j1, j1) = dW_j1^2 / 2, with
//   A = -1/(2 pi) sum_{r=1}^{p} 1/r [z1 (sqrt2 dW_j2 - z2) - z3 (sqrt2 dW_j1 - z4)]
//       + rho_p (mu1 dW_j2 - mu2 dW_j1),   rho_p = sqrt(1/12 - sum_{r<=p} 1/(2 pi^2 r^2)).
// Every z and mu is a fresh N(0, dt) draw per pair, as the reference's generators
// advance on every call.  Draw order: pairs j1 = M-1..1, j2 = j1-1..0; per pair one
// Philox call (4 normals) per r, then one call whose first two normals are mu1, mu2;
// calls start at 2.
inline double double_noise_rho(int p) {
    double s = 0.0;
    for (int r = 1; r <= p; ++r) s += 1.0 / (static_cast<double>(r) * r);
    return std::sqrt(1.0 / 12.0 - s / (2.0 * kPi * kPi));
}
template <class T, int M>
Mat<T, M, M> double_noise_matrix(uint64_t seed, uint64_t pid, uint64_t step, int p, const T& sqrtdt,
                                 const Vec<T, M>& dW) {
    const T sqrt2 = T(1.4142135623730951), inv2pi = T(0.15915494309189535);
    const T rho = T(double_noise_rho(p));
    Mat<T, M, M> J = Mat<T, M, M>::zero();
    uint32_t call = 2;
    for (int j1 = M; j1--;) {
        for (int j2 = j1; j2--;) {
            J(j1, j2) = (T(0.5) * dW[j1]) * dW[j2];
            J(j2, j1) = J(j1, j2);
            T tmp = T(0.0);
            if (p >= 1) {
                T sum = T(0.0);
                for (int r = 1; r <= p; ++r) {
                    double z[4];
                    philox_call_normals(seed, pid, step, call++, z);
                    const T z1 = T(z[0]) * sqrtdt, z2 = T(z[1]) * sqrtdt, z3 = T(z[2]) * sqrtdt, z4 = T(z[3]) * sqrtdt;
                    sum = sum + (T(1.0) / T(r)) * (z1 * (sqrt2 * dW[j2] - z2) - z3 * (sqrt2 * dW[j1] - z4));
                }
                tmp = -sum * inv2pi;
            }
            if (p >= 0) {
                double u[4];
                philox_call_normals(seed, pid, step, call++, u);
                tmp = tmp + rho * ((T(u[0]) * sqrtdt) * dW[j2] - (T(u[1]) * sqrtdt) * dW[j1]);
            }
            J(j1, j2) = J(j1, j2) + tmp;
            J(j2, j1) = J(j2, j1) - tmp;
        }
        J(j1, j1) = (T(0.5) * dW[j1]) * dW[j1];
    }
    return J;
}

// ====================================================================== simulation
struct SimSpec {
    int problem, aniso, solver;
    ProblemCfg cfg;
    int maxIter; double tol;
    bool exactJacobian;
    int doubleNoiseApprox;
    uint64_t steps, W; double dt;
    FieldEval field;
    uint64_t seed, pid_offset;
    bool injected;
    const double* dw;   // [S_int][M][N]
    uint64_t N;
};

// One particle: SingleParticleSimulator::startSimulation
// (Simulator/SingleParticleSimulator.h:129-159).  Writes K window means.
template <class P, class T>
void simulate_particle(const SimSpec& sp, const ParticleIn& pin, uint64_t p, double* traj /*[K][OUT]*/,
                       double* final_state, NewtonStats& nst) {
    P pr;
    pr.init(pin, sp.cfg);
    using Dep = typename P::Dep;
    constexpr int OUT = P::OUT, M = P::M;
    const uint64_t K = sp.steps / sp.W;
    const T dt = T(sp.dt);
    const double sqrt_dt = std::sqrt(sp.dt);
    Dep yi = pr.getStart(pin);
    {
        const Vec<T, OUT> o = pr.calculateOutputResult(yi);
        for (int c = 0; c < OUT; ++c) traj[c] = to_double(o[c]);
    }
    Vec<T, OUT> sum = Vec<T, OUT>::zero(), comp = Vec<T, OUT>::zero();
    uint64_t counter = 0;
    double z[8];
    for (uint64_t k = 1; k < K; ++k) {
        for (uint64_t l = 0; l < sp.W; ++l) {
            const uint64_t n = counter;  // integrated-step index (0-based)
            const double time = sp.dt * static_cast<double>(++counter);
            Vec<T, M> dW;
            if (sp.injected) {
                for (int j = 0; j < M; ++j) dW[j] = T(sp.dw[(n * M + j) * sp.N + p]);
            } else {
                philox_normals(sp.seed, sp.pid_offset + p, n, M, z);
                for (int j = 0; j < M; ++j) dW[j] = T(sqrt_dt * z[j]);
            }
            double B[3];
            V3<T> xi;
            if (sp.solver == SP_SOLVER_IMPLICIT_MIDPOINT) {
                sp.field.eval(time + 0.5 * sp.dt, B);  // Implicit_Midpoint.inl:59
                for (int i = 0; i < 3; ++i) xi[i] = T(B[i]);
                if constexpr (P::HasJacobian)
                    yi = Stepper<P, T>::implicit_midpoint(pr, yi, xi, dW, dt, sp.maxIter, sp.tol, sp.exactJacobian, nst);
            } else {
                sp.field.eval(time, B);  // field at t_{n+1} (SingleParticleSimulator.h:145-146)
                for (int i = 0; i < 3; ++i) xi[i] = T(B[i]);
                switch (sp.solver) {
                    case SP_SOLVER_EULER_MARUYAMA: yi = Stepper<P, T>::euler_maruyama(pr, yi, xi, dW, dt); break;
                    case SP_SOLVER_HEUN_NOT_CONSISTENT: {
                        philox_normals(sp.seed, sp.pid_offset + p, n, M, z, 2);
                        Vec<T, M> dW2;
                        for (int j = 0; j < M; ++j) dW2[j] = T(sqrt_dt * z[j]);
                        yi = Stepper<P, T>::heun_not_consistent(pr, yi, xi, dW, dW2, dt);
                        break;
                    }
                    case SP_SOLVER_WEAK_TEST:
                    case SP_SOLVER_EXPLICIT_STRONG_1: {
                        const T sqdt = T(sqrt_dt);
                        const Mat<T, M, M> J =
                            double_noise_matrix<T, M>(sp.seed, sp.pid_offset + p, n, sp.doubleNoiseApprox, sqdt, dW);
                        yi = sp.solver == SP_SOLVER_WEAK_TEST ? Stepper<P, T>::weak_test(pr, yi, xi, dW, J, dt, sqdt)
                                                              : Stepper<P, T>::explicit_strong_1(pr, yi, xi, dW, J, dt, sqdt);
                        break;
                    }
                    case SP_SOLVER_HEUN_STRONG: yi = Stepper<P, T>::heun(pr, yi, xi, dW, dt); break;
                    case SP_SOLVER_EULER_MARUYAMA_NORMALIZED:
                        yi = Stepper<P, T>::euler_maruyama_normalized(pr, yi, xi, dW, dt);
                        break;
                    default: yi = Stepper<P, T>::millstein(pr, yi, xi, dW, dt); break;
                }
            }
            // Kahan summation of the output (:148-153); comp is not reset between windows
            const Vec<T, OUT> o = pr.calculateOutputResult(yi);
            const Vec<T, OUT> y = o - comp;
            const Vec<T, OUT> t = sum + y;
            comp = (t - sum) - y;
            sum = t;
        }
        for (int c = 0; c < OUT; ++c) traj[k * OUT + c] = to_double(sum[c] / T(static_cast<double>(sp.W)));
        sum = Vec<T, OUT>::zero();  // std::swap with the zero-initialised result slot (:156)
    }
    if (final_state)
        for (int i = 0; i < P::D; ++i) final_state[i] = to_double(yi[i]);
}

inline ParticleIn particle_in(const sp_ensemble_desc& d, uint64_t p) {
    const sp_particles& q = d.particles;
    ParticleIn r{};
    r.radius = q.magnetic_radius[p];
    r.Ms = q.saturation_magnetisation[p];
    r.alpha = q.damping_constant[p];
    r.gamma = q.gyromagnetic_ratio[p];
    r.K = q.anisotropy_constant[p];
    r.rh = q.hydrodynamic_radius ? q.hydrodynamic_radius[p] : 0.0;
    r.viscosity = q.viscosity ? q.viscosity[p] : 0.0;
    r.temperature = d.temperature;
    for (int i = 0; i < 3; ++i) { r.euler[i] = q.orientation[3 * p + i]; r.mag[i] = q.magnetisation[3 * p + i]; }
    if (d.anisotropy == SP_ANISOTROPY_UNIAXIAL_CUBIC) {
        r.K2 = q.cubic_constant[p];
        for (int i = 0; i < 3; ++i) r.urot[i] = q.uniaxial_rotation[3 * p + i];
    }
    return r;
}

inline int out_dim(int problem) {
    switch (problem) {
        case SP_PROBLEM_NEEL: return 3;
        case SP_PROBLEM_NEEL_SPHERICAL: return 3;
        case SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL: return 9;
        case SP_PROBLEM_BROWN_AND_NEEL: return 6;
    }
    return 0;
}
inline int state_dim(int problem) {
    switch (problem) {
        case SP_PROBLEM_NEEL: return 3;
        case SP_PROBLEM_NEEL_SPHERICAL: return 2;
        case SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL: return 5;
        case SP_PROBLEM_BROWN_AND_NEEL: return 6;
    }
    return 0;
}

template <class T>
using SimFn = void (*)(const SimSpec&, const ParticleIn&, uint64_t, double*, double*, NewtonStats&);

template <class T>
SimFn<T> pick(int problem, int aniso) {
    const bool cubic = aniso == SP_ANISOTROPY_CUBIC;
    if (aniso == SP_ANISOTROPY_UNIAXIAL_CUBIC) {
        switch (problem) {
            case SP_PROBLEM_NEEL: return &simulate_particle<NeelProblem<T, UniaxialCubic<T>>, T>;
            case SP_PROBLEM_NEEL_SPHERICAL: return &simulate_particle<NeelSphericalProblem<T, UniaxialCubic<T>>, T>;
            case SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL:
                return &simulate_particle<BrownNeelEulerProblem<T, UniaxialCubic<T>>, T>;
        }
        return nullptr;  // not defined for the coupled Cartesian problem
    }
    switch (problem) {
        case SP_PROBLEM_NEEL:
            return cubic ? &simulate_particle<NeelProblem<T, Cubic<T>>, T> : &simulate_particle<NeelProblem<T, Uniaxial<T>>, T>;
        case SP_PROBLEM_NEEL_SPHERICAL:
            return cubic ? &simulate_particle<NeelSphericalProblem<T, Cubic<T>>, T>
                         : &simulate_particle<NeelSphericalProblem<T, Uniaxial<T>>, T>;
        case SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL:
            return cubic ? &simulate_particle<BrownNeelEulerProblem<T, Cubic<T>>, T>
                         : &simulate_particle<BrownNeelEulerProblem<T, Uniaxial<T>>, T>;
        case SP_PROBLEM_BROWN_AND_NEEL:
            return cubic ? &simulate_particle<BrownNeelProblem<T, Cubic<T>, true>, T>
                         : &simulate_particle<BrownNeelProblem<T, Uniaxial<T>, false>, T>;
    }
    return nullptr;
}

template <class T>
void weights_of(int problem, int aniso, const ParticleIn& pin, const ProblemCfg& cfg, double* w) {
    const bool cubic = aniso == SP_ANISOTROPY_CUBIC;
    switch (problem) {
        case SP_PROBLEM_NEEL: { NeelProblem<T, Uniaxial<T>> p; p.init(pin, cfg); p.weighting(w); break; }
        case SP_PROBLEM_NEEL_SPHERICAL: { NeelSphericalProblem<T, Uniaxial<T>> p; p.init(pin, cfg); p.weighting(w); break; }
        case SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL: { BrownNeelEulerProblem<T, Uniaxial<T>> p; p.init(pin, cfg); p.weighting(w); break; }
        case SP_PROBLEM_BROWN_AND_NEEL: { BrownNeelProblem<T, Uniaxial<T>, false> p; p.init(pin, cfg); p.weighting(w); break; }
    }
    (void)cubic;
}

SimSpec spec_of(const sp_ensemble_desc& d) {
    SimSpec s{};
    s.problem = d.problem; s.aniso = d.anisotropy; s.solver = d.solver;
    s.cfg.useRot = d.problem_settings.use_coordinate_transformation != 0;
    s.cfg.minAngle = d.problem_settings.min_angle_before_transformation;
    s.cfg.useBrownRot = d.problem_settings.use_euler_coordinate_transformation != 0;
    s.cfg.brownMinAngle = d.problem_settings.brown_min_angle_before_transformation;
    s.cfg.useNeelRot = d.problem_settings.use_spherical_coordinate_transformation != 0;
    s.cfg.neelMinAngle = d.problem_settings.neel_min_angle_before_transformation;
    s.cfg.simpleModel = d.problem_settings.use_simple_model != 0;
    s.maxIter = d.max_iteration; s.tol = d.accuracy_goal;
    s.exactJacobian = d.jacobian == SP_JACOBIAN_EXACT;
    s.doubleNoiseApprox = d.double_noise_approx;
    s.steps = d.number_of_steps; s.W = d.oversampling; s.dt = d.timestep;
    s.field.init(d.field);
    s.seed = d.seed; s.pid_offset = d.particle_id_offset;
    s.injected = d.noise == SP_NOISE_INJECTED;
    s.dw = d.injected_dw;
    s.N = d.n_particles;
    return s;
}

// Simulator/SingleParticleSimulator.h:236-273 (time and window-mean field)
void time_and_field(const SimSpec& s, double* times, double* fields) {
    const uint64_t K = s.steps / s.W;
    if (K == 0) return;
    double start = 0.0, end = 0.0;
    const double timeshift = s.dt * static_cast<double>(s.W) * 0.5;
    times[0] = start;
    s.field.eval(start, fields);
    uint64_t counter = 0;
    for (uint64_t k = 1; k < K; ++k) {
        double tmp[3] = {0.0, 0.0, 0.0};
        start = end + s.dt;
        for (uint64_t l = 0; l < s.W; ++l) {
            double B[3];
            s.field.eval(s.dt * static_cast<double>(++counter), B);
            for (int i = 0; i < 3; ++i) tmp[i] += B[i];
        }
        end = s.dt * static_cast<double>(counter) + start;
        for (int i = 0; i < 3; ++i) fields[3 * k + i] = tmp[i] / static_cast<double>(s.W);
        times[k] = (end - start) - timeshift;
    }
}

}  // namespace orc

using namespace orc;

extern "C" {

int oracle_abi_version(void) { return 6; }

// Runs the ensemble described by desc.  mean[K][OUT], weight[OUT], time[K],
// field[K][3], traj[N][K][OUT] and final_state[N][D] are optional (NULL).
// precision_mode: 0 = double, 1 = long double.  Returns 0 on success.
int oracle_simulate(const sp_ensemble_desc* d_in, double* mean, double* weight, double* time, double* field,
                    double* traj, double* final_state, uint64_t* newton_stats, int nthreads, int precision_mode) {
    if (!d_in || d_in->oversampling == 0 || d_in->number_of_steps < d_in->oversampling) return 1;
    std::unique_ptr<ProvidedArrays> provided;
    if (d_in->provider) provided = std::make_unique<ProvidedArrays>(*d_in);
    const sp_ensemble_desc* d = provided ? &provided->desc : d_in;
    if (d->solver == SP_SOLVER_IMPLICIT_MIDPOINT && d->problem == SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL) return 2;
    if (d->solver == SP_SOLVER_IMPLICIT_MIDPOINT && d->jacobian == SP_JACOBIAN_EXACT && d->problem != SP_PROBLEM_NEEL)
        return 3;
    if (!pick<double>(d->problem, d->anisotropy)) return 4;
    if (d->solver >= SP_SOLVER_HEUN_NOT_CONSISTENT && d->noise == SP_NOISE_INJECTED) return 5;
    if ((d->solver == SP_SOLVER_WEAK_TEST || d->solver == SP_SOLVER_EXPLICIT_STRONG_1) &&
        (d->double_noise_approx < -1 || d->double_noise_approx > 10))
        return 6;
    const SimSpec s = spec_of(*d);
    const int OUT = out_dim(d->problem), SD = state_dim(d->problem);
    const uint64_t K = s.steps / s.W, N = d->n_particles;
    if (time && field) time_and_field(s, time, field);
    else if (time || field) {
        std::vector<double> t(K), f(3 * K);
        time_and_field(s, t.data(), f.data());
        if (time) std::memcpy(time, t.data(), K * sizeof(double));
        if (field) std::memcpy(field, f.data(), 3 * K * sizeof(double));
    }
    // particles are processed in fixed blocks whose partial sums are added in
    // block order, so the result does not depend on the thread count
    const uint64_t BLK = 64;
    const uint64_t nblk = (N + BLK - 1) / BLK;
    std::vector<double> partial(mean ? nblk * K * OUT : 0, 0.0);
    std::vector<double> wsum_blk(nblk * OUT, 0.0);
    std::atomic<uint64_t> nit{0}, nunc{0}, next{0};
    auto worker = [&]() {
        std::vector<double> tr(K * OUT);
        for (;;) {
            const uint64_t b = next.fetch_add(1);
            if (b >= nblk) break;
            NewtonStats nst;
            for (uint64_t p = b * BLK; p < std::min<uint64_t>(N, (b + 1) * BLK); ++p) {
                const ParticleIn pin = particle_in(*d, p);
                double* trp = traj ? traj + p * K * OUT : tr.data();
                double* fs = final_state ? final_state + p * SD : nullptr;
                if (precision_mode == 1) pick<long double>(s.problem, s.aniso)(s, pin, p, trp, fs, nst);
                else pick<double>(s.problem, s.aniso)(s, pin, p, trp, fs, nst);
                double w[9];
                weights_of<double>(s.problem, s.aniso, pin, s.cfg, w);
                for (int c = 0; c < OUT; ++c) wsum_blk[b * OUT + c] += w[c];
                if (mean)
                    for (uint64_t k = 0; k < K; ++k)
                        for (int c = 0; c < OUT; ++c) partial[(b * K + k) * OUT + c] += w[c] * trp[k * OUT + c];
            }
            nit += nst.iterations; nunc += nst.unconverged;
        }
    };
    int nt = nthreads > 0 ? nthreads : static_cast<int>(std::thread::hardware_concurrency());
    if (nt < 1) nt = 1;
    nt = static_cast<int>(std::min<uint64_t>(static_cast<uint64_t>(nt), nblk));
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    std::vector<double> wsum(OUT, 0.0);
    for (uint64_t b = 0; b < nblk; ++b) for (int c = 0; c < OUT; ++c) wsum[c] += wsum_blk[b * OUT + c];
    if (weight) for (int c = 0; c < OUT; ++c) weight[c] = wsum[c];
    if (mean) {
        // MeanSimulationResult::normalize (Results/MeanSimulationResult.h:63-75)
        bool allzero = true;
        for (int c = 0; c < OUT; ++c) allzero = allzero && wsum[c] == 0.0;
        for (uint64_t k = 0; k < K; ++k)
            for (int c = 0; c < OUT; ++c) {
                double acc = 0.0;
                for (uint64_t b = 0; b < nblk; ++b) acc += partial[(b * K + k) * OUT + c];
                mean[k * OUT + c] = allzero ? acc : acc / wsum[c];
            }
    }
    if (newton_stats) { newton_stats[0] = nit.load(); newton_stats[1] = nunc.load(); }
    return 0;
}

// Unit normals of the shared Philox stream: out[n_steps][m][n].
void oracle_philox_normals(uint64_t seed, uint64_t pid0, uint64_t n, uint64_t step0, uint64_t nsteps, int m, double* out) {
    double z[8];
    for (uint64_t s = 0; s < nsteps; ++s)
        for (uint64_t p = 0; p < n; ++p) {
            philox_normals(seed, pid0 + p, step0 + s, m, z);
            for (int j = 0; j < m; ++j) out[(s * m + j) * n + p] = z[j];
        }
}

// Double noise matrices of particles pid0..pid0+n-1 at one step with the step's own
// Philox dW (unit normals x sqrt(dt)): dw[n][m], J[n][m][m].  m = 3 or 6.
void oracle_double_noise_matrix(uint64_t seed, uint64_t pid0, uint64_t n, uint64_t step, int p, double dt, int m,
                                double* dw, double* J) {
    const double sqdt = std::sqrt(dt);
    for (uint64_t i = 0; i < n; ++i) {
        double z[8];
        philox_normals(seed, pid0 + i, step, m, z);
        if (m == 3) {
            Vec<double, 3> w;
            for (int j = 0; j < 3; ++j) { w[j] = sqdt * z[j]; dw[i * 3 + j] = w[j]; }
            const Mat<double, 3, 3> Jm = double_noise_matrix<double, 3>(seed, pid0 + i, step, p, sqdt, w);
            for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) J[(i * 3 + r) * 3 + c] = Jm(r, c);
        } else {
            Vec<double, 6> w;
            for (int j = 0; j < 6; ++j) { w[j] = sqdt * z[j]; dw[i * 6 + j] = w[j]; }
            const Mat<double, 6, 6> Jm = double_noise_matrix<double, 6>(seed, pid0 + i, step, p, sqdt, w);
            for (int r = 0; r < 6; ++r) for (int c = 0; c < 6; ++c) J[(i * 6 + r) * 6 + c] = Jm(r, c);
        }
    }
}

// The particles of a provider: out[n][20] as sp_provide_particles writes them.
void oracle_provide_particles(const sp_ensemble_desc* d, double* out) {
    for (uint64_t p = 0; p < d->n_particles; ++p)
        provide_particle(*d->provider, d->particle_id_offset + p, d->problem, d->anisotropy, out + 20 * p);
}

// Raw Philox4x32-10 block for a given counter/key (known-answer tests).
void oracle_philox4x32_10(const uint32_t* ctr_in, const uint32_t* key, uint32_t* out) {
    uint32_t c[4] = {ctr_in[0], ctr_in[1], ctr_in[2], ctr_in[3]};
    philox4x32_10(c, key[0], key[1]);
    for (int i = 0; i < 4; ++i) out[i] = c[i];
}

// Neel parameters (ParameterCalculatorNeel.h:44-92): out = NF1, NF2, DriftPrefactor, NoisePrefactor, Damping
void oracle_neel_params(double radius, double Ms, double alpha, double gamma, double temperature, double* out) {
    const NeelParamsD p = calc_neel_params(radius, Ms, alpha, gamma, temperature);
    out[0] = p.NeelFactor1; out[1] = p.NeelFactor2; out[2] = p.DriftPrefactor; out[3] = p.NoisePrefactor; out[4] = p.Damping;
}
// Brown parameters (ParameterCalculatorBrown.h:39-58): out = BrownPrefactor, BrownDiffusion, Brown_F_Noise
void oracle_brown_params(double rh, double viscosity, double temperature, double* out) {
    const BrownParamsD p = calc_brown_params(rh, viscosity, temperature);
    out[0] = p.BrownPrefactor; out[1] = p.BrownDiffusion; out[2] = p.Brown_F_Noise;
}

// Uniaxial anisotropy pieces (UniaxialAnisotropy.h): field[3], jacobi[9] (row-major)
void oracle_uniaxial(double K, double Ms, double radius, const double* m, const double* axis, double* field, double* jac) {
    Uniaxial<double> u; u.init(K, Ms, sphere_volume(radius));
    V3<double> mm, n, z = V3<double>::zero();
    for (int i = 0; i < 3; ++i) { mm[i] = m[i]; n[i] = axis[i]; }
    const V3<double> h = u.getAnisotropyField(mm, z, z, n);
    const M3<double> J = u.getJacobiAnisotropyField(mm, z, z, n);
    for (int i = 0; i < 3; ++i) { field[i] = h[i]; for (int j = 0; j < 3; ++j) jac[3 * i + j] = J(i, j); }
}
// Cubic anisotropy pieces (CubicAnisotropy.h:110-193): field[3], torque[3]
void oracle_cubic(double K1, double Ms, double radius, const double* m, const double* x, const double* y, const double* z,
                  const double* statesin, const double* statecos, double* field, double* torque) {
    Cubic<double> cb; cb.init(K1, Ms, sphere_volume(radius));
    V3<double> mm, xx, yy, zz;
    for (int i = 0; i < 3; ++i) { mm[i] = m[i]; xx[i] = x[i]; yy[i] = y[i]; zz[i] = z[i]; }
    cb.prepareField(mm, xx, yy, zz);
    const V3<double> h = cb.getAnisotropyField(mm, xx, yy, zz);
    const V3<double> t = cb.getEffTorque(mm, xx, yy, zz, statesin, statecos);
    for (int i = 0; i < 3; ++i) { field[i] = h[i]; torque[i] = t[i]; }
}

// B(t) of a field description at n times: out[n][3]
void oracle_field_eval(const sp_field_desc* f, const double* times, uint64_t n, double* out) {
    FieldEval fe;
    fe.init(*f);
    for (uint64_t i = 0; i < n; ++i) fe.eval(times[i], out + 3 * i);
}

// Exact Neel (Cartesian) Jacobians at state m (the analytic Newton matrix of
// SP_JACOBIAN_EXACT): jdet[9] = d a / d m, jsto[9] = d (b(m) dW) / d m, row-major.
// props: radius, Ms, alpha, gamma, K, temperature
void oracle_neel_exact_jacobians(int aniso, const double* props, const double* euler, const double* m,
                                 const double* field, const double* dW, double* jdet, double* jsto) {
    ParticleIn pin{};
    pin.radius = props[0]; pin.Ms = props[1]; pin.alpha = props[2]; pin.gamma = props[3]; pin.K = props[4];
    pin.temperature = props[5];
    for (int i = 0; i < 3; ++i) { pin.euler[i] = euler[i]; pin.mag[i] = 0.0; }
    ProblemCfg cfg;
    auto run = [&](auto& pr) {
        pr.init(pin, cfg);
        V3<double> y, B, w;
        for (int i = 0; i < 3; ++i) { y[i] = m[i]; B[i] = field[i]; w[i] = dW[i]; }
        const auto Ja = pr.getJacobiDeterministicExact(y, B);
        const auto Jb = pr.getJacobiStochasticExact(y, w);
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) { jdet[3 * i + j] = Ja(i, j); jsto[3 * i + j] = Jb(i, j); }
    };
    if (aniso == SP_ANISOTROPY_CUBIC) { NeelProblem<double, Cubic<double>> p; run(p); }
    else { NeelProblem<double, Uniaxial<double>> p; run(p); }
}

// Evaluates one problem at one state the way the reference's unit tests do:
// prepareCalculations(state) (which may rotate it), then the requested pieces.
//  props: radius, Ms, alpha, gamma, K, rh, viscosity, temperature
//  settings: useRot, minAngle, useBrownRot, brownMin, useNeelRot, neelMin, simpleModel
//  outputs (any may be NULL): prepared[D], a[D], b[D*M], drift[D], jdet[D*D], jsto[D*D],
//  finished[D] (finishCalculations applied to the prepared state), rotated[2]
int oracle_eval_problem(int problem, int aniso, const double* props, const double* euler, const double* settings,
                        const double* state, const double* field, double dt, const double* dW,
                        double* prepared, double* a, double* b, double* drift, double* jdet, double* jsto,
                        double* finished, int* rotated, int finish_jacobi) {
    ParticleIn pin{};
    pin.radius = props[0]; pin.Ms = props[1]; pin.alpha = props[2]; pin.gamma = props[3]; pin.K = props[4];
    pin.rh = props[5]; pin.viscosity = props[6]; pin.temperature = props[7];
    for (int i = 0; i < 3; ++i) { pin.euler[i] = euler[i]; pin.mag[i] = 0.0; }
    ProblemCfg cfg;
    cfg.useRot = settings[0] != 0.0; cfg.minAngle = settings[1];
    cfg.useBrownRot = settings[2] != 0.0; cfg.brownMinAngle = settings[3];
    cfg.useNeelRot = settings[4] != 0.0; cfg.neelMinAngle = settings[5];
    cfg.simpleModel = settings[6] != 0.0;
    auto run = [&](auto& pr, bool) {
        using PR = std::decay_t<decltype(pr)>;
        constexpr int D = PR::D, M = PR::M;
        pr.init(pin, cfg);
        typename PR::Dep y;
        for (int i = 0; i < D; ++i) y[i] = state[i];
        pr.prepareCalculations(y);
        V3<double> B; for (int i = 0; i < 3; ++i) B[i] = field ? field[i] : 0.0;
        if (prepared) for (int i = 0; i < D; ++i) prepared[i] = y[i];
        if (a) { const auto v = pr.getDeterministicVector(y, B); for (int i = 0; i < D; ++i) a[i] = v[i]; }
        if (b) { const auto m = pr.getStochasticMatrix(y); for (int i = 0; i < D; ++i) for (int j = 0; j < M; ++j) b[i * M + j] = m(i, j); }
        if (drift) { const auto v = pr.getDrift(y); for (int i = 0; i < D; ++i) drift[i] = v[i]; }
        if constexpr (PR::HasJacobian) if (jdet || jsto) {
            pr.prepareJacobiCalculations(y);
            if (jdet) {
                auto J = pr.getJacobiDeterministic(y, B, dt);
                if (finish_jacobi) pr.finishJacobiCalculations(J);
                for (int i = 0; i < D; ++i) for (int j = 0; j < D; ++j) jdet[i * D + j] = J(i, j);
            }
            if (jsto) {
                Vec<double, M> w; for (int j = 0; j < M; ++j) w[j] = dW ? dW[j] : 0.0;
                auto J = pr.getJacobiStochastic(w);
                if (finish_jacobi) pr.finishJacobiCalculations(J);
                for (int i = 0; i < D; ++i) for (int j = 0; j < D; ++j) jsto[i * D + j] = J(i, j);
            }
        }
        if (finished) { auto f = y; pr.finishCalculations(f); for (int i = 0; i < D; ++i) finished[i] = f[i]; }
        return 0;
    };
    const bool cubic = aniso == SP_ANISOTROPY_CUBIC;
    int r = 0;
    switch (problem) {
        case SP_PROBLEM_NEEL:
            if (cubic) { NeelProblem<double, Cubic<double>> p; r = run(p, true); }
            else { NeelProblem<double, Uniaxial<double>> p; r = run(p, true); }
            break;
        case SP_PROBLEM_NEEL_SPHERICAL:
            if (cubic) { NeelSphericalProblem<double, Cubic<double>> p; r = run(p, true); if (rotated) rotated[0] = p.isRotated; }
            else { NeelSphericalProblem<double, Uniaxial<double>> p; r = run(p, true); if (rotated) rotated[0] = p.isRotated; }
            break;
        case SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL:
            if (cubic) { BrownNeelEulerProblem<double, Cubic<double>> p; r = run(p, false); if (rotated) { rotated[0] = p.bIsRotated; rotated[1] = p.nIsRotated; } }
            else { BrownNeelEulerProblem<double, Uniaxial<double>> p; r = run(p, false); if (rotated) { rotated[0] = p.bIsRotated; rotated[1] = p.nIsRotated; } }
            break;
        case SP_PROBLEM_BROWN_AND_NEEL:
            if (cubic) { BrownNeelProblem<double, Cubic<double>, true> p; r = run(p, true); }
            else { BrownNeelProblem<double, Uniaxial<double>, false> p; r = run(p, true); }
            break;
        default: return 1;
    }
    return r;
}

// Algorithmic work of the restated step formulas (RNG excluded): runs one
// particle for n_steps with the counting scalar and returns per-step averages
// out = {flops, divs, transcendentals, sqrts, newton_iterations}.
int oracle_count_ops(const sp_ensemble_desc* d, double* out) {
    if (!d) return 1;
    sp_ensemble_desc one = *d;
    one.n_particles = 1;
    one.noise = SP_NOISE_PHILOX;
    const SimSpec s = spec_of(one);
    const uint64_t K = s.steps / s.W;
    std::vector<double> tr(K * out_dim(d->problem));
    NewtonStats nst;
    const ParticleIn pin = particle_in(*d, 0);
    g_ops = OpCounts{};
    // field evaluation and noise generation are outside the counted arithmetic
    // because they run with doubles; only the Cnt-typed problem/solver math counts
    SimFn<Cnt> fn = pick<Cnt>(s.problem, s.aniso);
    if (!fn) return 2;
    fn(s, pin, 0, tr.data(), nullptr, nst);
    const double steps = static_cast<double>((K - 1) * s.W);
    out[0] = g_ops.flops / steps; out[1] = g_ops.divs / steps; out[2] = g_ops.transc / steps; out[3] = g_ops.sqrts / steps;
    out[4] = nst.iterations / steps;
    return 0;
}

}  // extern "C"
