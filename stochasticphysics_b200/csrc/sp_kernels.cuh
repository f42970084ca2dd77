// sp_kernels.cuh — kernel templates of the ensemble engine (sm_100a).
//
//  init_kernel      per-particle prefactors (FP64 formulas of
//                   Problems/Helpers/ParameterCalculator{Neel,Brown}.h), the
//                   initial state (getStart of each problem), sample 0 and the
//                   weights (getWeighting), reduced per warp
//  step_kernel      one chunk of steps for a list of particle tiles, one or two
//                   particles per thread: the state lives in registers, each warp
//                   stages the chunk's B(t) table (computed once per step in FP64 by
//                   field_chunk_kernel) in shared memory, the Wiener increments come
//                   from in-kernel Philox (or from HBM in injection mode, staged a few
//                   steps ahead in shared memory by bulk copies), each step's output sines and
//                   cosines carry to the next step's prepare, and each window's Kahan
//                   mean is reduced per warp in FP64 and stored in one coalesced store
//                   (SingleParticleSimulator.h:129-159, MeanSimulationResult.h:87-119)
//  reduce_kernel    per-warp window partials -> ensemble sums, fixed order
//  commit_kernel    advances the device step counter (graph replay)
//  field_window_kernel  window-mean field of the Results contract
//                   (SingleParticleSimulator.h:236-273)
#pragma once

#include "sp_physics.cuh"
#include "sp_stage.cuh"

namespace sp {

// ------------------------------------------------------------------ problem traits
template <int PROB, class R, int A> struct ProblemOf;
template <class R, int A> struct ProblemOf<kNeel, R, A> { using type = NeelCart<R, A>; static constexpr int P = param_count_of(kNeel, A); };
template <class R, int A> struct ProblemOf<kNeelSpherical, R, A> { using type = NeelSph<R, A>; static constexpr int P = param_count_of(kNeelSpherical, A); };
template <class R, int A> struct ProblemOf<kBrownNeelEuler, R, A> { using type = BrownNeelEuler<R, A>; static constexpr int P = param_count_of(kBrownNeelEuler, A); };
template <class R, int A> struct ProblemOf<kBrownNeel, R, A> { using type = BrownNeelCart<R, A>; static constexpr int P = param_count_of(kBrownNeel, A); };

// ------------------------------------------------------------------ FP64 parameter formulas
constexpr double kBoltzmann = 1.3806485279E-23;  // ParameterCalculatorNeel.h:43
constexpr double kPiD = 3.14159265358979323846;

__device__ __forceinline__ double sphere_volume(double r) { return 4.0 / 3.0 * kPiD * r * r * r; }

struct NeelP { double NF1, NF2, Dp, DN; };
// ParameterCalculatorNeel.h:44-92
__device__ __forceinline__ NeelP neel_params(double r, double Ms, double alpha, double gamma, double T) {
    NeelP p;
    const double moment = sphere_volume(r) * Ms;
    double diffsquare = 2.0 * alpha * kBoltzmann * T / (gamma * moment);
    if (isinf(diffsquare) || isnan(diffsquare)) diffsquare = 0.0;
    if (isinf(alpha)) { p.NF1 = 0.0; p.NF2 = 0.0; }
    else { p.NF1 = -gamma / (1.0 + alpha * alpha); p.NF2 = fabs(p.NF1) * alpha; }
    p.Dp = (diffsquare == 0.0) ? 0.0 : -1.0 * (p.NF1 * p.NF1) * (1.0 + alpha * alpha) * diffsquare;
    p.DN = sqrt(diffsquare);
    return p;
}
struct BrownP { double c, DB, cF; };
// ParameterCalculatorBrown.h:39-58
__device__ __forceinline__ BrownP brown_params(double rh, double eta, double T) {
    BrownP p;
    const double vh = sphere_volume(rh);
    p.c = 1.0 / (6.0 * eta * vh);
    p.DB = sqrt(2.0 * kBoltzmann * T * (6.0 * eta * vh));
    if (isinf(p.DB) || isnan(p.DB)) p.DB = 0.0;
    if (isnan(p.c)) p.c = 0.0;
    p.cF = p.c * p.DB;
    return p;
}
// NeelRelaxation.h:240-260 / ParticleStateInitializer.h:64-105
__device__ __forceinline__ void euler_axes(const double* e, double* x, double* y, double* z) {
    double sphi, cphi, stheta, ctheta, spsi, cpsi;
    sincos(e[0], &sphi, &cphi);
    sincos(e[1], &stheta, &ctheta);
    sincos(e[2], &spsi, &cpsi);
    const double cphicpsi = cphi * cpsi, sphicpsi = sphi * cpsi, cphispsi = cphi * spsi, sphispsi = sphi * spsi;
    x[0] = cphicpsi - ctheta * sphispsi; x[1] = -sphicpsi - ctheta * cphispsi; x[2] = stheta * spsi;
    y[0] = ctheta * sphicpsi + cphispsi; y[1] = ctheta * cphicpsi - sphispsi; y[2] = -stheta * cpsi;
    z[0] = stheta * sphi; z[1] = stheta * cphi; z[2] = ctheta;
}

// UniaxialCubicAnisotropy.hpp:57-83 calcRotation: rotation of the uniaxial part from its
// Euler angles, row-major
__device__ __forceinline__ void uniaxial_rotation(const double* e, double* Rm) {
    double sphi, cphi, stheta, ctheta, spsi, cpsi;
    sincos(e[0], &sphi, &cphi);
    sincos(e[1], &stheta, &ctheta);
    sincos(e[2], &spsi, &cpsi);
    const double cphicpsi = cphi * cpsi, sphicpsi = sphi * cpsi, cphispsi = cphi * spsi, sphispsi = sphi * spsi;
    Rm[0] = cphicpsi - ctheta * sphispsi; Rm[1] = -sphicpsi - ctheta * cphispsi; Rm[2] = stheta * spsi;
    Rm[3] = ctheta * sphicpsi + cphispsi; Rm[4] = ctheta * cphicpsi - sphispsi; Rm[5] = -stheta * cpsi;
    Rm[6] = stheta * sphi; Rm[7] = stheta * cphi; Rm[8] = ctheta;
}

// Fills params[k] (FP64) and the initial state y (FP64) of particle p.
template <int PROB, int A>
__device__ __forceinline__ void particle_setup(const RawParticles& rp, unsigned long long p, double* prm, double* y,
                                               double& moment) {
    const double r = rp.radius[p], Ms = rp.Ms[p], alpha = rp.alpha[p], gamma = rp.gamma[p], K = rp.K[p];
    const double V = sphere_volume(r);
    moment = V * Ms;
    const double e[3] = {rp.euler[3 * p], rp.euler[3 * p + 1], rp.euler[3 * p + 2]};
    const double mg[3] = {rp.mag[3 * p], rp.mag[3 * p + 1], rp.mag[3 * p + 2]};
    const NeelP np = neel_params(r, Ms, alpha, gamma, rp.temperature);
    const double pF = -2.0 * K / Ms;  // UniaxialAnisotropy.h:71-77, CubicAnisotropy.h:93
    if constexpr (PROB == kNeel || PROB == kNeelSpherical) {
        double x[3], yy[3], z[3];
        euler_axes(e, x, yy, z);
        if constexpr (PROB == kNeel) {
            prm[0] = np.NF1; prm[1] = np.NF2; prm[2] = np.Dp; prm[3] = np.NF1 * np.DN; prm[4] = np.NF2 * np.DN;
            prm[5] = pF; prm[6] = 2.0 * alpha;
            for (int i = 0; i < 3; ++i) { prm[7 + i] = z[i]; prm[10 + i] = x[i]; prm[13 + i] = yy[i]; }
            const double n = sqrt(mg[0] * mg[0] + mg[1] * mg[1] + mg[2] * mg[2]);  // NeelRelaxation.h:283
            y[0] = mg[0] / n; y[1] = mg[1] / n; y[2] = mg[2] / n;
        } else {
            prm[0] = np.NF1; prm[1] = np.NF2; prm[2] = np.Dp; prm[3] = np.DN; prm[4] = pF; prm[5] = 2.0 * alpha;
            for (int i = 0; i < 3; ++i) { prm[6 + i] = z[i]; prm[9 + i] = x[i]; prm[12 + i] = yy[i]; }
            y[0] = acos(mg[2]); y[1] = atan2(mg[1], mg[0]);  // ParticleStateInitializer.h:132-144
        }
        if constexpr (A == kUniaxialCubic) {
            // cubic field prefactor and the uniaxial axis R^T z (UniaxialCubicAnisotropy.hpp:104-110)
            const int o = (PROB == kNeel) ? kParamsNeel : kParamsNeelSph;
            double Rm[9];
            uniaxial_rotation(rp.urot + 3 * p, Rm);
            prm[o] = -2.0 * rp.K2[p] / Ms;
            for (int i = 0; i < 3; ++i) prm[o + 1 + i] = Rm[0 * 3 + i] * z[0] + Rm[1 * 3 + i] * z[1] + Rm[2 * 3 + i] * z[2];
        }
    } else {
        const BrownP bp = brown_params(rp.rh[p], rp.viscosity[p], rp.temperature);
        const double a = np.NF1, b = np.NF2, DN = np.DN;
        const double d = bp.c * moment;  // BrownAndNeelRelaxationEulerSpherical.h:390
        const double bpd = b + d;
        const double cT = bp.c * (-2.0 * K * V);  // c * torque prefactor (UniaxialAnisotropy.h:79-85)
        if constexpr (PROB == kBrownNeelEuler) {
            prm[0] = a; prm[1] = bpd; prm[2] = d; prm[3] = cT; prm[4] = pF; prm[5] = bp.cF;
            prm[6] = d * DN; prm[7] = bpd * DN; prm[8] = a * DN;
            prm[9] = a * d * (DN * DN); prm[10] = 0.25 * (d * DN) * (d * DN); prm[11] = 0.5 * bp.cF * bp.cF;
            prm[12] = 0.5 * bp.cF * bp.cF + 0.5 * (a * a + bpd * bpd) * (DN * DN);
            y[0] = e[0]; y[1] = e[1]; y[2] = e[2];  // BrownAndNeelRelaxationEulerSpherical.h:741-753
            y[3] = acos(mg[2]); y[4] = atan2(mg[1], mg[0]);
            if constexpr (A == kUniaxialCubic) {
                // cubic field and torque prefactors and the uniaxial rotation R
                // (UniaxialCubicAnisotropy.hpp:104-121: field with R^T z, torque of R m)
                prm[13] = -2.0 * rp.K2[p] / Ms;
                prm[14] = bp.c * (-2.0 * rp.K2[p] * V);
                uniaxial_rotation(rp.urot + 3 * p, prm + 15);
            }
        } else {
            const bool simple = rp.simple_model != 0;
            prm[0] = a; prm[1] = bpd; prm[2] = d; prm[3] = cT; prm[4] = pF; prm[5] = bp.cF;
            prm[6] = simple ? 0.0 : d * DN;
            prm[7] = (simple ? b : bpd) * DN;
            prm[8] = a * DN;
            prm[9] = bp.cF * bp.cF;
            prm[10] = simple ? 0.0 : d * a * (DN * DN);
            prm[11] = simple ? 0.0 : 0.5 * d * d * (DN * DN);
            prm[12] = simple ? (a * a + b * b) * (DN * DN) : bp.cF * bp.cF + (a * a + bpd * bpd) * (DN * DN);
            prm[13] = simple ? 0.0 : bp.cF;
            // BrownAndNeelRelaxation.inl:278-324 with given orientation and magnetisation
            double sa, ca, sb, cb, sg, cg;
            sincos(e[0], &sa, &ca); sincos(e[1], &sb, &cb); sincos(e[2], &sg, &cg);
            double n[3] = {ca * cg - sa * cb * sg, -ca * sg - sa * cb * cg, sa * sb};
            const double nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            const double mm = sqrt(mg[0] * mg[0] + mg[1] * mg[1] + mg[2] * mg[2]);
            for (int i = 0; i < 3; ++i) { y[i] = n[i] / nn; y[3 + i] = mg[i] / mm; }
        }
    }
}

template <int PROB>
__device__ __forceinline__ double weight_of(int c, double moment) {
    if constexpr (PROB == kBrownNeel) return c < 3 ? 1.0 : moment;  // BrownAndNeelRelaxation.h:152-159
    else return moment;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ------------------------------------------------------------------ init
// partial slot 0 <- weighted sample 0, slot 1 <- weights (per warp)
template <int PROB, class R, int A>
__global__ void __launch_bounds__(kMaxBlock) init_kernel(const EnsDev* __restrict__ ens, RawParticles rp) {
    using Prob = typename ProblemOf<PROB, R, A>::type;
    constexpr int D = Prob::D, OUT = Prob::OUT, P = ProblemOf<PROB, R, A>::P;
    const EnsDev& e = *ens;
    const unsigned long long p = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const unsigned long long Np = e.Np;
    if (p >= Np) return;
    const bool active = p < e.n;
    R* state = static_cast<R*>(e.state);
    R* ks = static_cast<R*>(e.ksum);
    R* kc = static_cast<R*>(e.kcomp);
    R* prm = const_cast<R*>(static_cast<const R*>(e.params));
    double yd[D], pd[P > 0 ? P : 1], moment = 0.0;
    if (active) {
        particle_setup<PROB, A>(rp, p, pd, yd, moment);
    } else {
        for (int i = 0; i < D; ++i) yd[i] = 0.0;
        for (int i = 0; i < P; ++i) pd[i] = 0.0;
    }
    R y[D];
    for (int i = 0; i < D; ++i) { y[i] = static_cast<R>(yd[i]); state[i * Np + p] = y[i]; }
    for (int i = 0; i < P; ++i) prm[i * Np + p] = static_cast<R>(pd[i]);
    const_cast<double*>(e.moment)[p] = moment;
    for (int c = 0; c < OUT; ++c) { ks[c * Np + p] = R(0); kc[c * Np + p] = R(0); }
    if (e.slo)
        for (int i = 0; i < D; ++i) static_cast<R*>(e.slo)[i * Np + p] = R(0);
    e.status[p] = 0;
    R o[OUT];
    Prob::out(y, o);
    const unsigned long long warp = p >> 5;
    const int lane = threadIdx.x & 31;
    for (int c = 0; c < OUT; ++c) {
        const double w = active ? weight_of<PROB>(c, moment) : 0.0;
        const double vo = active ? static_cast<double>(o[c]) : 0.0;
        if (e.traj && active && (p + 1) % e.traj_stride == 0)
            e.traj[static_cast<unsigned long long>(c) * e.traj_n + (p + 1) / e.traj_stride - 1] = vo;
        const double s0 = warp_sum(w * vo), s1 = warp_sum(w);
        if (lane == 0) {
            e.partial[(warp * e.slots + 0) * OUT + c] = s0;
            e.partial[(warp * e.slots + 1) * OUT + c] = s1;
        }
    }
}

// ------------------------------------------------------------------ window sums
// Kahan summation of each step's output over a window (SingleParticleSimulator.h:148-153);
// the compensation carries over from one window to the next, the sum restarts.
template <class R, int OUT>
struct WindowSum {
    R sum[OUT], comp[OUT];
    __device__ __forceinline__ void set(int c, R s, R k) { sum[c] = s; comp[c] = k; }
    __device__ __forceinline__ R get_sum(int c) const { return sum[c]; }
    __device__ __forceinline__ R get_comp(int c) const { return comp[c]; }
    __device__ __forceinline__ void clear_sum(int c) { sum[c] = R(0); }
    __device__ __forceinline__ void add(const R* o) {
#pragma unroll
        for (int c = 0; c < OUT; ++c) {
            const R yv = o[c] - comp[c];
            const R tv = sum[c] + yv;
            comp[c] = (tv - sum[c]) - yv;
            sum[c] = tv;
        }
    }
};
// FP32: two outputs per 64-bit register, both updated by one paired instruction
// (add/sub.rn.f32x2); each lane rounds exactly as the scalar form does.
__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float2 unpack2(unsigned long long v) {
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
    return make_float2(lo, hi);
}
__device__ __forceinline__ unsigned long long add2(unsigned long long a, unsigned long long b) {
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long sub2(unsigned long long a, unsigned long long b) {
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
template <int OUT>
struct WindowSum<float, OUT> {
    static constexpr int NP = (OUT + 1) / 2;
    unsigned long long sum[NP] = {}, comp[NP] = {};  // an odd OUT leaves a zero lane
    __device__ __forceinline__ void set(int c, float s, float k) {
        const float2 a = unpack2(sum[c / 2]), b = unpack2(comp[c / 2]);
        sum[c / 2] = (c & 1) ? pack2(a.x, s) : pack2(s, a.y);
        comp[c / 2] = (c & 1) ? pack2(b.x, k) : pack2(k, b.y);
    }
    __device__ __forceinline__ float get_sum(int c) const {
        const float2 a = unpack2(sum[c / 2]);
        return (c & 1) ? a.y : a.x;
    }
    __device__ __forceinline__ float get_comp(int c) const {
        const float2 a = unpack2(comp[c / 2]);
        return (c & 1) ? a.y : a.x;
    }
    __device__ __forceinline__ void clear_sum(int c) {
        const float2 a = unpack2(sum[c / 2]);
        sum[c / 2] = (c & 1) ? pack2(a.x, 0.0f) : pack2(0.0f, a.y);
    }
    __device__ __forceinline__ void add(const float* o) {
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const unsigned long long v = pack2(o[2 * k], 2 * k + 1 < OUT ? o[2 * k + 1] : 0.0f);
            const unsigned long long yv = sub2(v, comp[k]);
            const unsigned long long tv = add2(sum[k], yv);
            comp[k] = sub2(sub2(tv, sum[k]), yv);
            sum[k] = tv;
        }
    }
};

// ------------------------------------------------------------------ step
// One tile = blockDim.x * PPT particles of one ensemble; thread t integrates particles
// first + k blockDim.x + t, k < PPT.  With PPT = 2 each thread carries two independent
// step chains, which the scheduler interleaves (instruction-level parallelism in a
// latency-bound loop).  Each particle runs the same source arithmetic for every PPT; the
// instantiations are compiled separately, so results agree to rounding.
//
// Resident CTAs of kMaxBlock threads the compiler must allow per SM (0: its own choice,
// as without the bound; an explicit 1 lets it take up to 255 registers, which made the
// FP32 kernels 25 % slower at 163-167 registers instead of 128).  The FP64 explicit steps
// of Brown+Neel Euler/spherical use about 230-255 registers left alone (8 warps per SM, whose FP64
// dependency chains leave the issue slots idle: the leading stall is `wait`); held to 128
// registers they spill some state to local memory, which L1 serves, and run 16 warps per
// SM: 25-31 % more particle-steps/s for an ensemble that fills the GPU (FP64 Millstein,
// 262144 particles: 9.2e9 against 7.0e9; caps of 96, 112, 144 and 200 registers were
// slower).  The Brown+Neel Cartesian ones (168-182 registers left alone) gain 12-22 % the
// same way (Heun, 262144 particles: 2.43e10 against 2.13e10); the Neel kernels need no more
// than 128 registers anyway.  Of the implicit-midpoint kernels (222-235 registers left
// alone) the exact-Jacobian one gains 16 % (cubic Neel, 262144 particles: 6.13e9 against
// 5.27e9) and the reference-matrix one, whose 20 Newton iterations spill more, loses 5 %,
// so only the former is bound.  Register allocation does not change the arithmetic.
template <int PROB, class R, int SOLVER, bool INJECT, int PPT>
constexpr int step_min_blocks() {
    return (sizeof(R) == 8 && !INJECT && PPT == 1 &&
            (SOLVER == kEulerMaruyama || SOLVER == kHeun || SOLVER == kMillstein || SOLVER == kEulerMaruyamaNormalized ||
             SOLVER == kImplicitMidpointExact))
               ? 2
               : 0;
}
template <int PROB, class R, int A, int SOLVER, bool INJECT, int PPT>
__global__ void __launch_bounds__(kMaxBlock / PPT, (step_min_blocks<PROB, R, SOLVER, INJECT, PPT>()))
    step_kernel(const EnsDev* __restrict__ ensembles, const TileDesc* __restrict__ tiles, int ntiles) {
    using Prob = typename ProblemOf<PROB, R, A>::type;
    using St = Stepper<Prob, R, SOLVER>;
    constexpr int D = Prob::D, Mn = Prob::Mn, OUT = Prob::OUT;
    // per-warp copy of the chunk's field table: warps never wait on each other
    // (a CTA-wide barrier every tile made fast warps wait for slow ones).  Injected kernels
    // stage 32 steps at a time, leaving shared memory to the increments' ring.
    constexpr int FT = INJECT ? 32 : kFieldTile;
    __shared__ R sBw[kMaxBlock / 32][FT][3];
    R(*const sB)[3] = sBw[threadIdx.x >> 5];
    // injection mode: each warp's ring of staged increments (dynamic shared memory)
    using Stream = DwStream<R, Mn>;
    static_assert(!INJECT || PPT == 1, "injected increments are staged for one particle per thread");
    Stream dws;
    if constexpr (INJECT) {
        extern __shared__ __align__(128) unsigned char sp_dyn_smem[];
        __shared__ uint64_t sbar[kMaxBlock / 32][Stream::kStages];
        const int warp = threadIdx.x >> 5;
        dws.init(reinterpret_cast<R*>(sp_dyn_smem + static_cast<size_t>(warp) * Stream::kStages * Stream::kStageBytes),
                 sbar[warp]);
    }

    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const TileDesc td = tiles[t];
        const EnsDev& e = ensembles[td.ens];
        const unsigned long long s0 = e.ctl->step_done, tgt = e.ctl->step_target;
        const unsigned long long nsteps = tgt > s0 ? min(e.chunk, tgt - s0) : 0ull;
        if (nsteps == 0) continue;  // uniform across the CTA
        const unsigned long long Np = e.Np, W = e.W;
        unsigned long long p[PPT];
        bool active[PPT];
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            p[k] = td.first + static_cast<unsigned long long>(k) * blockDim.x + threadIdx.x;
            active[k] = p[k] < e.n;
        }
        const double dt_d = e.dt;
        const R dt = static_cast<R>(dt_d);
        const R sqdt = static_cast<R>(e.sqrt_dt);
        const R m2dt = static_cast<R>(-2.0 * dt_d);  // FP32 Box-Muller radius scale
        const unsigned long long seed = e.seed;
        const R* ftab = static_cast<const R*>(e.ftab);
        Rot<R> rot;
        rot.rb = e.rot_brown != 0; rot.rn = e.rot_neel != 0;
        rot.min1 = static_cast<R>(e.min1); rot.max1 = static_cast<R>(e.max1);
        rot.min2 = static_cast<R>(e.min2); rot.max2 = static_cast<R>(e.max2);

        R y[PPT][D];
        R lo[PPT][D];  // FP32 form: the carried rounding errors of the slowly moving components
        WindowSum<R, OUT> acc[PPT];
        typename Prob::Par q[PPT];
        typename Prob::Trig tr[PPT];  // sincos of y, carried from each step's output to the next prepare
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            if (active[k]) {
                const R* state = static_cast<const R*>(e.state);
                const R* ks = static_cast<const R*>(e.ksum);
                const R* kc = static_cast<const R*>(e.kcomp);
#pragma unroll
                for (int i = 0; i < D; ++i) y[k][i] = state[i * Np + p[k]];
#pragma unroll
                for (int c = 0; c < OUT; ++c) acc[k].set(c, ks[c * Np + p[k]], kc[c * Np + p[k]]);
                q[k] = Prob::load(static_cast<const R*>(e.params), Np, p[k]);
            } else {
#pragma unroll
                for (int i = 0; i < D; ++i) y[k][i] = R(0);
#pragma unroll
                for (int c = 0; c < OUT; ++c) acc[k].set(c, R(0), R(0));
                q[k] = Prob::load(static_cast<const R*>(e.params), Np, td.first);  // any valid slot; results are discarded
            }
            Prob::trig(y[k], tr[k]);
            const R* slo = static_cast<const R*>(e.slo);
#pragma unroll
            for (int i = 0; i < D; ++i) lo[k][i] = (slo && active[k]) ? slo[i * Np + p[k]] : R(0);
        }
        NewtonCount nc{0u, 0u};
        // W < 2^31 (validated); the window position fits 32 bits.  Values used only
        // at a window end (once per W steps) are re-read there instead of being kept
        // live in registers across the step loop.
        unsigned int wpos = static_cast<unsigned int>(s0 % W);
        const unsigned int W32 = static_cast<unsigned int>(W);
        // injected increments stream from HBM: the warp's rows of the tile's first steps go
        // in flight now (the warp's 32 particles start at the tile's first + 32 warp)
        if constexpr (INJECT)
            dws.begin(static_cast<const R*>(e.dw), Np, td.first + (threadIdx.x & ~31u), e.dw_chunk ? 0ull : s0, nsteps);

        for (unsigned long long t0 = 0; t0 < nsteps; t0 += FT) {
            const int len = static_cast<int>(min(static_cast<unsigned long long>(FT), nsteps - t0));
            __syncwarp();
            for (int i = threadIdx.x & 31; i < 3 * len; i += 32) (&sB[0][0])[i] = ftab[3 * t0 + i];
            __syncwarp();
            // one step of every particle of the thread; winj: the injected increments
            auto one_step = [&](int i, const R (*winj)[Mn]) {
                const unsigned long long g = s0 + t0 + i;
                const R B[3] = {sB[i][0], sB[i][1], sB[i][2]};
#pragma unroll
                for (int k = 0; k < PPT; ++k) {
                    if (!active[k]) continue;
                    const unsigned long long pid = e.pid_offset + p[k];
                    R w[Mn];
                    if constexpr (INJECT) {
#pragma unroll
                        for (int j = 0; j < Mn; ++j) w[j] = winj[k][j];
                    } else {
                        philox_increments<R, Mn, Prob::kCalledMath>(seed, pid, g, sqdt, m2dt, w);
                    }
                    if constexpr (SOLVER == kHeunNotConsistent) {
                        R w2[Mn];
                        philox_normals<R, Mn>(seed, pid, g, w2, 2u);
#pragma unroll
                        for (int j = 0; j < Mn; ++j) w2[j] = w2[j] * sqdt;
                        St::step_heun_nc(q[k], rot, y[k], B, w, w2, dt, tr[k]);
                    } else if constexpr (uses_double_noise(SOLVER)) {
                        R An[Mn * (Mn - 1) / 2];
                        double_noise_antisym<R, Mn>(seed, pid, g, e.dna, static_cast<R>(e.rho), sqdt, w, An);
                        if constexpr (SOLVER == kWeakTest) St::step_weak(q[k], rot, y[k], B, w, An, dt, sqdt, tr[k]);
                        else St::step_es1(q[k], rot, y[k], B, w, An, dt, sqdt, tr[k]);
                    } else {
                        St::step(q[k], rot, y[k], B, w, dt, e.max_iter, e.tol, nc, tr[k],
                                 M<R>::kCompensatedState ? lo[k] : nullptr);
                    }
                    R o[OUT];
                    Prob::out_t(y[k], o, tr[k]);
                    acc[k].add(o);
                }
                if (++wpos == W32) {  // window end: uniform across the CTA
                    wpos = 0;
                    const unsigned long long kw = (g + 1) / W;
                    const int slot = static_cast<int>(kw - s0 / W - 1);
                    double* const traj = e.traj;
#pragma unroll
                    for (int k = 0; k < PPT; ++k) {
                        const double mom = active[k] ? e.moment[p[k]] : 0.0;
                        double* const partial = e.partial + ((p[k] >> 5) * e.slots + slot) * OUT;
                        // recorded particles: every traj_stride-th (the reference's Save_intervall)
                        const bool rec = traj && active[k] && (p[k] + 1) % e.traj_stride == 0;
                        const unsigned long long ti = rec ? (p[k] + 1) / e.traj_stride - 1 : 0;
                        // the butterfly leaves every lane with the same sums; lane c keeps
                        // component c, and the warp writes its OUT sums in one coalesced store
                        const int lane = threadIdx.x & 31;
                        double mine = 0.0;
#pragma unroll
                        for (int c = 0; c < OUT; ++c) {
                            const R v = active[k] ? acc[k].get_sum(c) / static_cast<R>(static_cast<double>(W)) : R(0);
                            acc[k].clear_sum(c);
                            const double vd = static_cast<double>(v);
                            if (rec) traj[(kw * OUT + c) * e.traj_n + ti] = vd;
                            const double ws = warp_sum(active[k] ? weight_of<PROB>(c, mom) * vd : 0.0);
                            if (lane == c) mine = ws;
                        }
                        if (lane < OUT) partial[lane] = mine;
                    }
                }
            };
            if constexpr (INJECT) {
                for (int i = 0; i < len; ++i) {
                    R cur[PPT][Mn];
                    if (!dws.next(cur[0])) break;  // a stage timed out (uniform across the warp)
                    one_step(i, cur);
                }
                if (!dws.ok) break;
            } else {
                for (int i = 0; i < len; ++i) one_step(i, nullptr);
            }
        }
        if constexpr (INJECT) {
            if (!dws.ok) {  // report, wait for the copies still in flight, leave the results unwritten
                if ((threadIdx.x & 31) == 0) atomicExch(&e.ctl->fault, 1ull);
                dws.drain();
                return;
            }
        }
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            if (active[k]) {
                R* state = static_cast<R*>(e.state);
                R* ks = static_cast<R*>(e.ksum);
                R* kc = static_cast<R*>(e.kcomp);
                bool finite = true;
#pragma unroll
                for (int i = 0; i < D; ++i) {
                    state[i * Np + p[k]] = y[k][i];
                    finite = finite && M<R>::finite(y[k][i]);
                }
                if (e.slo) {
                    R* slo = static_cast<R*>(e.slo);
#pragma unroll
                    for (int i = 0; i < D; ++i) slo[i * Np + p[k]] = lo[k][i];
                }
#pragma unroll
                for (int c = 0; c < OUT; ++c) { ks[c * Np + p[k]] = acc[k].get_sum(c); kc[c * Np + p[k]] = acc[k].get_comp(c); }
                if (!finite) e.status[p[k]] = 1;
            }
        }
        if constexpr (SOLVER == kImplicitMidpoint || SOLVER == kImplicitMidpointExact) {
            unsigned int it = nc.iterations, un = nc.unconverged;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) { it += __shfl_xor_sync(0xffffffffu, it, o); un += __shfl_xor_sync(0xffffffffu, un, o); }
            if ((threadIdx.x & 31) == 0) {
                atomicAdd(&e.ctl->newton_iterations, static_cast<unsigned long long>(it));
                atomicAdd(&e.ctl->newton_unconverged, static_cast<unsigned long long>(un));
            }
        }
    }
}

// ------------------------------------------------------------------ reductions
// grid (slots*OUT, n_ens); block kReduceThreads.  mode 0: windows completed in
// the current chunk -> msum[k]; mode 1 (after init): slot 0 -> msum[0], slot 1 -> wsum.
template <int OUT>
__global__ void __launch_bounds__(kReduceThreads) reduce_kernel(const EnsDev* __restrict__ ensembles, int mode) {
    const EnsDev& e = ensembles[blockIdx.y];
    const int slot = blockIdx.x / OUT, c = blockIdx.x % OUT;
    if (slot >= e.slots) return;
    double* dst;
    if (mode == 0) {
        const unsigned long long s0 = e.ctl->step_done, tgt = e.ctl->step_target;
        const unsigned long long nsteps = tgt > s0 ? min(e.chunk, tgt - s0) : 0ull;
        const unsigned long long nwin = (s0 + nsteps) / e.W - s0 / e.W;
        if (static_cast<unsigned long long>(slot) >= nwin) return;
        dst = e.msum + (s0 / e.W + 1 + slot) * OUT + c;
    } else {
        if (slot > 1) return;
        dst = (slot == 0) ? e.msum + c : e.wsum + c;
    }
    // warps holding at least one particle; the step kernel's tiles cover exactly these
    // (the 256-padding beyond them is never written after init)
    const unsigned long long nwarps = (e.n + 31) >> 5;
    double acc = 0.0;
    for (unsigned long long w = threadIdx.x; w < nwarps; w += blockDim.x) acc += e.partial[(w * e.slots + slot) * OUT + c];
    __shared__ double red[kReduceThreads];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kReduceThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *dst = red[0];
}

// B(t) for every step of the current chunk of each ensemble (grid.y = ensemble):
// t = (n+1) dt (SingleParticleSimulator.h:145), + dt/2 for ImplicitMidpoint
// (Implicit_Midpoint.inl:59); phase and sine in FP64, stored as Real.
template <class R>
__global__ void field_chunk_kernel(const EnsDev* __restrict__ ensembles, int midpoint) {
    const EnsDev& e = ensembles[blockIdx.y];
    const unsigned long long s0 = e.ctl->step_done, tgt = e.ctl->step_target;
    const unsigned long long nsteps = tgt > s0 ? min(e.chunk, tgt - s0) : 0ull;
    const unsigned long long i = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nsteps) return;
    const double t = e.dt * static_cast<double>(s0 + i + 1) + (midpoint ? 0.5 * e.dt : 0.0);
    double B[3];
    field_eval(e.field, t, B);
    R* f = static_cast<R*>(e.ftab) + 3 * i;
    f[0] = static_cast<R>(B[0]); f[1] = static_cast<R>(B[1]); f[2] = static_cast<R>(B[2]);
}

// Pregenerated noise: the Wiener increments of the current chunk of each ensemble
// (grid.y = ensemble), drawn exactly as the in-kernel path draws them (philox_increments:
// the same Philox counters and the same arithmetic), into dw [chunk][Mn][Np]; the
// injected step kernel then reads them instead of drawing them on its own step chain.
// One thread per (step, particle), particles fastest (coalesced stores).
template <int PROB, class R, int A>
__global__ void __launch_bounds__(256) noise_chunk_kernel(const EnsDev* __restrict__ ensembles) {
    using Prob = typename ProblemOf<PROB, R, A>::type;
    constexpr int Mn = Prob::Mn;
    const EnsDev& e = ensembles[blockIdx.y];
    const unsigned long long s0 = e.ctl->step_done, tgt = e.ctl->step_target;
    const unsigned long long nsteps = tgt > s0 ? min(e.chunk, tgt - s0) : 0ull;
    const unsigned long long n = e.n, Np = e.Np, total = nsteps * n;
    R* const dw = static_cast<R*>(e.dw);
    const R sqdt = static_cast<R>(e.sqrt_dt);
    const R m2dt = static_cast<R>(-2.0 * e.dt);
    for (unsigned long long i = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        const unsigned long long j = i / n, p = i - j * n;
        R w[Mn];
        philox_increments<R, Mn, Prob::kCalledMath>(e.seed, e.pid_offset + p, s0 + j, sqdt, m2dt, w);
#pragma unroll
        for (int m = 0; m < Mn; ++m) dw[(j * Mn + m) * Np + p] = w[m];
    }
}

template <class R, int Mn>
__global__ void debug_normals_kernel(unsigned long long seed, unsigned long long pid0, unsigned long long n,
                                     unsigned long long step0, unsigned long long nsteps, double* out) {
    const unsigned long long idx = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= n * nsteps) return;
    const unsigned long long s = idx / n, p = idx % n;
    R z[Mn];
    philox_normals<R, Mn>(seed, pid0 + p, step0 + s, z);
    for (int j = 0; j < Mn; ++j) out[(s * Mn + j) * n + p] = static_cast<double>(z[j]);
}

}  // namespace sp
