// sp_types.h — data shared by the host runtime and the sm_100a kernels.
//
// Device memory of one ensemble (structure of arrays, particle index fastest,
// Np = n rounded up to a multiple of kPad so every tile is full in memory):
//   state   [D][Np]      Real   SDE state y (D = 3, 2, 5, 6)
//   ksum    [OUT][Np]    Real   Kahan running window sum of the outputs
//   kcomp   [OUT][Np]    Real   Kahan compensation (persists across windows)
//   slo     [D][Np]      float  FP32 form only: rounding errors the state update carries
//   params  [P][Np]      Real   derived per-particle prefactors (see kParams*)
//   moment  [Np]         double Ms*V, the reference's getWeighting
//   partial [warps][slots][OUT] double  per-warp weighted window means of one chunk
//   msum    [K][OUT]     double weighted ensemble sums of every sample
//   traj    [K][OUT][Nt] double optional window means of every s-th particle (Nt = n / s)
//   dw      [S][M][Np]   Real   optional injected Wiener increments
//   ftab    [chunk][3]   Real   B(t) of each step of the current chunk (FP64 phase, once per ensemble)
#pragma once

#include <stdint.h>

namespace sp {

constexpr int kPad = 256;           // particle padding = largest block size
constexpr int kMaxBlock = 256;
constexpr int kFieldTile = 128;     // steps of B(t) each warp stages in shared memory at a time
constexpr int kReduceThreads = 256; // threads per (sample, component) in the window reduction

enum ProblemId : int { kNeel = 0, kNeelSpherical = 1, kBrownNeelEuler = 2, kBrownNeel = 3 };
enum AnisoId : int { kUniaxial = 0, kCubic = 1, kUniaxialCubic = 2 };
enum SolverId : int { kEulerMaruyama = 0, kHeun = 1, kMillstein = 2, kImplicitMidpoint = 3, kEulerMaruyamaNormalized = 4 };
// kernel-table slot of ImplicitMidpoint with the analytic Newton matrix (SP_JACOBIAN_EXACT)
constexpr int kImplicitMidpointExact = 5;
// kernel-table slots of SP_SOLVER_HEUN_NOT_CONSISTENT, _WEAK_TEST, _EXPLICIT_STRONG_1 (5, 6, 7)
constexpr int kHeunNotConsistent = 6;
constexpr int kWeakTest = 7;
constexpr int kExplicitStrong1 = 8;
constexpr bool uses_double_noise(int slot) { return slot == kWeakTest || slot == kExplicitStrong1; }

// number of derived parameters per problem
constexpr int kParamsNeel = 16;
constexpr int kParamsNeelSph = 15;
constexpr int kParamsBrownNeelEuler = 13;
constexpr int kParamsBrownNeel = 14;
// extra parameters of the uniaxial+cubic anisotropy: Neel problems keep the cubic
// field prefactor and the rotated uniaxial axis; the Euler problem adds the cubic
// torque prefactor and the 3x3 rotation (its body axes move)
constexpr int kParamsUniaxialCubicNeel = 4;
constexpr int kParamsUniaxialCubicEuler = 11;
__host__ __device__ constexpr int param_count_of(int problem, int aniso) {
    return problem == kNeel            ? kParamsNeel + (aniso == kUniaxialCubic ? kParamsUniaxialCubicNeel : 0)
           : problem == kNeelSpherical ? kParamsNeelSph + (aniso == kUniaxialCubic ? kParamsUniaxialCubicNeel : 0)
           : problem == kBrownNeelEuler ? kParamsBrownNeelEuler + (aniso == kUniaxialCubic ? kParamsUniaxialCubicEuler : 0)
                                        : kParamsBrownNeel;
}

struct FieldParams {
    int type;  // sp_field_type
    int pad;
    double offset[3];     // RECTANGULAR: the shifted offset of the alternating form
    double amplitude[3];  // RECTANGULAR: doubled when alternating
    double omega[3];      // 2*pi*frequency
    double phase[3];
    double periode, half_periode;
    double time_offset;   // RECTANGULAR: the shifted time offset of the alternating form
    double inv_tau;       // RECTANGULAR: 1/Tau (max double for Tau ~ 0)
    double max_field[3];  // RECTANGULAR: amplitude * (1 - exp(-periode/(2 tau)))
    double sinc_a;        // SINC: 11 / (periode / 2)
};

// Control block of one ensemble, advanced by the commit kernel so that a
// captured chunk graph can be replayed without changing kernel arguments.
struct EnsCtl {
    unsigned long long step_done;    // integrated steps completed
    unsigned long long step_target;  // integrate up to this step
    unsigned long long newton_iterations;
    unsigned long long newton_unconverged;
    unsigned long long fault;  // non-zero: a staged copy of injected increments did not arrive in time
};

struct EnsDev {
    // geometry
    unsigned long long n, Np, K, W, S;  // particles, padded, samples, window, integrated steps
    unsigned long long chunk;           // steps per chunk
    unsigned long long seed, pid_offset;
    double dt, sqrt_dt;
    FieldParams field;
    // solver / problem settings
    int max_iter;
    int dna;        // WeakTest / ExplicitStrong_1: order p of the double-integral approximation
    double rho;     // sqrt(1/12 - sum_{r<=p} 1/(2 pi^2 r^2)) (DoubleNoiseMatrix.h sqrtpp)
    int rot_brown;  // NeelSpherical: rotation enabled; BrownNeelEuler: Brown rotation enabled
    int rot_neel;   // BrownNeelEuler: Neel rotation enabled
    int slots;      // partial slots per chunk (max windows completing in a chunk)
    double tol;
    double min1, max1, min2, max2;  // rotation thresholds
    // buffers
    void* state;
    void* ksum;
    void* kcomp;
    void* slo;      // FP32 form: [D][Np] carried rounding errors of the state (nullptr in FP64)
    const void* params;
    const double* moment;
    void* dw;       // Wiener increments [rows][Mn][Np]: injected (every step) or pregenerated
    int dw_chunk;   // 1: dw holds only the current chunk's increments (row 0 = its first step)
    double* partial;
    double* msum;   // [K][OUT] weighted ensemble sums
    double* wsum;   // [OUT] summed weights
    double* traj;   // [K][OUT][traj_n] window means of particles traj_stride-1, 2 traj_stride-1, ...
    unsigned long long traj_stride, traj_n;
    void* ftab;     // [chunk][3] Real: B(t) of every step of the current chunk
    unsigned char* status;
    EnsCtl* ctl;
};

// One CTA's worth of particles of one ensemble.
struct TileDesc {
    unsigned int ens;    // index into the EnsDev array
    unsigned int first;  // first particle of the tile
};

// raw per-particle properties as uploaded (FP64, [n] or [n][3])
struct RawParticles {
    const double* radius;
    const double* Ms;
    const double* alpha;
    const double* gamma;
    const double* K;
    const double* rh;
    const double* viscosity;
    const double* euler;  // [n][3]
    const double* mag;    // [n][3]
    const double* K2;     // uniaxial+cubic: K_cubic
    const double* urot;   // uniaxial+cubic: [n][3] Euler angles of the uniaxial axis
    double temperature;
    int simple_model;
};

}  // namespace sp
