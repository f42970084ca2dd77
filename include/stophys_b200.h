/*
 * stophys_b200.h — C ABI of the B200 ensemble SDE engine.
 *
 * The engine replaces the reference's per-particle simulation loop for a whole
 * ensemble.  In the reference every particle gets its own
 * SingleParticleSimulator<Solver,Field>, created and run by
 * SimulationManager::singleSimulationTask
 *   (Particle_Simulation/Simulator/SimulationManager.h:126-160)
 * which calls doSimulation -> startSimulation
 *   (Particle_Simulation/Simulator/SingleParticleSimulator.h:109-159,221-227)
 * and folds each particle's window-mean trajectory into the moment-weighted
 * ensemble mean (Particle_Simulation/Results/MeanSimulationResult.h:87-119).
 * The reference's binary plug-in point is the per-ISA shared library exporting
 * SimulationManager<PREC,ISA> (Particle_Simulation/app/StoPhys_arch.cpp.in:4,
 * selected in Particle_Simulation/app/StoPhysApp_MultiArch.cpp:27-75); this ABI
 * is the B200 backend a maintainer registers beside AVX/AVX2/AVX512.
 *
 * Conventions
 *  - Every call returns sp_status; no C++ exception crosses the ABI.  The text
 *    of the last error on the calling thread is returned by sp_last_error().
 *  - All arrays passed in are HOST pointers owned by the caller.  The library
 *    copies what it needs to the device and owns all device memory.
 *  - Units and signs follow the reference's .ini contract: SI units, fields in
 *    tesla, gyromagnetic ratio positive for the electron, and the reference's
 *    anisotropy sign (uniaxial H = (-2K/Ms)(m.n)n, so K < 0 is an easy axis).
 */
#ifndef STOPHYS_B200_H
#define STOPHYS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SP_ABI_VERSION 9u

#if defined(_WIN32)
#define SP_API __declspec(dllexport)
#else
#define SP_API __attribute__((visibility("default")))
#endif

typedef enum sp_status {
    SP_OK = 0,
    SP_ERR_INVALID_ARG = 1,       /* malformed or out-of-range description */
    SP_ERR_UNSUPPORTED_COMBO = 2, /* e.g. ImplicitMidpoint on a problem without Jacobian */
    SP_ERR_OUT_OF_MEMORY = 3,
    SP_ERR_ADMISSION_REFUSED = 4, /* request larger than the server's memory budget */
    SP_ERR_DEVICE_TIMEOUT = 5,
    SP_ERR_NUMERIC_FAULT = 6,     /* non-finite state detected (see sp_stats) */
    SP_ERR_CUDA = 7,
    SP_ERR_NOT_READY = 8,
    SP_ERR_NOT_FOUND = 9,
    SP_ERR_CANCELLED = 10,
    SP_ERR_NO_DEVICE = 11
} sp_status;

/* Problems the reference registers (Particle_Simulation/Problems/Problems.h:6-9,
 * enum IProblem in Particle_Simulation/Settings/ProblemSettings.h). */
typedef enum sp_problem {
    SP_PROBLEM_NEEL = 0,                          /* NeelRelaxation: m in R^3         */
    SP_PROBLEM_NEEL_SPHERICAL = 1,                /* NeelRelaxationSpherical: (theta, phi) */
    SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL = 2,/* Euler ZXZ (phi,theta,psi) + Neel (theta,phi) */
    SP_PROBLEM_BROWN_AND_NEEL = 3                 /* BrownAndNeelRelaxation: (n, m) in R^6 */
} sp_problem;

/* Particle_Simulation/Problems/Anisotropy/AnisotropyList.h:45 */
typedef enum sp_anisotropy {
    SP_ANISOTROPY_UNIAXIAL = 0,
    SP_ANISOTROPY_CUBIC = 1,
    /* UniaxialCubicAnisotropy.hpp: a uniaxial part whose axis is the particle's z axis
     * rotated by uniaxial_rotation (Euler ZXZ), plus a cubic part on the particle axes;
     * anisotropy_constant = K_uniaxial, cubic_constant = K_cubic.  Not for the coupled
     * Cartesian problem, where the reference's cubic torque is evaluated with zero Euler
     * angles and divides by sin(0). */
    SP_ANISOTROPY_UNIAXIAL_CUBIC = 2
} sp_anisotropy;

/* Particle_Simulation/Fields/FieldList.h:48 */
typedef enum sp_field_type {
    SP_FIELD_ZERO = 0,
    SP_FIELD_CONSTANT = 1,
    SP_FIELD_SINUSOIDAL = 2,
    SP_FIELD_LISSAJOUS = 3,
    SP_FIELD_TRIANGULAR = 4,
    SP_FIELD_RECTANGULAR = 5,
    SP_FIELD_SINC = 6
} sp_field_type;

/* Particle_Simulation/Settings/SolverSettings.h:39 (ISolver) */
typedef enum sp_solver {
    SP_SOLVER_EULER_MARUYAMA = 0,
    SP_SOLVER_HEUN_STRONG = 1,
    SP_SOLVER_MILLSTEIN = 2,
    SP_SOLVER_IMPLICIT_MIDPOINT = 3,
    SP_SOLVER_EULER_MARUYAMA_NORMALIZED = 4, /* EulerMaruyama_Normalized.inl:40-56 */
    /* The next three exist in the reference but are switched off in its manager
     * (SimulationManager.h:325-328).  They take in-kernel (Philox) noise only.
     * Each evaluates its support points in the chart prepareCalculations chose for
     * y_n and finishes once, like HEUN_STRONG. */
    SP_SOLVER_HEUN_NOT_CONSISTENT = 5, /* Heun_NotConsistent.inl:35-47: two independent dW */
    SP_SOLVER_WEAK_TEST = 6,           /* WeakTest.inl:18-63 + double noise matrix        */
    SP_SOLVER_EXPLICIT_STRONG_1 = 7    /* Explicit_Strong_1.inl:20-78 + double noise matrix */
} sp_solver;

typedef enum sp_precision {
    SP_PRECISION_FP64 = 0, /* plain drop-in: FP64 throughout                         */
    SP_PRECISION_FP32 = 1  /* FP32 stepping; FP64 time, field phase, ensemble sums,
                              Newton acceptance test                                 */
} sp_precision;

/* Newton matrix of ImplicitMidpoint, S = -I + dt/2 J_a + 1/2 J_b at the midpoint
 * (Implicit_Midpoint.inl:83-98).  REFERENCE uses the problems' own Jacobians as
 * the reference defines them (NeelRelaxation.h:134-190 with its -2 alpha/dt [m]x
 * term and the b Jacobian's cross-product part only; CubicAnisotropy.h:228-236
 * J_H = I; BrownAndNeelRelaxation.h:178-187 J = 0), so the iteration matches the
 * reference step for step.  EXACT uses the analytic Jacobians of a(y) and
 * b(y)·dW (Neel Cartesian, uniaxial and cubic): the same fixed point, reached in
 * fewer iterations (quadratic convergence); other problems refuse it. */
typedef enum sp_jacobian {
    SP_JACOBIAN_REFERENCE = 0,
    SP_JACOBIAN_EXACT = 1
} sp_jacobian;

typedef enum sp_noise {
    SP_NOISE_PHILOX = 0,   /* counter-based Philox4x32-10 + Box-Muller, in-kernel    */
    SP_NOISE_INJECTED = 1  /* Wiener increments supplied by the caller (parity mode) */
} sp_noise;

/* Per-particle physical properties, host structure-of-arrays of length
 * n_particles each.  Keys mirror Magnetic_Properties / Hydrodynamic_Properties
 * (Particle_Simulation/Properties/MagneticProperties.h:207-216,
 *  Particle_Simulation/Properties/HydrodynamicProperties.h:52-56) and the
 * initialisation settings (Particle_Simulation/Settings/ParticleSimulationInitSettings.h:30-38)
 * with Use_random_initial_* = false: orientation and magnetisation are given. */
typedef struct sp_particles {
    const double* magnetic_radius;          /* m                                  */
    const double* saturation_magnetisation; /* A/m                                */
    const double* damping_constant;         /* alpha                              */
    const double* gyromagnetic_ratio;       /* rad/(s T)                          */
    const double* anisotropy_constant;      /* K_uniaxial or K1_cubic, J/m^3      */
    const double* hydrodynamic_radius;      /* m; Brown problems only (else NULL) */
    const double* viscosity;                /* Pa s; Brown problems only          */
    const double* orientation;              /* [n][3] Euler angles phi,theta,psi (ZXZ) */
    const double* magnetisation;            /* [n][3] initial magnetisation direction  */
    const double* cubic_constant;           /* UNIAXIAL_CUBIC only: K_cubic, J/m^3 (else NULL) */
    const double* uniaxial_rotation;        /* UNIAXIAL_CUBIC only: [n][3] Euler angles of the
                                               uniaxial axis (Uniaxial_Rotation; else NULL)  */
} sp_particles;

/* External field B(t) in tesla.
 *   ZERO:        B = 0
 *   CONSTANT:    B = offset                                  (ConstantField.h:43)
 *   SINUSOIDAL:  B = amplitude*sin(2 pi frequency[0] t + phase[0]) + offset
 *                                                            (SinusoidalField.h:47-51)
 *   LISSAJOUS:   B_i = offset_i + amplitude_i*sin(2 pi frequency_i t + phase_i)
 *                                                            (LissajousField.h:98-101)
 *   TRIANGULAR:  piecewise linear in the position p = (t + time_offset) mod periode
 *                (TriangularField.h:52-70)
 *   RECTANGULAR: exponential rise / decay with time constant tau in each half
 *                period, optionally alternating (RectangularField.h:30-63)
 *   SINC:        B = amplitude*sinc^2(pi a p) + offset, a = 22/periode,
 *                p = (t mod periode) - periode/2                (SincField.h:38-48) */
typedef struct sp_field_desc {
    int32_t type;        /* sp_field_type                         */
    int32_t alternating; /* RECTANGULAR: Alternating              */
    double offset[3];
    double amplitude[3];
    double frequency[3];
    double phase[3];
    double periode;      /* TRIANGULAR / RECTANGULAR / SINC: Periode (s) */
    double time_offset;  /* TRIANGULAR / RECTANGULAR: TimeOffset (s)     */
    double tau;          /* RECTANGULAR: Tau (s)                          */
} sp_field_desc;

/* Problem_Settings (Particle_Simulation/Settings/ProblemSettings.h:119-206). */
typedef struct sp_problem_settings {
    int32_t use_coordinate_transformation;            /* NeelSpherical             */
    int32_t use_euler_coordinate_transformation;      /* BrownAndNeelEulerSpherical */
    int32_t use_spherical_coordinate_transformation;  /* BrownAndNeelEulerSpherical */
    int32_t use_simple_model;                         /* BrownAndNeel (Cartesian)   */
    double min_angle_before_transformation;           /* rad                        */
    double brown_min_angle_before_transformation;     /* rad                        */
    double neel_min_angle_before_transformation;      /* rad                        */
} sp_problem_settings;

/* ---- device-side particle provider -------------------------------------
 * Particle properties and initial states drawn on the device instead of being
 * passed in: the reference's provider (Provider/ParticleProvider.h:194-217) selects a
 * particle template per particle, its ParticleSimulationSettings
 * (Settings/ParticleSimulationSettings.h:51-152, Properties/Anisotropy/Uniaxial.hpp:41-85)
 * apply the size and anisotropy distributions, and the problem's initialiser draws
 * random orientations and magnetisations (NeelRelaxation.h:226-283,
 * BrownAndNeelRelaxation.inl:288-315, ParticleStateInitializer.h:50-123).  Draws come
 * from Philox4x32-10 keyed by the provider's seed, so a provided ensemble is
 * reproducible; the reference's generators are seeded from std::random_device. */
typedef enum sp_distribution {
    SP_DIST_DELTA = 0,
    SP_DIST_NORMAL = 1,    /* N(mean, sigma)                                  */
    SP_DIST_LOGNORMAL = 2  /* lognormal with the given mean and sigma          */
} sp_distribution;

typedef struct sp_dist {
    int32_t type;     /* sp_distribution                                                    */
    int32_t relative; /* 1: value * X, X from (1, width); 0: drawn around the value itself  */
    double width;     /* relative sigma, or for radius/shell sigma/mean, for K the sigma    */
} sp_dist;

typedef struct sp_particle_template {
    double weight;  /* Particle_Numbers entry: selection weight, or count when sequential */
    double magnetic_radius, saturation_magnetisation, damping_constant, gyromagnetic_ratio;
    double anisotropy_constant, hydrodynamic_radius, viscosity;
    double cubic_constant;          /* uniaxial+cubic only                              */
    double orientation[3];          /* Initial_particle_orientation (Euler ZXZ)         */
    double magnetisation[3];        /* Initial_magnetisation_direction                  */
    double uniaxial_rotation[3];    /* uniaxial+cubic only                              */
    int32_t random_orientation;     /* Use_random_initial_particle_orientation          */
    int32_t random_magnetisation;   /* Use_random_initial_particle_magnetisation        */
    int32_t random_uniaxial_rotation; /* UseRandomCubicOrientation (uniaxial+cubic)     */
    int32_t reserved;
    sp_dist magnetic_radius_dist, hydrodynamic_shell_dist, anisotropy_dist, cubic_dist;
} sp_particle_template;

typedef struct sp_provider_desc {
    uint64_t seed;        /* key of the provider's draws                                  */
    int32_t n_templates;  /* 1..64                                                        */
    int32_t sequential;   /* 1: fill each template's count in order, then template 0
                             (Use_discrete_distribution_to_select_particle = false); 0: draw
                             each particle's template with probability weight / sum      */
    const sp_particle_template* templates;
} sp_provider_desc;

typedef struct sp_ensemble_desc {
    uint32_t abi_version; /* SP_ABI_VERSION */
    int32_t problem;      /* sp_problem     */
    int32_t anisotropy;   /* sp_anisotropy  */
    int32_t solver;       /* sp_solver      */
    int32_t precision;    /* sp_precision   */
    int32_t noise;        /* sp_noise       */
    sp_problem_settings problem_settings;
    int32_t max_iteration;       /* Solver_Settings Max_Iterations (ImplicitMidpoint) */
    int32_t record_trajectories; /* 0: none; s >= 1: keep the window means of every s-th
                                    particle (ensemble indices s-1, 2s-1, ...: the reference's
                                    Save_intervall rule, SimulationResultManager.h:117-118), 1 =
                                    every particle (parity runs); read as sp_result.trajectories */
    int32_t jacobian;            /* sp_jacobian (ImplicitMidpoint only)               */
    int32_t double_noise_approx; /* Solver_Settings Approximation_of_double_noise_integral
                                    (WeakTest, ExplicitStrong_1.0): order p of the double
                                    Stratonovich integral approximation, -1..10
                                    (SimulationManager.h:503-525, DoubleNoiseMatrix.h) */
    double accuracy_goal;        /* Solver_Settings Accuracy_Goal (ImplicitMidpoint)  */
    uint64_t number_of_steps;    /* Simulation_Settings Number_of_steps               */
    uint64_t oversampling;       /* Simulation_Settings OverSampling (window W)       */
    double timestep;             /* Simulation_Settings Timestep (s)                  */
    double temperature;          /* K                                                 */
    sp_field_desc field;
    uint64_t n_particles;
    sp_particles particles;
    uint64_t seed;               /* Philox key                                        */
    uint64_t particle_id_offset; /* global id of particle 0 (shards keep one stream)  */
    /* SP_NOISE_INJECTED only: Wiener increments dW (already scaled by sqrt(dt)),
     * layout [integrated_steps][noise_dim][n_particles] with
     * integrated_steps = (number_of_steps/oversampling - 1) * oversampling. */
    const double* injected_dw;
    /* Optional: when set, `particles` is ignored and every particle is drawn on the
     * device by this provider (particle i of the provider is particle_id_offset + i). */
    const sp_provider_desc* provider;
} sp_ensemble_desc;

/* Outputs.  n_samples = number_of_steps / oversampling (SingleParticleSimulator.h:125);
 * sample 0 is the initial state, sample k>=1 the Kahan mean over window k.
 * Any pointer may be NULL to skip that output. */
typedef struct sp_result {
    double* mean;         /* [n_samples][out_dim] moment-weighted ensemble mean           */
    double* weight;       /* [out_dim] summed weights (Ms*V per component)                */
    double* time;         /* [n_samples] window-centre times (SingleParticleSimulator.h:236-273) */
    double* field;        /* [n_samples][3] window-mean field                             */
    double* trajectories; /* [n_particles / s][n_samples][out_dim] window means of the
                             particles record_trajectories = s selects (all when s = 1)  */
    double* final_state;  /* [n_particles][state_dim] state after the last step           */
    double* weighted_sum; /* [n_samples][out_dim] the un-normalised sums sum_p w_p r_p[k] that
                             MeanSimulationResult accumulates before normalize divides them by
                             the weight (Results/MeanSimulationResult.h:87-119); what shards of
                             one ensemble exchange to be merged (sp_merge_shards)              */
} sp_result;

typedef struct sp_stats {
    uint64_t particle_steps;      /* integrated particle-steps                       */
    uint64_t nonfinite_particles; /* particles whose state became NaN/Inf            */
    uint64_t newton_iterations;   /* ImplicitMidpoint: total Newton iterations       */
    uint64_t newton_unconverged;  /* ImplicitMidpoint: steps that hit Max_Iterations */
    uint64_t kernel_launches;     /* device kernels launched for this ensemble       */
    double device_ms;             /* device time of the stepping kernels             */
    /* host-clock phases of the call or request, ms: waiting for admission (server only),
       set-up (device buffers, particle upload, initial state), integration (first launch
       to the last chunk complete) and read-back of the results */
    double queue_ms, setup_ms, run_ms, readback_ms;
} sp_stats;

typedef struct sp_context sp_context;
typedef struct sp_ensemble sp_ensemble;
typedef struct sp_server sp_server;

/* ---- metadata --------------------------------------------------------- */
SP_API const char* sp_last_error(void);
SP_API uint32_t sp_abi_version(void);
/* State / noise / output dimensions of a problem (GeneralSDEDimension of each
 * problem: NeelRelaxation.h:24-25, NeelRelaxationSpherical.h:29-30,
 * BrownAndNeelRelaxationEulerSpherical.h:36-37, BrownAndNeelRelaxation.h:68-69). */
SP_API sp_status sp_query_dims(int32_t problem, int32_t* state_dim, int32_t* noise_dim, int32_t* out_dim);
/* Validates a description without touching the device. */
SP_API sp_status sp_validate(const sp_ensemble_desc* desc);
/* Total kernels this process launched through the library. */
SP_API uint64_t sp_kernel_launch_count(void);

/* ---- shards -------------------------------------------------------------
 * Merges the results of shards of one ensemble (the same description split by
 * particle_id_offset, e.g. one shard per GPU) into the result of the whole: the
 * reference folds every particle into MeanSimulationResult::operator+= (weighted
 * result and weight added, Results/MeanSimulationResult.h:87-119) and normalize()
 * divides by the summed weight unless it is all zero (:63-75).  Inputs are each
 * shard's weighted_sum [n_samples][out_dim] and weight [out_dim] (sp_result);
 * they are added in FP64 in shard order.  Outputs (any may be NULL): mean_out
 * [n_samples][out_dim], weighted_sum_out [n_samples][out_dim], weight_out
 * [out_dim].  Host memory only; needs no device. */
SP_API sp_status sp_merge_shards(int32_t n_shards, uint64_t n_samples, int32_t out_dim,
                                 const double* const* weighted_sums, const double* const* weights,
                                 double* mean_out, double* weighted_sum_out, double* weight_out);

/* ---- context ----------------------------------------------------------- */
SP_API sp_status sp_create(sp_context** ctx, int32_t device);
SP_API sp_status sp_destroy(sp_context* ctx);

/* ---- synchronous drop-in ----------------------------------------------
 * Runs the whole ensemble: replaces SimulationManager::StartSimulationManager's
 * fan-out of singleSimulationTask over all particles
 * (Particle_Simulation/Simulator/SimulationManager.h:549-574) and the
 * MeanSimulationResult accumulation.  Host in, host out. */
SP_API sp_status sp_simulate(sp_context* ctx, const sp_ensemble_desc* desc, sp_result* out, sp_stats* stats);

/* ---- device-resident ensembles ----------------------------------------
 * sp_ensemble_create copies inputs to the device and builds the initial
 * state; sp_ensemble_advance integrates further steps (in chunks, on the
 * given CUDA stream, NULL = the context's stream); sp_ensemble_read waits and
 * copies results out.  State stays on the device between calls. */
SP_API sp_status sp_ensemble_create(sp_context* ctx, const sp_ensemble_desc* desc, sp_ensemble** ens);
SP_API sp_status sp_ensemble_advance(sp_ensemble* ens, uint64_t n_steps, void* cuda_stream);
SP_API sp_status sp_ensemble_steps_done(const sp_ensemble* ens, uint64_t* steps_done, uint64_t* steps_total);
SP_API sp_status sp_ensemble_read(sp_ensemble* ens, sp_result* out, sp_stats* stats);
SP_API sp_status sp_ensemble_destroy(sp_ensemble* ens);
/* Bytes of device memory an ensemble of this description holds. */
SP_API sp_status sp_ensemble_footprint(const sp_ensemble_desc* desc, uint64_t* bytes);

/* ---- continuous-batching server ----------------------------------------- */
typedef struct sp_server_config {
    uint64_t memory_budget_bytes; /* admission limit on device bytes of admitted requests */
    uint64_t chunk_steps;         /* steps per scheduling round; 0 = the tuned chunk
                                     capped at 4000 steps (whole windows).  Admitted
                                     requests are grouped by kernel; each group runs its
                                     rounds on its own stream at its own pace;
                                     requests join and leave a group only between its
                                     rounds (a request whose kind's group is mid-round
                                     starts a second group of its kind), so the round
                                     bounds how long a request that finishes mid-round
                                     waits to be read back.  A round runs as chunk
                                     launches of at most 1000 steps (whole windows where
                                     a window fits)                                      */
    int32_t max_active;           /* cap on concurrently admitted requests (0 = none)     */
    int32_t groups_per_kind;      /* (ABI 9) groups of one kernel kind that may run at
                                     once (0 = 2): a request whose kind has that many
                                     groups mid-round joins the least full at its next
                                     round; below the cap it starts a group at once     */
} sp_server_config;

typedef enum sp_request_state {
    SP_REQUEST_QUEUED = 0,
    SP_REQUEST_RUNNING = 1,
    SP_REQUEST_DONE = 2,
    SP_REQUEST_FAILED = 3,
    SP_REQUEST_CANCELLED = 4
} sp_request_state;

SP_API sp_status sp_server_create(sp_context* ctx, const sp_server_config* cfg, sp_server** srv);
/* The description (and every array it points to) is copied at submit. */
SP_API sp_status sp_server_submit(sp_server* srv, const sp_ensemble_desc* desc, uint64_t* request_id);
/* Submits descs[0..n) at once: each is checked and copied as by sp_server_submit, then all
 * are queued under one lock, so an idle server admits them together and their first
 * rounds overlap (submitted one by one, the first can start alone before the next is
 * queued).  All or nothing: if any is refused, none is queued and the error text names
 * its index.  request_ids[i] receives the id of descs[i]. */
SP_API sp_status sp_server_submit_many(sp_server* srv, const sp_ensemble_desc* descs, int32_t n, uint64_t* request_ids);
SP_API sp_status sp_server_poll(sp_server* srv, uint64_t request_id, int32_t* state);
/* Blocks up to timeout_ms (<0: forever) and copies results of a finished request.
 * A finished, failed or cancelled request is reported once: afterwards its id is
 * unknown (SP_ERR_NOT_FOUND).  SP_ERR_NOT_READY leaves it pending. */
SP_API sp_status sp_server_wait(sp_server* srv, uint64_t request_id, double timeout_ms, sp_result* out,
                         sp_stats* stats, double* latency_ms);
SP_API sp_status sp_server_cancel(sp_server* srv, uint64_t request_id);
SP_API sp_status sp_server_destroy(sp_server* srv);

/* ---- test hooks ------------------------------------------------------------
 * Writes the unit normals the kernels draw for particles
 * [particle_id, particle_id+n) and steps [step0, step0+n_steps) into
 * out[n_steps][noise_dim][n] (FP64 values; FP32 draws are widened). */
SP_API sp_status sp_debug_philox_normals(sp_context* ctx, uint64_t seed, uint64_t particle_id, uint64_t n,
                                  uint64_t step0, uint64_t n_steps, int32_t noise_dim,
                                  int32_t precision, double* out);

/* Measured dense FMA throughput of this device (TFLOP/s, 2 flops per FMA) for
 * precision SP_PRECISION_FP64 or SP_PRECISION_FP32: the denominator of the
 * issue roofline the engine's kernels are reported against. */
SP_API sp_status sp_measure_fma_peak(sp_context* ctx, int32_t precision, double* tflops);

/* ---- autotuner ----------------------------------------------------------
 * No counterpart in the reference (its thread pool has no launch shape).
 * Launch shape of one kernel key (problem, anisotropy, solver, precision,
 * noise): particles per CTA tile, particles per thread (1, or 2 for the FP32
 * kernels: the CTA then has block / 2 threads, each integrating two particles
 * whose step chains interleave), persistent grid (CTAs = resident CTAs x SMs
 * striding over the tiles) or one CTA per tile, and SDE steps per captured chunk. */
typedef struct sp_launch_config {
    int32_t block;
    int32_t persistent;
    uint64_t chunk_steps;
    double particle_steps_per_s; /* measured rate of this shape on the probe */
    int32_t particles_per_thread;
    int32_t reserved0;
} sp_launch_config;
/* Times every candidate shape on a probe of desc (its first
 * min(n_particles, probe_particles) particles; 0 = 65536) with CUDA events and
 * caches the fastest for desc's kernel key in this process; every later
 * ensemble, sp_simulate and server group of that key uses it.  best and
 * candidates[max_candidates] (optional) receive the winner and the timings;
 * *n_candidates the number timed.  SP_NOISE_INJECTED descriptions are refused. */
SP_API sp_status sp_autotune(sp_context* ctx, const sp_ensemble_desc* desc, uint64_t probe_particles,
                             sp_launch_config* best, sp_launch_config* candidates, int32_t max_candidates,
                             int32_t* n_candidates);
/* Launch shape the library uses for desc now (tuned or default). */
SP_API sp_status sp_launch_config_for(sp_context* ctx, const sp_ensemble_desc* desc, sp_launch_config* out);
/* sp_ensemble_create with the caller's launch shape (shape NULL = the tuned or default
 * one): block 32, 64, 128 or 256; persistent 0 or 1; chunk_steps >= 1, rounded down to
 * whole windows (at least one); particles_per_thread 1 or 2 (2 falls back to 1 where the
 * kernel key has no two-particle form or the block is under 64); particle_steps_per_s
 * and reserved0 are ignored.  Results do not depend on the shape.  Ensembles advanced
 * side by side on separate streams run faster with short chunks (about 1000 steps): a
 * chunk launch ends with its CTAs draining, and the SMs they free go to the other
 * ensembles' CTAs only when those have launches in flight, where a lone ensemble is
 * fastest with the longer chunk the autotuner picks.
 * Small FP64 ensembles with SP_NOISE_PHILOX (at most 8 x 32 particles per SM) draw each
 * chunk's increments in a separate parallel kernel before the step kernel (the same
 * Philox stream, bit-identical results, about half the per-step latency); their chunk
 * is shortened where needed so that this buffer stays within 256 MB.  sp_simulate and
 * sp_ensemble_* do this; server groups always draw in the step kernel. */
SP_API sp_status sp_ensemble_create_shaped(sp_context* ctx, const sp_ensemble_desc* desc, const sp_launch_config* shape,
                                           sp_ensemble** ens);
/* Write / read (merge) the tuned shapes of this process as text, one key per
 * line; reset forgets them all (defaults apply again). */
SP_API sp_status sp_tuning_save(const char* path);
SP_API sp_status sp_tuning_load(const char* path);
SP_API sp_status sp_tuning_reset(void);

/* ---- provider ------------------------------------------------------------
 * The particles `desc->provider` draws for this description, copied to the host:
 * out[n_particles][20] with columns magnetic_radius, saturation_magnetisation,
 * damping_constant, gyromagnetic_ratio, anisotropy_constant, hydrodynamic_radius,
 * viscosity, orientation[3], magnetisation[3] (unit), cubic_constant,
 * uniaxial_rotation[3], template index, reserved. */
SP_API sp_status sp_provide_particles(sp_context* ctx, const sp_ensemble_desc* desc, double* out);

/* ---- allocation-free run ----------------------------------------------------
 * No counterpart in the reference: an addition for hosts whose plug-ins may not
 * allocate device memory while they run (real-time or embedded control loops,
 * hosts that pre-reserve and account all GPU memory, sandboxes that forbid
 * cudaMalloc after start-up).  Runs the whole ensemble like sp_simulate, on
 * cuda_stream (NULL = the legacy default stream), asynchronously, and allocates
 * nothing: the caller passes the per-particle inputs as DEVICE pointers
 * (device_particles, same layout as sp_particles; desc->particles is ignored)
 * and receives mean [n_samples][out_dim] and weight [out_dim] in DEVICE memory,
 * valid once the stream has completed.  Every internal buffer lives in one
 * static device array of 32 MiB that each GPU loading the library holds until
 * exit; ensembles needing more are refused with SP_ERR_INVALID_ARG.  Philox noise
 * only, no trajectories.  The first call on a device resolves the array's
 * address (make it before any stream capture) and keeps it for the life of the
 * device's context: after cudaDeviceReset the library must be reloaded before
 * this entry point is used again.  Calls overlapping on the GPU share the array
 * and race. */
SP_API sp_status sp_simulate_noalloc(const sp_ensemble_desc* desc, const sp_particles* device_particles,
                                     double* device_mean, double* device_weight, void* cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* STOPHYS_B200_H */
