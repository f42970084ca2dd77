"""GPU parity: the sm_100a kernels, called through the C ABI, against the CPU oracle.

Bars (stated per test):
  injection mode (same Wiener increments on both sides), FP64:
      per-trajectory window means within 1e-9 relative (floor 1e-3 absolute scale),
      ensemble mean within 1e-10 absolute (the mean magnetisation is O(1)).
      Strict: every (problem, solver, anisotropy) over 1000 integrated steps on the
      particles whose oracle agrees with its own long-double run to 1e-11.
      Whole ensembles: where the dynamics amplify round-off (particles crossing saddles,
      e.g. cubic anisotropy at ~1 kT barriers) the FP64 oracle itself drifts from its
      long-double run; there the bar is 20x that spread, over the longest horizon on
      which it stays at or below 1e-7 (asserted; the bar and horizon are printed).
  in-kernel Philox, FP64: the same 32-bit Philox words as the oracle; normals
      within 1e-14 relative, trajectories within 1e-9
  FP32 form: ensemble mean within 1e-3 of the FP64 kernel on the same noise, with a
      standard error of at most 3e-4 and no bias beyond 4 standard errors
"""
import dataclasses
import math

import numpy as np
import pytest

import oracle
import stochasticphysics_b200 as sp
from stochasticphysics_b200 import provider
from stochasticphysics_b200._abi import Anisotropy, FieldSpec, Jacobian, Noise, Precision, Problem, Solver

pytestmark = pytest.mark.gpu

REL_TRAJ = 1e-9
ABS_MEAN = 1e-10


@pytest.fixture(scope="module")
def ctx():
    c = sp.Context(0)
    yield c
    c.close()


def small_spec(problem, solver, aniso=Anisotropy.Uniaxial, n=67, steps=1000, W=50, seed=11, **kw):
    """Small ensemble of the given kind with config-like parameters."""
    if problem == Problem.BrownAndNeelEulerSpherical:
        base = provider.brown_neel_relaxation(n=n, steps=steps, oversampling=W, seed=seed)
    elif problem == Problem.BrownAndNeel:
        base = provider.brown_neel_relaxation(n=n, steps=steps, oversampling=W, seed=seed)
        base = dataclasses.replace(base, problem=Problem.BrownAndNeel,
                                   magnetisation=provider.along_axis_random_sign(
                                       np.random.default_rng(seed), provider.easy_axis(Problem.BrownAndNeel, base.orientation)))
    elif problem == Problem.NeelSpherical:
        base = provider.neel_relaxation(n=n, steps=steps, oversampling=W, seed=seed)
        base = dataclasses.replace(base, problem=Problem.NeelSpherical, use_coordinate_transformation=True,
                                   min_angle_before_transformation=math.pi / 36)
    else:
        base = provider.neel_relaxation(n=n, steps=steps, oversampling=W, seed=seed)
    if aniso == Anisotropy.Cubic:
        # start on a <111> easy direction: a <100> start is an unstable equilibrium for K1 < 0,
        # where round-off differences grow exponentially
        m0 = base.magnetisation
        if problem != Problem.BrownAndNeel:
            m0 = provider.along_axis_random_sign(np.random.default_rng(seed + 1),
                                                 provider.cubic_easy_direction(problem, base.orientation))
        base = dataclasses.replace(base, anisotropy=Anisotropy.Cubic, anisotropy_constant=np.full(n, -1.1e4),
                                   magnetisation=m0)
    return dataclasses.replace(base, solver=solver, **kw)


def compare(gpu, ref, rel=REL_TRAJ, mean_abs=ABS_MEAN):
    # particles that run away to NaN/Inf must do so identically on both sides
    bad_g = ~np.isfinite(gpu.trajectories).all(axis=(1, 2))
    bad_r = ~np.isfinite(ref["trajectories"]).all(axis=(1, 2))
    np.testing.assert_array_equal(bad_g, bad_r)
    ok = ~bad_r
    t_err = np.max(np.abs(gpu.trajectories[ok] - ref["trajectories"][ok]) /
                   np.maximum(np.abs(ref["trajectories"][ok]), 1e-3))
    if bad_r.any():
        return t_err, 0.0
    m_err = np.max(np.abs(gpu.mean - ref["mean"]))
    assert t_err < rel, f"per-trajectory relative error {t_err:.3e}"
    assert m_err < mean_abs, f"ensemble-mean error {m_err:.3e}"
    np.testing.assert_allclose(gpu.weight, ref["weight"], rtol=1e-13)
    np.testing.assert_allclose(gpu.time, ref["time"], rtol=1e-15, atol=0)
    np.testing.assert_allclose(gpu.field, ref["field"], rtol=1e-12, atol=1e-16)
    return t_err, m_err


RELAX_CAP = 1e-7    # the largest relaxed per-trajectory bar any whole-ensemble test may apply
LD_STRICT = 1e-11   # oracle double-vs-long-double spread of the particles of the strict tests
MIN_WINDOWS = 5     # a relaxed comparison covers at least the initial state and 4 windows


def ld_spread(spec, ref):
    """Per-particle, per-window relative spread of the oracle's double run against its own
    long-double run (inf where either is non-finite), shape [n][windows]."""
    ld = oracle.simulate(spec, trajectories=True, long_double=True)
    t, tl = ref["trajectories"], ld["trajectories"]
    with np.errstate(invalid="ignore"):
        e = np.max(np.abs(t - tl) / np.maximum(np.abs(tl), 1e-3), axis=2)
    e[~(np.isfinite(t).all(axis=2) & np.isfinite(tl).all(axis=2))] = np.inf
    return e, ld


def conditioned_bars(spec, ref, label=""):
    """Bars and horizon of a whole-ensemble comparison: the strict 1e-9 / 1e-10, or 20x the
    oracle's own double-vs-long-double spread when that is larger, over the longest run of
    windows on which the relaxed per-trajectory bar stays at or below RELAX_CAP.  Returns
    (trajectory bar, mean bar, windows)."""
    e, ld = ld_spread(spec, ref)
    per_window = np.max(e, axis=0)
    cum = np.maximum.accumulate(per_window)
    k = int(np.searchsorted(cum, RELAX_CAP / 20, side="right"))
    assert k >= MIN_WINDOWS, f"{label}: the oracle is ill-conditioned from window {k} on (spread {cum[k]:.1e})"
    rel = max(REL_TRAJ, 20 * float(cum[k - 1]))
    m_ld = float(np.max(np.abs(ref["mean"][:k] - ld["mean"][:k])))
    mabs = max(ABS_MEAN, 20 * m_ld)
    assert rel <= RELAX_CAP and mabs <= RELAX_CAP
    print(f"{label}: bars {rel:.1e} / {mabs:.1e} over {k} of {len(cum)} windows")
    return rel, mabs, k


def first_windows(res, k):
    """The first k windows of a GPU result or an oracle record (later windows cannot change them)."""
    if isinstance(res, dict):
        return {**res, "trajectories": res["trajectories"][:, :k], "mean": res["mean"][:k],
                "time": res["time"][:k], "field": res["field"][:k]}
    return dataclasses.replace(res, trajectories=res.trajectories[:, :k], mean=res.mean[:k], time=res.time[:k],
                               field=res.field[:k])


def select_particles(spec, idx):
    """The particles idx (with their injected increments) as an ensemble of their own."""
    idx = np.asarray(idx)
    kw = {}
    for name in ("magnetic_radius", "saturation_magnetisation", "damping_constant", "gyromagnetic_ratio",
                 "anisotropy_constant", "hydrodynamic_radius", "viscosity", "cubic_constant"):
        v = getattr(spec, name)
        kw[name] = None if v is None else np.asarray(v)[idx]
    for name in ("orientation", "magnetisation", "uniaxial_rotation"):
        v = getattr(spec, name)
        kw[name] = None if v is None else np.asarray(v).reshape(-1, 3)[idx]
    m = spec.dims[1]
    kw["injected_dw"] = np.ascontiguousarray(np.asarray(spec.injected_dw).reshape(-1, m, spec.n)[:, :, idx])
    return dataclasses.replace(spec, n=len(idx), **kw)


@pytest.mark.parametrize("problem,solver", [(Problem.Neel, Solver.Heun_Strong), (Problem.Neel, Solver.EulerMaruyama),
                                            (Problem.NeelSpherical, Solver.Millstein),
                                            (Problem.BrownAndNeelEulerSpherical, Solver.EulerMaruyama),
                                            (Problem.Neel, Solver.Implicit_Midpoint)])
def test_cubic_short_horizon_strict(ctx, problem, solver):
    """Cubic anisotropy over a horizon where the FP64 oracle is itself accurate (400 steps):
    the strict 1e-9 / 1e-10 bars."""
    spec = provider.with_injected_noise(small_spec(problem, solver, Anisotropy.Cubic, steps=400, W=40), seed=3)
    gpu = ctx.simulate(spec, trajectories=True)
    ref = oracle.simulate(spec, trajectories=True)
    compare(gpu, ref)


EXPLICIT = [Solver.EulerMaruyama, Solver.Heun_Strong, Solver.Millstein]
PROBLEMS = [Problem.Neel, Problem.NeelSpherical, Problem.BrownAndNeelEulerSpherical, Problem.BrownAndNeel]
CASES = [(p, s, a) for p in PROBLEMS for s in EXPLICIT for a in (Anisotropy.Uniaxial, Anisotropy.Cubic)]
CASES += [(Problem.Neel, Solver.Implicit_Midpoint, Anisotropy.Uniaxial),
          (Problem.Neel, Solver.Implicit_Midpoint, Anisotropy.Cubic),
          (Problem.NeelSpherical, Solver.Implicit_Midpoint, Anisotropy.Uniaxial),
          (Problem.BrownAndNeel, Solver.Implicit_Midpoint, Anisotropy.Uniaxial)]


def injection_case(problem, solver, aniso, steps=1050, W=50):
    """The injection-mode ensemble of one (problem, solver, anisotropy): 67 particles,
    (steps / W - 1) W integrated steps (1000 by default)."""
    kw = {}
    if problem == Problem.BrownAndNeel and solver == Solver.EulerMaruyama:
        # EM without renormalisation amplifies the precession by sqrt(1 + (w dt)^2) per step;
        # at dt = 1e-11 |m| runs away (test_runaway_particles_match covers that regime)
        kw["timestep"] = 1e-12
    if problem == Problem.NeelSpherical and solver == Solver.Implicit_Midpoint:
        # with the coordinate rotation on, finish() returns phi in (-pi, pi] and the Newton
        # residual jumps by 2 pi: the reference formulation is only usable without rotation
        kw["use_coordinate_transformation"] = False
    spec = small_spec(problem, solver, aniso, steps=steps, W=W, **kw)
    if problem == Problem.NeelSpherical and solver == Solver.Implicit_Midpoint:
        # without the rotation, 1/sin(theta) near a pole leaves Newton unconverged and the
        # oracle's double and long-double runs part within the first window: keep the easy
        # axes (and the moments along them) within 60 degrees of the equator
        e = np.array(spec.orientation, copy=True)
        e[:, 1] = np.arccos(np.random.default_rng(4).uniform(-0.5, 0.5, spec.n))
        sign = np.sign(np.sum(np.asarray(spec.magnetisation) * provider.easy_axis(problem, spec.orientation), axis=1))
        spec = dataclasses.replace(spec, orientation=e, magnetisation=provider.easy_axis(problem, e) * sign[:, None])
    spec = provider.with_injected_noise(spec, seed=3)
    if solver == Solver.Implicit_Midpoint:
        spec = dataclasses.replace(spec, max_iteration=20, accuracy_goal=1e-10)
    return spec


CASE_IDS = [f"{p.name}-{s.name}-{a.name}" for p, s, a in CASES]


@pytest.mark.parametrize("problem,solver,aniso", CASES, ids=CASE_IDS)
def test_injection_parity_fp64_strict(ctx, problem, solver, aniso):
    """The strict bars, 1e-9 per trajectory and 1e-10 on the ensemble mean, over 1000
    integrated steps for every case: on the particles (at least 16) whose oracle run agrees
    with its own long-double run to LD_STRICT in every window."""
    spec = injection_case(problem, solver, aniso)
    assert spec.integrated_steps >= 1000
    e, _ = ld_spread(spec, oracle.simulate(spec, trajectories=True))
    good = np.where(np.max(e, axis=1) <= LD_STRICT)[0]
    assert len(good) >= 16, f"only {len(good)} well-conditioned particles"
    sub = select_particles(spec, good)
    gpu = ctx.simulate(sub, trajectories=True, final_state=True)
    ref = oracle.simulate(sub, trajectories=True, final_state=True)
    t_err, m_err = compare(gpu, ref)
    print(f"strict on {len(good)} of {spec.n} particles: trajectory {t_err:.1e}, mean {m_err:.1e}")
    assert gpu.stats["nonfinite_particles"] == 0


@pytest.mark.parametrize("problem,solver,aniso", CASES, ids=CASE_IDS)
def test_injection_parity_fp64(ctx, problem, solver, aniso):
    """The whole ensemble of every case, with the conditioned bars (at most RELAX_CAP)."""
    spec = injection_case(problem, solver, aniso)
    gpu = ctx.simulate(spec, trajectories=True, final_state=True)
    ref = oracle.simulate(spec, trajectories=True, final_state=True)
    rel, mabs, k = conditioned_bars(spec, ref, f"{problem.name}-{solver.name}-{aniso.name}")
    compare(first_windows(gpu, k), first_windows(ref, k), rel=rel, mean_abs=mabs)
    assert gpu.stats["nonfinite_particles"] == 0
    if solver == Solver.Implicit_Midpoint:
        assert gpu.stats["newton_iterations"] > 0
        # converged roots agree; iteration counts may differ by a few per run
        assert abs(gpu.stats["newton_iterations"] - ref["newton_iterations"]) <= 0.01 * ref["newton_iterations"] + 5


@pytest.mark.parametrize("aniso", [Anisotropy.Uniaxial, Anisotropy.Cubic])
def test_exact_jacobian_parity_fp64(ctx, aniso):
    """ImplicitMidpoint with the analytic Newton matrix: same bars as the reference
    mode, every step converged, iteration counts as in the oracle."""
    spec = provider.with_injected_noise(small_spec(Problem.Neel, Solver.Implicit_Midpoint, aniso), seed=3)
    spec = dataclasses.replace(spec, max_iteration=20, accuracy_goal=1e-10, jacobian=Jacobian.Exact)
    gpu = ctx.simulate(spec, trajectories=True, final_state=True)
    ref = oracle.simulate(spec, trajectories=True, final_state=True)
    rel, mabs, k = conditioned_bars(spec, ref, f"exact-{aniso.name}")
    compare(first_windows(gpu, k), first_windows(ref, k), rel=rel, mean_abs=mabs)
    assert gpu.stats["newton_unconverged"] == 0 and ref["newton_unconverged"] == 0
    assert abs(gpu.stats["newton_iterations"] - ref["newton_iterations"]) <= 0.01 * ref["newton_iterations"] + 5
    assert gpu.stats["newton_iterations"] <= 4.1 * spec.n * spec.integrated_steps


def test_exact_jacobian_fp32_state_with_fp64_acceptance(ctx):
    """The stiff cubic ImplicitMidpoint workload in the FP32 form (FP32 state, FP64
    residual acceptance) against the all-FP64 kernel, both with the exact Newton matrix.
    Particles hop between cubic easy axes (~1 kT barriers), so FP32 and FP64 paths on
    the same noise decorrelate by chaos as they do for the explicit steppers: the first
    window must agree closely, every window within 4 two-sample standard errors."""
    base = dataclasses.replace(provider.cubic_implicit(n=4096, steps=3000, oversampling=100),
                               jacobian=Jacobian.Exact)
    r64 = ctx.simulate(base)
    r32 = ctx.simulate(dataclasses.replace(base, precision=Precision.FP32))
    steps = base.n * base.integrated_steps
    assert r64.stats["newton_unconverged"] == 0
    assert r32.stats["newton_unconverged"] <= 1e-3 * steps
    d = np.abs(r32.mean - r64.mean)
    assert d[1].max() < 1e-4
    assert d.max() < 4 * math.sqrt(2.0 / (3.0 * base.n))


FIELDS = {
    "triangular": FieldSpec.triangular((0.0, 0.0, 0.01), 2e-9, 3e-10, (1e-3, 0.0, 0.0)),
    "rectangular": FieldSpec.rectangular((0.0, 0.004, 0.01), 2e-9, 1e-10, 3e-10, False),
    "rectangular_alternating": FieldSpec.rectangular((0.0, 0.004, 0.01), 2e-9, 1e-10, 3e-10, True),
    "sinc": FieldSpec.sinc((0.0, 0.0, 0.02), 2e-9, (0.0, 1e-3, 0.0)),
}


@pytest.mark.parametrize("name", list(FIELDS))
def test_field_waveform_parity(ctx, name):
    """Triangular, rectangular (plain and alternating) and sinc fields: the FP64 field
    table and the window-mean field against the oracle, and a Heun run driven by them
    (200 steps per period, 5 periods)."""
    spec = dataclasses.replace(small_spec(Problem.Neel, Solver.Heun_Strong, steps=1000, W=50), field=FIELDS[name])
    spec = provider.with_injected_noise(spec, seed=4)
    gpu = ctx.simulate(spec, trajectories=True)
    ref = oracle.simulate(spec, trajectories=True)
    rel, mabs, k = conditioned_bars(spec, ref, name)
    compare(first_windows(gpu, k), first_windows(ref, k), rel=rel, mean_abs=mabs)
    # the field table is independent of the dynamics: all windows at the field bar
    np.testing.assert_allclose(gpu.field, ref["field"], rtol=1e-12, atol=1e-16)
    assert np.ptp(ref["field"][1:], axis=0).max() > 1e-3  # the waveform actually varies


@pytest.mark.parametrize("problem", [Problem.Neel, Problem.BrownAndNeel, Problem.NeelSpherical])
def test_euler_maruyama_normalized_parity(ctx, problem):
    """EulerMaruyama_Normalized: EulerMaruyama followed by the problem's normalize
    (unit |m|, and |n| for the coupled Cartesian problem; no-op in spherical
    coordinates), at a step where plain EulerMaruyama runs away for BrownAndNeel."""
    spec = provider.with_injected_noise(small_spec(problem, Solver.EulerMaruyama_Normalized), seed=3)
    gpu = ctx.simulate(spec, trajectories=True, final_state=True)
    ref = oracle.simulate(spec, trajectories=True, final_state=True)
    rel, mabs, k = conditioned_bars(spec, ref, f"normalized-{problem.name}")
    compare(first_windows(gpu, k), first_windows(ref, k), rel=rel, mean_abs=mabs)
    assert gpu.stats["nonfinite_particles"] == 0
    if problem != Problem.NeelSpherical:
        fs = gpu.final_state.reshape(spec.n, -1, 3)
        np.testing.assert_allclose(np.linalg.norm(fs, axis=2), 1.0, rtol=1e-14)


UC_CASES = [(p, s) for p in (Problem.Neel, Problem.NeelSpherical, Problem.BrownAndNeelEulerSpherical)
            for s in (Solver.EulerMaruyama, Solver.Heun_Strong)] + [(Problem.Neel, Solver.Implicit_Midpoint)]


@pytest.mark.parametrize("problem,solver", UC_CASES, ids=[f"{p.name}-{s.name}" for p, s in UC_CASES])
def test_uniaxial_cubic_parity(ctx, problem, solver):
    """Uniaxial+cubic anisotropy (rotated uniaxial axis, K_u and K_c both set,
    per-particle rotations) against the oracle on the same increments."""
    base = small_spec(problem, solver)
    rng = np.random.default_rng(8)
    spec = dataclasses.replace(base, anisotropy=Anisotropy.UniaxialCubic, anisotropy_constant=np.full(base.n, -8e3),
                               cubic_constant=np.full(base.n, -4e3),
                               uniaxial_rotation=rng.uniform(0, 2 * math.pi, (base.n, 3)))
    if solver == Solver.Implicit_Midpoint:
        spec = dataclasses.replace(spec, max_iteration=20, accuracy_goal=1e-10)
    spec = provider.with_injected_noise(spec, seed=3)
    gpu = ctx.simulate(spec, trajectories=True)
    ref = oracle.simulate(spec, trajectories=True)
    label = f"uniaxial-cubic-{problem.name}-{solver.name}"
    rel, mabs, k = conditioned_bars(spec, ref, label)
    compare(first_windows(gpu, k), first_windows(ref, k), rel=rel, mean_abs=mabs)
    if solver == Solver.Implicit_Midpoint:
        ex = dataclasses.replace(spec, jacobian=Jacobian.Exact)
        rex = oracle.simulate(ex, trajectories=True)
        rel, mabs, k = conditioned_bars(ex, rex, label + "-exact")
        compare(first_windows(ctx.simulate(ex, trajectories=True), k), first_windows(rex, k), rel=rel, mean_abs=mabs)


def test_runaway_particles_match(ctx):
    """Brown+Neel Cartesian with EulerMaruyama at dt = 1e-11: |m| is not renormalised in the
    reference's solver, so some particles diverge; the same particles diverge on both sides."""
    spec = provider.with_injected_noise(small_spec(Problem.BrownAndNeel, Solver.EulerMaruyama), seed=3)
    gpu = ctx.simulate(spec, trajectories=True)
    ref = oracle.simulate(spec, trajectories=True)
    compare(gpu, ref)
    n_bad = int((~np.isfinite(ref["trajectories"]).all(axis=(1, 2))).sum())
    assert n_bad > 0 and gpu.stats["nonfinite_particles"] == n_bad


def test_philox_normals_bit_layout(ctx):
    for m in (3, 6):
        dev = ctx.philox_normals(seed=0x5EED0001, pid0=17, n=300, step0=123456, nsteps=40, noise_dim=m, precision=0)
        cpu = oracle.philox_normals(0x5EED0001, 17, 300, 123456, 40, m)
        np.testing.assert_allclose(dev, cpu, rtol=1e-13, atol=1e-14)
        f32 = ctx.philox_normals(seed=0x5EED0001, pid0=17, n=300, step0=123456, nsteps=40, noise_dim=m, precision=1)
        # FP32 draws use the same Philox words; SFU log/sincos keep them within ~1e-5 of the FP64 draws
        assert np.max(np.abs(f32 - cpu)) < 2e-5


@pytest.mark.parametrize("problem,solver", [(Problem.Neel, Solver.Heun_Strong),
                                            (Problem.BrownAndNeelEulerSpherical, Solver.Millstein)])
def test_philox_mode_parity_fp64(ctx, problem, solver):
    spec = small_spec(problem, solver, n=129, steps=2000, W=100)
    gpu = ctx.simulate(spec, trajectories=True)
    ref = oracle.simulate(spec, trajectories=True)
    compare(gpu, ref)


def test_config_shaped_parity(ctx):
    """The three single-ensemble workloads at reduced size, injection mode."""
    for spec in (provider.neel_relaxation(n=256, steps=3000, oversampling=100),
                 provider.brown_neel_relaxation(n=96, steps=3000, oversampling=100),
                 provider.cubic_implicit(n=96, steps=600, oversampling=100)):
        spec = provider.with_injected_noise(spec, seed=5)
        gpu = ctx.simulate(spec, trajectories=True)
        ref = oracle.simulate(spec, trajectories=True)
        compare(gpu, ref)


@pytest.mark.parametrize("n,steps,W", [(1, 500, 50), (33, 1050, 100), (300, 100, 100), (40, 999, 333)])
def test_edge_sizes(ctx, n, steps, W):
    """one particle, ragged warps, a single sample (no integrated steps), steps % W != 0"""
    spec = provider.with_injected_noise(small_spec(Problem.Neel, Solver.Heun_Strong, n=n, steps=steps, W=W), seed=9)
    gpu = ctx.simulate(spec, trajectories=True)
    ref = oracle.simulate(spec, trajectories=True)
    assert gpu.mean.shape == (steps // W, 3)
    compare(gpu, ref)


def test_chunked_advance_equals_one_shot(ctx):
    """advancing in odd-sized pieces (windows straddle the pieces) gives identical results"""
    spec = small_spec(Problem.BrownAndNeelEulerSpherical, Solver.Heun_Strong, n=100, steps=2000, W=100,
                      record_trajectories=True)
    one = ctx.simulate(spec, trajectories=True)
    with ctx.ensemble(spec) as e:
        done, total = e.steps()
        assert (done, total) == (0, 1900)
        while done < total:
            e.advance(37)
            done, _ = e.steps()
        r = e.read(trajectories=True)
    np.testing.assert_array_equal(r.mean, one.mean)
    np.testing.assert_array_equal(r.trajectories, one.trajectories)


FP32_CASES = [(Problem.Neel, Solver.Heun_Strong, 65536, 21000), (Problem.Neel, Solver.Millstein, 65536, 21000),
              (Problem.NeelSpherical, Solver.Heun_Strong, 65536, 21000),
              (Problem.NeelSpherical, Solver.EulerMaruyama, 65536, 21000),
              (Problem.BrownAndNeelEulerSpherical, Solver.Millstein, 524288, 31000),
              (Problem.BrownAndNeelEulerSpherical, Solver.Heun_Strong, 524288, 31000),
              (Problem.BrownAndNeel, Solver.EulerMaruyama_Normalized, 65536, 21000)]


@pytest.mark.parametrize("problem,solver,n,steps", FP32_CASES,
                         ids=[f"{p.name}-{s.name}-{n}" for p, s, n, _ in FP32_CASES])
def test_fp32_ensemble_mean_within_1e_3(ctx, problem, solver, n, steps):
    """The FP32 form against the FP64 kernel on the same Philox noise, the qualifier of the
    headline metric: the moment-weighted mean magnetisation (saturation value 1) of the FP32
    ensemble within 1e-3 of the FP64 one in every window and component.  The ensemble runs
    as 16 shards with global particle ids, merged (sp_merge_shards); the spread of the
    shards' differences gives the standard error, whose root mean square over the windows
    must be at most 3e-4 (and its largest single estimate at most 4.5e-4) so that a 1e-3
    error is resolved, and the difference averaged over the windows must be within 4 standard
    errors of zero (no bias; a plainly rounded FP32 state update of the slow Brown angles
    gave -4e-4, about 5 standard errors, on the headline workload).  The first window
    agrees pathwise (1e-4).  The coupled Cartesian problem runs EulerMaruyama_Normalized:
    its other explicit steppers let |m| run away to overflow within these horizons, as the
    reference's do."""
    shards = 16
    spec = small_spec(problem, solver, n=n, steps=steps, W=1000)
    k = n // shards
    parts = [spec.subset(i * k, (i + 1) * k) for i in range(shards)]
    res = {}
    for prec in (Precision.FP64, Precision.FP32):
        with ctx.server() as srv:
            ids = srv.submit_many([dataclasses.replace(p, precision=prec) for p in parts])
            res[prec] = [srv.wait(i)[0] for i in ids]
    merged = {prec: sp.merge_shards([r.weighted_sum for r in rs], [r.weight for r in rs])[0] for prec, rs in res.items()}
    cols = slice(spec.dims[2] - 3, spec.dims[2])
    d = (merged[Precision.FP32] - merged[Precision.FP64])[1:, cols]
    per_shard = np.stack([(a.mean - b.mean)[1:, cols] for a, b in zip(res[Precision.FP32], res[Precision.FP64])])
    se = per_shard.std(axis=0, ddof=1) / math.sqrt(shards)
    bias, bias_se = d.mean(axis=0), per_shard.mean(axis=1).std(axis=0, ddof=1) / math.sqrt(shards)
    label = f"{problem.name}/{solver.name}"
    rms_se = float(np.sqrt(np.mean(se ** 2)))
    print(f"{label}: max {np.abs(d).max():.2e}, rms se {rms_se:.2e}, max se {se.max():.2e}, bias {bias} +- {bias_se}")
    assert np.isfinite(d).all(), f"{label}: non-finite mean"
    assert np.abs(d[0]).max() < 1e-4, f"{label}: first-window FP32 error {np.abs(d[0]).max():.2e}"
    assert np.abs(d).max() <= 1e-3, f"{label}: FP32 mean error {np.abs(d).max():.2e}"
    assert rms_se <= 3e-4 and se.max() <= 4.5e-4, f"{label}: standard error {rms_se:.2e} cannot resolve 1e-3"
    assert np.all(np.abs(bias) <= 4 * bias_se + 1e-5), f"{label}: FP32 bias {bias} (se {bias_se})"


def test_fp32_difference_is_unbiased_path_noise(ctx):
    """Why the FP32 and FP64 means part after the first windows.  Brown+Neel Euler Heun,
    4096 particles x 1e5 steps, same Philox stream.  Each particle's FP32 path drifts from
    its FP64 path by accumulated rounding (median of the largest window difference about
    2e-3), with random sign across particles, so the drift averages out of the ensemble
    mean; and a small fraction of particles take a different path altogether (a barrier
    crossing in one run and not the other), as an FP64 run started from Euler angles
    perturbed by 1e-7 rad, FP32 rounding size, also shows.  The mean difference is
    therefore Monte-Carlo, bounded by the two-sample standard error, not an FP32 bias."""
    n = 4096
    spec = small_spec(Problem.BrownAndNeelEulerSpherical, Solver.Heun_Strong, n=n, steps=100000, W=1000)
    rng = np.random.default_rng(5)
    pert = dataclasses.replace(spec, orientation=spec.orientation + 1e-7 * rng.standard_normal(spec.orientation.shape))
    r64 = ctx.simulate(spec, trajectories=True)
    r64p = ctx.simulate(pert, trajectories=True)
    r32 = ctx.simulate(dataclasses.replace(spec, precision=Precision.FP32), trajectories=True)
    diff32 = r32.trajectories[:, :, 6:9] - r64.trajectories[:, :, 6:9]
    d32 = np.abs(diff32).max(axis=(1, 2))
    dp = np.abs(r64p.trajectories[:, :, 6:9] - r64.trajectories[:, :, 6:9]).max(axis=(1, 2))
    assert np.median(d32) < 1e-2 and np.median(dp) < 1e-5
    divp = (dp > 0.1).mean()
    assert 0 < divp < 0.02, f"perturbed FP64 diverged fraction {divp:.4f}"
    last = diff32[:, -1, :]  # signed per-particle difference in the last window
    assert np.all(np.abs(last.mean(axis=0)) < 4 * last.std(axis=0) / math.sqrt(n))
    se = math.sqrt(2.0 / (3.0 * n))
    assert np.abs(r32.mean[:, 6:9] - r64.mean[:, 6:9]).max() < 4 * se


@pytest.mark.parametrize("problem,solver", [(Problem.Neel, Solver.Heun_Strong),
                                            (Problem.BrownAndNeelEulerSpherical, Solver.EulerMaruyama)])
def test_philox_mean_within_three_standard_errors_of_independent_noise(ctx, problem, solver):
    """The in-kernel RNG against independent noise, as the reference's own generator would
    be: the FP64 GPU run with Philox increments and the oracle run with independently drawn
    (injected) increments of the same particles agree window by window within 3 standard
    errors of the paired difference (per particle: GPU window mean minus oracle window
    mean); at most 2 % of the (window, component) pairs may exceed 3 and none 5."""
    n = 4096
    spec = small_spec(problem, solver, n=n, steps=5000, W=250)
    gpu = ctx.simulate(spec, trajectories=True)
    ref = oracle.simulate(provider.with_injected_noise(spec, seed=77), trajectories=True)
    d = gpu.trajectories[:, 1:, -3:] - ref["trajectories"][:, 1:, -3:]
    z = np.abs(d.mean(axis=0)) / (d.std(axis=0) / math.sqrt(n))
    assert (z > 3).mean() <= 0.02 and z.max() < 5, f"max z {z.max():.2f}, share above 3 {(z > 3).mean():.3f}"


LANGEVIN = [(p, prec) for p in (Problem.Neel, Problem.NeelSpherical, Problem.BrownAndNeelEulerSpherical)
            for prec in (Precision.FP64, Precision.FP32)]


@pytest.mark.parametrize("problem,precision", LANGEVIN, ids=[f"{p.name}-{q.name}" for p, q in LANGEVIN])
def test_langevin_equilibrium(ctx, problem, precision):
    """Zero anisotropy, constant field, Heun: <m.B/|B|> -> coth(xi) - 1/xi with
    xi = Ms V |B| / (kB T), for every problem that carries a magnetisation direction and in
    both precisions (the Euler problem's magnetisation is outputs 7-9).  Heun, because the
    reference's Millstein formula (Millstein.inl:43, D |dW|^2) does not keep this
    equilibrium (test_oracle_cpu.py pins that)."""
    n, B = 16384, 0.01
    rng = np.random.default_rng(21)
    v = rng.standard_normal((n, 3))
    m0 = v / np.linalg.norm(v, axis=1, keepdims=True)
    if problem == Problem.BrownAndNeelEulerSpherical:
        base = provider.brown_neel_relaxation(n=n, steps=60000, oversampling=1000, solver=Solver.Heun_Strong)
        base = dataclasses.replace(base, magnetic_radius=np.full(n, 10e-9), hydrodynamic_radius=np.full(n, 30e-9))
    else:
        base = provider.neel_relaxation(n=n, steps=60000, oversampling=1000, solver=Solver.Heun_Strong)
        if problem == Problem.NeelSpherical:
            base = dataclasses.replace(base, problem=problem, use_coordinate_transformation=True,
                                       min_angle_before_transformation=math.pi / 36)
    spec = dataclasses.replace(base, anisotropy_constant=np.zeros(n), magnetisation=m0, precision=precision,
                               field=sp.FieldSpec.constant((0.0, 0.0, B)))
    r = ctx.simulate(spec)
    V = 4.0 / 3.0 * math.pi * (10e-9) ** 3
    xi = 4.8e5 * V * B / (1.3806485279e-23 * 295.0)
    langevin = 1.0 / math.tanh(xi) - 1.0 / xi
    tail = r.mean[30:, -1]  # m_z after ~5 relaxation times
    se = 1.0 / math.sqrt(3.0 * n)  # per-window standard error bound (|m_z| <= 1, variance <= 1/3)
    assert abs(tail.mean() - langevin) < 3 * se + 2e-3, (tail.mean(), langevin)


def test_nonfinite_particle_is_flagged(ctx):
    spec = small_spec(Problem.Neel, Solver.EulerMaruyama, n=64, steps=500, W=50)
    mag = np.array(spec.magnetisation, copy=True)
    mag[5] = 0.0  # normalising a zero vector gives NaN (NeelRelaxation.h:283)
    r = ctx.simulate(dataclasses.replace(spec, magnetisation=mag))
    assert r.stats["nonfinite_particles"] == 1


def test_server_alone_equals_in_mix(ctx):
    """Continuous batching: a request's result is identical alone and sharing launches."""
    a = small_spec(Problem.Neel, Solver.Heun_Strong, n=3000, steps=30000, W=1000, seed=1)
    b = small_spec(Problem.Neel, Solver.Heun_Strong, n=5000, steps=50000, W=1000, seed=2)
    c = small_spec(Problem.BrownAndNeelEulerSpherical, Solver.Millstein, n=2000, steps=20000, W=1000, seed=3)
    alone = ctx.simulate(a)
    with ctx.server(chunk_steps=5000) as srv:
        ib = srv.submit(b)
        ia = srv.submit(a)
        ic = srv.submit(c)
        ra, lat_a = srv.wait(ia)
        rb, _ = srv.wait(ib)
        rc, _ = srv.wait(ic)
    np.testing.assert_array_equal(ra.mean, alone.mean)
    np.testing.assert_array_equal(rb.mean, ctx.simulate(b).mean)
    np.testing.assert_array_equal(rc.mean, ctx.simulate(c).mean)
    assert lat_a > 0
