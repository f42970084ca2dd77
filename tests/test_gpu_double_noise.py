"""GPU parity of the solvers the reference switches off in its manager
(SimulationManager.h:325-328): Heun_NotConsistent (Heun_NotConsistent.inl:35-47),
WeakTest (WeakTest.inl:18-63) and ExplicitStrong_1.0 (Explicit_Strong_1.inl:20-78),
the last two with the double noise matrix of order p (DoubleNoiseMatrix.h).

They take in-kernel Philox noise only: dW from calls 0-1 of each step, dW2 or the
double-noise draws from calls 2 and up, on the device and in the oracle alike.
Bars: FP64 per-trajectory window means within 1e-9 relative and the ensemble mean
within 1e-10 (or 20x the oracle's double-vs-long-double spread where the dynamics
amplify round-off); FP32 as the other solvers' FP32 check.
"""
import dataclasses
import math

import numpy as np
import pytest

import oracle
import stochasticphysics_b200 as sp
from stochasticphysics_b200 import provider
from stochasticphysics_b200._abi import Anisotropy, Noise, Precision, Problem, Solver
from stochasticphysics_b200.lib import SPError
from test_gpu_parity import compare, conditioned_bars, first_windows, small_spec

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = sp.Context(0)
    yield c
    c.close()


HNC, WT, ES1 = Solver.Heun_NotConsistent, Solver.WeakTest, Solver.ExplicitStrong_1
U, C, UC = Anisotropy.Uniaxial, Anisotropy.Cubic, Anisotropy.UniaxialCubic
CASES = [
    (Problem.Neel, HNC, U, -1), (Problem.Neel, ES1, U, -1), (Problem.Neel, ES1, C, 2),
    (Problem.Neel, WT, U, 0), (Problem.Neel, WT, UC, 10),
    (Problem.NeelSpherical, HNC, U, -1), (Problem.NeelSpherical, ES1, U, 1), (Problem.NeelSpherical, WT, U, 3),
    (Problem.BrownAndNeelEulerSpherical, HNC, U, -1), (Problem.BrownAndNeelEulerSpherical, ES1, U, 3),
    (Problem.BrownAndNeelEulerSpherical, WT, U, 10),
    (Problem.BrownAndNeel, HNC, U, -1), (Problem.BrownAndNeel, ES1, U, 1),
]


def case_spec(problem, solver, aniso, p, **kw):
    spec = small_spec(problem, solver, aniso=U if aniso == UC else aniso, **kw)
    if aniso == UC:
        rng = np.random.default_rng(8)
        spec = dataclasses.replace(spec, anisotropy=UC, anisotropy_constant=np.full(spec.n, -8e3),
                                   cubic_constant=np.full(spec.n, -4e3),
                                   uniaxial_rotation=rng.uniform(0, 2 * math.pi, (spec.n, 3)))
    return dataclasses.replace(spec, double_noise_approx=p)


@pytest.mark.parametrize("problem,solver,aniso,p", CASES,
                         ids=[f"{a.name}-{b.name}-{c.name}-p{d}" for a, b, c, d in CASES])
def test_reference_disabled_solver_parity_fp64(ctx, problem, solver, aniso, p):
    spec = case_spec(problem, solver, aniso, p)
    gpu = ctx.simulate(spec, trajectories=True)
    ref = oracle.simulate(spec, trajectories=True)
    rel, mabs, k = conditioned_bars(spec, ref, f"{problem.name}-{solver.name}-{aniso.name}-p{p}")
    compare(first_windows(gpu, k), first_windows(ref, k), rel=rel, mean_abs=mabs)


@pytest.mark.parametrize("problem,solver,p", [(Problem.Neel, HNC, -1), (Problem.Neel, ES1, 4),
                                              (Problem.BrownAndNeelEulerSpherical, ES1, 0)])
def test_reference_disabled_solver_fp32_close_to_fp64(ctx, problem, solver, p):
    """FP32 stepping vs FP64 on the same Philox words: first window within 1e-4 and
    every window within 4 standard errors of the difference of two means."""
    n = 4096
    spec = dataclasses.replace(small_spec(problem, solver, n=n, steps=20000, W=1000), double_noise_approx=p)
    r64 = ctx.simulate(spec)
    r32 = ctx.simulate(dataclasses.replace(spec, precision=Precision.FP32))
    d = np.abs(r32.mean[:, -3:] - r64.mean[:, -3:])
    assert np.max(d[1]) < 1e-4, f"first-window FP32 error {np.max(d[1]):.2e}"
    assert np.nanmax(d) < 4 * math.sqrt(2.0 / (3.0 * n)), f"FP32 mean error {np.nanmax(d):.2e}"


def test_weak_test_fp32_close_to_fp64_before_it_runs_away(ctx):
    """WeakTest adds (b(S+) + b(S-)) dW once per support pair (WeakTest.inl:47-52), so |m|
    grows without bound: a third of the particles overflow within 1000 steps at dt = 1e-11.
    FP32 and FP64 are compared over the first 400 steps, window by window, within 1e-3."""
    spec = dataclasses.replace(small_spec(Problem.Neel, WT, n=4096, steps=500, W=100), double_noise_approx=1)
    r64 = ctx.simulate(spec)
    r32 = ctx.simulate(dataclasses.replace(spec, precision=Precision.FP32))
    assert np.isfinite(r64.mean).all() and np.isfinite(r32.mean).all()
    d = np.abs(r32.mean - r64.mean)
    assert np.max(d[1]) < 1e-4 and np.max(d) < 1e-3, f"FP32 mean error {np.max(d):.2e}"


def test_double_noise_order_changes_the_path(ctx):
    """The order p selects the draws: p = -1 and p = 3 share dW but not the paths."""
    a = ctx.simulate(case_spec(Problem.Neel, ES1, U, -1), trajectories=True).trajectories
    b = ctx.simulate(case_spec(Problem.Neel, ES1, U, 3), trajectories=True).trajectories
    np.testing.assert_array_equal(a[:, 0], b[:, 0])
    assert np.abs(a[:, 1:] - b[:, 1:]).max() > 0


def test_refusals(ctx):
    spec = provider.with_injected_noise(case_spec(Problem.Neel, ES1, U, 1), seed=3)
    with pytest.raises(SPError, match="Philox"):
        ctx.simulate(spec)
    with pytest.raises(SPError, match="double_noise_approx"):
        ctx.simulate(case_spec(Problem.Neel, WT, U, 11))
    assert spec.noise == Noise.Injected
