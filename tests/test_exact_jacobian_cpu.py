"""The analytic Newton matrix of ImplicitMidpoint (SP_JACOBIAN_EXACT), on the CPU.

The reference's Neel Jacobians are approximations (a -2 alpha/dt [m]x stand-in for
the damping derivative, no derivative of the projection part of b, and J_H = I for
cubic anisotropy: NeelRelaxation.h:134-190, CubicAnisotropy.h:228-236); Newton
still converges to the same root where it converges at all, only more slowly.
The exact mode differentiates a(m) and b(m) dW analytically.  Checked here:
  - against central finite differences of the oracle's own a(m) and b(m) dW;
  - the oracle's ImplicitMidpoint in both modes: same states within the Newton
    tolerance where the reference mode converges, far fewer iterations, and
    convergence for cubic anisotropy where the reference mode never converges.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import oracle
from stochasticphysics_b200 import provider
from stochasticphysics_b200._abi import Anisotropy, DescHolder, Jacobian, Problem, Solver
from stochasticphysics_b200.lib import load

PROPS = [11e-9, 4.8e5, 0.07, 1.76e11, -1.1e4, 295.0]  # radius, Ms, alpha, gamma, K, T


def _a_and_bw(aniso, euler, m, field, dW):
    props8 = PROPS[:5] + [0.0, 0.0, PROPS[5]]
    out = oracle.eval_problem(int(Problem.Neel), int(aniso), props8, euler, [0] * 7, m, field=field, dW=dW)
    return out["a"], out["b"] @ np.asarray(dW)


@pytest.mark.parametrize("aniso", [Anisotropy.Uniaxial, Anisotropy.Cubic])
def test_exact_jacobians_match_finite_differences(aniso):
    rng = np.random.default_rng(5)
    for _ in range(8):
        euler = rng.uniform(0, 2 * np.pi, 3)
        m = rng.standard_normal(3)
        m *= rng.uniform(0.8, 1.2) / np.linalg.norm(m)  # off the unit sphere too: |m| drifts in the reference
        field = rng.uniform(-0.02, 0.02, 3)
        dW = rng.standard_normal(3) * np.sqrt(1e-10)
        jd, js = oracle.neel_exact_jacobians(int(aniso), PROPS, euler, m, field, dW)
        h = 1e-6
        fd_a, fd_b = np.zeros((3, 3)), np.zeros((3, 3))
        for j in range(3):
            e = np.zeros(3); e[j] = h
            ap, bp = _a_and_bw(aniso, euler, m + e, field, dW)
            am, bm = _a_and_bw(aniso, euler, m - e, field, dW)
            fd_a[:, j] = (ap - am) / (2 * h)
            fd_b[:, j] = (bp - bm) / (2 * h)
        np.testing.assert_allclose(jd, fd_a, rtol=1e-6, atol=1e-8 * np.abs(fd_a).max())
        np.testing.assert_allclose(js, fd_b, rtol=1e-6, atol=1e-8 * np.abs(fd_b).max())


def _im(spec, jac):
    s = dataclasses.replace(spec, jacobian=jac)
    return oracle.simulate(s, trajectories=True)


def test_exact_mode_reaches_the_reference_root_in_fewer_iterations():
    spec = provider.neel_relaxation(n=64, steps=2000, oversampling=100, solver=Solver.Implicit_Midpoint)
    spec = dataclasses.replace(spec, max_iteration=20, accuracy_goal=1e-10)
    ref = _im(spec, Jacobian.Reference)
    ex = _im(spec, Jacobian.Exact)
    steps = spec.n * spec.integrated_steps
    assert ref["newton_unconverged"] == 0 and ex["newton_unconverged"] == 0
    assert ex["newton_iterations"] < 0.5 * ref["newton_iterations"]
    assert ex["newton_iterations"] <= 4 * steps
    # both accept within 1e-10 of the same implicit-midpoint root
    np.testing.assert_allclose(ex["trajectories"], ref["trajectories"], rtol=0, atol=1e-8)


def test_exact_mode_converges_for_cubic_anisotropy():
    spec = provider.cubic_implicit(n=64, steps=2000, oversampling=100)
    ref = _im(spec, Jacobian.Reference)
    ex = _im(spec, Jacobian.Exact)
    steps = spec.n * spec.integrated_steps
    assert ref["newton_unconverged"] == steps  # J_H = I: the reference iteration never meets 1e-10
    assert ex["newton_unconverged"] == 0
    assert ex["newton_iterations"] <= 4.1 * steps  # vs 20 per step in the reference mode
    assert np.all(np.isfinite(ex["trajectories"]))


@pytest.mark.parametrize("problem,expect", [(Problem.Neel, 0), (Problem.NeelSpherical, 2), (Problem.BrownAndNeel, 2)])
def test_validation_of_the_jacobian_mode(problem, expect):
    spec = provider.neel_relaxation(n=8, steps=200, oversampling=100, solver=Solver.Implicit_Midpoint)
    kw = {}
    if problem == Problem.BrownAndNeel:
        kw = {"hydrodynamic_radius": np.full(8, 3e-8), "viscosity": np.full(8, 1e-3)}
    spec = dataclasses.replace(spec, problem=problem, jacobian=Jacobian.Exact, max_iteration=20,
                               accuracy_goal=1e-10, **kw)
    assert load().sp_validate(DescHolder(spec).byref()) == expect
    h = DescHolder(spec)
    h.desc.jacobian = 7
    assert load().sp_validate(h.byref()) == 1
