"""CPU checks of the solvers the reference switches off in its manager
(SimulationManager.h:325-328) and of the double noise matrix, on the oracle alone.

Heun_NotConsistent (Heun_NotConsistent.inl:35-47), WeakTest (WeakTest.inl:18-63) and
ExplicitStrong_1.0 (Explicit_Strong_1.inl:20-78), the latter two with
DoubleNoiseMatrix.h.  The reference seeds these generators from std::random_device,
so nothing pins their draws; the checks are the matrix's structure and moments, the
deterministic limits, and one step restated from the problem pieces.
"""
import dataclasses
import math

import numpy as np
import pytest

import oracle
from stochasticphysics_b200 import provider
from stochasticphysics_b200._abi import FieldSpec, Problem, Solver


def s_p(p):
    return sum(1.0 / (r * r) for r in range(1, p + 1))


@pytest.mark.parametrize("m", [3, 6])
@pytest.mark.parametrize("p", [-1, 0, 1, 4, 10])
def test_double_noise_matrix_structure(m, p):
    """J = dW dW^T / 2 + A with A antisymmetric, diagonal dW^2 / 2, A = 0 for p = -1;
    dW is the step's own Philox increment."""
    dt = 1e-11
    dw, J = oracle.double_noise_matrix(0x5EED, 100, 500, 77, p, dt, m)
    sym = 0.5 * (J + J.transpose(0, 2, 1))
    np.testing.assert_allclose(sym, 0.5 * dw[:, :, None] * dw[:, None, :], rtol=0, atol=1e-12 * dt)
    np.testing.assert_array_equal(np.diagonal(J, axis1=1, axis2=2), 0.5 * dw * dw)
    A = 0.5 * (J - J.transpose(0, 2, 1))
    if p == -1:
        assert not A.any()
    else:
        assert np.all(A[:, np.triu_indices(m, 1)[0], np.triu_indices(m, 1)[1]] != 0)
    z = oracle.philox_normals(0x5EED, 100, 500, 77, 1, m)[0].T
    np.testing.assert_allclose(dw, z * math.sqrt(dt), rtol=1e-15)


@pytest.mark.parametrize("p", [0, 1, 3, 10])
def test_double_noise_antisymmetric_moments(p):
    """The reference's formula with N(0, dt) draws: E[A] = 0, E[A dW] = 0 and
    Var[A] = dt^2 (1/6 + S_p / (2 pi^2)), S_p = sum_{r<=p} 1/r^2 (two rho_p^2 dt^2
    from the mu term, 6 dt^2 / (4 pi^2 r^2) per Fourier term)."""
    dt = 1.0
    n = 40000
    dw, J = oracle.double_noise_matrix(0x5EED0002, 0, n, 5, p, dt, 3)
    A = np.concatenate([J[:, 1, 0], J[:, 2, 0], J[:, 2, 1]]) - np.concatenate(
        [0.5 * dw[:, 1] * dw[:, 0], 0.5 * dw[:, 2] * dw[:, 0], 0.5 * dw[:, 2] * dw[:, 1]])
    var = (1.0 / 6.0 + s_p(p) / (2 * math.pi ** 2)) * dt ** 2
    assert abs(A.var() / var - 1) < 0.03
    assert abs(A.mean()) < 5 * math.sqrt(var / A.size)
    w0 = np.concatenate([dw[:, 0], dw[:, 0], dw[:, 1]])
    assert abs(np.mean(A * w0)) < 5 * math.sqrt(var * dt / A.size)


def _zero_t(problem, solver, **kw):
    if problem == Problem.BrownAndNeelEulerSpherical:
        base = provider.brown_neel_relaxation(n=16, steps=400, oversampling=20, seed=4)
    else:
        base = provider.neel_relaxation(n=16, steps=400, oversampling=20, seed=4)
        if problem == Problem.NeelSpherical:
            base = dataclasses.replace(base, problem=Problem.NeelSpherical, use_coordinate_transformation=True,
                                       min_angle_before_transformation=math.pi / 36)
    return dataclasses.replace(base, temperature=0.0, solver=solver, **kw)


@pytest.mark.parametrize("problem", [Problem.Neel, Problem.NeelSpherical, Problem.BrownAndNeelEulerSpherical])
def test_zero_temperature_limits(problem):
    """With b = 0 and D = 0: ExplicitStrong_1.0 is EulerMaruyama and Heun_NotConsistent
    is Heun_Strong, bit for bit, whatever the double-noise order."""
    em = oracle.simulate(_zero_t(problem, Solver.EulerMaruyama), trajectories=True)["trajectories"]
    heun = oracle.simulate(_zero_t(problem, Solver.Heun_Strong), trajectories=True)["trajectories"]
    for p in (-1, 0, 3):
        es1 = oracle.simulate(_zero_t(problem, Solver.ExplicitStrong_1, double_noise_approx=p), trajectories=True)
        np.testing.assert_array_equal(es1["trajectories"], em)
    hnc = oracle.simulate(_zero_t(problem, Solver.Heun_NotConsistent), trajectories=True)["trajectories"]
    np.testing.assert_array_equal(hnc, heun)
    assert np.abs(em - heun).max() > 0


def _one_step_spec(solver, p=-1):
    base = provider.neel_relaxation(n=6, steps=2, oversampling=1, dt=1e-11, seed=9)
    return dataclasses.replace(base, solver=solver, double_noise_approx=p, seed=0xABC, particle_id_offset=40,
                               field=FieldSpec.constant((0.004, -0.002, 0.006)))


def _pieces(spec, i):
    props = [spec.magnetic_radius[i], spec.saturation_magnetisation[i], spec.damping_constant[i],
             spec.gyromagnetic_ratio[i], spec.anisotropy_constant[i], 0.0, 0.0, spec.temperature]
    euler = spec.orientation[i]

    def ev(y):
        r = oracle.eval_problem(int(Problem.Neel), 0, props, euler, [0] * 7, y, field=spec.field.offset)
        return r["a"], r["b"], r["drift"]
    return ev


@pytest.mark.parametrize("solver,p", [(Solver.Heun_NotConsistent, -1), (Solver.ExplicitStrong_1, -1),
                                      (Solver.ExplicitStrong_1, 2), (Solver.WeakTest, 0), (Solver.WeakTest, 5)])
def test_one_step_restated_from_problem_pieces(solver, p):
    """One Neel Cartesian step composed here from a(y), b(y), D(y) of the problem and
    the oracle's dW / dW2 / J equals the oracle's stepper."""
    spec = _one_step_spec(solver, p)
    got = oracle.simulate(spec, trajectories=True)["trajectories"][:, 1, :]
    dt, sq = spec.timestep, math.sqrt(spec.timestep)
    for i in range(spec.n):
        ev = _pieces(spec, i)
        pid = spec.particle_id_offset + i
        y = np.asarray(spec.magnetisation[i], dtype=float)
        dw = sq * oracle.philox_normals(spec.seed, pid, 1, 0, 1, 3)[0, :, 0]
        a, b, d = ev(y)
        if solver == Solver.Heun_NotConsistent:
            dw2 = sq * _call_normals(spec.seed, pid, 0, 2)[:3]  # dW2: Philox call 2
            s = y + (a + d) * dt + b @ dw
            a2, b2, d2 = ev(s)
            want = y + 0.5 * (a2 + d2 + a + d) * dt + 0.5 * (b2 + b) @ dw2
        else:
            dw_j, J = oracle.double_noise_matrix(spec.seed, pid, 1, 0, p, dt, 3)
            np.testing.assert_array_equal(dw_j[0], dw)
            J = J[0]
            t = y + a * dt
            corr = np.zeros(3)
            add = np.zeros(3)
            for j in range(3):
                bp = ev(t + b[:, j] * sq)[1]
                bm = ev(t - b[:, j] * sq)[1]
                corr += (bp - bm) @ J[:, j]
                add += (bp + bm) @ dw
            if solver == Solver.ExplicitStrong_1:
                want = corr / sq + t + b @ dw
            else:
                as_ = ev(t + b @ dw)[0]
                tt = (corr / sq + add) / 4 + 0.5 * (b @ dw)
                y2 = y + 0.5 * as_ * dt + 0.5 * a * dt + tt
                want = y + 0.5 * ev(y2)[0] * dt + 0.5 * a * dt + tt
        np.testing.assert_allclose(got[i], want, rtol=1e-12, atol=1e-15)


def _call_normals(seed, pid, step, call):
    """Normals of Philox call `call`: the counter's top byte selects the call."""
    ctr = [step & 0xFFFFFFFF, step >> 32, pid & 0xFFFFFFFF, ((pid >> 32) & 0xFFFFFF) | (call << 24)]
    w = oracle.philox4x32_10(ctr, [seed & 0xFFFFFFFF, seed >> 32])
    u = [(x + 0.5) * 2.0 ** -32 for x in w]
    r0, r1 = math.sqrt(-2 * math.log(u[0])), math.sqrt(-2 * math.log(u[2]))
    return np.array([r0 * math.cos(2 * math.pi * u[1]), r0 * math.sin(2 * math.pi * u[1]),
                     r1 * math.cos(2 * math.pi * u[3]), r1 * math.sin(2 * math.pi * u[3])])


def test_injected_noise_and_orders_are_refused():
    spec = _one_step_spec(Solver.ExplicitStrong_1, 11)
    with pytest.raises(RuntimeError, match="code 6"):
        oracle.simulate(spec)
    spec = provider.with_injected_noise(_one_step_spec(Solver.WeakTest, 1))
    with pytest.raises(RuntimeError, match="code 5"):
        oracle.simulate(spec)
