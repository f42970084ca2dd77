"""Device-side provider restated in the oracle (CPU): template selection, the size and
anisotropy distributions, the random initial states of each problem, determinism and
shard consistency, and that a provided ensemble simulates like the same particles
passed explicitly."""
import dataclasses
import math

import numpy as np
import pytest

import oracle
from stochasticphysics_b200 import provider
from stochasticphysics_b200._abi import (Anisotropy, DistSpec, Distribution, EnsembleSpec, ParticleTemplateSpec, Problem,
                                         ProviderSpec, Solver)

R, MS, ALPHA, GAMMA = 1e-8, 4.8e5, 0.1, 1.76e11


def tpl(**kw):
    base = dict(magnetic_radius=R, saturation_magnetisation=MS, damping_constant=ALPHA, gyromagnetic_ratio=GAMMA,
                anisotropy_constant=-1e4, hydrodynamic_radius=3e-8, viscosity=1e-3)
    base.update(kw)
    return ParticleTemplateSpec(**base)


def spec_for(prov, n, problem=Problem.Neel, aniso=Anisotropy.Uniaxial, offset=0):
    return EnsembleSpec(problem=problem, n=n, magnetic_radius=None, saturation_magnetisation=None,
                        damping_constant=None, gyromagnetic_ratio=None, anisotropy_constant=None, orientation=None,
                        magnetisation=None, number_of_steps=300, oversampling=100, timestep=1e-11,
                        anisotropy=aniso, provider=prov, particle_id_offset=offset, solver=Solver.Heun_Strong)


def test_sequential_selection_fills_counts_then_uses_the_first():
    prov = ProviderSpec([tpl(weight=3), tpl(weight=5, magnetic_radius=2e-8)], seed=1, sequential=True)
    p = oracle.provide_particles(spec_for(prov, 12))
    np.testing.assert_array_equal(p[:, 17], [0, 0, 0, 1, 1, 1, 1, 1, 0, 0, 0, 0])
    np.testing.assert_array_equal(p[:, 0], np.where(p[:, 17] == 1, 2e-8, R))
    # shards keep the global particle index: particles 5..11 alone give rows 5..11
    q = oracle.provide_particles(spec_for(prov, 7, offset=5))
    np.testing.assert_array_equal(q, p[5:])


def test_discrete_selection_follows_weights():
    prov = ProviderSpec([tpl(weight=1), tpl(weight=3)], seed=2)
    p = oracle.provide_particles(spec_for(prov, 20000))
    share = (p[:, 17] == 1).mean()
    assert abs(share - 0.75) < 4 * math.sqrt(0.75 * 0.25 / 20000)


def test_distributions():
    t = tpl(magnetic_radius_dist=DistSpec(Distribution.Lognormal, 0.1),
            hydrodynamic_shell_dist=DistSpec(Distribution.Normal, 0.05),
            anisotropy_dist=DistSpec(Distribution.Normal, 2000.0, relative=False))
    p = oracle.provide_particles(spec_for(ProviderSpec([t], seed=3), 40000))
    n = len(p)
    r, K, rh = p[:, 0], p[:, 4], p[:, 5]
    x = r / R
    assert abs(x.mean() - 1) < 4 * 0.1 / math.sqrt(n) and abs(x.std() / 0.1 - 1) < 0.03 and (x > 0).all()
    shell = (rh - r) / (3e-8 - r)
    assert abs(shell.mean() - 1) < 4 * 0.05 / math.sqrt(n) and abs(shell.std() / 0.05 - 1) < 0.03
    assert abs(K.mean() + 1e4) < 4 * 2000 / math.sqrt(n) and abs(K.std() / 2000 - 1) < 0.03
    np.testing.assert_array_equal(p[:, 1], MS)


@pytest.mark.parametrize("problem", [Problem.Neel, Problem.NeelSpherical, Problem.BrownAndNeelEulerSpherical,
                                     Problem.BrownAndNeel])
def test_random_initial_states_follow_each_problem(problem):
    t = tpl(random_orientation=True, random_magnetisation=True)
    p = oracle.provide_particles(spec_for(ProviderSpec([t], seed=4), 30000, problem=problem))
    e, m = p[:, 7:10], p[:, 10:13]
    n = len(p)
    np.testing.assert_allclose(np.linalg.norm(m, axis=1), 1.0, rtol=1e-14)
    if problem in (Problem.Neel, Problem.BrownAndNeel):  # N(0,1)^3 normalised: uniform on the sphere
        assert np.all(np.abs((m ** 2).mean(axis=0) - 1 / 3) < 4 * math.sqrt(4 / 45 / n))
    else:  # theta uniform in [0, pi)
        th = np.arccos(np.clip(m[:, 2], -1, 1))
        assert abs(th.mean() - math.pi / 2) < 4 * math.pi / math.sqrt(12 * n)
    if problem == Problem.Neel:
        assert e.min() >= 0 and e.max() < 2 * math.pi and e[:, 1].max() > 1.9 * math.pi
    elif problem == Problem.BrownAndNeel:
        a, b, g = e[:, 0], e[:, 1], e[:, 2]
        axis = np.stack([np.cos(a) * np.cos(g) - np.sin(a) * np.cos(b) * np.sin(g),
                         -np.cos(a) * np.sin(g) - np.sin(a) * np.cos(b) * np.cos(g), np.sin(a) * np.sin(b)], axis=1)
        np.testing.assert_allclose(np.linalg.norm(axis, axis=1), 1.0, rtol=1e-12)
        assert np.all(np.abs((axis ** 2).mean(axis=0) - 1 / 3) < 4 * math.sqrt(4 / 45 / n))
    else:
        assert e[:, 1].max() < math.pi and e[:, 0].max() > 1.9 * math.pi


def test_uniaxial_cubic_templates():
    t = tpl(cubic_constant=-5e3, cubic_dist=DistSpec(Distribution.Normal, 0.1), random_uniaxial_rotation=True)
    p = oracle.provide_particles(spec_for(ProviderSpec([t], seed=5), 5000, aniso=Anisotropy.UniaxialCubic))
    kc = p[:, 13] / -5e3
    assert abs(kc.mean() - 1) < 4 * 0.1 / math.sqrt(len(p))
    assert p[:, 14].max() > 1.9 * math.pi and p[:, 15].max() < math.pi
    fixed = oracle.provide_particles(spec_for(ProviderSpec([tpl(uniaxial_rotation=(0.1, 0.2, 0.3))], seed=5), 4,
                                              aniso=Anisotropy.UniaxialCubic))
    np.testing.assert_array_equal(fixed[:, 14:17], [[0.1, 0.2, 0.3]] * 4)


def test_seed_and_provided_simulation_equal_explicit_particles():
    t = tpl(random_orientation=True, random_magnetisation=True, magnetic_radius_dist=DistSpec(Distribution.Lognormal, 0.1))
    a = oracle.provide_particles(spec_for(ProviderSpec([t], seed=7), 64))
    b = oracle.provide_particles(spec_for(ProviderSpec([t], seed=7), 64))
    c = oracle.provide_particles(spec_for(ProviderSpec([t], seed=8), 64))
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, c)
    spec = provider.with_injected_noise(spec_for(ProviderSpec([t], seed=7), 64), seed=1)
    explicit = dataclasses.replace(spec, provider=None, magnetic_radius=a[:, 0], saturation_magnetisation=a[:, 1],
                                   damping_constant=a[:, 2], gyromagnetic_ratio=a[:, 3], anisotropy_constant=a[:, 4],
                                   orientation=a[:, 7:10], magnetisation=a[:, 10:13])
    np.testing.assert_array_equal(oracle.simulate(spec)["mean"], oracle.simulate(explicit)["mean"])
