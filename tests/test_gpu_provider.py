"""Device-side provider on the GPU: the particles the kernel draws against the oracle's
restatement of the same draws, and a provided ensemble against the same particles
passed explicitly (alone and through the server)."""
import dataclasses

import numpy as np
import pytest

import oracle
import stochasticphysics_b200 as sp
from stochasticphysics_b200._abi import (Anisotropy, DistSpec, Distribution, ParticleTemplateSpec, Problem, ProviderSpec,
                                         Solver)
from test_provider_cpu import spec_for, tpl

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = sp.Context(0)
    yield c
    c.close()


TEMPLATES = [tpl(weight=2, random_orientation=True, random_magnetisation=True,
                 magnetic_radius_dist=DistSpec(Distribution.Lognormal, 0.1),
                 hydrodynamic_shell_dist=DistSpec(Distribution.Normal, 0.05),
                 anisotropy_dist=DistSpec(Distribution.Normal, 0.2)),
             tpl(weight=1, magnetic_radius=1.3e-8, magnetisation=(0.0, 0.6, 0.8), orientation=(0.3, 0.2, 0.1))]


@pytest.mark.parametrize("problem", [Problem.Neel, Problem.NeelSpherical, Problem.BrownAndNeelEulerSpherical,
                                     Problem.BrownAndNeel])
@pytest.mark.parametrize("sequential", [False, True])
def test_device_draws_match_the_oracle(ctx, problem, sequential):
    spec = spec_for(ProviderSpec(TEMPLATES, seed=11, sequential=sequential), 5000, problem=problem, offset=17)
    dev = ctx.provide_particles(spec)
    ref = oracle.provide_particles(spec)
    np.testing.assert_array_equal(dev[:, 17], ref[:, 17])  # template of every particle
    np.testing.assert_allclose(dev, ref, rtol=1e-13, atol=1e-15)


def test_uniaxial_cubic_draws(ctx):
    t = [tpl(cubic_constant=-5e3, cubic_dist=DistSpec(Distribution.Normal, 0.1), random_uniaxial_rotation=True,
             random_magnetisation=True)]
    spec = spec_for(ProviderSpec(t, seed=12), 3000, problem=Problem.BrownAndNeelEulerSpherical,
                    aniso=Anisotropy.UniaxialCubic)
    np.testing.assert_allclose(ctx.provide_particles(spec), oracle.provide_particles(spec), rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize("problem", [Problem.Neel, Problem.BrownAndNeelEulerSpherical])
def test_provided_ensemble_equals_explicit_particles(ctx, problem):
    spec = dataclasses.replace(spec_for(ProviderSpec(TEMPLATES, seed=13), 4096, problem=problem),
                               number_of_steps=3000, oversampling=500)
    p = ctx.provide_particles(spec)
    explicit = dataclasses.replace(spec, provider=None, magnetic_radius=p[:, 0], saturation_magnetisation=p[:, 1],
                                   damping_constant=p[:, 2], gyromagnetic_ratio=p[:, 3], anisotropy_constant=p[:, 4],
                                   hydrodynamic_radius=p[:, 5], viscosity=p[:, 6], orientation=p[:, 7:10],
                                   magnetisation=p[:, 10:13])
    a = ctx.simulate(spec)
    b = ctx.simulate(explicit)
    np.testing.assert_array_equal(a.mean, b.mean)
    np.testing.assert_array_equal(a.weight, b.weight)
    with sp.Server(ctx) as srv:
        rid = srv.submit(spec)
        c, _ = srv.wait(rid)
    np.testing.assert_array_equal(c.mean, a.mean)
