"""The paired FP32 form: two Brown+Neel particles per thread in f32x2 arithmetic.

Thread t of a 128-particle tile integrates particles t and t + 64 with every add,
multiply and fused multiply-add shared between them (csrc/sp_kernels_x2.cuh).  A
particle's chart (the Euler and Neel coordinate rotations near a pole) is decided per
lane, so a particle's result may not depend on its partner: particles whose partners
are replaced, including by partners that sit near a pole and take the rotated charts,
keep their trajectories bit for bit.  Against the one-particle kernel the arithmetic
fuses differently, so the two agree to FP32 round-off.
"""
import dataclasses
import math

import numpy as np
import pytest

import stochasticphysics_b200 as sp
from stochasticphysics_b200 import provider
from stochasticphysics_b200._abi import Precision, Solver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = sp.Context(0)
    yield c
    c.close()


def shape(ppt):
    return {"block": 128, "persistent": 0, "chunk_steps": 1000, "particles_per_thread": ppt}


def run(ctx, spec, ppt):
    with ctx.ensemble(spec, shape=shape(ppt)) as e:
        e.advance(spec.integrated_steps)
        return e.read(trajectories=True)


@pytest.mark.parametrize("solver", [Solver.Millstein, Solver.Heun_Strong, Solver.EulerMaruyama,
                                    Solver.EulerMaruyama_Normalized])
def test_partner_does_not_change_a_particle(ctx, solver):
    base = dataclasses.replace(provider.brown_neel_relaxation(n=512, steps=3000, oversampling=100, solver=solver,
                                                              precision=Precision.FP32), record_trajectories=1)
    # lanes y of every tile (particles 64..127 of each 128) get other particles; half of
    # them start 2 degrees from a pole of both charts, so their steps take the rotated path
    idx = np.arange(base.n)
    partner = (idx % 128) >= 64
    rng = np.random.default_rng(12)
    e = np.array(base.orientation, copy=True)
    m = np.array(base.magnetisation, copy=True)
    e[partner] = provider.isotropic_euler(rng, int(partner.sum()))
    near = partner & (idx % 2 == 0)
    e[near, 1] = math.radians(2.0)
    m[near] = [math.sin(math.radians(1.5)), 0.0, math.cos(math.radians(1.5))]
    other = dataclasses.replace(base, orientation=e, magnetisation=m)
    a = run(ctx, base, 2)
    b = run(ctx, other, 2)
    np.testing.assert_array_equal(a.trajectories[~partner], b.trajectories[~partner])
    assert not np.array_equal(a.trajectories[partner], b.trajectories[partner])


@pytest.mark.parametrize("solver", [Solver.Millstein, Solver.Heun_Strong])
def test_paired_agrees_with_one_particle_per_thread(ctx, solver):
    """The first window to FP32 round-off (1e-5 per trajectory), and the ensemble mean
    of 16384 particles over 20 windows within 1e-3 of the one-particle kernel."""
    spec = dataclasses.replace(provider.brown_neel_relaxation(n=16384, steps=2100, oversampling=100, solver=solver,
                                                              precision=Precision.FP32), record_trajectories=1)
    one = run(ctx, spec, 1)
    two = run(ctx, spec, 2)
    np.testing.assert_allclose(two.trajectories[:, 1], one.trajectories[:, 1], rtol=0, atol=1e-5)
    assert np.abs(two.mean - one.mean).max() < 1e-3
    np.testing.assert_array_equal(two.weight, one.weight)


def test_paired_against_fp64(ctx):
    """Paired FP32 against the FP64 kernel on the same Philox noise: first window within
    1e-4 per trajectory."""
    spec = dataclasses.replace(provider.brown_neel_relaxation(n=4096, steps=1100, oversampling=100,
                                                              solver=Solver.Heun_Strong), record_trajectories=1)
    r64 = ctx.simulate(spec, trajectories=True)
    r32 = run(ctx, dataclasses.replace(spec, precision=Precision.FP32), 2)
    assert np.abs(r32.trajectories[:, 1] - r64.trajectories[:, 1]).max() < 1e-4
