"""Pregenerated noise: a small FP64 ensemble with in-kernel Philox noise draws each chunk's
increments in a separate kernel (the same Philox counters and arithmetic) and integrates
them with the injected step kernel.  The results must be bit-identical to the in-kernel
path, which the server always takes; the extra kernel shows in the launch count."""
import dataclasses
import math

import numpy as np
import pytest

import stochasticphysics_b200 as sp
from stochasticphysics_b200._abi import Anisotropy, Problem, Solver

from test_gpu_parity import small_spec

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = sp.Context(0)
    yield c
    c.close()


CASES = [
    (Problem.Neel, Solver.Heun_Strong),
    (Problem.Neel, Solver.EulerMaruyama),
    (Problem.NeelSpherical, Solver.Millstein),
    (Problem.BrownAndNeelEulerSpherical, Solver.Millstein),
    (Problem.BrownAndNeelEulerSpherical, Solver.Heun_Strong),
    (Problem.BrownAndNeel, Solver.Heun_Strong),
    (Problem.Neel, Solver.Implicit_Midpoint),
]


@pytest.mark.parametrize("problem,solver", CASES)
def test_pregenerated_noise_equals_in_kernel_noise(ctx, problem, solver):
    spec = small_spec(problem, solver, n=1000, steps=6000, W=200, seed=5)
    alone = ctx.simulate(spec)  # small FP64 ensemble: pregenerated noise
    with ctx.server() as srv:  # the server's groups draw in the kernel
        served = srv.wait(srv.submit(spec))[0]
    np.testing.assert_array_equal(alone.mean, served.mean)
    np.testing.assert_array_equal(alone.weight, served.weight)


@pytest.mark.parametrize("problem,aniso", [(Problem.Neel, Anisotropy.UniaxialCubic),
                                           (Problem.BrownAndNeelEulerSpherical, Anisotropy.Cubic)])
def test_pregenerated_noise_other_anisotropies(ctx, problem, aniso):
    if aniso == Anisotropy.UniaxialCubic:
        base = small_spec(problem, Solver.Heun_Strong, n=700, steps=3000, W=100, seed=9)
        rng = np.random.default_rng(9)
        spec = dataclasses.replace(base, anisotropy=Anisotropy.UniaxialCubic,
                                   anisotropy_constant=np.full(base.n, -8e3), cubic_constant=np.full(base.n, -4e3),
                                   uniaxial_rotation=rng.uniform(0, 2 * math.pi, (base.n, 3)))
    else:
        spec = small_spec(problem, Solver.Heun_Strong, aniso=aniso, n=700, steps=3000, W=100, seed=9)
    alone = ctx.simulate(spec)
    with ctx.server() as srv:
        served = srv.wait(srv.submit(spec))[0]
    np.testing.assert_array_equal(alone.mean, served.mean)


def test_pregenerated_noise_in_short_chunks(ctx):
    """30 000 Brown+Neel particles (6 increments each per step): the pregenerated chunk is
    cut to 185 steps to keep its buffer within 256 MB, so windows of 100 steps straddle the
    chunks; the result still equals the in-kernel path's."""
    spec = small_spec(Problem.BrownAndNeelEulerSpherical, Solver.Heun_Strong, n=30000, steps=1200, W=100, seed=8)
    alone = ctx.simulate(spec)
    with ctx.server() as srv:
        served = srv.wait(srv.submit(spec))[0]
    np.testing.assert_array_equal(alone.mean, served.mean)
    np.testing.assert_array_equal(alone.weight, served.weight)


def test_only_small_ensembles_pregenerate(ctx):
    """Up to eight warps per SM, two per scheduler (8 x 32 x SMs particles), the ensemble
    runs one noise launch more per chunk; above it draws in the kernel.  Same kernel key, so the
    same chunk length for both sizes."""
    sms = 148
    small = small_spec(Problem.Neel, Solver.Heun_Strong, n=1000, steps=4000, W=200, seed=6)
    large = small_spec(Problem.Neel, Solver.Heun_Strong, n=8 * 32 * sms + 32, steps=4000, W=200, seed=6)
    chunk = min(ctx.launch_config(small)["chunk_steps"], small.integrated_steps)
    chunks = -(-small.integrated_steps // chunk)
    a = ctx.simulate(small)
    b = ctx.simulate(large)
    assert a.stats["kernel_launches"] == b.stats["kernel_launches"] + chunks
