"""Shards of one ensemble, run separately through the library and merged.

Each shard keeps its particles' global ids (particle_id_offset), so it draws the
same Philox increments as the whole ensemble; its un-normalised window sums
(sp_result.weighted_sum) and weights fold into the whole ensemble's result with
sp_merge_shards, the restatement of MeanSimulationResult::operator+= and
normalize (Particle_Simulation/Results/MeanSimulationResult.h:63-119).  Shard
cuts inside a warp change only how the FP64 partial sums are grouped, so the
merged mean equals the whole run within 1e-13 relative.
"""
import numpy as np
import pytest

import stochasticphysics_b200 as sp
from stochasticphysics_b200 import merge_shards, provider
from stochasticphysics_b200._abi import Precision, Solver
from stochasticphysics_b200.lib import load

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    # default launch shapes: one particle per thread for every shard size, so each
    # particle runs the same compiled step in the whole ensemble and in its shard
    load().sp_tuning_reset()
    c = sp.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("precision", [Precision.FP64, Precision.FP32])
def test_simulated_shards_merge_to_the_whole_ensemble(ctx, precision):
    spec = provider.brown_neel_relaxation(n=1000, steps=5000, oversampling=500, solver=Solver.Heun_Strong,
                                          precision=precision)
    whole = ctx.simulate(spec)
    np.testing.assert_allclose(whole.weighted_sum, whole.mean * whole.weight[None, :], rtol=1e-15)
    cuts = (0, 13, 300, 301, 777, 1000)  # inside warps, a one-particle shard
    parts = [ctx.simulate(spec.subset(lo, hi)) for lo, hi in zip(cuts[:-1], cuts[1:])]
    mean, total, weight = merge_shards([p.weighted_sum for p in parts], [p.weight for p in parts])
    np.testing.assert_allclose(mean, whole.mean, rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(total, whole.weighted_sum, rtol=1e-13, atol=1e-30)
    np.testing.assert_allclose(weight, whole.weight, rtol=1e-13)


def test_served_shards_merge_to_the_whole_ensemble(ctx):
    """The server returns the same sums: shards submitted together (batched into shared
    launches) merge to the whole ensemble run alone."""
    spec = provider.neel_relaxation(n=4096, steps=3000, oversampling=100, solver=Solver.Millstein)
    whole = ctx.simulate(spec)
    with ctx.server() as srv:
        ids = srv.submit_many([spec.subset(i * 1024, (i + 1) * 1024) for i in range(4)])
        parts = [srv.wait(i)[0] for i in ids]
    mean, _, weight = merge_shards([p.weighted_sum for p in parts], [p.weight for p in parts])
    np.testing.assert_allclose(mean, whole.mean, rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(weight, whole.weight, rtol=1e-13)
