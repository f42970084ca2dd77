"""sp_merge_shards on the host: the shard merge of MeanSimulationResult::operator+=.

The reference adds every particle's weighted window means and its weight into
one MeanSimulationResult and normalize() divides the sums by the summed weight,
leaving them as they are when every weight is zero
(Particle_Simulation/Results/MeanSimulationResult.h:63-119).  The library's
merge does the same over whole shards, so shards of one ensemble, each
integrated separately with its global particle ids, merge into the result of
the whole ensemble.  No GPU: shard results come from the oracle.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import stochasticphysics_b200 as sp
from stochasticphysics_b200 import merge_shards, provider
from stochasticphysics_b200._abi import Problem, Solver
from stochasticphysics_b200.lib import load


def test_merge_adds_sums_and_weights_then_normalises():
    rng = np.random.default_rng(3)
    sums = [rng.standard_normal((7, 9)) for _ in range(3)]
    weights = [rng.uniform(1, 2, 9) for _ in range(3)]
    mean, total, w = merge_shards(sums, weights)
    np.testing.assert_array_equal(total, (sums[0] + sums[1]) + sums[2])
    np.testing.assert_array_equal(w, (weights[0] + weights[1]) + weights[2])
    np.testing.assert_array_equal(mean, total / w[None, :])


def test_all_zero_weights_leave_the_sums_unnormalised():
    sums = [np.ones((3, 3)), 2 * np.ones((3, 3))]
    mean, total, w = merge_shards(sums, [np.zeros(3), np.zeros(3)])
    np.testing.assert_array_equal(mean, 3 * np.ones((3, 3)))
    np.testing.assert_array_equal(w, np.zeros(3))


def test_merge_refuses_bad_arguments():
    lib = load()
    dp = C.POINTER(C.c_double)
    a = np.zeros((2, 3))
    w = np.zeros(3)
    arr = (dp * 1)(a.ctypes.data_as(dp))
    warr = (dp * 1)(w.ctypes.data_as(dp))
    assert lib.sp_merge_shards(0, 2, 3, arr, warr, None, None, None) == int(sp.Status.INVALID_ARG)
    assert lib.sp_merge_shards(1, 2, 0, arr, warr, None, None, None) == int(sp.Status.INVALID_ARG)
    assert lib.sp_merge_shards(1, 2, 3, None, warr, None, None, None) == int(sp.Status.INVALID_ARG)
    null = (dp * 1)()
    assert lib.sp_merge_shards(1, 2, 3, arr, null, None, None, None) == int(sp.Status.INVALID_ARG)
    assert b"shard 0" in lib.sp_last_error()
    with pytest.raises(ValueError):
        merge_shards([np.zeros((2, 3))], [np.zeros(2)])


@pytest.mark.parametrize("problem,cuts", [(Problem.Neel, (0, 37, 38, 100)),
                                          (Problem.BrownAndNeelEulerSpherical, (0, 50, 100))])
def test_uneven_oracle_shards_merge_to_the_whole(problem, cuts):
    if problem == Problem.Neel:
        spec = provider.neel_relaxation(n=100, steps=600, oversampling=100, solver=Solver.Heun_Strong)
    else:
        spec = provider.brown_neel_relaxation(n=100, steps=600, oversampling=100, solver=Solver.Millstein)
    whole = oracle.simulate(spec)
    parts = [oracle.simulate(spec.subset(lo, hi)) for lo, hi in zip(cuts[:-1], cuts[1:])]
    mean, _, w = merge_shards([p["mean"] * p["weight"] for p in parts], [p["weight"] for p in parts])
    np.testing.assert_allclose(mean, whole["mean"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(w, whole["weight"], rtol=1e-13)
