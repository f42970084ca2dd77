"""Autotuner on the GPU: timings, cache, and launch-shape independence of results.

The ensemble mean is reduced per warp in a fixed order, so no launch shape
(CTA size, persistent grid, chunk length) may change a single bit of the result.
Two particles per thread (FP32) run each particle's steps through a separately
compiled kernel; the test states how close it is to one particle per thread.
"""
import dataclasses

import numpy as np
import pytest

import stochasticphysics_b200 as sp
from stochasticphysics_b200 import provider
from stochasticphysics_b200._abi import Precision, Solver
from stochasticphysics_b200.lib import SPError

pytestmark = pytest.mark.gpu


@pytest.fixture
def ctx():
    sp.Context.tuning_reset()
    c = sp.Context(0)
    yield c
    c.close()
    sp.Context.tuning_reset()


def test_autotune_picks_the_fastest_candidate(ctx):
    spec = provider.brown_neel_relaxation(n=65536, steps=200000, oversampling=1000, solver=Solver.Millstein,
                                          precision=Precision.FP32)
    out = ctx.autotune(spec, probe_particles=32768)
    best, cands = out["best"], out["candidates"]
    assert len(cands) >= 4
    assert all(c["particle_steps_per_s"] > 0 for c in cands)
    top = max(c["particle_steps_per_s"] for c in cands)
    assert best["particle_steps_per_s"] >= 0.98 * top
    # the winning shape keeps the shortest chunk within 2 % of the best rate
    shape = ("block", "persistent", "particles_per_thread")
    same = [c for c in cands if all(c[k] == best[k] for k in shape)]
    assert {c["chunk_steps"] for c in same} >= {1000, 2000, 10000, 40000}
    assert best["chunk_steps"] == min(c["chunk_steps"] for c in same if c["particle_steps_per_s"] >= 0.98 * top)
    used = ctx.launch_config(spec)
    assert (used["block"], used["persistent"], used["chunk_steps"]) == (best["block"], best["persistent"],
                                                                         best["chunk_steps"])


@pytest.mark.parametrize("shape", ["0/0/0/0/0 64 1 3000", "0/0/0/0/0 256 0 1000", "0/0/0/0/0 32 1 500"])
def test_results_do_not_depend_on_the_launch_shape(ctx, tmp_path, shape):
    spec = provider.neel_relaxation(n=5000, steps=6000, oversampling=100, solver=Solver.EulerMaruyama)
    key = f"{int(spec.problem)}/{int(spec.anisotropy)}/{int(spec.solver)}/{int(spec.precision)}/{int(spec.noise)}"
    assert key == "0/0/0/0/0"
    ref = ctx.simulate(spec)
    f = tmp_path / "shape.txt"
    f.write_text(shape + " 0\n")
    sp.Context.tuning_load(f)
    got = ctx.simulate(spec)
    block, persistent, chunk = (int(v) for v in shape.split()[1:4])
    used = ctx.launch_config(spec)
    assert (used["persistent"], used["chunk_steps"]) == (persistent, chunk)
    np.testing.assert_array_equal(got.mean, ref.mean)
    np.testing.assert_array_equal(got.weight, ref.weight)


@pytest.mark.parametrize("problem,solver,persistent", [("neel", Solver.Heun_Strong, 0), ("brown_neel", Solver.Millstein, 0),
                                                      ("brown_neel", Solver.Heun_Strong, 1),
                                                      ("neel", Solver.Implicit_Midpoint, 1)])
def test_two_particles_per_thread(ctx, tmp_path, problem, solver, persistent):
    """FP32 with two particles per thread against one: each particle runs the same source
    arithmetic in another instantiation, so the first window agrees to FP32 round-off
    (1e-5 per trajectory); afterwards a few particles near a saddle part as FP32 and FP64
    runs do, so the ensemble mean of the 20 windows is checked within 1e-3, and the
    autotuner may choose either shape."""
    make = provider.neel_relaxation if problem == "neel" else provider.brown_neel_relaxation
    spec = make(n=40000, steps=2100, oversampling=100, solver=solver, precision=Precision.FP32)
    key = f"{int(spec.problem)}/{int(spec.anisotropy)}/{int(spec.solver)}/1/0"
    f = tmp_path / "shape.txt"
    f.write_text(f"{key} 128 {persistent} 1000 0 1\n")
    sp.Context.tuning_load(f)
    one = ctx.simulate(spec, trajectories=True)
    assert ctx.launch_config(spec)["particles_per_thread"] == 1
    f.write_text(f"{key} 128 {persistent} 1000 0 2\n")
    sp.Context.tuning_load(f)
    assert ctx.launch_config(spec)["particles_per_thread"] == 2
    two = ctx.simulate(spec, trajectories=True)
    np.testing.assert_allclose(two.trajectories[:, :2], one.trajectories[:, :2], rtol=0, atol=1e-5)
    assert np.abs(two.mean - one.mean).max() < 1e-3
    np.testing.assert_array_equal(two.weight, one.weight)
    with sp.Server(ctx) as srv:  # the server's group launch takes the same shape
        res = srv.wait(srv.submit(spec))[0]
    np.testing.assert_allclose(res.mean, two.mean, rtol=0, atol=1e-6)


def test_tuned_shapes_reach_the_server(ctx, tmp_path):
    spec = provider.neel_relaxation(n=3000, steps=4000, oversampling=100, solver=Solver.Heun_Strong)
    ref = ctx.simulate(spec)
    f = tmp_path / "shape.txt"
    f.write_text("0/0/1/0/0 64 1 2000 0\n")
    sp.Context.tuning_load(f)
    other = dataclasses.replace(spec, seed=spec.seed + 1)
    with sp.Server(ctx) as srv:
        ids = [srv.submit(spec), srv.submit(other)]
        res = [srv.wait(i)[0] for i in ids]
    np.testing.assert_array_equal(res[0].mean, ref.mean)
    assert not np.array_equal(res[1].mean, ref.mean)


def test_shaped_ensemble_equals_the_tuned_one(ctx):
    """sp_ensemble_create_shaped: the caller's CTA size, grid form and chunk (rounded down
    to whole windows) change no bit of the result; invalid shapes are refused."""
    spec = provider.brown_neel_relaxation(n=5000, steps=8000, oversampling=1000, solver=Solver.Heun_Strong,
                                          precision=Precision.FP32)
    shape = {"block": 64, "persistent": 1, "chunk_steps": 1500, "particles_per_thread": 1}
    with ctx.ensemble(spec) as a, ctx.ensemble(spec, shape=shape) as b:
        for e in (a, b):
            e.advance(3000)
            e.advance(3000)
        ra, rb = a.read(), b.read()
    np.testing.assert_array_equal(rb.mean, ra.mean)
    np.testing.assert_array_equal(rb.weight, ra.weight)
    for bad in ({"block": 96}, {"persistent": 2}, {"chunk_steps": 0}, {"particles_per_thread": 3}):
        with pytest.raises(SPError, match="shape"):
            ctx.ensemble(spec, shape=dict(shape, **bad))
