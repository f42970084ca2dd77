"""Server life cycle on the GPU: admission refusal, queueing behind max_active, wait
timeouts, cancellation while queued and while running, and results handed over once."""
import dataclasses

import numpy as np
import pytest

import stochasticphysics_b200 as sp
from stochasticphysics_b200 import provider
from stochasticphysics_b200._abi import RequestState, Solver, Status

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = sp.Context(0)
    yield c
    c.close()


def small(n=2000, steps=4000, seed=1):
    return provider.neel_relaxation(n=n, steps=steps, oversampling=100, solver=Solver.Heun_Strong, seed=seed)


def test_admission_refused_when_the_request_exceeds_the_budget(ctx):
    with sp.Server(ctx, memory_budget_bytes=1 << 20) as srv:
        with pytest.raises(sp.SPError) as e:
            srv.submit(small(n=200000))
        assert e.value.status == Status.ADMISSION_REFUSED


def test_wait_timeout_then_result_once(ctx):
    long = small(n=65536, steps=200000)
    with sp.Server(ctx) as srv:
        rid = srv.submit(long)
        with pytest.raises(sp.SPError) as e:
            srv.wait(rid, timeout_ms=1.0)
        assert e.value.status == Status.NOT_READY
        res, lat = srv.wait(rid)
        assert lat > 0 and res.mean.shape == (long.n_samples, 3)
        assert res.stats["particle_steps"] == long.n * long.integrated_steps
        with pytest.raises(sp.SPError) as e2:
            srv.wait(rid)
        assert e2.value.status == Status.NOT_FOUND


def test_queue_behind_max_active_and_cancel(ctx):
    with sp.Server(ctx, max_active=1) as srv:
        first = srv.submit(small(n=65536, steps=300000, seed=2))
        queued = srv.submit(small(seed=3))
        assert srv.poll(queued) == RequestState.QUEUED
        srv.cancel(queued)
        with pytest.raises(sp.SPError) as e:
            srv.wait(queued)
        assert e.value.status == Status.CANCELLED
        assert srv.poll(first) in (RequestState.QUEUED, RequestState.RUNNING)
        srv.cancel(first)
        with pytest.raises(sp.SPError) as e2:
            srv.wait(first)
        assert e2.value.status == Status.CANCELLED
        # the server keeps serving after cancellations
        spec = small(seed=4)
        done = srv.submit(spec)
        res, _ = srv.wait(done)
        np.testing.assert_array_equal(res.mean, ctx.simulate(spec).mean)


def test_many_requests_release_their_memory(ctx):
    """Host copies are dropped at admission and results at hand-over, so a long
    stream of requests does not accumulate state in the server."""
    with sp.Server(ctx) as srv:
        for k in range(3):
            ids = [srv.submit(small(n=1000, steps=1000, seed=10 * k + j)) for j in range(20)]
            for i in ids:
                srv.wait(i)
            for i in ids:
                with pytest.raises(sp.SPError):
                    srv.poll(i)


def test_submit_many_queues_all_or_nothing(ctx):
    """sp_server_submit_many: every result equals its own sp_simulate; a refused
    description (here over the budget) queues none and names its index."""
    specs = [small(n=3000, steps=6000, seed=21), small(n=5000, steps=3000, seed=22),
             provider.brown_neel_relaxation(n=2000, steps=5000, oversampling=1000, solver=Solver.Millstein, seed=23)]
    with sp.Server(ctx) as srv:
        ids = srv.submit_many(specs)
        assert len(set(ids)) == 3
        for rid, spec in zip(ids, specs):
            np.testing.assert_array_equal(srv.wait(rid)[0].mean, ctx.simulate(spec).mean)
    with sp.Server(ctx, memory_budget_bytes=1 << 20) as srv:
        with pytest.raises(sp.SPError, match="request 1") as e:
            srv.submit_many([small(n=100), small(n=200000)])
        assert e.value.status == Status.ADMISSION_REFUSED


@pytest.mark.parametrize("groups_per_kind", [1, 2, 3])
def test_groups_per_kind_leave_results_unchanged(ctx, groups_per_kind):
    """Requests of one kind arriving while that kind's group is mid-round either start a
    group of their own or join a running one at its next round (sp_server_config.
    groups_per_kind); each result is bit-identical to the request run alone."""
    import time
    specs = [small(n=3000 + 500 * i, steps=40000, seed=10 + i) for i in range(4)]
    with sp.Server(ctx, chunk_steps=2000, groups_per_kind=groups_per_kind) as srv:
        ids = []
        for s in specs:
            ids.append(srv.submit(s))
            time.sleep(0.003)  # the earlier requests' groups are mid-round
        got = [srv.wait(i)[0] for i in ids]
    for s, r in zip(specs, got):
        np.testing.assert_array_equal(r.mean, ctx.simulate(s).mean)
        np.testing.assert_array_equal(r.weight, ctx.simulate(s).weight)


def test_negative_groups_per_kind_is_refused(ctx):
    with pytest.raises(sp.SPError) as ei:
        sp.Server(ctx, groups_per_kind=-1)
    assert ei.value.status == Status.INVALID_ARG
