"""sp_simulate_noalloc against sp_simulate, through the C ABI.

sp_simulate_noalloc serves hosts whose plug-ins may not allocate device memory
while they run (real-time control loops, hosts that pre-reserve and account all
GPU memory, sandboxes that forbid cudaMalloc after start-up): the caller hands
in device buffers it already owns, and the library works inside one static
32 MiB device array.  This file is collected last so a failure here cannot hide
the results of the other tests; it passes alone in a fresh process too.

Each call's ensemble mean must match sp_simulate's within the ensemble-mean
tolerance the parity tests use (1e-10 absolute); the weights within 1e-13
relative.  Consecutive calls with different ensembles check that whatever the
previous call left in the shared array does not leak into the next result.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import stochasticphysics_b200 as sp
from stochasticphysics_b200 import provider
from stochasticphysics_b200._abi import DescHolder, Precision, Solver, sp_particles
from stochasticphysics_b200.lib import load

pytestmark = pytest.mark.gpu

ABS_MEAN = 1e-10


def _dptr(t):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))


def _run_noalloc(spec, torch):
    holder = DescHolder(spec)
    dev = {k: torch.from_numpy(v).cuda() for k, v in holder.arrays.items() if v is not None}
    dp = sp_particles()
    for k, t in dev.items():
        setattr(dp, k, _dptr(t))
    _, _, od = spec.dims
    mean = torch.full((spec.n_samples, od), float("nan"), dtype=torch.float64, device="cuda")
    weight = torch.full((od,), float("nan"), dtype=torch.float64, device="cuda")
    rc = load().sp_simulate_noalloc(holder.byref(), C.byref(dp), _dptr(mean), _dptr(weight), None)
    assert rc == 0, load().sp_last_error().decode()
    torch.cuda.synchronize()
    return mean.cpu().numpy(), weight.cpu().numpy()


def test_noalloc_matches_simulate_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    first = provider.brown_neel_relaxation(n=3000, steps=12000, oversampling=1000, solver=Solver.Millstein,
                                           precision=Precision.FP32)
    second = provider.neel_relaxation(n=1500, steps=5000, oversampling=100, solver=Solver.Heun_Strong,
                                      precision=Precision.FP64)
    with sp.Context(0) as ctx:
        refs = [ctx.simulate(first), ctx.simulate(second)]
    for spec, ref in ((first, refs[0]), (second, refs[1]), (first, refs[0])):
        mean, weight = _run_noalloc(spec, torch)
        assert np.max(np.abs(mean - ref.mean)) <= ABS_MEAN
        np.testing.assert_allclose(weight, ref.weight, rtol=1e-13)


def test_noalloc_refuses_oversized_ensembles():
    pytest.importorskip("torch")
    spec = dataclasses.replace(provider.brown_neel_relaxation(n=400000, steps=3000, oversampling=1000))
    holder = DescHolder(spec)
    dp = sp_particles()
    dummy = C.cast(C.c_void_p(16), C.POINTER(C.c_double))  # never dereferenced: refused before any launch
    for k, _ in sp_particles._fields_:
        setattr(dp, k, dummy)
    rc = load().sp_simulate_noalloc(holder.byref(), C.byref(dp), dummy, dummy, None)
    assert rc == int(sp.Status.INVALID_ARG)
    msg = load().sp_last_error().decode()
    assert "bytes of scratch" in msg and str(32 << 20) in msg
