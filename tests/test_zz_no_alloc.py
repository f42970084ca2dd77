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
import math

import numpy as np
import pytest

import stochasticphysics_b200 as sp
from stochasticphysics_b200 import provider
from stochasticphysics_b200._abi import Anisotropy, DescHolder, Precision, Problem, Solver, sp_particles
from stochasticphysics_b200.lib import load

pytestmark = pytest.mark.gpu

ABS_MEAN = 1e-10


def _dptr(t):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))


def _run_noalloc(spec, torch, stream=None):
    """One sp_simulate_noalloc call; `stream` (a torch.cuda.Stream) orders every copy and
    launch of the call, and the inputs are made on it so nothing runs ahead of them."""
    holder = DescHolder(spec)
    if stream is not None:
        with torch.cuda.stream(stream):
            return _run_noalloc_on(holder, spec, torch, stream)
    return _run_noalloc_on(holder, spec, torch, None)


def _run_noalloc_on(holder, spec, torch, stream):
    dev = {k: torch.from_numpy(v).cuda() for k, v in holder.arrays.items() if v is not None}
    dp = sp_particles()
    for k, t in dev.items():
        setattr(dp, k, _dptr(t))
    _, _, od = spec.dims
    mean = torch.full((spec.n_samples, od), float("nan"), dtype=torch.float64, device="cuda")
    weight = torch.full((od,), float("nan"), dtype=torch.float64, device="cuda")
    handle = None if stream is None else C.c_void_p(stream.cuda_stream)
    rc = load().sp_simulate_noalloc(holder.byref(), C.byref(dp), _dptr(mean), _dptr(weight), handle)
    assert rc == 0, load().sp_last_error().decode()
    if stream is not None:
        stream.synchronize()
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


def _uniaxial_cubic(spec):
    rng = np.random.default_rng(8)
    return dataclasses.replace(spec, anisotropy=Anisotropy.UniaxialCubic, anisotropy_constant=np.full(spec.n, -8e3),
                               cubic_constant=np.full(spec.n, -4e3),
                               uniaxial_rotation=rng.uniform(0, 2 * math.pi, (spec.n, 3)))


def _neel_spherical(spec):
    return dataclasses.replace(spec, problem=Problem.NeelSpherical, use_coordinate_transformation=True,
                               min_angle_before_transformation=math.pi / 36)


PATHS = {
    # the caller's K_cubic and uniaxial rotation arrays reach the kernels as device pointers
    "neel-uniaxial-cubic-fp64": lambda: _uniaxial_cubic(
        provider.neel_relaxation(n=700, steps=3000, oversampling=100, solver=Solver.Heun_Strong)),
    "brown-neel-euler-uniaxial-cubic-fp32": lambda: _uniaxial_cubic(
        provider.brown_neel_relaxation(n=900, steps=4000, oversampling=500, solver=Solver.Heun_Strong,
                                       precision=Precision.FP32)),
    # the spherical problems' rotation settings are copied into the descriptor by hand
    "neel-spherical-fp64": lambda: _neel_spherical(
        provider.neel_relaxation(n=800, steps=3000, oversampling=100, solver=Solver.EulerMaruyama)),
    "brown-neel-euler-fp64": lambda: provider.brown_neel_relaxation(n=600, steps=3000, oversampling=300,
                                                                    solver=Solver.Millstein),
}


@pytest.mark.parametrize("name", list(PATHS))
def test_noalloc_matches_simulate_per_path(name):
    torch = pytest.importorskip("torch")
    spec = PATHS[name]()
    with sp.Context(0) as ctx:
        ref = ctx.simulate(spec)
    mean, weight = _run_noalloc(spec, torch)
    assert np.max(np.abs(mean - ref.mean)) <= ABS_MEAN
    np.testing.assert_allclose(weight, ref.weight, rtol=1e-13)


def test_noalloc_on_a_caller_stream_twice():
    """Every clear, the descriptor write and every launch go to the caller's stream: two
    calls in a row on a non-default stream, each read only after that stream completes."""
    torch = pytest.importorskip("torch")
    spec = provider.neel_relaxation(n=2000, steps=4000, oversampling=100, solver=Solver.Millstein,
                                    precision=Precision.FP32)
    with sp.Context(0) as ctx:
        ref = ctx.simulate(spec)
    st = torch.cuda.Stream()
    for _ in range(2):
        mean, weight = _run_noalloc(spec, torch, stream=st)
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
