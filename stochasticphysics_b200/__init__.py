"""B200 engine for ensemble SDE integration of magnetic nanoparticles.

Drop-in for the per-particle simulation loop of Neumann-A/StochasticPhysics
(Neel, Neel-spherical and coupled Brown+Neel problems; uniaxial and cubic
anisotropy; zero, constant, sinusoidal and Lissajous fields; EulerMaruyama,
Heun, Millstein and ImplicitMidpoint steppers) behind the C ABI in
include/stophys_b200.h.
"""
from ._abi import (Anisotropy, DistSpec, Distribution, EnsembleSpec, FieldSpec, FieldType, Jacobian,  # noqa: F401
                   Noise, ParticleTemplateSpec, Precision, ProviderSpec,
                   Problem, RequestState, Solver, Status, DIMS)
from .lib import SPError, load  # noqa: F401
from .simulator import Context, DeviceEnsemble, Server, SimulationResult, kernel_launch_count, merge_shards  # noqa: F401

__all__ = ["Anisotropy", "DistSpec", "Distribution", "ParticleTemplateSpec", "ProviderSpec", "EnsembleSpec", "FieldSpec", "FieldType", "Jacobian", "Noise", "Precision", "Problem", "RequestState",
           "Solver", "Status", "DIMS", "SPError", "load", "Context", "DeviceEnsemble", "Server", "SimulationResult",
           "kernel_launch_count", "merge_shards"]
