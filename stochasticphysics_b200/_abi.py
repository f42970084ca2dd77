"""ctypes mirror of include/stophys_b200.h.

Plain data only: structures, enums and a builder that turns numpy arrays into
an ``sp_ensemble_desc`` whose pointers stay valid while the returned object
lives.  Loading the shared library happens in :mod:`stochasticphysics_b200.lib`.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from enum import IntEnum
from typing import Optional

import numpy as np

ABI_VERSION = 9


class Status(IntEnum):
    OK = 0
    INVALID_ARG = 1
    UNSUPPORTED_COMBO = 2
    OUT_OF_MEMORY = 3
    ADMISSION_REFUSED = 4
    DEVICE_TIMEOUT = 5
    NUMERIC_FAULT = 6
    CUDA = 7
    NOT_READY = 8
    NOT_FOUND = 9
    CANCELLED = 10
    NO_DEVICE = 11


class Problem(IntEnum):
    """Reference problem names (Particle_Simulation/Problems/Problems.h:6-9)."""
    Neel = 0
    NeelSpherical = 1
    BrownAndNeelEulerSpherical = 2
    BrownAndNeel = 3


class Anisotropy(IntEnum):
    Uniaxial = 0
    Cubic = 1
    UniaxialCubic = 2


class FieldType(IntEnum):
    Zero = 0
    Constant = 1
    Sinusoidal = 2
    Lissajous = 3
    Triangular = 4
    Rectangular = 5
    Sinc = 6


class Solver(IntEnum):
    EulerMaruyama = 0
    Heun_Strong = 1
    Millstein = 2
    Implicit_Midpoint = 3
    EulerMaruyama_Normalized = 4
    # switched off in the reference's manager (SimulationManager.h:325-328); in-kernel noise only
    Heun_NotConsistent = 5
    WeakTest = 6
    ExplicitStrong_1 = 7


class Precision(IntEnum):
    FP64 = 0
    FP32 = 1


class Noise(IntEnum):
    Philox = 0
    Injected = 1


class Jacobian(IntEnum):
    Reference = 0
    Exact = 1


class RequestState(IntEnum):
    QUEUED = 0
    RUNNING = 1
    DONE = 2
    FAILED = 3
    CANCELLED = 4


# (state_dim, noise_dim, out_dim) per problem
DIMS = {
    Problem.Neel: (3, 3, 3),
    Problem.NeelSpherical: (2, 3, 3),
    Problem.BrownAndNeelEulerSpherical: (5, 6, 9),
    Problem.BrownAndNeel: (6, 6, 6),
}

_dp = C.POINTER(C.c_double)


class sp_particles(C.Structure):
    _fields_ = [
        ("magnetic_radius", _dp),
        ("saturation_magnetisation", _dp),
        ("damping_constant", _dp),
        ("gyromagnetic_ratio", _dp),
        ("anisotropy_constant", _dp),
        ("hydrodynamic_radius", _dp),
        ("viscosity", _dp),
        ("orientation", _dp),
        ("magnetisation", _dp),
        ("cubic_constant", _dp),
        ("uniaxial_rotation", _dp),
    ]


class sp_field_desc(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("alternating", C.c_int32),
        ("offset", C.c_double * 3),
        ("amplitude", C.c_double * 3),
        ("frequency", C.c_double * 3),
        ("phase", C.c_double * 3),
        ("periode", C.c_double),
        ("time_offset", C.c_double),
        ("tau", C.c_double),
    ]


class sp_problem_settings(C.Structure):
    _fields_ = [
        ("use_coordinate_transformation", C.c_int32),
        ("use_euler_coordinate_transformation", C.c_int32),
        ("use_spherical_coordinate_transformation", C.c_int32),
        ("use_simple_model", C.c_int32),
        ("min_angle_before_transformation", C.c_double),
        ("brown_min_angle_before_transformation", C.c_double),
        ("neel_min_angle_before_transformation", C.c_double),
    ]


class sp_dist(C.Structure):
    _fields_ = [("type", C.c_int32), ("relative", C.c_int32), ("width", C.c_double)]


class sp_particle_template(C.Structure):
    _fields_ = [
        ("weight", C.c_double),
        ("magnetic_radius", C.c_double), ("saturation_magnetisation", C.c_double),
        ("damping_constant", C.c_double), ("gyromagnetic_ratio", C.c_double),
        ("anisotropy_constant", C.c_double), ("hydrodynamic_radius", C.c_double), ("viscosity", C.c_double),
        ("cubic_constant", C.c_double),
        ("orientation", C.c_double * 3), ("magnetisation", C.c_double * 3), ("uniaxial_rotation", C.c_double * 3),
        ("random_orientation", C.c_int32), ("random_magnetisation", C.c_int32),
        ("random_uniaxial_rotation", C.c_int32), ("reserved", C.c_int32),
        ("magnetic_radius_dist", sp_dist), ("hydrodynamic_shell_dist", sp_dist),
        ("anisotropy_dist", sp_dist), ("cubic_dist", sp_dist),
    ]


class sp_provider_desc(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("n_templates", C.c_int32), ("sequential", C.c_int32),
                ("templates", C.POINTER(sp_particle_template))]


class sp_ensemble_desc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("problem", C.c_int32),
        ("anisotropy", C.c_int32),
        ("solver", C.c_int32),
        ("precision", C.c_int32),
        ("noise", C.c_int32),
        ("problem_settings", sp_problem_settings),
        ("max_iteration", C.c_int32),
        ("record_trajectories", C.c_int32),
        ("jacobian", C.c_int32),
        ("double_noise_approx", C.c_int32),
        ("accuracy_goal", C.c_double),
        ("number_of_steps", C.c_uint64),
        ("oversampling", C.c_uint64),
        ("timestep", C.c_double),
        ("temperature", C.c_double),
        ("field", sp_field_desc),
        ("n_particles", C.c_uint64),
        ("particles", sp_particles),
        ("seed", C.c_uint64),
        ("particle_id_offset", C.c_uint64),
        ("injected_dw", _dp),
        ("provider", C.POINTER(sp_provider_desc)),
    ]


class sp_result(C.Structure):
    _fields_ = [
        ("mean", _dp),
        ("weight", _dp),
        ("time", _dp),
        ("field", _dp),
        ("trajectories", _dp),
        ("final_state", _dp),
        ("weighted_sum", _dp),
    ]


class sp_stats(C.Structure):
    _fields_ = [
        ("particle_steps", C.c_uint64),
        ("nonfinite_particles", C.c_uint64),
        ("newton_iterations", C.c_uint64),
        ("newton_unconverged", C.c_uint64),
        ("kernel_launches", C.c_uint64),
        ("device_ms", C.c_double),
        ("queue_ms", C.c_double),
        ("setup_ms", C.c_double),
        ("run_ms", C.c_double),
        ("readback_ms", C.c_double),
    ]


class sp_launch_config(C.Structure):
    _fields_ = [
        ("block", C.c_int32),
        ("persistent", C.c_int32),
        ("chunk_steps", C.c_uint64),
        ("particle_steps_per_s", C.c_double),
        ("particles_per_thread", C.c_int32),
        ("reserved0", C.c_int32),
    ]

    def to_dict(self) -> dict:
        return {"block": int(self.block), "persistent": int(self.persistent), "chunk_steps": int(self.chunk_steps),
                "particles_per_thread": int(self.particles_per_thread),
                "particle_steps_per_s": float(self.particle_steps_per_s)}


class sp_server_config(C.Structure):
    _fields_ = [
        ("memory_budget_bytes", C.c_uint64),
        ("chunk_steps", C.c_uint64),
        ("max_active", C.c_int32),
        ("groups_per_kind", C.c_int32),
    ]


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def _f64(a, n: Optional[int] = None, shape=None) -> np.ndarray:
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if n is not None and arr.ndim == 0:
        arr = np.full(n, float(arr), dtype=np.float64)
    if shape is not None:
        arr = np.ascontiguousarray(arr.reshape(shape))
    return arr


@dataclass
class FieldSpec:
    """External field B(t) in tesla (Properties/Fields/{Sinusoidal,Lissajous}.hpp)."""
    type: FieldType = FieldType.Zero
    offset: tuple = (0.0, 0.0, 0.0)
    amplitude: tuple = (0.0, 0.0, 0.0)
    frequency: tuple = (0.0, 0.0, 0.0)
    phase: tuple = (0.0, 0.0, 0.0)
    periode: float = 0.0       # triangular / rectangular / sinc
    time_offset: float = 0.0   # triangular / rectangular
    tau: float = 0.0           # rectangular
    alternating: bool = False  # rectangular

    @staticmethod
    def sinusoidal(amplitude, frequency, phase=0.0, offset=(0.0, 0.0, 0.0)) -> "FieldSpec":
        return FieldSpec(FieldType.Sinusoidal, tuple(offset), tuple(amplitude), (frequency, 0.0, 0.0), (phase, 0.0, 0.0))

    @staticmethod
    def lissajous(amplitude, frequencies, phases=(0.0, 0.0, 0.0), offset=(0.0, 0.0, 0.0)) -> "FieldSpec":
        return FieldSpec(FieldType.Lissajous, tuple(offset), tuple(amplitude), tuple(frequencies), tuple(phases))

    @staticmethod
    def constant(offset) -> "FieldSpec":
        return FieldSpec(FieldType.Constant, tuple(offset))

    @staticmethod
    def triangular(amplitude, periode, time_offset=0.0, offset=(0.0, 0.0, 0.0)) -> "FieldSpec":
        return FieldSpec(FieldType.Triangular, tuple(offset), tuple(amplitude), periode=periode, time_offset=time_offset)

    @staticmethod
    def rectangular(amplitude, periode, tau, time_offset=0.0, alternating=False, offset=(0.0, 0.0, 0.0)) -> "FieldSpec":
        return FieldSpec(FieldType.Rectangular, tuple(offset), tuple(amplitude), periode=periode,
                         time_offset=time_offset, tau=tau, alternating=alternating)

    @staticmethod
    def sinc(amplitude, periode, offset=(0.0, 0.0, 0.0)) -> "FieldSpec":
        return FieldSpec(FieldType.Sinc, tuple(offset), tuple(amplitude), periode=periode)

    def to_c(self) -> sp_field_desc:
        f = sp_field_desc()
        f.type = int(self.type)
        for i in range(3):
            f.offset[i] = float(self.offset[i])
            f.amplitude[i] = float(self.amplitude[i])
            f.frequency[i] = float(self.frequency[i])
            f.phase[i] = float(self.phase[i])
        f.periode = float(self.periode)
        f.time_offset = float(self.time_offset)
        f.tau = float(self.tau)
        f.alternating = int(bool(self.alternating))
        return f


class Distribution(IntEnum):
    Delta = 0
    Normal = 1
    Lognormal = 2


@dataclass
class DistSpec:
    """One size or anisotropy distribution (ParticleSimulationSettings.h:62-101)."""
    type: Distribution = Distribution.Delta
    width: float = 0.0
    relative: bool = True

    def to_c(self) -> sp_dist:
        return sp_dist(int(self.type), int(bool(self.relative)), float(self.width))


@dataclass
class ParticleTemplateSpec:
    """One particle template of the device-side provider (a Particle_List entry)."""
    magnetic_radius: float
    saturation_magnetisation: float
    damping_constant: float
    gyromagnetic_ratio: float
    anisotropy_constant: float
    weight: float = 1.0
    hydrodynamic_radius: float = 0.0
    viscosity: float = 0.0
    cubic_constant: float = 0.0
    orientation: tuple = (0.0, 0.0, 0.0)
    magnetisation: tuple = (0.0, 0.0, 1.0)
    uniaxial_rotation: tuple = (0.0, 0.0, 0.0)
    random_orientation: bool = False
    random_magnetisation: bool = False
    random_uniaxial_rotation: bool = False
    magnetic_radius_dist: DistSpec = field(default_factory=DistSpec)
    hydrodynamic_shell_dist: DistSpec = field(default_factory=DistSpec)
    anisotropy_dist: DistSpec = field(default_factory=DistSpec)
    cubic_dist: DistSpec = field(default_factory=DistSpec)

    def to_c(self) -> sp_particle_template:
        t = sp_particle_template()
        for k in ("weight", "magnetic_radius", "saturation_magnetisation", "damping_constant", "gyromagnetic_ratio",
                  "anisotropy_constant", "hydrodynamic_radius", "viscosity", "cubic_constant"):
            setattr(t, k, float(getattr(self, k)))
        for k in ("orientation", "magnetisation", "uniaxial_rotation"):
            v = getattr(self, k)
            for i in range(3):
                getattr(t, k)[i] = float(v[i])
        for k in ("random_orientation", "random_magnetisation", "random_uniaxial_rotation"):
            setattr(t, k, int(bool(getattr(self, k))))
        for k in ("magnetic_radius_dist", "hydrodynamic_shell_dist", "anisotropy_dist", "cubic_dist"):
            setattr(t, k, getattr(self, k).to_c())
        return t


@dataclass
class ProviderSpec:
    """Device-side provider: particles drawn on the GPU from these templates."""
    templates: list
    seed: int = 0
    sequential: bool = False


@dataclass
class EnsembleSpec:
    """Everything one ensemble simulation needs; mirrors sp_ensemble_desc.

    Per-particle properties are arrays of length ``n`` (scalars broadcast);
    ``orientation`` holds ZXZ Euler angles (n, 3), ``magnetisation`` the
    initial magnetisation directions (n, 3).
    """
    problem: Problem
    n: int
    magnetic_radius: np.ndarray
    saturation_magnetisation: np.ndarray
    damping_constant: np.ndarray
    gyromagnetic_ratio: np.ndarray
    anisotropy_constant: np.ndarray
    orientation: np.ndarray
    magnetisation: np.ndarray
    number_of_steps: int
    oversampling: int
    timestep: float
    temperature: float = 295.0
    hydrodynamic_radius: Optional[np.ndarray] = None
    viscosity: Optional[np.ndarray] = None
    anisotropy: Anisotropy = Anisotropy.Uniaxial
    solver: Solver = Solver.Heun_Strong
    precision: Precision = Precision.FP64
    noise: Noise = Noise.Philox
    field: FieldSpec = field(default_factory=FieldSpec)
    seed: int = 0
    particle_id_offset: int = 0
    max_iteration: int = 20
    accuracy_goal: float = 1e-10
    use_coordinate_transformation: bool = False
    min_angle_before_transformation: float = 0.0
    use_euler_coordinate_transformation: bool = False
    brown_min_angle_before_transformation: float = 0.0
    use_spherical_coordinate_transformation: bool = False
    neel_min_angle_before_transformation: float = 0.0
    use_simple_model: bool = False
    injected_dw: Optional[np.ndarray] = None
    record_trajectories: int = 0  # 0/False: none; s (True = 1): every s-th particle's window means
    jacobian: Jacobian = Jacobian.Reference
    double_noise_approx: int = -1                    # WeakTest / ExplicitStrong_1: order p, -1..10
    cubic_constant: Optional[np.ndarray] = None      # UniaxialCubic: K_cubic (n)
    uniaxial_rotation: Optional[np.ndarray] = None   # UniaxialCubic: Euler angles of the uniaxial axis (n, 3)
    provider: Optional[ProviderSpec] = None          # particles drawn on the device (arrays unused)

    @property
    def dims(self):
        return DIMS[Problem(self.problem)]

    @property
    def n_samples(self) -> int:
        return int(self.number_of_steps // self.oversampling)

    @property
    def integrated_steps(self) -> int:
        return max(self.n_samples - 1, 0) * int(self.oversampling)

    def subset(self, lo: int, hi: int) -> "EnsembleSpec":
        """Particles [lo, hi) as their own ensemble with unchanged global ids."""
        import dataclasses
        kw = {}
        for name in ("magnetic_radius", "saturation_magnetisation", "damping_constant", "gyromagnetic_ratio",
                     "anisotropy_constant", "hydrodynamic_radius", "viscosity", "cubic_constant"):
            v = getattr(self, name)
            kw[name] = None if v is None else np.asarray(v)[lo:hi]
        kw["orientation"] = np.asarray(self.orientation).reshape(-1, 3)[lo:hi]
        kw["magnetisation"] = np.asarray(self.magnetisation).reshape(-1, 3)[lo:hi]
        if self.uniaxial_rotation is not None:
            kw["uniaxial_rotation"] = np.asarray(self.uniaxial_rotation).reshape(-1, 3)[lo:hi]
        if self.injected_dw is not None:
            m = self.dims[1]
            kw["injected_dw"] = np.asarray(self.injected_dw).reshape(-1, m, self.n)[:, :, lo:hi]
        return dataclasses.replace(self, n=hi - lo, particle_id_offset=self.particle_id_offset + lo, **kw)


class DescHolder:
    """An sp_ensemble_desc plus the numpy buffers its pointers refer to."""

    def __init__(self, spec: EnsembleSpec):
        n = int(spec.n)
        opt = lambda v, **kw: None if v is None else _f64(v, **kw)  # noqa: E731
        self.arrays = {
            "magnetic_radius": opt(spec.magnetic_radius, n=n),
            "saturation_magnetisation": opt(spec.saturation_magnetisation, n=n),
            "damping_constant": opt(spec.damping_constant, n=n),
            "gyromagnetic_ratio": opt(spec.gyromagnetic_ratio, n=n),
            "anisotropy_constant": opt(spec.anisotropy_constant, n=n),
            "hydrodynamic_radius": opt(spec.hydrodynamic_radius, n=n),
            "viscosity": opt(spec.viscosity, n=n),
            "orientation": opt(spec.orientation, shape=(n, 3)),
            "magnetisation": opt(spec.magnetisation, shape=(n, 3)),
            "cubic_constant": None if spec.cubic_constant is None else _f64(spec.cubic_constant, n),
            "uniaxial_rotation": None if spec.uniaxial_rotation is None else _f64(spec.uniaxial_rotation, shape=(n, 3)),
        }
        self.dw = None if spec.injected_dw is None else _f64(spec.injected_dw)
        d = sp_ensemble_desc()
        d.abi_version = ABI_VERSION
        d.problem = int(spec.problem)
        d.anisotropy = int(spec.anisotropy)
        d.solver = int(spec.solver)
        d.precision = int(spec.precision)
        d.noise = int(spec.noise)
        ps = d.problem_settings
        ps.use_coordinate_transformation = int(bool(spec.use_coordinate_transformation))
        ps.use_euler_coordinate_transformation = int(bool(spec.use_euler_coordinate_transformation))
        ps.use_spherical_coordinate_transformation = int(bool(spec.use_spherical_coordinate_transformation))
        ps.use_simple_model = int(bool(spec.use_simple_model))
        ps.min_angle_before_transformation = float(spec.min_angle_before_transformation)
        ps.brown_min_angle_before_transformation = float(spec.brown_min_angle_before_transformation)
        ps.neel_min_angle_before_transformation = float(spec.neel_min_angle_before_transformation)
        d.max_iteration = int(spec.max_iteration)
        d.record_trajectories = int(spec.record_trajectories)
        d.jacobian = int(spec.jacobian)
        d.double_noise_approx = int(spec.double_noise_approx)
        d.accuracy_goal = float(spec.accuracy_goal)
        d.number_of_steps = int(spec.number_of_steps)
        d.oversampling = int(spec.oversampling)
        d.timestep = float(spec.timestep)
        d.temperature = float(spec.temperature)
        d.field = spec.field.to_c()
        d.n_particles = n
        p = d.particles
        for k, v in self.arrays.items():
            setattr(p, k, _ptr(v))
        d.seed = int(spec.seed) & 0xFFFFFFFFFFFFFFFF
        d.particle_id_offset = int(spec.particle_id_offset)
        d.injected_dw = _ptr(self.dw)
        self.provider = self.templates = None
        if spec.provider is not None:
            pv = spec.provider
            self.templates = (sp_particle_template * len(pv.templates))(*[t.to_c() for t in pv.templates])
            self.provider = sp_provider_desc(int(pv.seed) & 0xFFFFFFFFFFFFFFFF, len(pv.templates), int(bool(pv.sequential)),
                                             C.cast(self.templates, C.POINTER(sp_particle_template)))
            d.provider = C.pointer(self.provider)
        self.desc = d
        self.spec = spec

    def byref(self):
        return C.byref(self.desc)


class ResultBuffers:
    """numpy outputs wired into an sp_result."""

    def __init__(self, spec: EnsembleSpec, trajectories: bool = False, final_state: bool = False):
        k, (sd, _, od) = spec.n_samples, spec.dims
        self.mean = np.zeros((k, od))
        self.weight = np.zeros(od)
        self.time = np.zeros(k)
        self.field = np.zeros((k, 3))
        self.weighted_sum = np.zeros((k, od))
        stride = max(1, int(spec.record_trajectories))  # the recorded particles: every stride-th
        self.trajectories = np.zeros((spec.n // stride, k, od)) if trajectories else None
        self.final_state = np.zeros((spec.n, sd)) if final_state else None
        r = sp_result()
        r.mean = _ptr(self.mean)
        r.weight = _ptr(self.weight)
        r.time = _ptr(self.time)
        r.field = _ptr(self.field)
        r.weighted_sum = _ptr(self.weighted_sum)
        r.trajectories = _ptr(self.trajectories)
        r.final_state = _ptr(self.final_state)
        self.c = r

    def as_dict(self):
        d = {"mean": self.mean, "weight": self.weight, "time": self.time, "field": self.field,
             "weighted_sum": self.weighted_sum}
        if self.trajectories is not None:
            d["trajectories"] = self.trajectories
        if self.final_state is not None:
            d["final_state"] = self.final_state
        return d
