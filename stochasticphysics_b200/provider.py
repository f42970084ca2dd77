"""Per-particle parameter sets: the Provider role of the reference.

The reference draws particle properties per simulation in
ParticleSimulationSettings::getNewParticleProperties
(Particle_Simulation/Settings/ParticleSimulationSettings.h:51-152) and hands
them out through ParticleProvider::getProvidedObject
(Particle_Simulation/Provider/ParticleProvider.h:194-217).  Its random
initial orientations are neither seedable nor isotropic
(Problems/NeelRelaxation.h:225-235, Problems/Helpers/ParticleStateInitializer.h:42-62),
so this module generates seeded, explicitly isotropic / Haar-uniform Euler
angles and passes them through the boundary with Use_random_initial_* = false.

Workloads (seeded synthetic inputs; no dataset exists):
  neel_relaxation          1024 monodisperse magnetite particles, Cartesian Neel, Heun
  brown_neel_relaxation    65536 polydisperse particles, Brown+Neel Euler/spherical
  cubic_implicit           262144 particles, cubic anisotropy, ImplicitMidpoint
  batched_sets             256 parameter sets of uneven size and length
  serving_request          one Poisson-arriving request of the serving workload
"""
from __future__ import annotations

import math

import numpy as np

from ._abi import (Anisotropy, EnsembleSpec, FieldSpec, Noise, Precision, Problem, Solver)

GAMMA = 1.76e11      # rad/(s T)
MS_MAGNETITE = 4.8e5  # A/m
T_ROOM = 295.0       # K


def isotropic_euler(rng: np.random.Generator, n: int) -> np.ndarray:
    """ZXZ Euler angles with phi, psi ~ U[0, 2pi) and cos(theta) ~ U[-1, 1]: the body
    axes are a Haar-uniform rotation, so every body axis is isotropic on the sphere."""
    phi = rng.uniform(0.0, 2 * math.pi, n)
    theta = np.arccos(rng.uniform(-1.0, 1.0, n))
    psi = rng.uniform(0.0, 2 * math.pi, n)
    return np.stack([phi, theta, psi], axis=1)


def easy_axis(problem: Problem, euler: np.ndarray) -> np.ndarray:
    """The uniaxial easy axis each problem derives from the Euler angles."""
    ph, th, ps = euler[:, 0], euler[:, 1], euler[:, 2]
    if problem in (Problem.Neel, Problem.NeelSpherical):
        # zAxis of calculateParticleAxes (Problems/NeelRelaxation.h:259)
        return np.stack([np.sin(th) * np.sin(ph), np.sin(th) * np.cos(ph), np.cos(th)], axis=1)
    if problem == Problem.BrownAndNeelEulerSpherical:
        # third column of the cached Euler rotation (BrownAndNeelRelaxationEulerSpherical.h:211-217)
        return np.stack([np.sin(th) * np.sin(ps), -np.sin(th) * np.cos(ps), np.cos(th)], axis=1)
    # BrownAndNeelRelaxation.inl:304-307 (first column of the rotation applied to (1,0,0))
    a, b, g = ph, th, ps
    return np.stack([np.cos(a) * np.cos(g) - np.sin(a) * np.cos(b) * np.sin(g),
                     -np.cos(a) * np.sin(g) - np.sin(a) * np.cos(b) * np.cos(g),
                     np.sin(a) * np.sin(b)], axis=1)


def body_axes(problem: Problem, euler: np.ndarray):
    """Body x, y, z axes (world coordinates) as each problem derives them from the Euler angles."""
    ph, th, ps = euler[:, 0], euler[:, 1], euler[:, 2]
    cph, sph, cth, sth, cps, sps = np.cos(ph), np.sin(ph), np.cos(th), np.sin(th), np.cos(ps), np.sin(ps)
    if problem == Problem.BrownAndNeelEulerSpherical:
        # columns of the cached Euler rotation (BrownAndNeelRelaxationEulerSpherical.h:209-217)
        x = np.stack([cph * cps - cth * sph * sps, cth * sph * cps + cph * sps, sth * sph], axis=1)
        y = np.stack([-sph * cps - cth * cph * sps, cth * cph * cps - sph * sps, sth * cph], axis=1)
        z = np.stack([sth * sps, -sth * cps, cth], axis=1)
    else:
        # calculateParticleAxes (Problems/NeelRelaxation.h:257-259)
        x = np.stack([cph * cps - cth * sph * sps, -sph * cps - cth * cph * sps, sth * sps], axis=1)
        y = np.stack([cth * sph * cps + cph * sps, cth * cph * cps - sph * sps, -sth * cps], axis=1)
        z = np.stack([sth * sph, sth * cph, cth], axis=1)
    return x, y, z


def cubic_easy_direction(problem: Problem, euler: np.ndarray) -> np.ndarray:
    """A <111> body diagonal: an easy direction of cubic anisotropy with K1 < 0."""
    x, y, z = body_axes(problem, euler)
    return (x + y + z) / math.sqrt(3.0)


def along_axis_random_sign(rng: np.random.Generator, axis: np.ndarray) -> np.ndarray:
    sign = np.where(rng.uniform(size=axis.shape[0]) < 0.5, -1.0, 1.0)
    return axis * sign[:, None]


def lognormal_radius(rng: np.random.Generator, n: int, median: float, sigma: float) -> np.ndarray:
    return median * np.exp(sigma * rng.standard_normal(n))


def neel_relaxation(n: int = 1024, steps: int = 1_000_000, oversampling: int = 100, dt: float = 1e-11,
                    solver: Solver = Solver.Heun_Strong, precision: Precision = Precision.FP64,
                    seed: int = 0x5EED0001) -> EnsembleSpec:
    """Plain Neel relaxation: Cartesian LLG, uniaxial K = 1e4 J/m^3 easy axis (reference
    sign: K = -1e4), r = 10 nm, alpha = 0.1, 10 mT sinusoidal along z at 100 kHz."""
    rng = np.random.default_rng(seed)
    euler = isotropic_euler(rng, n)
    m0 = along_axis_random_sign(rng, easy_axis(Problem.Neel, euler))
    return EnsembleSpec(
        problem=Problem.Neel, n=n, magnetic_radius=np.full(n, 10e-9), saturation_magnetisation=np.full(n, MS_MAGNETITE),
        damping_constant=np.full(n, 0.1), gyromagnetic_ratio=np.full(n, GAMMA), anisotropy_constant=np.full(n, -1e4),
        orientation=euler, magnetisation=m0, number_of_steps=steps, oversampling=oversampling, timestep=dt,
        temperature=T_ROOM, solver=solver, precision=precision, seed=seed,
        field=FieldSpec.sinusoidal((0.0, 0.0, 0.010), 1e5))


def brown_neel_relaxation(n: int = 65536, steps: int = 4_000_000, oversampling: int = 1000, dt: float = 1e-11,
                          solver: Solver = Solver.Millstein, precision: Precision = Precision.FP64,
                          seed: int = 0x5EED0002) -> EnsembleSpec:
    """Coupled Brown+Neel (Euler angles + Neel spherical), lognormal cores (median 10 nm,
    sigma 0.1), hydrodynamic radius = core + 20 nm, eta = 1e-3 Pa s, K ~ U[5e3, 2e4] J/m^3
    easy axis, alpha = 0.1, 20 mT at 25 kHz; both coordinate rotations on at pi/36."""
    rng = np.random.default_rng(seed)
    r = lognormal_radius(rng, n, 10e-9, 0.1)
    euler = isotropic_euler(rng, n)
    m0 = along_axis_random_sign(rng, easy_axis(Problem.BrownAndNeelEulerSpherical, euler))
    K = -rng.uniform(5e3, 2e4, n)
    return EnsembleSpec(
        problem=Problem.BrownAndNeelEulerSpherical, n=n, magnetic_radius=r,
        saturation_magnetisation=np.full(n, MS_MAGNETITE), damping_constant=np.full(n, 0.1),
        gyromagnetic_ratio=np.full(n, GAMMA), anisotropy_constant=K, hydrodynamic_radius=r + 20e-9,
        viscosity=np.full(n, 1e-3), orientation=euler, magnetisation=m0, number_of_steps=steps,
        oversampling=oversampling, timestep=dt, temperature=T_ROOM, solver=solver, precision=precision, seed=seed,
        field=FieldSpec.sinusoidal((0.0, 0.0, 0.020), 2.5e4),
        use_euler_coordinate_transformation=True, brown_min_angle_before_transformation=math.pi / 36,
        use_spherical_coordinate_transformation=True, neel_min_angle_before_transformation=math.pi / 36)


def cubic_implicit(n: int = 262144, steps: int = 2_000_000, oversampling: int = 1000, dt: float = 1e-10,
                   precision: Precision = Precision.FP64, seed: int = 0x5EED0003) -> EnsembleSpec:
    """Stiff path: Cartesian Neel with cubic K1 = -1.1e4 J/m^3 (standard sign, passed
    unchanged), Haar-random axes, alpha = 0.05, lognormal cores (median 12 nm, sigma 0.15),
    12 mT at 25 kHz, ImplicitMidpoint with tolerance 1e-10 and 20 iterations."""
    rng = np.random.default_rng(seed)
    r = lognormal_radius(rng, n, 12e-9, 0.15)
    euler = isotropic_euler(rng, n)
    # start on a <111> body diagonal, an easy direction for K1 < 0 (a <100> start would sit
    # on an unstable equilibrium)
    m0 = along_axis_random_sign(rng, cubic_easy_direction(Problem.Neel, euler))
    return EnsembleSpec(
        problem=Problem.Neel, n=n, magnetic_radius=r, saturation_magnetisation=np.full(n, MS_MAGNETITE),
        damping_constant=np.full(n, 0.05), gyromagnetic_ratio=np.full(n, GAMMA), anisotropy_constant=np.full(n, -1.1e4),
        anisotropy=Anisotropy.Cubic, orientation=euler, magnetisation=m0, number_of_steps=steps,
        oversampling=oversampling, timestep=dt, temperature=T_ROOM, solver=Solver.Implicit_Midpoint,
        precision=precision, seed=seed, max_iteration=20, accuracy_goal=1e-10,
        field=FieldSpec.sinusoidal((0.0, 0.0, 0.012), 2.5e4))


def _loguniform(rng, lo, hi):
    return float(math.exp(rng.uniform(math.log(lo), math.log(hi))))


def batched_sets(count: int = 256, seed: int = 0x5EED0004, precision: Precision = Precision.FP32,
                 step_scale: float = 1.0, n_scale: float = 1.0, oversampling: int = 1000,
                 lissajous: bool = False, problems=(Problem.Neel,)) -> list:
    """Parameter sets with N ~ logU[1e3, 6.4e4], S ~ logU[1e5, 1e7] (times step_scale),
    |B| ~ U[1, 25] mT, f ~ logU[1e4, 1e6] Hz, K ~ U[5e3, 3e4] J/m^3 easy axis,
    alpha ~ U[0.02, 0.3], core radius lognormal (median U[8, 14] nm, sigma 0.1);
    solvers alternate Heun / Millstein."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        n = max(32, int(round(_loguniform(rng, 1e3, 6.4e4) * n_scale)))
        steps = max(2 * oversampling, int(round(_loguniform(rng, 1e5, 1e7) * step_scale / oversampling)) * oversampling)
        amp = rng.uniform(1e-3, 25e-3)
        freq = _loguniform(rng, 1e4, 1e6)
        K = rng.uniform(5e3, 3e4)
        alpha = rng.uniform(0.02, 0.3)
        r_med = rng.uniform(8e-9, 14e-9)
        problem = problems[int(rng.integers(len(problems)))]
        sub = np.random.default_rng(int(rng.integers(1 << 62)))
        r = lognormal_radius(sub, n, r_med, 0.1)
        euler = isotropic_euler(sub, n)
        m0 = along_axis_random_sign(sub, easy_axis(problem, euler))
        if lissajous:
            fld = FieldSpec.lissajous((0.012, 0.012, 0.0), (25250.0, 26040.0, 0.0))
        else:
            fld = FieldSpec.sinusoidal((0.0, 0.0, amp), freq)
        brown = problem in (Problem.BrownAndNeel, Problem.BrownAndNeelEulerSpherical)
        specs.append(EnsembleSpec(
            problem=problem, n=n, magnetic_radius=r, saturation_magnetisation=np.full(n, MS_MAGNETITE),
            damping_constant=np.full(n, alpha), gyromagnetic_ratio=np.full(n, GAMMA),
            anisotropy_constant=np.full(n, -K), hydrodynamic_radius=(r + 20e-9) if brown else None,
            viscosity=np.full(n, 1e-3) if brown else None, orientation=euler, magnetisation=m0,
            number_of_steps=steps, oversampling=oversampling, timestep=1e-11, temperature=T_ROOM,
            solver=Solver.Heun_Strong if i % 2 == 0 else Solver.Millstein, precision=precision,
            seed=int(sub.integers(1 << 62)), field=fld,
            use_euler_coordinate_transformation=brown, brown_min_angle_before_transformation=math.pi / 36,
            use_spherical_coordinate_transformation=brown, neel_min_angle_before_transformation=math.pi / 36))
    return specs


def with_injected_noise(spec: EnsembleSpec, seed: int = 1234) -> EnsembleSpec:
    """Same ensemble, Wiener increments drawn on the host (parity mode)."""
    import dataclasses
    rng = np.random.default_rng(seed)
    m = spec.dims[1]
    dw = rng.standard_normal((spec.integrated_steps, m, spec.n)) * math.sqrt(spec.timestep)
    return dataclasses.replace(spec, noise=Noise.Injected, injected_dw=dw)
