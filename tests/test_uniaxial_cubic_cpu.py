"""Uniaxial+cubic anisotropy (UniaxialCubicAnisotropy.hpp) in the oracle and the driver.

Reductions that must hold exactly in the restatement: with K_cubic = 0 and no
uniaxial rotation it is the uniaxial anisotropy; with K_uniaxial = 0 it is the
cubic anisotropy.  With a rotation, the Neel (Cartesian) problem's uniaxial axis is
R^T z, so it equals a uniaxial particle whose easy axis was rotated the same way.
"""
import dataclasses
import math
from pathlib import Path

import numpy as np
import pytest

import oracle
from stochasticphysics_b200 import provider, settings
from stochasticphysics_b200._abi import Anisotropy, DescHolder, Problem, Solver
from stochasticphysics_b200.lib import load


def _base(problem, solver=Solver.Heun_Strong, n=24):
    if problem == Problem.BrownAndNeelEulerSpherical:
        s = provider.brown_neel_relaxation(n=n, steps=600, oversampling=100)
    else:
        s = provider.neel_relaxation(n=n, steps=600, oversampling=100)
        if problem == Problem.NeelSpherical:
            s = dataclasses.replace(s, problem=problem, use_coordinate_transformation=True,
                                    min_angle_before_transformation=math.pi / 36)
    return provider.with_injected_noise(dataclasses.replace(s, solver=solver), seed=6)


def _uc(spec, k_cubic, urot):
    return dataclasses.replace(spec, anisotropy=Anisotropy.UniaxialCubic, cubic_constant=np.full(spec.n, k_cubic),
                               uniaxial_rotation=np.tile(np.asarray(urot, dtype=float), (spec.n, 1)))


PROBLEMS = [Problem.Neel, Problem.NeelSpherical, Problem.BrownAndNeelEulerSpherical]


@pytest.mark.parametrize("problem", PROBLEMS)
def test_reduces_to_uniaxial(problem):
    base = _base(problem)
    a = oracle.simulate(base, trajectories=True)
    b = oracle.simulate(_uc(base, 0.0, (0.0, 0.0, 0.0)), trajectories=True)
    np.testing.assert_array_equal(a["trajectories"], b["trajectories"])


@pytest.mark.parametrize("problem", PROBLEMS)
def test_reduces_to_cubic(problem):
    base = _base(problem)
    cub = dataclasses.replace(base, anisotropy=Anisotropy.Cubic, anisotropy_constant=np.full(base.n, -1.1e4))
    uc = _uc(dataclasses.replace(base, anisotropy_constant=np.zeros(base.n)), -1.1e4, (0.4, 0.9, 1.3))
    a = oracle.simulate(cub, trajectories=True)
    b = oracle.simulate(uc, trajectories=True)
    np.testing.assert_allclose(b["trajectories"], a["trajectories"], rtol=0, atol=1e-13)


def _rotation(e):
    sphi, cphi, st, ct, sps, cps = math.sin(e[0]), math.cos(e[0]), math.sin(e[1]), math.cos(e[1]), math.sin(e[2]), math.cos(e[2])
    cc, sc, cs, ss = cphi * cps, sphi * cps, cphi * sps, sphi * sps
    return np.array([[cc - ct * ss, -sc - ct * cs, st * sps], [ct * sc + cs, ct * cc - ss, -st * cps],
                     [st * sphi, st * cphi, ct]])


def test_rotated_uniaxial_axis_in_the_neel_problem():
    """Neel (Cartesian), K_cubic = 0: the easy axis is R^T z.  A uniaxial particle whose
    body axes give that z (Euler angles solved for it) follows the same path."""
    base = _base(Problem.Neel, n=8)
    urot = (0.3, 1.1, -0.7)
    Rm = _rotation(urot)
    euler = np.asarray(base.orientation).reshape(-1, 3)
    new_euler = []
    for e in euler:
        sphi, cphi, st, ct, sps, cps = (math.sin(e[0]), math.cos(e[0]), math.sin(e[1]), math.cos(e[1]),
                                        math.sin(e[2]), math.cos(e[2]))
        z = np.array([st * sphi, st * cphi, ct])  # body z of the ZXZ angles (NeelRelaxation.h:240-260)
        zr = Rm.T @ z
        theta = math.acos(max(-1.0, min(1.0, zr[2])))
        phi = math.atan2(zr[0], zr[1])
        new_euler.append((phi, theta, 0.0))
    uni = dataclasses.replace(base, orientation=np.array(new_euler))
    a = oracle.simulate(uni, trajectories=True)
    b = oracle.simulate(_uc(base, 0.0, urot), trajectories=True)
    np.testing.assert_allclose(b["trajectories"], a["trajectories"], rtol=0, atol=1e-12)


def test_validation():
    base = _uc(_base(Problem.Neel), -1e4, (0.1, 0.2, 0.3))
    assert load().sp_validate(DescHolder(base).byref()) == 0
    missing = dataclasses.replace(base, cubic_constant=None)
    assert load().sp_validate(DescHolder(missing).byref()) == 1
    bn = provider.brown_neel_relaxation(n=8, steps=200, oversampling=100)
    bn = _uc(dataclasses.replace(bn, problem=Problem.BrownAndNeel), -1e4, (0, 0, 0))
    assert load().sp_validate(DescHolder(bn).byref()) == 2


def test_driver_reads_uniaxialcubic_particles(tmp_path):
    ini = Path(__file__).resolve().parent / "data" / "ini"
    (tmp_path / "uc_particle.ini").write_text("""
[Particle_Properties]
Temperature = 295
[Particle_Properties.Magnetic_Properties]
Magnetic_radius = 1.0e-08
Saturation_magnetisation = 4.8e+05
Damping_constant = 0.1
Gyromagnetic_ratio = 1.76e+11
Type_of_anisotropy = 'uniaxialcubic'
Uniaxial_Rotation = {0.1, 0.2, 0.3}
[Particle_Properties.Magnetic_Properties.Anisotropy.Uniaxial_Part]
K_uniaxial = -1.0e+04
[Particle_Properties.Magnetic_Properties.Anisotropy.Cubic_Part]
K_cubic = -5.0e+03
[Particle_Simulation_Initialization]
Use_random_initial_particle_orientation = FALSE
Use_random_initial_particle_magnetisation = FALSE
Initial_particle_orientation = {0.0, 0.0, 0.0}
Initial_magnetisation_direction = {0.0, 0.0, 1.0}
[Particle_Simulation_Settings.Anisotropy_Distribution]
UseRandomCubicOrientation = FALSE
[Particle_Simulation_Settings.Anisotropy_Distribution.Uniaxial_Distribution]
Distribution_type = 'delta'
Sigma_K_uniaxial = 0.0
Use_relative_distribution_width = TRUE
[Particle_Simulation_Settings.Anisotropy_Distribution.Cubic_Distribution]
Distribution_type = 'normal'
Sigma_K_cubic = 0.1
Use_relative_distribution_width = TRUE
""")
    text = (ini / "legacy_neel_spherical.ini").read_text()
    text = text.replace("Small='legacy_particle_small.ini'\nLarge='legacy_particle_large.ini'", "Small='uc_particle.ini'")
    text = text.replace("Small = 3\nLarge = 5", "Small = 10")
    (tmp_path / "run.ini").write_text(text)
    d = settings.describe_ini(tmp_path / "run.ini")
    assert Anisotropy(d["anisotropy"]) == Anisotropy.UniaxialCubic
    p = d["particles"]
    np.testing.assert_array_equal(p["anisotropy_constant"], [-1e4] * 10)
    kc = np.array(p["cubic_constant"])
    assert np.all(kc != -5e3) and np.all(np.abs(kc / -5e3 - 1) < 0.6)
    np.testing.assert_array_equal(p["uniaxial_rotation"], [[0.1, 0.2, 0.3]] * 10)
    spec = settings.load_ini(tmp_path / "run.ini")
    assert spec.anisotropy == Anisotropy.UniaxialCubic and spec.cubic_constant.shape == (10,)
    assert load().sp_validate(DescHolder(spec).byref()) == 0
