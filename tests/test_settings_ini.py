""".ini settings and the particle provider of the command-line driver (CPU).

The driver follows the reference's settings readers and provider
(Settings/SimulationManagerSettings.h:126-186, Provider/ParticleProvider.h:194-217,
Settings/ParticleSimulationSettings.h:51-152); `-print` runs all of it without a
GPU.  Fixtures under tests/data/ini cover the older field layout of the
reference's example files and the current key names.
"""
import math
from pathlib import Path

import numpy as np
import pytest

from stochasticphysics_b200 import settings
from stochasticphysics_b200._abi import (Anisotropy, DescHolder, FieldType, Precision, Problem, Solver)
from stochasticphysics_b200.lib import load

INI = Path(__file__).resolve().parent / "data" / "ini"


@pytest.fixture(scope="module", autouse=True)
def driver():
    if not settings.APP.exists():
        from stochasticphysics_b200.build import build
        build()
    assert settings.APP.exists()


def test_older_layout_field_problem_and_solver():
    d = settings.describe_ini(INI / "legacy_neel_spherical.ini")
    assert Problem(d["problem"]) == Problem.NeelSpherical
    assert Solver(d["solver"]) == Solver.Heun_Strong
    assert Anisotropy(d["anisotropy"]) == Anisotropy.Uniaxial
    f = d["field"]
    assert FieldType(f["type"]) == FieldType.Sinusoidal
    assert f["offset"] == [1e-5, -3e-5, 2e-5]          # Amplitude_1
    assert f["amplitude"] == [0.0, 1.2e-2, 0.0]         # Amplitude_2
    assert f["frequency"][0] == 1e4 and f["phase"][0] == 0.25
    assert d["problem_settings"]["use_coordinate_transformation"] == 1
    assert d["problem_settings"]["min_angle_before_transformation"] == 0.1  # "% rad" is a comment
    assert (d["number_of_steps"], d["oversampling"], d["timestep"]) == (2000, 100, 2e-12)
    assert d["temperature"] == 300 and d["savefile"] == "legacy_result.mat"


def test_sequential_provider_fills_counts_in_list_order():
    """Without the discrete distribution the provider hands out Small x3, Large x5,
    then the first template again without counting it (ParticleProvider.h:201-213)."""
    d = settings.describe_ini(INI / "legacy_neel_spherical.ini")
    p = d["particles"]
    assert d["used_particle_numbers"] == {"Small": 3, "Large": 5}
    r = np.array(p["magnetic_radius"])
    np.testing.assert_array_equal(r, [8e-9] * 3 + [1.2e-8] * 5 + [8e-9] * 2)
    np.testing.assert_array_equal(p["anisotropy_constant"], [-2e3] * 3 + [-1.5e3] * 5 + [-2e3] * 2)
    # delta distributions keep every property; the shell is rebuilt around the radius
    np.testing.assert_allclose(p["hydrodynamic_radius"], 3e-8, rtol=1e-15)
    m = np.array(p["magnetisation"])
    np.testing.assert_allclose(m[:3], [[0, 0.6, 0.8]] * 3, rtol=1e-15)
    np.testing.assert_allclose(m[3:8], [[0, 0, 1]] * 5, rtol=1e-15)  # {0,0,2} normalised
    np.testing.assert_allclose(p["orientation"], [[0.3, 0.2, 0.1]] * 10, rtol=1e-15)


def test_current_layout_lissajous_and_solver_settings():
    d = settings.describe_ini(INI / "current_brown_neel.ini")
    assert Problem(d["problem"]) == Problem.BrownAndNeel
    assert Solver(d["solver"]) == Solver.Millstein
    assert (d["max_iteration"], d["accuracy_goal"]) == (50, 1e-11)
    f = d["field"]
    assert FieldType(f["type"]) == FieldType.Lissajous
    assert f["offset"] == [0, 0, 1e-3] and f["amplitude"] == [1e-2, 2e-2, 0]
    assert f["frequency"] == [2.5e4, 2.6e4, 0] and f["phase"] == [0, math.pi / 2, 0]


def test_discrete_selection_follows_particle_numbers():
    d = settings.describe_ini(INI / "current_brown_neel.ini")
    used = d["used_particle_numbers"]
    n = d["n_particles"]
    assert used["Particle_1"] + used["Particle_2"] == n == 4000
    share = used["Particle_1"] / n  # weights 3 : 1
    assert abs(share - 0.75) < 4 * math.sqrt(0.75 * 0.25 / n)


def test_size_and_anisotropy_distributions():
    """Relative widths: radius ~ r0 * lognormal(mean 1, sd 0.1); shell around the
    drawn radius ~ (rh0 - r) * N(1, 0.05); K ~ K0 * N(1, 0.2)."""
    d = settings.describe_ini(INI / "current_brown_neel.ini")
    p = d["particles"]
    r = np.array(p["magnetic_radius"])
    rh = np.array(p["hydrodynamic_radius"])
    K = np.array(p["anisotropy_constant"])
    small = np.array(p["saturation_magnetisation"]) == 4.8e5  # template 1 (template 2 has 4.9e5)
    for sel, r0, rh0 in ((small, 1e-8, 2.5e-8), (~small, 1.4e-8, 3e-8)):
        x = r[sel] / r0
        m = x.size
        assert abs(x.mean() - 1) < 4 * 0.1 / math.sqrt(m)
        assert abs(x.std() / 0.1 - 1) < 0.15
        assert np.all(x > 0)
        shell = (rh[sel] - r[sel]) / (rh0 - r[sel])
        assert abs(shell.mean() - 1) < 4 * 0.05 / math.sqrt(m)
        assert abs(shell.std() / 0.05 - 1) < 0.15
    k = K / -1e4
    assert abs(k.mean() - 1) < 4 * 0.2 / math.sqrt(k.size)
    assert abs(k.std() / 0.2 - 1) < 0.1


def test_random_cartesian_state_is_uniform_on_the_sphere():
    """BrownAndNeel: magnetisation N(0,1)^3 normalised; the particle axis too,
    handed over as ZXZ angles whose rotated x axis is that direction
    (BrownAndNeelRelaxation.inl:288-315)."""
    d = settings.describe_ini(INI / "current_brown_neel.ini")
    p = d["particles"]
    m = np.array(p["magnetisation"])
    e = np.array(p["orientation"])
    a, b, g = e[:, 0], e[:, 1], e[:, 2]
    axis = np.stack([np.cos(a) * np.cos(g) - np.sin(a) * np.cos(b) * np.sin(g),
                     -np.cos(a) * np.sin(g) - np.sin(a) * np.cos(b) * np.cos(g),
                     np.sin(a) * np.sin(b)], axis=1)
    n = len(m)
    for v in (m, axis):
        np.testing.assert_allclose(np.linalg.norm(v, axis=1), 1.0, rtol=1e-14)
        assert np.all(np.abs(v.mean(axis=0)) < 4 / math.sqrt(3 * n))
        # uniform on the sphere: each coordinate uniform on [-1, 1], E[x^2] = 1/3
        assert np.all(np.abs((v ** 2).mean(axis=0) - 1 / 3) < 4 * math.sqrt(4 / 45 / n))


def test_random_spherical_state_follows_the_reference_angles():
    """Spherical problems draw phi ~ U[0, 2pi), theta ~ U[0, pi) for the
    magnetisation and (U2pi, Upi, U2pi) Euler angles (ParticleStateInitializer.h:50-56,
    113-123) — uniform in the angles, not on the sphere."""
    d = settings.describe_ini(INI / "current_neel_spherical_random.ini")
    p = d["particles"]
    m = np.array(p["magnetisation"])
    theta = np.arccos(np.clip(m[:, 2], -1, 1))
    n = len(theta)
    assert abs(theta.mean() - math.pi / 2) < 4 * math.pi / math.sqrt(12 * n)
    assert abs(theta.var() / (math.pi ** 2 / 12) - 1) < 0.1
    e = np.array(p["orientation"])
    assert e[:, 0].max() < 2 * math.pi and e[:, 1].max() < math.pi and e.min() >= 0
    assert e[:, 1].max() > 0.95 * math.pi and e[:, 0].max() > 1.9 * math.pi
    assert FieldType(d["field"]["type"]) == FieldType.Constant and d["field"]["offset"] == [0, 0, 5e-3]


def test_seed_makes_the_provider_deterministic():
    a = settings.describe_ini(INI / "current_brown_neel.ini", seed=7)
    b = settings.describe_ini(INI / "current_brown_neel.ini", seed=7)
    c = settings.describe_ini(INI / "current_brown_neel.ini", seed=8)
    assert a["particles"] == b["particles"]
    assert a["particles"]["magnetic_radius"] != c["particles"]["magnetic_radius"]


def test_spec_from_ini_builds_a_valid_description():
    spec = settings.load_ini(INI / "current_brown_neel.ini", seed=3, precision=Precision.FP32)
    assert spec.n == 4000 and spec.seed == 3 and spec.precision == Precision.FP32
    assert spec.hydrodynamic_radius is not None and spec.orientation.shape == (4000, 3)
    h = DescHolder(spec)
    assert load().sp_validate(h.byref()) == 0, load().sp_last_error().decode()
    legacy = settings.load_ini(INI / "legacy_neel_spherical.ini")
    assert legacy.hydrodynamic_radius is None  # Neel problems pass no Brown properties
    assert load().sp_validate(DescHolder(legacy).byref()) == 0


@pytest.mark.parametrize("edit, message", [
    (("'Heun_Strong'", "'Implicit_Midpoint_GSL'"), "unsupported Solver 'Implicit_Midpoint_GSL'"),
    (("'Heun_Strong'", "'WeakTest'"), "missing key Approximation_of_double_noise_integral"),
    (("Timestep = 2.0e-12", ""), "missing key Timestep"),
    (("'legacy_particle_large.ini'", "'no_such_particle.ini'"), "cannot open"),
    (("Type_of_field = 'sinusoidal'", "Type_of_field = 'sawtooth'"), "unsupported Type_of_field"),
    (("Type_of_field = 'sinusoidal'", "Type_of_field = 'triangular'"), "finite periode > 0"),
    (("Oversampling = 100", "Oversampling = 3000"), "oversampling"),
])
def test_invalid_settings_are_reported(tmp_path, edit, message):
    text = (INI / "legacy_neel_spherical.ini").read_text()
    assert edit[0] in text
    for name in ("legacy_particle_small.ini", "legacy_particle_large.ini"):
        (tmp_path / name).write_text((INI / name).read_text())
    bad = tmp_path / "bad.ini"
    bad.write_text(text.replace(edit[0], edit[1]))
    with pytest.raises(settings.SettingsError, match=message):
        settings.describe_ini(bad)


@pytest.mark.parametrize("name, solver", [("WeakTest", Solver.WeakTest), ("ExplicitStrong_1.0", Solver.ExplicitStrong_1),
                                          ("Heun_NotConsistent", Solver.Heun_NotConsistent)])
def test_reference_disabled_solvers_parse(tmp_path, name, solver):
    """SolverSettings.cpp:18-20 names; Approximation_of_double_noise_integral is read for
    WeakTest and ExplicitStrong_1.0 only (SolverSettings.h:113-116), -1 otherwise."""
    text = (INI / "legacy_neel_spherical.ini").read_text()
    for f in ("legacy_particle_small.ini", "legacy_particle_large.ini"):
        (tmp_path / f).write_text((INI / f).read_text())
    text = text.replace("'Heun_Strong'", f"'{name}'\nApproximation_of_double_noise_integral = 3")
    (tmp_path / "s.ini").write_text(text)
    spec = settings.load_ini(tmp_path / "s.ini")
    assert spec.solver == solver
    assert spec.double_noise_approx == (-1 if solver == Solver.Heun_NotConsistent else 3)
    assert load().sp_validate(DescHolder(spec).byref()) == 0, load().sp_last_error().decode()


def test_system_matrix_voxels_and_fields():
    """SystemMatrixSettings.h: voxel size (stop - start) / (slices - 1), x fastest,
    offset = configured offset + Startfield + size * voxel; files *_Vox_x_y_z.*"""
    d = settings.describe_sysmatrix(INI / "legacy_neel_spherical.ini", INI / "sysmatrix_2x3.ini", seed=100)
    assert d["Number_of_voxels"] == 6
    assert d["System_Matrix_Settings"]["Voxel_Size"] == [4e-3, 1e-3, 0.0]
    vox = [v["Voxel"] for v in d["Voxels"]]
    assert vox == [[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [0, 2, 0], [1, 2, 0]]
    base = np.array([1e-5, -3e-5, 2e-5])  # Amplitude_1 of the particle run
    for i, v in enumerate(d["Voxels"]):
        x, y, z = v["Voxel"]
        np.testing.assert_allclose(v["Offset_Field"], base + [-2e-3 + 4e-3 * x, -1e-3 + 1e-3 * y, 0.0], rtol=0, atol=1e-18)
        assert v["Seed"] == 100 + i
        assert v["File"] == f"legacy_result_Vox_{x}_{y}_{z}.mat"


def test_system_matrix_start_stop_voxels_follow_the_reference_count():
    """Use_start_stop_Voxel: walk from Start_Voxel in x-fastest order for
    getNumberVoxelsToSimulate voxels (SystemMatrixSettings.h:159-215); with
    Start.x > Stop.x the count is |dz| nx ny + |dy| nx - |dx|."""
    d = settings.describe_sysmatrix(INI / "legacy_neel_spherical.ini", INI / "sysmatrix_start_stop.ini")
    vox = [tuple(v["Voxel"]) for v in d["Voxels"]]
    assert d["Number_of_voxels"] == len(vox) == 1 * 16 + 2 * 4 - 1
    lin = [x + 4 * y + 16 * z for x, y, z in vox]
    assert lin == list(range(2 + 4 * 1, 2 + 4 * 1 + 23))


@pytest.mark.parametrize("text, message", [
    ("Startfield = {0,0,0}\nStopfield = {1,0,0}\nSlices = {1,1,1}\n", "Unable to calculate VoxelSize"),
    ("Startfield = {0,0,0}\nStopfield = {0,0,0}\nSlices = {0,1,1}\n", "at least one"),
    ("Startfield = {0,0,0}\nSlices = {1,1,1}\n", "missing key Stopfield"),
])
def test_invalid_system_matrix_settings(tmp_path, text, message):
    f = tmp_path / "sm.ini"
    f.write_text("[System_Matrix_Settings]\n" + text)
    with pytest.raises(settings.SettingsError, match=message):
        settings.describe_sysmatrix(INI / "legacy_neel_spherical.ini", f)
