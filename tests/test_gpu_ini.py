""".ini runs on the GPU: the command-line driver against the Python API and the oracle.

`stophys_b200 -parfile:<ini>` (the reference's application entry point,
Simulator/SimulationApplication.cpp:29-158) must give the same Mean_Results as
Context.simulate on the EnsembleSpec the same .ini and seed describe — the same
library call on the same inputs, so equal bit for bit — and the CPU oracle's
ensemble mean within the FP64 Philox-mode parity bar (1e-10 absolute).
"""
import dataclasses
from pathlib import Path

import numpy as np
import pytest

import oracle
import stochasticphysics_b200 as sp
from stochasticphysics_b200 import settings

pytestmark = pytest.mark.gpu

INI = Path(__file__).resolve().parent / "data" / "ini"
ABS_MEAN = 1e-10


def _copy(tmp_path, main, n, particles):
    for name in particles:
        (tmp_path / name).write_text((INI / name).read_text())
    text = (INI / main).read_text()
    lines = [f"Number_of_simulations = {n}" if ln.startswith("Number_of_simulations") else ln
             for ln in text.splitlines()]
    out = tmp_path / main
    out.write_text("\n".join(lines) + "\n")
    return out


@pytest.mark.parametrize("main, n, particles", [
    ("legacy_neel_spherical.ini", 10, ("legacy_particle_small.ini", "legacy_particle_large.ini")),
    ("current_brown_neel.ini", 256, ("current_particle.ini", "current_particle_b.ini")),
])
def test_ini_run_matches_api_and_oracle(tmp_path, main, n, particles):
    path = _copy(tmp_path, main, n, particles)
    rec = settings.run_ini(path, seed=21)["Mean_Results"]
    spec = settings.load_ini(path, seed=21)
    with sp.Context(0) as ctx:
        api = ctx.simulate(spec)
    mean = np.array(rec["Results"], dtype=float)
    np.testing.assert_array_equal(mean, api.mean)
    np.testing.assert_array_equal(np.array(rec["Weight"], dtype=float), api.weight)
    np.testing.assert_array_equal(np.array(rec["Time"], dtype=float), api.time)
    np.testing.assert_array_equal(np.array(rec["Field"], dtype=float), api.field)
    ref = oracle.simulate(spec)
    assert np.all(np.isfinite(ref["mean"]))
    assert np.max(np.abs(mean - ref["mean"])) <= ABS_MEAN


@pytest.mark.parametrize("solver", ["ExplicitStrong_1.0", "WeakTest", "Heun_NotConsistent"])
def test_reference_disabled_solvers_run_from_ini(tmp_path, solver):
    """The solvers the reference's manager switches off, selected by name in an .ini
    (with Approximation_of_double_noise_integral where it is read): the driver's run
    equals the API run of the same description and the oracle's mean."""
    path = _copy(tmp_path, "legacy_neel_spherical.ini", 10, ("legacy_particle_small.ini", "legacy_particle_large.ini"))
    path.write_text(path.read_text().replace("'Heun_Strong'", f"'{solver}'\nApproximation_of_double_noise_integral = 2"))
    rec = settings.run_ini(path, seed=5)["Mean_Results"]
    spec = settings.load_ini(path, seed=5)
    with sp.Context(0) as ctx:
        api = ctx.simulate(spec)
    mean = np.array(rec["Results"], dtype=float)
    np.testing.assert_array_equal(mean, api.mean)
    ref = oracle.simulate(spec)
    ok = np.isfinite(ref["mean"]).all(axis=1)
    assert np.max(np.abs(mean[ok] - ref["mean"][ok])) <= 1e-9


def test_system_matrix_sweep_equals_per_voxel_runs(tmp_path):
    """Every voxel of the batched sweep equals a separate run of the same voxel
    description (same offset field, same Philox key) bit for bit."""
    path = _copy(tmp_path, "legacy_neel_spherical.ini", 40, ("legacy_particle_small.ini", "legacy_particle_large.ini"))
    sm = INI / "sysmatrix_2x3.ini"
    rec = settings.run_ini(path, seed=9, sysmatrix=sm)
    assert rec["Number_of_voxels"] == 6
    base = settings.load_ini(path, seed=9)
    with sp.Context(0) as ctx:
        for i, v in enumerate(rec["Voxels"]):
            f = base.field
            spec = dataclasses.replace(base, seed=9 + i, field=sp.FieldSpec(f.type, tuple(v["Offset_Field"]), f.amplitude,
                                                                            f.frequency, f.phase))
            alone = ctx.simulate(spec)
            np.testing.assert_array_equal(np.array(v["Mean_Results"]["Results"], dtype=float), alone.mean)
            np.testing.assert_array_equal(np.array(v["Mean_Results"]["Field"], dtype=float), alone.field)


def test_device_provider_run_agrees_statistically(tmp_path):
    """-device-provider draws the particles on the GPU from the .ini's templates: a
    different sample of the same distributions, so the mean agrees within Monte-Carlo
    error with the host-provider run, and the drawn sizes follow the templates."""
    path = _copy(tmp_path, "current_brown_neel.ini", 4000, ("current_particle.ini", "current_particle_b.ini"))
    host = settings.run_ini(path, seed=5)
    dev = settings.run_ini(path, seed=5, device_provider=True)
    a = np.array(host["Mean_Results"]["Results"], dtype=float)
    b = np.array(dev["Mean_Results"]["Results"], dtype=float)
    assert np.all(np.isfinite(b))
    se = np.sqrt(2.0 / (3.0 * 4000))
    assert np.max(np.abs(a - b)) < 5 * se
    mp = dev["Mean_Results"]["Mean_Properties"]
    # templates 1e-8 and 1.4e-8 m at weights 3:1, lognormal 10 %: mean 1.1e-8 m
    assert abs(mp["Magnetic_radius"] / 1.1e-8 - 1) < 0.02
    assert dev["Stats"]["particle_steps"] == host["Stats"]["particle_steps"]


@pytest.mark.parametrize("extra_files", [False, True])
def test_single_simulation_results_match_the_oracle(tmp_path, extra_files):
    """Save_single_simulations: every 3rd particle's window means, written by the driver
    (Results/SimulationResultManager.h:115-149), equal the oracle's trajectories of those
    particles within the Philox-mode parity bar, with the particle's own weight Ms V."""
    import json
    import math

    main = _copy(tmp_path, "legacy_neel_spherical.ini", 10, ("legacy_particle_small.ini", "legacy_particle_large.ini"))
    text = main.read_text().replace(
        "[Result_Settings]\nSavefile='legacy_result.mat'",
        "[Result_Settings]\nSavefile='legacy_result.mat'\nSave_single_simulations = TRUE\nSave_intervall = 3\n"
        "Single_simulations_savefile = 'singles/one.mat'\n"
        f"Use_extra_file_for_single_simulations = {'TRUE' if extra_files else 'FALSE'}")
    main.write_text(text)
    (tmp_path / "singles").mkdir()
    rec = settings.run_ini(main, seed=21, cwd=tmp_path)
    spec = settings.load_ini(main, seed=21)
    ref = oracle.simulate(spec, trajectories=True)
    for c in (3, 6, 9):
        name = f"Simulation_{c}"
        f = tmp_path / "singles" / (f"{name}.json" if extra_files else "one.json")
        single = json.loads(f.read_text())[name]
        res = np.array(single["Results"], dtype=float)
        assert np.max(np.abs(res - ref["trajectories"][c - 1])) < 1e-9
        moment = spec.saturation_magnetisation[c - 1] * 4.0 / 3.0 * math.pi * spec.magnetic_radius[c - 1] ** 3
        np.testing.assert_allclose(single["Weight"], [moment] * 3, rtol=1e-14)
        np.testing.assert_array_equal(np.array(single["Time"], dtype=float), np.array(rec["Mean_Results"]["Time"]))
        assert single["UsedProperties"]["Magnetic_radius"] == spec.magnetic_radius[c - 1]
    if extra_files:
        assert sorted(p.name for p in (tmp_path / "singles").iterdir()) == [
            "Simulation_3.json", "Simulation_6.json", "Simulation_9.json"]


def test_strided_trajectories_equal_the_selected_particles(tmp_path):
    """record_trajectories = s keeps every s-th particle's window means only."""
    from stochasticphysics_b200 import provider
    spec = dataclasses.replace(provider.neel_relaxation(n=100, steps=2000, oversampling=100), record_trajectories=7)
    with sp.Context(0) as ctx:
        strided = ctx.simulate(spec, trajectories=True)
        full = ctx.simulate(dataclasses.replace(spec, record_trajectories=1), trajectories=True)
    assert strided.trajectories.shape == (14, spec.n_samples, 3)
    np.testing.assert_array_equal(strided.trajectories, full.trajectories[6::7])
    np.testing.assert_array_equal(strided.mean, full.mean)
