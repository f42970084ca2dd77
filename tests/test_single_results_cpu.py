"""Single-simulation results of the .ini driver: selection and file names (CPU).

The reference's result manager writes every Save_intervall-th single result as
the named value <Save_single_name_prefix>_<counter>, into
Single_simulations_savefile or, with Use_extra_file_for_single_simulations, into
one file per result named after it, and refuses a single-results file equal to
Savefile (Particle_Simulation/Results/SimulationResultManager.h:115-149; keys
Settings/ResultSettings.h:90-118).  The driver counts results in particle order
and writes JSON; `-print` reports the selection without a GPU.
"""
from pathlib import Path

import pytest

from stochasticphysics_b200 import settings

INI = Path(__file__).resolve().parent / "data" / "ini"
PARTICLES = ("legacy_particle_small.ini", "legacy_particle_large.ini")


@pytest.fixture(scope="module", autouse=True)
def driver():
    if not settings.APP.exists():
        from stochasticphysics_b200.build import build
        build()


def ini_with(tmp_path, result_lines):
    for name in PARTICLES:
        (tmp_path / name).write_text((INI / name).read_text())
    text = (INI / "legacy_neel_spherical.ini").read_text()
    text = text.replace("[Result_Settings]\nSavefile='legacy_result.mat'",
                        "[Result_Settings]\nSavefile='legacy_result.mat'\n" + "\n".join(result_lines))
    out = tmp_path / "main.ini"
    out.write_text(text)
    return out


def test_every_interval_th_particle_into_one_file(tmp_path):
    path = ini_with(tmp_path, ["Save_single_simulations = TRUE", "Save_intervall = 3",
                               "Save_single_name_prefix = 'Sim'", "Single_simulations_savefile = 'out/singles.mat'",
                               "Use_extra_file_for_single_simulations = FALSE"])
    sel = settings.describe_ini(path)["single_results"]
    assert [s["particle"] for s in sel] == [2, 5, 8]  # counters 3, 6, 9 of 10 particles
    assert [s["name"] for s in sel] == ["Sim_3", "Sim_6", "Sim_9"]
    assert {s["file"] for s in sel} == {"out/singles.json"}  # JSON archive in place of the .mat


def test_extra_file_per_result_beside_the_configured_file(tmp_path):
    path = ini_with(tmp_path, ["Save_single_simulations = TRUE", "Save_intervall = 4",
                               "Single_simulations_savefile = 'res/single_base.json'",
                               "Use_extra_file_for_single_simulations = TRUE"])
    sel = settings.describe_ini(path)["single_results"]
    assert [(s["particle"], s["name"], s["file"]) for s in sel] == [
        (3, "Simulation_4", "res/Simulation_4.json"), (7, "Simulation_8", "res/Simulation_8.json")]


def test_defaults_and_switched_off(tmp_path):
    path = ini_with(tmp_path, ["Save_single_simulations = FALSE", "Save_intervall = 1"])
    assert settings.describe_ini(path)["single_results"] == []
    path = ini_with(tmp_path, ["Save_single_simulations = TRUE"])  # interval 1: every particle
    sel = settings.describe_ini(path)["single_results"]
    assert [s["name"] for s in sel] == [f"Simulation_{c}" for c in range(1, 11)]
    assert sel[0]["file"] == "ResultsSingle.json"


def test_interval_beyond_the_ensemble_selects_nothing(tmp_path):
    path = ini_with(tmp_path, ["Save_single_simulations = TRUE", "Save_intervall = 11",
                               "Single_simulations_savefile = 'legacy_result.mat'"])
    # nothing is written, so the same-file rule has nothing to refuse (as in the reference)
    assert settings.describe_ini(path)["single_results"] == []


def test_same_file_as_the_mean_result_is_refused(tmp_path):
    path = ini_with(tmp_path, ["Save_single_simulations = TRUE", "Save_intervall = 2",
                               "Single_simulations_savefile = 'legacy_result.mat'"])
    with pytest.raises(settings.SettingsError, match="same file currently not supported"):
        settings.describe_ini(path)


def test_bad_interval_is_refused(tmp_path):
    path = ini_with(tmp_path, ["Save_single_simulations = TRUE", "Save_intervall = 0"])
    with pytest.raises(settings.SettingsError, match="Save_intervall"):
        settings.describe_ini(path)
