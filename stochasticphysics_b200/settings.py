"""SimulationManagerSettings .ini files as EnsembleSpec, and .ini runs.

The parser and the particle provider live in one place, the command-line
driver `stophys_b200` (app/stophys_b200_app.cpp), which follows the
reference's settings and provider code
(Particle_Simulation/Settings/SimulationManagerSettings.h:126-186,
Provider/ParticleProvider.h:194-217, Settings/ParticleSimulationSettings.h:51-152).
`load_ini` runs it with `-print` (no GPU) and turns the description it prints
into an EnsembleSpec; `run_ini` runs the whole simulation through it and
returns the "Mean_Results" record (Results/MeanSimulationResult.h:131-141).
"""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import numpy as np

from ._abi import Anisotropy, EnsembleSpec, FieldSpec, FieldType, Noise, Precision, Problem, Solver

APP = Path(__file__).resolve().parent / "stophys_b200"


class SettingsError(RuntimeError):
    """The driver rejected the settings; the message is its own."""


def _driver() -> Path:
    if not APP.exists():
        raise FileNotFoundError(f"{APP} is not built; run `make -C {APP.parent / 'csrc'}`")
    return APP


def _call(args, timeout, cwd=None):
    p = subprocess.run([str(_driver()), *args], capture_output=True, text=True, timeout=timeout, cwd=cwd)
    if p.returncode != 0:
        raise SettingsError(p.stderr.strip() or f"stophys_b200 exited with {p.returncode}")
    return p.stdout


def _flags(path, seed, precision):
    return [f"-parfile:{path}", f"-seed:{int(seed)}",
            "-precision:fp32" if Precision(precision) == Precision.FP32 else "-precision:fp64"]


def describe_ini(path, seed: int = 0x5EED, precision: Precision = Precision.FP64, timeout: float = 120.0) -> dict:
    """The parsed description and every provided particle, as the driver prints it, with
    the single-simulation results the Result_Settings select (particle, name, file)."""
    return json.loads(_call(_flags(path, seed, precision) + ["-print"], timeout))


def spec_from_description(d: dict) -> EnsembleSpec:
    p = d["particles"]
    q = d["problem_settings"]
    f = d["field"]
    problem = Problem(d["problem"])
    brown = problem in (Problem.BrownAndNeelEulerSpherical, Problem.BrownAndNeel)
    arr = lambda k: np.asarray(p[k], dtype=np.float64)  # noqa: E731
    return EnsembleSpec(
        problem=problem, n=int(d["n_particles"]),
        magnetic_radius=arr("magnetic_radius"), saturation_magnetisation=arr("saturation_magnetisation"),
        damping_constant=arr("damping_constant"), gyromagnetic_ratio=arr("gyromagnetic_ratio"),
        anisotropy_constant=arr("anisotropy_constant"),
        orientation=arr("orientation").reshape(-1, 3), magnetisation=arr("magnetisation").reshape(-1, 3),
        hydrodynamic_radius=arr("hydrodynamic_radius") if brown else None,
        viscosity=arr("viscosity") if brown else None,
        number_of_steps=int(d["number_of_steps"]), oversampling=int(d["oversampling"]), timestep=float(d["timestep"]),
        temperature=float(d["temperature"]), anisotropy=Anisotropy(d["anisotropy"]), solver=Solver(d["solver"]),
        precision=Precision(d["precision"]), noise=Noise.Philox,
        field=FieldSpec(FieldType(f["type"]), tuple(f["offset"]), tuple(f["amplitude"]), tuple(f["frequency"]),
                        tuple(f["phase"]), periode=float(f["periode"]), time_offset=float(f["time_offset"]),
                        tau=float(f["tau"]), alternating=bool(f["alternating"])),
        max_iteration=int(d["max_iteration"]), accuracy_goal=float(d["accuracy_goal"]),
        double_noise_approx=int(d.get("double_noise_approx", -1)),
        use_coordinate_transformation=bool(q["use_coordinate_transformation"]),
        min_angle_before_transformation=float(q["min_angle_before_transformation"]),
        use_euler_coordinate_transformation=bool(q["use_euler_coordinate_transformation"]),
        brown_min_angle_before_transformation=float(q["brown_min_angle_before_transformation"]),
        use_spherical_coordinate_transformation=bool(q["use_spherical_coordinate_transformation"]),
        neel_min_angle_before_transformation=float(q["neel_min_angle_before_transformation"]),
        use_simple_model=bool(q["use_simple_model"]),
        cubic_constant=arr("cubic_constant") if "cubic_constant" in p else None,
        uniaxial_rotation=arr("uniaxial_rotation").reshape(-1, 3) if "uniaxial_rotation" in p else None,
    )


def load_ini(path, seed: int = 0x5EED, precision: Precision = Precision.FP64) -> EnsembleSpec:
    """EnsembleSpec of a SimulationManagerSettings .ini (particles drawn with `seed`).

    The spec's Philox key is `seed` too, so `Context.simulate(load_ini(p, s))`
    equals `run_ini(p, s)`.
    """
    spec = spec_from_description(describe_ini(path, seed, precision))
    spec.seed = int(seed)
    return spec


def run_ini(path, seed: int = 0x5EED, precision: Precision = Precision.FP64, device: int = 0,
            timeout: float = 3600.0, sysmatrix=None, device_provider: bool = False, cwd=None) -> dict:
    """Runs the .ini on `device` through the driver; returns its JSON record.  With
    `sysmatrix` (a System_Matrix_Settings .ini) it runs the voxel sweep: one
    ensemble per voxel, offset field moved to the voxel's field, Philox key
    seed + voxel number, all batched through the server.  Single-simulation result
    files (Save_single_simulations) are written relative to `cwd`."""
    extra = [f"-sysmatrix:{sysmatrix}"] if sysmatrix else []
    if device_provider:  # particles drawn on the GPU from the same templates
        extra.append("-device-provider")
    return json.loads(_call(_flags(path, seed, precision) + extra + [f"-device:{int(device)}"], timeout, cwd=cwd))


def describe_sysmatrix(path, sysmatrix, seed: int = 0x5EED, timeout: float = 120.0) -> dict:
    """Voxels, their offset fields, keys and file names of a system-matrix sweep (no GPU)."""
    return json.loads(_call(_flags(path, seed, Precision.FP64) + [f"-sysmatrix:{sysmatrix}", "-print"], timeout))
