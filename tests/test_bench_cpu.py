"""bench.py on the CPU: the CPU-baseline sample and the reference arm.

Only whole windows are integrated (sample 0 is the initial state), so a CPU sample
must be sized in windows; a sample shorter than the workload's window would time set-up
alone.  The reference arm must print one JSON line with the driver's keys.
"""
import json
import subprocess
import sys
from pathlib import Path

import bench

ROOT = Path(__file__).resolve().parents[1]


def test_cpu_sample_integrates_the_steps_it_reports():
    for steps in (300, 2000):
        r = bench.cpu_baseline(steps_sample=steps, n=64)
        assert r["value"] > 0 and f"x {steps} integrated steps" in r["sample"]


def test_reference_arm_prints_one_json_line():
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "3",
                        "--n-particles", "512"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr
    lines = [ln for ln in p.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun the reference arm runs on rank 0 alone; the other ranks exit 0 silently."""
    import os
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "3", "--n-particles", "512"], capture_output=True, text=True, timeout=600, cwd=ROOT,
                       env=env)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""


def test_bench_workloads_integrate_whole_windows():
    """Every workload the bench times integrates a positive number of whole windows, the
    count its rates are computed from."""
    from stochasticphysics_b200 import provider
    from stochasticphysics_b200._abi import Precision, Problem
    specs = bench.workload_specs(256, 2 * 4 * 10000 + 2000, Precision.FP32, 0)
    specs += provider.batched_sets(count=64, step_scale=0.02)
    specs += provider.batched_sets(count=64, step_scale=0.006, lissajous=True,
                                   problems=(Problem.Neel, Problem.BrownAndNeelEulerSpherical))
    for s in specs:
        assert s.integrated_steps > 0 and s.integrated_steps % s.oversampling == 0
        assert s.number_of_steps >= 2 * s.oversampling


def test_co_scheduled_shape_passes_the_shape_checks():
    """The bench's side-by-side ensembles take the tuned (here: default) shape with
    CO_CHUNK-step chunks; sp_ensemble_create_shaped accepts it (it stops only at the
    missing context)."""
    import ctypes as C
    from stochasticphysics_b200._abi import DescHolder, Precision, sp_launch_config
    from stochasticphysics_b200.lib import load
    lib = load()
    for spec in bench.workload_specs(bench.N_PER_GPU, 4 * bench.CHUNK, Precision.FP32, 0):
        out = sp_launch_config()
        assert lib.sp_launch_config_for(None, DescHolder(spec).byref(), C.byref(out)) == 0
        shape = dict(out.to_dict(), chunk_steps=bench.CO_CHUNK)
        lc = sp_launch_config(block=shape["block"], persistent=shape["persistent"], chunk_steps=shape["chunk_steps"],
                              particles_per_thread=shape["particles_per_thread"])
        h = C.c_void_p()
        assert lib.sp_ensemble_create_shaped(None, DescHolder(spec).byref(), C.byref(lc), C.byref(h)) == 1
        assert "ctx is NULL" in lib.sp_last_error().decode()
