"""Autotuner cache on the CPU: load / save / reset and the shape lookup.

sp_autotune itself times kernels (GPU test in test_gpu_tuning.py); the cache it
fills is plain host state keyed by problem/anisotropy/solver/precision/noise.
"""
import ctypes as C

import pytest

from stochasticphysics_b200 import provider
from stochasticphysics_b200._abi import DescHolder, Precision, Solver, sp_launch_config
from stochasticphysics_b200.lib import load


def _shape(spec):
    out = sp_launch_config()
    assert load().sp_launch_config_for(None, DescHolder(spec).byref(), C.byref(out)) == 0, load().sp_last_error()
    return out.to_dict()


@pytest.fixture(autouse=True)
def clean_cache():
    load().sp_tuning_reset()
    yield
    load().sp_tuning_reset()


def test_defaults_without_tuning():
    spec = provider.brown_neel_relaxation(n=65536, steps=20000, oversampling=1000, precision=Precision.FP32)
    s = _shape(spec)
    # CTA size halved from 256 until there are >= 2 CTAs per SM (148 SMs), down to 32
    assert s == {"block": 128, "persistent": 0, "chunk_steps": 10000, "particles_per_thread": 1,
                 "particle_steps_per_s": 0.0}
    small = provider.brown_neel_relaxation(n=4000, steps=20000, oversampling=1000)
    assert _shape(small)["block"] == 32


def test_loaded_shape_applies_to_its_key_only(tmp_path):
    bn = provider.brown_neel_relaxation(n=65536, steps=20000, oversampling=1000, solver=Solver.Millstein,
                                        precision=Precision.FP32)
    key = f"{int(bn.problem)}/{int(bn.anisotropy)}/{int(bn.solver)}/{int(bn.precision)}/{int(bn.noise)}"
    f = tmp_path / "tune.txt"
    f.write_text(f"{key} 128 1 30000 1.5e10\n")
    assert load().sp_tuning_load(str(f).encode()) == 0
    assert _shape(bn) == {"block": 128, "persistent": 1, "chunk_steps": 30000, "particles_per_thread": 1,
                          "particle_steps_per_s": 1.5e10}
    heun = provider.brown_neel_relaxation(n=65536, steps=20000, oversampling=1000, solver=Solver.Heun_Strong,
                                          precision=Precision.FP32)
    assert _shape(heun)["persistent"] == 0 and _shape(heun)["block"] == 128
    # chunks stay whole windows; small ensembles still cover the SMs
    odd = provider.brown_neel_relaxation(n=65536, steps=70000, oversampling=7000, solver=Solver.Millstein,
                                         precision=Precision.FP32)
    assert _shape(odd)["chunk_steps"] == 28000
    tiny = provider.brown_neel_relaxation(n=5000, steps=20000, oversampling=1000, solver=Solver.Millstein,
                                          precision=Precision.FP32)
    assert _shape(tiny)["block"] == 32


def test_particles_per_thread(tmp_path):
    """Two particles per thread are kept for FP32 in-kernel-noise keys with tiles of at
    least 64 particles, and fall back to one otherwise (FP64 has no such kernel)."""
    f32 = provider.brown_neel_relaxation(n=65536, steps=20000, oversampling=1000, solver=Solver.Millstein,
                                         precision=Precision.FP32)
    f64 = provider.brown_neel_relaxation(n=65536, steps=20000, oversampling=1000, solver=Solver.Millstein)
    tiny = provider.brown_neel_relaxation(n=5000, steps=20000, oversampling=1000, solver=Solver.Millstein,
                                          precision=Precision.FP32)
    k32 = f"{int(f32.problem)}/{int(f32.anisotropy)}/{int(f32.solver)}/1/0"
    k64 = f"{int(f64.problem)}/{int(f64.anisotropy)}/{int(f64.solver)}/0/0"
    f = tmp_path / "tune.txt"
    f.write_text(f"{k32} 128 0 10000 3e10 2\n{k64} 128 0 10000 6e9 2\n")
    assert load().sp_tuning_load(str(f).encode()) == 0
    assert _shape(f32)["particles_per_thread"] == 2
    assert _shape(f64)["particles_per_thread"] == 1
    assert _shape(tiny)["block"] == 32 and _shape(tiny)["particles_per_thread"] == 1
    g = tmp_path / "saved.txt"
    assert load().sp_tuning_save(str(g).encode()) == 0
    assert f"{k32} 128 0 10000 3e+10 2" in g.read_text()


def test_save_load_roundtrip_and_reset(tmp_path):
    a = tmp_path / "a.txt"
    a.write_text("0/0/1/1/0 64 0 20000 2e10\n2/0/2/0/0 256 1 10000 4e9\n")
    assert load().sp_tuning_load(str(a).encode()) == 0
    b = tmp_path / "b.txt"
    assert load().sp_tuning_save(str(b).encode()) == 0
    assert sorted(b.read_text().split("\n")) == sorted(["0/0/1/1/0 64 0 20000 2e+10 1", "2/0/2/0/0 256 1 10000 4e+09 1",
                                                         ""])
    load().sp_tuning_reset()
    c = tmp_path / "c.txt"
    assert load().sp_tuning_save(str(c).encode()) == 0
    assert c.read_text() == ""


@pytest.mark.parametrize("text", ["0/0/1/1 64 0 100 1\n", "0/0/1/1/0 48 0 100 1\n", "0/0/1/1/0 64 0\n",
                                  "0/0/1/1/0 64 0 0 1\n", "0/0/1/1/0 64 0 100 1 3\n"])
def test_malformed_tuning_files_are_refused(tmp_path, text):
    f = tmp_path / "bad.txt"
    f.write_text(text)
    assert load().sp_tuning_load(str(f).encode()) == 1
    assert load().sp_tuning_load(str(tmp_path / "missing.txt").encode()) == 1


def test_shaped_create_checks_the_shape_before_the_device():
    """sp_ensemble_create_shaped refuses malformed shapes before it needs a context, so
    the checks run here without a GPU; a well-formed shape then needs the context."""
    spec = provider.brown_neel_relaxation(n=4096, steps=20000, oversampling=1000, precision=Precision.FP32)
    good = dict(block=64, persistent=1, chunk_steps=1500, particles_per_thread=2)
    h = C.c_void_p()
    lib = load()
    cases = [({}, "ctx is NULL"), ({"block": 96}, "shape.block"), ({"persistent": 2}, "shape.persistent"),
             ({"chunk_steps": 0}, "shape.chunk_steps"), ({"particles_per_thread": 0}, "shape.particles_per_thread")]
    for change, message in cases:
        lc = sp_launch_config(**dict(good, **change))
        assert lib.sp_ensemble_create_shaped(None, DescHolder(spec).byref(), C.byref(lc), C.byref(h)) == 1
        assert message in lib.sp_last_error().decode()
    lc = sp_launch_config(**good)
    assert lib.sp_ensemble_create_shaped(None, DescHolder(spec).byref(), C.byref(lc), None) == 1
    assert "ens is NULL" in lib.sp_last_error().decode()
