"""ctypes front-end of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY.  The oracle is the checker: it may be imported by
tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and by
nothing in the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from stochasticphysics_b200._abi import DescHolder, EnsembleSpec

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
_lib = None
_dp = C.POINTER(C.c_double)


def build(force: bool = False) -> Path:
    """Compile liboracle.so with the committed Makefile."""
    if force or not LIB_PATH.exists():
        subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        L.oracle_simulate.restype = C.c_int
        L.oracle_simulate.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_uint64), C.c_int, C.c_int]
        L.oracle_philox_normals.restype = None
        L.oracle_philox_normals.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_int, _dp]
        L.oracle_philox4x32_10.restype = None
        L.oracle_philox4x32_10.argtypes = [C.POINTER(C.c_uint32)] * 3
        L.oracle_neel_params.restype = None
        L.oracle_neel_params.argtypes = [C.c_double] * 5 + [_dp]
        L.oracle_brown_params.restype = None
        L.oracle_brown_params.argtypes = [C.c_double] * 3 + [_dp]
        L.oracle_uniaxial.restype = None
        L.oracle_uniaxial.argtypes = [C.c_double] * 3 + [_dp] * 4
        L.oracle_cubic.restype = None
        L.oracle_cubic.argtypes = [C.c_double] * 3 + [_dp] * 8
        L.oracle_eval_problem.restype = C.c_int
        L.oracle_eval_problem.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_double, _dp,
                                          _dp, _dp, _dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_int), C.c_int]
        L.oracle_provide_particles.restype = None
        L.oracle_provide_particles.argtypes = [C.c_void_p, _dp]
        L.oracle_field_eval.restype = None
        L.oracle_field_eval.argtypes = [C.c_void_p, _dp, C.c_uint64, _dp]
        L.oracle_neel_exact_jacobians.restype = None
        L.oracle_neel_exact_jacobians.argtypes = [C.c_int] + [_dp] * 7
        L.oracle_double_noise_matrix.restype = None
        L.oracle_double_noise_matrix.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_int, C.c_double,
                                                 C.c_int, _dp, _dp]
        L.oracle_count_ops.restype = C.c_int
        L.oracle_count_ops.argtypes = [C.c_void_p, _dp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def simulate(spec: EnsembleSpec, trajectories: bool = False, final_state: bool = False, threads: int = 0,
             long_double: bool = False) -> dict:
    """Run the ensemble on the CPU; returns mean, weight, time, field (+ optional per-particle outputs)."""
    h = DescHolder(spec)
    k = spec.n_samples
    sd, _, od = spec.dims
    out = {"mean": np.zeros((k, od)), "weight": np.zeros(od), "time": np.zeros(k), "field": np.zeros((k, 3))}
    tr = np.zeros((spec.n, k, od)) if trajectories else None
    fs = np.zeros((spec.n, sd)) if final_state else None
    ns = (C.c_uint64 * 2)()
    rc = lib().oracle_simulate(C.addressof(h.desc), _p(out["mean"]), _p(out["weight"]), _p(out["time"]),
                               _p(out["field"]), _p(tr), _p(fs), ns, int(threads), 1 if long_double else 0)
    if rc != 0:
        raise RuntimeError(f"oracle_simulate failed with code {rc}")
    if tr is not None:
        out["trajectories"] = tr
    if fs is not None:
        out["final_state"] = fs
    out["newton_iterations"] = int(ns[0])
    out["newton_unconverged"] = int(ns[1])
    return out


def philox_normals(seed: int, pid0: int, n: int, step0: int, nsteps: int, m: int) -> np.ndarray:
    out = np.zeros((nsteps, m, n))
    lib().oracle_philox_normals(seed, pid0, n, step0, nsteps, m, _p(out))
    return out


def double_noise_matrix(seed: int, pid0: int, n: int, step: int, p: int, dt: float, m: int):
    """(dW[n][m], J[n][m][m]) of WeakTest / ExplicitStrong_1.0 at one step."""
    dw = np.zeros((n, m))
    J = np.zeros((n, m, m))
    lib().oracle_double_noise_matrix(seed, pid0, n, step, p, dt, m, _p(dw), _p(J))
    return dw, J


def philox4x32_10(ctr, key) -> list:
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().oracle_philox4x32_10(c, k, o)
    return list(o)


def neel_params(radius, Ms, alpha, gamma, temperature) -> dict:
    o = np.zeros(5)
    lib().oracle_neel_params(radius, Ms, alpha, gamma, temperature, _p(o))
    return dict(zip(["NeelFactor1", "NeelFactor2", "DriftPrefactor", "NoisePrefactor", "Damping"], o.tolist()))


def brown_params(rh, viscosity, temperature) -> dict:
    o = np.zeros(3)
    lib().oracle_brown_params(rh, viscosity, temperature, _p(o))
    return dict(zip(["BrownPrefactor", "BrownDiffusion", "Brown_F_Noise"], o.tolist()))


def uniaxial(K, Ms, radius, m, axis):
    f, j = np.zeros(3), np.zeros(9)
    lib().oracle_uniaxial(K, Ms, radius, _p(np.asarray(m, float)), _p(np.asarray(axis, float)), _p(f), _p(j))
    return f, j.reshape(3, 3)


def cubic(K1, Ms, radius, m, x, y, z, statesin, statecos):
    f, t = np.zeros(3), np.zeros(3)
    a = [np.ascontiguousarray(v, dtype=float) for v in (m, x, y, z, statesin, statecos)]
    lib().oracle_cubic(K1, Ms, radius, *[_p(v) for v in a], _p(f), _p(t))
    return f, t


STATE_DIM = {0: 3, 1: 2, 2: 5, 3: 6}
NOISE_DIM = {0: 3, 1: 3, 2: 6, 3: 6}


def eval_problem(problem: int, aniso: int, props, euler, settings, state, field=None, dt=0.0, dW=None,
                 finish_jacobi: bool = False) -> dict:
    """prepareCalculations(state) then every problem piece, as the reference unit tests do."""
    d, m = STATE_DIM[problem], NOISE_DIM[problem]
    props = np.ascontiguousarray(props, dtype=float)
    euler = np.ascontiguousarray(euler, dtype=float)
    settings = np.ascontiguousarray(settings, dtype=float)
    state = np.ascontiguousarray(state, dtype=float)
    fld = None if field is None else np.ascontiguousarray(field, dtype=float)
    w = None if dW is None else np.ascontiguousarray(dW, dtype=float)
    out = {"prepared": np.zeros(d), "a": np.zeros(d), "b": np.zeros((d, m)), "drift": np.zeros(d),
           "jdet": np.zeros((d, d)), "jsto": np.zeros((d, d)), "finished": np.zeros(d)}
    rot = (C.c_int * 2)()
    rc = lib().oracle_eval_problem(problem, aniso, _p(props), _p(euler), _p(settings), _p(state), _p(fld), dt, _p(w),
                                   _p(out["prepared"]), _p(out["a"]), _p(out["b"]), _p(out["drift"]),
                                   _p(out["jdet"]), _p(out["jsto"]), _p(out["finished"]), rot,
                                   1 if finish_jacobi else 0)
    if rc != 0:
        raise RuntimeError(f"oracle_eval_problem failed ({rc})")
    out["rotated"] = (bool(rot[0]), bool(rot[1]))
    return out


def provide_particles(spec: EnsembleSpec) -> np.ndarray:
    """The particles spec.provider draws: [n][20] as sp_provide_particles writes them."""
    h = DescHolder(spec)
    out = np.zeros((int(spec.n), 20))
    lib().oracle_provide_particles(C.addressof(h.desc), _p(out))
    return out


def field_eval(field, times) -> np.ndarray:
    """B(t) [len(times)][3] of a FieldSpec."""
    f = field.to_c()
    t = np.ascontiguousarray(times, dtype=float)
    out = np.zeros((t.size, 3))
    lib().oracle_field_eval(C.addressof(f), _p(t), t.size, _p(out))
    return out


def neel_exact_jacobians(aniso: int, props, euler, m, field, dW):
    """Analytic d a/d m and d (b(m) dW)/d m of the Neel (Cartesian) problem.
    props: radius, Ms, alpha, gamma, K, temperature."""
    arr = [np.ascontiguousarray(v, dtype=float) for v in (props, euler, m, field, dW)]
    jd, js = np.zeros((3, 3)), np.zeros((3, 3))
    lib().oracle_neel_exact_jacobians(int(aniso), *[_p(a) for a in arr], _p(jd), _p(js))
    return jd, js


def count_ops(spec: EnsembleSpec) -> dict:
    """Per-step adds+muls (FMA = 2), divisions, transcendentals, sqrts, Newton iterations."""
    h = DescHolder(spec)
    o = np.zeros(5)
    rc = lib().oracle_count_ops(C.addressof(h.desc), _p(o))
    if rc != 0:
        raise RuntimeError(f"oracle_count_ops failed ({rc})")
    return dict(zip(["flops", "divs", "transcendentals", "sqrts", "newton_iterations"], o.tolist()))


def cpu_threads() -> int:
    return os.cpu_count() or 1
