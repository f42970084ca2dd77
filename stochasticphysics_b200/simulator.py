"""Host-side mirror of the reference's simulation interface, over the C ABI.

``Context.simulate`` is the drop-in for the reference's per-particle loop
(SimulationManager::StartSimulationManager fanning out singleSimulationTask,
Particle_Simulation/Simulator/SimulationManager.h:549-574, plus the
MeanSimulationResult accumulation): one call integrates the whole ensemble
and returns the Results contract {Time, Field, Results (mean), Weight}
(Particle_Simulation/Results/MeanSimulationResult.h:131-141).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from ._abi import (DescHolder, EnsembleSpec, RequestState, ResultBuffers, sp_ensemble_desc, sp_launch_config, sp_result,
                   sp_server_config, sp_stats)
from .lib import check, load


@dataclass
class SimulationResult:
    time: np.ndarray
    field: np.ndarray
    mean: np.ndarray
    weight: np.ndarray
    trajectories: Optional[np.ndarray] = None
    final_state: Optional[np.ndarray] = None
    stats: dict = field(default_factory=dict)
    # un-normalised sum_p w_p r_p[k]: what shards of one ensemble exchange (merge_shards)
    weighted_sum: Optional[np.ndarray] = None


def _stats_dict(st: sp_stats) -> dict:
    return {"particle_steps": st.particle_steps, "nonfinite_particles": st.nonfinite_particles,
            "newton_iterations": st.newton_iterations, "newton_unconverged": st.newton_unconverged,
            "kernel_launches": st.kernel_launches, "device_ms": st.device_ms, "queue_ms": st.queue_ms,
            "setup_ms": st.setup_ms, "run_ms": st.run_ms, "readback_ms": st.readback_ms}


def _result(buf: ResultBuffers, st: sp_stats) -> SimulationResult:
    return SimulationResult(time=buf.time, field=buf.field, mean=buf.mean, weight=buf.weight,
                            trajectories=buf.trajectories, final_state=buf.final_state, stats=_stats_dict(st),
                            weighted_sum=buf.weighted_sum)


def merge_shards(weighted_sums, weights):
    """Ensemble mean, weighted sums and weights of the union of shards of one description
    (sp_merge_shards: MeanSimulationResult::operator+= over the shards in order, then
    normalize; Particle_Simulation/Results/MeanSimulationResult.h:63-119).  Inputs are each
    shard's ``weighted_sum`` [n_samples][out_dim] and ``weight`` [out_dim]."""
    sums = [np.ascontiguousarray(s, dtype=np.float64) for s in weighted_sums]
    ws = [np.ascontiguousarray(w, dtype=np.float64) for w in weights]
    if not sums or len(sums) != len(ws):
        raise ValueError("one weight vector per shard is needed")
    k, od = sums[0].shape
    if any(s.shape != (k, od) for s in sums) or any(w.shape != (od,) for w in ws):
        raise ValueError("every shard needs weighted_sum [n_samples][out_dim] and weight [out_dim] of one shape")
    dp = C.POINTER(C.c_double)
    sp_arr = (dp * len(sums))(*[s.ctypes.data_as(dp) for s in sums])
    w_arr = (dp * len(ws))(*[w.ctypes.data_as(dp) for w in ws])
    mean, tot, wt = np.zeros((k, od)), np.zeros((k, od)), np.zeros(od)
    check(load().sp_merge_shards(len(sums), k, od, sp_arr, w_arr, mean.ctypes.data_as(dp), tot.ctypes.data_as(dp),
                                 wt.ctypes.data_as(dp)))
    return mean, tot, wt


class Context:
    """One CUDA device.  Owns a library context (sp_create/sp_destroy)."""

    def __init__(self, device: int = 0):
        self._lib = load()
        h = C.c_void_p()
        check(self._lib.sp_create(C.byref(h), device))
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            check(self._lib.sp_destroy(self.handle))
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    # -------------------------------------------------------------- synchronous drop-in
    def simulate(self, spec: EnsembleSpec, trajectories: bool = False, final_state: bool = False) -> SimulationResult:
        h = DescHolder(spec)
        buf = ResultBuffers(spec, trajectories=trajectories, final_state=final_state)
        st = sp_stats()
        check(self._lib.sp_simulate(self.handle, h.byref(), C.byref(buf.c), C.byref(st)))
        return _result(buf, st)

    def ensemble(self, spec: EnsembleSpec, shape: Optional[dict] = None) -> "DeviceEnsemble":
        """A device-resident ensemble; `shape` (keys block, persistent, chunk_steps,
        particles_per_thread, as :meth:`launch_config` returns them) replaces the tuned
        launch shape (sp_ensemble_create_shaped)."""
        return DeviceEnsemble(self, spec, shape)

    def server(self, memory_budget_bytes: int = 0, chunk_steps: int = 0, max_active: int = 0) -> "Server":
        return Server(self, memory_budget_bytes, chunk_steps, max_active)

    def philox_normals(self, seed: int, pid0: int, n: int, step0: int, nsteps: int, noise_dim: int,
                       precision: int = 0) -> np.ndarray:
        out = np.zeros((nsteps, noise_dim, n))
        check(self._lib.sp_debug_philox_normals(self.handle, seed, pid0, n, step0, nsteps, noise_dim, precision,
                                                out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def fma_peak_tflops(self, precision: int) -> float:
        """Measured FMA throughput of the device (TFLOP/s); precision 0 = FP64, 1 = FP32."""
        v = C.c_double()
        check(self._lib.sp_measure_fma_peak(self.handle, int(precision), C.byref(v)))
        return float(v.value)

    def autotune(self, spec: EnsembleSpec, probe_particles: int = 65536) -> dict:
        """Times the candidate launch shapes for spec's kernel key on a probe of its
        particles and caches the fastest in this process (sp_autotune)."""
        best = sp_launch_config()
        cands = (sp_launch_config * 16)()
        n = C.c_int32()
        check(self._lib.sp_autotune(self.handle, DescHolder(spec).byref(), int(probe_particles), C.byref(best),
                                    cands, 16, C.byref(n)))
        return {"best": best.to_dict(), "candidates": [cands[i].to_dict() for i in range(min(n.value, 16))]}

    def launch_config(self, spec: EnsembleSpec) -> dict:
        """Launch shape the library uses for spec now (tuned or default)."""
        out = sp_launch_config()
        check(self._lib.sp_launch_config_for(self.handle, DescHolder(spec).byref(), C.byref(out)))
        return out.to_dict()

    @staticmethod
    def tuning_save(path) -> None:
        check(load().sp_tuning_save(str(path).encode()))

    @staticmethod
    def tuning_load(path) -> None:
        check(load().sp_tuning_load(str(path).encode()))

    @staticmethod
    def tuning_reset() -> None:
        check(load().sp_tuning_reset())

    def provide_particles(self, spec: EnsembleSpec) -> np.ndarray:
        """The particles spec.provider draws on the device: [n][20] columns magnetic_radius,
        saturation_magnetisation, damping_constant, gyromagnetic_ratio, anisotropy_constant,
        hydrodynamic_radius, viscosity, orientation[3], magnetisation[3], cubic_constant,
        uniaxial_rotation[3], template index, reserved[2]."""
        out = np.zeros((int(spec.n), 20))
        check(self._lib.sp_provide_particles(self.handle, DescHolder(spec).byref(),
                                             out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    @staticmethod
    def footprint(spec: EnsembleSpec) -> int:
        h = DescHolder(spec)
        v = C.c_uint64()
        check(load().sp_ensemble_footprint(h.byref(), C.byref(v)))
        return int(v.value)


class DeviceEnsemble:
    """A device-resident ensemble: inputs uploaded once, advanced chunk by chunk."""

    def __init__(self, ctx: Context, spec: EnsembleSpec, shape: Optional[dict] = None):
        self.ctx, self.spec = ctx, spec
        self._lib = ctx._lib
        self._holder = DescHolder(spec)
        h = C.c_void_p()
        if shape is None:
            check(self._lib.sp_ensemble_create(ctx.handle, self._holder.byref(), C.byref(h)))
        else:
            lc = sp_launch_config(block=int(shape["block"]), persistent=int(shape["persistent"]),
                                  chunk_steps=int(shape["chunk_steps"]),
                                  particles_per_thread=int(shape.get("particles_per_thread", 1)))
            check(self._lib.sp_ensemble_create_shaped(ctx.handle, self._holder.byref(), C.byref(lc), C.byref(h)))
        self.handle = h

    def advance(self, n_steps: int, stream: Optional[int] = None) -> None:
        check(self._lib.sp_ensemble_advance(self.handle, int(n_steps), C.c_void_p(stream or 0)))

    def steps(self):
        d, t = C.c_uint64(), C.c_uint64()
        check(self._lib.sp_ensemble_steps_done(self.handle, C.byref(d), C.byref(t)))
        return int(d.value), int(t.value)

    def read(self, trajectories: bool = False, final_state: bool = False) -> SimulationResult:
        buf = ResultBuffers(self.spec, trajectories=trajectories, final_state=final_state)
        st = sp_stats()
        check(self._lib.sp_ensemble_read(self.handle, C.byref(buf.c), C.byref(st)))
        return _result(buf, st)

    def close(self):
        if self.handle:
            check(self._lib.sp_ensemble_destroy(self.handle))
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


class Server:
    """Continuous-batching server (sp_server_*): submit at any time, wait for results."""

    def __init__(self, ctx: Context, memory_budget_bytes: int = 0, chunk_steps: int = 0, max_active: int = 0,
                 groups_per_kind: int = 0):
        self.ctx = ctx
        self._lib = ctx._lib
        cfg = sp_server_config()
        cfg.memory_budget_bytes = int(memory_budget_bytes)
        cfg.chunk_steps = int(chunk_steps)
        cfg.max_active = int(max_active)
        cfg.groups_per_kind = int(groups_per_kind)
        h = C.c_void_p()
        check(self._lib.sp_server_create(ctx.handle, C.byref(cfg), C.byref(h)))
        self.handle = h
        self._specs = {}

    def submit(self, spec: EnsembleSpec) -> int:
        holder = DescHolder(spec)
        rid = C.c_uint64()
        check(self._lib.sp_server_submit(self.handle, holder.byref(), C.byref(rid)))
        self._specs[int(rid.value)] = spec
        return int(rid.value)

    def submit_many(self, specs) -> list:
        """Queues all specs at once (sp_server_submit_many): an idle server admits them
        together.  All or nothing."""
        holders = [DescHolder(sp_) for sp_ in specs]
        arr = (sp_ensemble_desc * len(holders))(*[h.desc for h in holders])
        rids = (C.c_uint64 * len(holders))()
        check(self._lib.sp_server_submit_many(self.handle, arr, len(holders), rids))
        out = [int(r) for r in rids]
        for rid, spec in zip(out, specs):
            self._specs[rid] = spec
        return out

    def poll(self, rid: int) -> RequestState:
        s = C.c_int32()
        check(self._lib.sp_server_poll(self.handle, rid, C.byref(s)))
        return RequestState(s.value)

    def wait(self, rid: int, timeout_ms: float = -1.0):
        spec = self._specs[rid]
        buf = ResultBuffers(spec)
        st = sp_stats()
        lat = C.c_double()
        check(self._lib.sp_server_wait(self.handle, rid, float(timeout_ms), C.byref(buf.c), C.byref(st), C.byref(lat)))
        return _result(buf, st), float(lat.value)

    def cancel(self, rid: int) -> None:
        check(self._lib.sp_server_cancel(self.handle, rid))

    def close(self):
        if self.handle:
            check(self._lib.sp_server_destroy(self.handle))
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def kernel_launch_count() -> int:
    return int(load().sp_kernel_launch_count())
