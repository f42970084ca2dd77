"""Benchmark: particle-steps/s of ensemble SDE integration on B200.

Workload (one GPU, weak scaling across GPUs): the coupled Brown+Neel relaxation,
BrownAndNeelEulerSpherical with the Milstein and Heun steppers, 65536 polydisperse
particles per GPU (lognormal cores, median 10 nm, sigma 0.1; hydrodynamic radius
= core + 20 nm; eta = 1e-3 Pa s; K ~ U[5e3, 2e4] J/m^3; alpha = 0.1; T = 295 K;
20 mT at 25 kHz; dt = 1e-11 s; samples every 1000 steps).  Inputs are seeded
synthetic data with those distributions.

One bench step = one chunk of 10000 SDE steps for both ensembles (Milstein and
Heun) on the device-resident state, i.e. 2 x 65536 x 10000 particle-steps.

  value        FP32 form (FP32 stepping; FP64 time, field phase, window and ensemble
               sums), device-resident, the two ensembles side by side on two streams in
               1000-step chunk launches, CUDA-event timed, max over ranks
  fp64_plain   the same steps with the plain FP64 kernel
  e2e          the same metric through the public C ABI with host buffers: per step
               both ensembles submitted together to the server (sp_server_submit_many;
               upload, 10000 steps, results back); sp_simulate one after the other is
               reported beside it
  cpu_baseline the CPU oracle (restatement of the reference formulas) on all host
               cores, rank 0 only, on a bounded sample of the same workload
  serving      continuous-batching leg (N=1): Poisson arrivals of mixed Neel /
               BrownAndNeelEulerSpherical requests (batched-set distributions, 2D
               Lissajous field) through sp_server_*, FP32; p50/p99 latency,
               aggregate particle-steps/s, and the same requests one at a time in
               FP64 as the serial baseline
  batched      256 Neel parameter sets (uneven N and S, the stated sizes: about 8e12
               particle-steps) submitted at once, batched per kernel key into shared
               launches (N=1)
  serving_overload  the serving arrivals with full-length requests for a fixed window:
               saturated rate, requests in flight over time, latency of those finished
  plain_neel_1024  the 1024-particle FP64 Neel run of 1e6 steps (latency-bound small
               ensemble), whole run on the device and end to end, beside the CPU
  stiff        the cubic ImplicitMidpoint workload (262144 particles, dt = 1e-10 s):
               FP64 with the reference's Newton matrix, FP64 and FP32 with the exact one
  injected     injection mode (caller-supplied dW read from HBM every step), Neel Heun,
               65536 particles, FP64 and FP32: particle-steps/s and dW GB/s vs HBM peak
  ensemble_sizes  the workload one ensemble at a time at 16k to 1M particles, FP32 and
               FP64 (a 65536-particle ensemble alone does not fill the GPU)
  --impl reference  runs that CPU restatement as the reference arm

Launch shapes come from the autotuner (sp_autotune) unless --no-autotune.

Run:  python bench.py [--gpus N --steps K --warmup W]
      torchrun --nproc-per-node N bench.py --gpus N ...
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CHUNK = 10000          # SDE steps per bench step
# Steps per chunk launch of the co-scheduled ensembles: a launch ends with its CTAs
# draining, and the other ensemble's next launch fills the SMs so freed; the tuned (lone
# ensemble) chunk of 10000-40000 steps leaves them idle for longer.
CO_CHUNK = 1000
N_PER_GPU = 65536
METRIC = "particle-steps/s/GPU: FP32 served vs FP64 plain at <=1e-3 mean-M error; p99 ms"
UNIT = "particle-steps/s"
THROTTLE_BITS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
                 0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown", 0x2: "applications_clocks_setting",
                 0x1: "gpu_idle"}


def workload_specs(n, steps, precision, rank):
    from stochasticphysics_b200 import provider
    from stochasticphysics_b200._abi import Solver
    specs = []
    for solver in (Solver.Millstein, Solver.Heun_Strong):
        s = provider.brown_neel_relaxation(n=n * (rank + 1), steps=steps, oversampling=1000, solver=solver,
                                           precision=precision)
        specs.append(s.subset(n * rank, n * (rank + 1)))  # global particle ids: shards of one ensemble
    return specs


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index):
        self.index, self.samples, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 4:
                try:
                    self.samples.append((float(parts[0]), float(parts[1]), float(parts[2]), int(parts[3], 16)))
                except ValueError:
                    pass

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        busy = [s for s in self.samples if s[2] > 200.0] or self.samples
        reasons = set()
        for s in busy:
            for bit, name in THROTTLE_BITS.items():
                if s[3] & bit and name != "gpu_idle":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(s[0] for s in busy), "sm_max_mhz": max(s[1] for s in busy),
                "power_w_max": max(s[2] for s in busy), "samples": len(busy), "reasons": sorted(reasons)}


def profiled_traffic_per_particle():
    """DRAM bytes per particle per step-kernel launch from the committed ncu summary
    (dram__bytes_read.sum + dram__bytes_write.sum of one capture, divided by the
    captured launch's particles); the traffic of a launch scales with particles, not
    steps (state, Kahan sums and prefactors are read once and written once)."""
    import re
    path = ROOT / "profiles" / "step_kernel_brown_neel_euler_65536.md"
    try:
        m = re.search(r"traffic_bytes_per_particle_per_launch:\s*([0-9.eE+-]+)", path.read_text())
    except OSError:
        return None, None
    return (float(m.group(1)), path.name) if m else (None, None)


def profiled_instructions(prefix=""):
    """Thread-instructions per particle-step of the step kernels (Millstein, Heun), from the
    committed ncu summary: FP32 (prefix "") or FP64 (prefix "fp64_")."""
    import re
    path = ROOT / "profiles" / "step_kernel_instruction_counts_65536.md"
    try:
        text = path.read_text()
    except OSError:
        return None, None
    m = re.search(rf"thread_instructions_per_particle_step_{prefix}millstein:\s*([0-9.]+)", text)
    h = re.search(rf"thread_instructions_per_particle_step_{prefix}heun:\s*([0-9.]+)", text)
    return ((float(m.group(1)), float(h.group(1))) if m and h else None), path.name


def profiled_pipes():
    """FP64-pipe and FP32 FMA-pipe utilisation of the step kernels (ncu
    sm__pipe_fp64_cycles_active / sm__inst_executed_pipe_fma, pct of peak) from the
    committed ncu summary, keyed "<precision>_<solver>"."""
    import re
    path = ROOT / "profiles" / "step_kernel_brown_neel_euler_65536.md"
    try:
        text = path.read_text()
    except OSError:
        return None
    out = {m.group(1): float(m.group(2)) for m in re.finditer(r"pipe_pct_(\w+):\s*([0-9.]+)", text)}
    return out or None


def serving_leg(ctx, seconds, rate, step_scale, seed=0x5EED0005, serial_sample=48, chunk_steps=0):
    """Poisson arrivals of mixed Neel / BrownAndNeelEulerSpherical requests with the
    batched-set distributions and the 2D Lissajous field, served by the continuous-
    batching server in FP32; latency = submit -> result ready (server clock).  The
    same requests, one at a time through the plain FP64 path (every k-th request, at
    most serial_sample), give the serial baseline and the FP32-vs-FP64 mean error."""
    import numpy as np

    import stochasticphysics_b200 as sp
    from stochasticphysics_b200 import provider
    from stochasticphysics_b200._abi import Precision, Problem

    rng = np.random.default_rng(seed)
    arrivals = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > seconds:
            break
        arrivals.append(t)
    specs = provider.batched_sets(count=len(arrivals), seed=seed, precision=Precision.FP32, step_scale=step_scale,
                                  lissajous=True, problems=(Problem.Neel, Problem.BrownAndNeelEulerSpherical))
    free, _ = __import__("torch").cuda.mem_get_info()
    budget = int(min(150e9, 0.8 * free))
    ids = [None] * len(specs)
    with sp.Server(ctx, memory_budget_bytes=budget, chunk_steps=chunk_steps) as srv:
        def submitter():
            t0 = time.perf_counter()
            for i, (ta, spec) in enumerate(zip(arrivals, specs)):
                d = t0 + ta - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                ids[i] = srv.submit(spec)
        th = threading.Thread(target=submitter)
        t_start = time.perf_counter()
        th.start()
        lat, served, phases = [], [], []
        for i in range(len(specs)):
            while ids[i] is None:
                time.sleep(0.0005)
            res, ms = srv.wait(ids[i])
            lat.append(ms)
            served.append(res.mean)
            phases.append([res.stats[k] for k in ("queue_ms", "setup_ms", "run_ms", "readback_ms")])
        t_end = time.perf_counter()
        th.join()
    ps = [s.n * s.integrated_steps for s in specs]
    k = max(1, len(specs) // serial_sample)
    sample = list(range(0, len(specs), k))[:serial_sample]
    serial_s, errs = 0.0, []
    for i in sample:
        s64 = dataclasses.replace(specs[i], precision=Precision.FP64)
        t = time.perf_counter()
        r64 = ctx.simulate(s64)
        serial_s += time.perf_counter() - t
        cols = slice(6, 9) if specs[i].problem == Problem.BrownAndNeelEulerSpherical else slice(0, 3)
        d = float(np.max(np.abs(served[i][:, cols] - r64.mean[:, cols])))
        errs.append((d, d / math.sqrt(2.0 / (3.0 * specs[i].n))))
    lat_s = sorted(lat)
    ph = np.array(phases)
    slowest = np.argsort(lat)[::-1][:max(1, len(lat) // 100)]
    breakdown = {
        "p50_ms": {k: float(np.percentile(ph[:, j], 50)) for j, k in enumerate(("queue", "setup", "run", "readback"))},
        "p99_ms": {k: float(np.percentile(ph[:, j], 99)) for j, k in enumerate(("queue", "setup", "run", "readback"))},
        "slowest_1pct": [{"latency_ms": float(lat[i]), "queue_ms": float(ph[i, 0]), "setup_ms": float(ph[i, 1]),
                          "run_ms": float(ph[i, 2]), "readback_ms": float(ph[i, 3]), "particles": int(specs[i].n),
                          "steps": int(specs[i].integrated_steps), "problem": specs[i].problem.name}
                         for i in slowest],
        "note": "server host clock per request: queue = submit -> admission, setup = upload and init, run = the "
                "rounds until its last window, readback = result copy; run covers the rounds the request shares "
                "with the others in flight",
    }
    return {
        "requests": len(specs), "arrival_rate_per_s": rate, "arrival_window_s": seconds,
        "p50_ms": float(np.percentile(lat_s, 50)), "p99_ms": float(np.percentile(lat_s, 99)),
        "max_ms": float(lat_s[-1]), "latency_breakdown": breakdown, "value": sum(ps) / (t_end - t_start), "unit": UNIT,
        "offered_particle_steps_per_s": sum(ps) / seconds, "memory_budget_bytes": budget,
        "serial_fp64": {"value": sum(ps[i] for i in sample) / serial_s, "unit": UNIT, "requests": len(sample),
                        "note": "same requests one at a time through sp_simulate in FP64 (every k-th request)"},
        "fp32_vs_fp64_mean_m": {"max_abs_diff": max(e[0] for e in errs),
                                "max_diff_over_two_sample_se": max(e[1] for e in errs)},
        "workload": f"Poisson {rate}/s for {seconds} s; N ~ logU[1e3, 6.4e4], S ~ logU[1e5, 1e7] x {step_scale} "
                    "(whole windows of 1000 steps, >= 2 windows); Neel or BrownAndNeelEulerSpherical (p = 1/2), "
                    "Heun / Millstein alternating, FP32; Lissajous 12 mT at 25.25 kHz (x) and 26.04 kHz (y); "
                    "dt = 1e-11 s",
    }


def plain_fp64_rate(ctx, specs, max_steps):
    """The plain FP64 drop-in on the given requests one at a time (sp_simulate, FP64, each
    run cut to at most max_steps integrated steps in whole windows: a long request's rate
    does not depend on its length): particle-steps/s of the whole sample."""
    from stochasticphysics_b200._abi import Precision
    ps, sec = 0, 0.0
    for s in specs:
        W = s.oversampling
        steps = min(s.number_of_steps, (max_steps // W + 1) * W)
        r = dataclasses.replace(s, precision=Precision.FP64, number_of_steps=steps)
        t = time.perf_counter()
        ctx.simulate(r)
        sec += time.perf_counter() - t
        ps += r.n * r.integrated_steps
    return ps / sec


def overload_leg(ctx, arrival_s=2.0, observe_s=30.0, rate=50.0, seed=0x5EED0005):
    """The serving workload at its stated size: Poisson arrivals at `rate`/s for `arrival_s`
    seconds of full-length requests (N ~ logU[1e3, 6.4e4], S ~ logU[1e5, 1e7], Neel or
    BrownAndNeelEulerSpherical, Lissajous field, FP32).  The offered load, about 50 x 1.5e4 x
    2.15e6 = 1.6e12 particle-steps/s, is some 30x what one B200 integrates, so the server
    saturates: reported are the particle-steps it completes per second over a fixed
    observation window, the requests in flight (admitted or queued) sampled every 0.5 s, and
    the latencies of the requests that finish inside the window; the rest are cancelled."""
    import numpy as np

    import stochasticphysics_b200 as sp
    from stochasticphysics_b200 import provider
    from stochasticphysics_b200._abi import Precision, Problem, RequestState

    rng = np.random.default_rng(seed)
    arrivals, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > arrival_s:
            break
        arrivals.append(t)
    specs = provider.batched_sets(count=len(arrivals), seed=seed, precision=Precision.FP32, step_scale=1.0,
                                  lissajous=True, problems=(Problem.Neel, Problem.BrownAndNeelEulerSpherical))
    work = [s.n * s.integrated_steps for s in specs]
    free, _ = __import__("torch").cuda.mem_get_info()
    budget = int(min(150e9, 0.8 * free))
    ids = [None] * len(specs)
    depth, done, lat = [], {}, []
    with sp.Server(ctx, memory_budget_bytes=budget) as srv:
        t0 = time.perf_counter()
        nxt = 0
        next_sample = 0.0
        while True:
            now = time.perf_counter() - t0
            while nxt < len(specs) and arrivals[nxt] <= now:
                ids[nxt] = srv.submit(specs[nxt])
                nxt += 1
            for i in range(nxt):
                if i in done:
                    continue
                if srv.poll(ids[i]) == RequestState.DONE:
                    _, ms = srv.wait(ids[i])
                    done[i] = now
                    lat.append(ms)
            if now >= next_sample:
                depth.append((round(now, 2), nxt - len(done)))
                next_sample += 0.5
            if now >= observe_s or (nxt == len(specs) and len(done) == len(specs)):
                break
            time.sleep(0.005)
        t_end = time.perf_counter() - t0
        # partial progress of the requests still running counts toward the throughput
        in_flight = [i for i in range(nxt) if i not in done]
        for i in in_flight:
            srv.cancel(ids[i])
        for i in in_flight:
            try:
                srv.wait(ids[i])
            except sp.SPError:
                pass
    completed = sum(work[i] for i in done)
    lat_s = sorted(lat)
    plain64 = plain_fp64_rate(ctx, specs[:12], 100000)
    return {"requests": len(specs), "arrival_rate_per_s": rate, "arrival_window_s": arrival_s,
            "observe_window_s": observe_s, "wall_s": t_end,
            "offered_particle_steps_per_s": sum(work) / arrival_s,
            "completed_requests": len(done), "completed_particle_steps": completed,
            "saturated_value": completed / t_end, "unit": UNIT,
            "p50_ms_completed": float(np.percentile(lat_s, 50)) if lat_s else None,
            "p99_ms_completed": float(np.percentile(lat_s, 99)) if lat_s else None,
            "in_flight_over_time": depth, "memory_budget_bytes": budget,
            "plain_fp64": {"value": plain64, "unit": UNIT,
                           "note": "the first 12 requests one at a time through sp_simulate in FP64, each cut "
                                   "to 1e5 steps"},
            "served_over_plain_fp64": completed / t_end / plain64,
            "note": "completed_particle_steps counts finished requests only (the cancelled ones' partial "
                    "work is not included), so saturated_value is a lower bound on the integration rate",
            "workload": f"Poisson {rate}/s for {arrival_s} s, full-length requests (step_scale 1.0): "
                        "N ~ logU[1e3, 6.4e4], S ~ logU[1e5, 1e7], Neel or BrownAndNeelEulerSpherical, "
                        "Heun / Millstein, FP32, Lissajous 12 mT at 25.25 / 26.04 kHz, dt = 1e-11 s"}


def batched_leg(ctx, count, step_scale, seed=0x5EED0004, serial_sample=16):
    """Parameter-set batch: `count` Neel ensembles with the batched-set distributions
    (N ~ logU[1e3, 6.4e4], S ~ logU[1e5, 1e7] x step_scale, Heun / Millstein
    alternating, FP32), all submitted at once to the server, which runs each kernel
    key's members as one launch per chunk over a shared tile work-list.  Launch shapes
    from the autotuner.  The same sets one at a time (every k-th, FP32) give the
    unbatched rate."""
    import stochasticphysics_b200 as sp
    from stochasticphysics_b200 import provider
    from stochasticphysics_b200._abi import Precision

    specs = provider.batched_sets(count=count, seed=seed, precision=Precision.FP32, step_scale=step_scale)
    for s in specs[:2]:
        ctx.autotune(s, probe_particles=32768)
    ps = sum(s.n * s.integrated_steps for s in specs)
    free, _ = __import__("torch").cuda.mem_get_info()
    with sp.Server(ctx, memory_budget_bytes=int(min(150e9, 0.8 * free))) as srv:
        t = time.perf_counter()
        ids = [srv.submit(s) for s in specs]
        lat = [srv.wait(i)[1] for i in ids]
        wall = time.perf_counter() - t
    k = max(1, count // serial_sample)
    sample = specs[::k][:serial_sample]
    t = time.perf_counter()
    for s in sample:
        ctx.simulate(s)
    serial_s = time.perf_counter() - t
    plain64 = plain_fp64_rate(ctx, sample, 100000)
    return {"sets": count, "value": ps / wall, "unit": UNIT, "wall_s": wall, "particle_steps": ps,
            "plain_fp64": {"value": plain64, "unit": UNIT, "sets": len(sample),
                           "note": "the same sampled sets one at a time through sp_simulate in FP64, each cut "
                                   "to 1e5 steps"},
            "batched_over_plain_fp64": ps / wall / plain64,
            "step_scale": step_scale,
            "max_latency_ms": max(lat),
            "launch_shapes": {s.solver.name: ctx.launch_config(s) for s in specs[:2]},
            "one_at_a_time": {"value": sum(s.n * s.integrated_steps for s in sample) / serial_s, "sets": len(sample)},
            "workload": f"Neel, N ~ logU[1e3, 6.4e4], S ~ logU[1e5, 1e7] x {step_scale}, |B| ~ U[1, 25] mT, "
                        "f ~ logU[1e4, 1e6] Hz, K ~ U[5e3, 3e4] J/m^3, alpha ~ U[0.02, 0.3], Heun / Millstein "
                        "alternating, FP32, W = 1000, dt = 1e-11 s"}


def plain_neel_leg(ctx, torch, cpu_steps=20000):
    """The plain Neel workload as the reference runs it: 1024 particles, FP64 Heun, the
    whole run of 1e6 steps with a sample every 100 steps (one field period at 100 kHz).
    A small ensemble: 32 warps, so each step's latency, not throughput, sets the time.
    Timed on the device (resident, CUDA events) and end to end through sp_simulate;
    the CPU restatement runs the first `cpu_steps` steps of the same particles on all
    host cores for comparison."""
    import oracle
    from stochasticphysics_b200 import provider
    from stochasticphysics_b200._abi import Precision

    spec = provider.neel_relaxation()
    st = torch.cuda.Stream()
    with ctx.ensemble(spec) as e:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        e.advance(spec.integrated_steps, st.cuda_stream)
        b.record(st)
        torch.cuda.synchronize()
        dev_s = a.elapsed_time(b) / 1e3
        res = e.read()
    t = time.perf_counter()
    ctx.simulate(spec)
    e2e_s = time.perf_counter() - t
    ps = spec.n * spec.integrated_steps
    with ctx.ensemble(dataclasses.replace(spec, precision=Precision.FP32)) as e:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        e.advance(spec.integrated_steps, st.cuda_stream)
        b.record(st)
        torch.cuda.synchronize()
        fp32_s = a.elapsed_time(b) / 1e3
    cpu = dataclasses.replace(spec, number_of_steps=cpu_steps + 100)
    t = time.perf_counter()
    oracle.simulate(cpu, threads=os.cpu_count() or 1)
    cpu_s = time.perf_counter() - t
    cpu_rate = spec.n * cpu_steps / cpu_s
    return {"value": ps / dev_s, "unit": UNIT, "run_s": dev_s, "e2e_run_s": e2e_s,
            "fp32": {"value": ps / fp32_s, "run_s": fp32_s},
            "nonfinite_particles": res.stats["nonfinite_particles"],
            "note": "the Cartesian Heun step does not renormalise |m| (the reference's own norm handling); "
                    "at dt = 1e-11 s the precession step omega dt is ~0.09, |m| drifts and some particles "
                    "overflow within 1e6 steps on the CPU restatement too, so the late windows of the mean "
                    "are not finite; the figure is a timing of the configuration as specified",
            "cpu": {"value": cpu_rate, "unit": UNIT, "cores": os.cpu_count() or 1,
                    "estimated_run_s": ps / cpu_rate, "sample": f"1024 particles x {cpu_steps} steps"},
            "workload": "neel_relaxation: Neel, FP64 Heun, 1024 particles, K = 1e4 J/m^3 easy axis, r = 10 nm, "
                        "alpha = 0.1, 10 mT at 100 kHz, dt = 1e-11 s, 1e6 steps, sample every 100 steps"}


def stiff_leg(ctx, torch, n=262144, timed_steps=2000):
    """The stiff cubic workload (ImplicitMidpoint, Newton tolerance 1e-10, at most 20
    iterations; 262144 Neel particles with cubic K1 = -1.1e4, dt = 1e-10 s) in three
    forms: FP64 with the reference's Newton matrix (the drop-in), FP64 with the exact
    Newton matrix, and the FP32 state with FP64 acceptance and the exact matrix.
    Device-resident, CUDA-event timed after one warm-up chunk."""
    from stochasticphysics_b200 import provider
    from stochasticphysics_b200._abi import Jacobian, Precision

    out = {}
    st = torch.cuda.Stream()
    for name, prec, jac in (("fp64_reference_jacobian", Precision.FP64, Jacobian.Reference),
                            ("fp64_exact_jacobian", Precision.FP64, Jacobian.Exact),
                            ("fp32_exact_jacobian", Precision.FP32, Jacobian.Exact)):
        spec = dataclasses.replace(provider.cubic_implicit(n=n, steps=timed_steps + 2000, oversampling=1000),
                                   precision=prec, jacobian=jac)
        with ctx.ensemble(spec) as e:
            e.advance(1000, st.cuda_stream)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            e.advance(timed_steps, st.cuda_stream)
            b.record(st)
            torch.cuda.synchronize()
            r = e.read()
        ms = a.elapsed_time(b)
        ps = r.stats["particle_steps"]
        out[name] = {"value": n * timed_steps / (ms / 1e3), "unit": UNIT,
                     "newton_iterations_per_step": r.stats["newton_iterations"] / ps,
                     "unconverged_fraction": r.stats["newton_unconverged"] / ps}
    out["workload"] = (f"cubic_implicit: Neel, cubic K1 = -1.1e4 J/m^3, Haar axes, alpha = 0.05, r ~ 12 nm lognormal "
                       f"(sigma 0.15), 12 mT at 25 kHz, dt = 1e-10 s, ImplicitMidpoint tol 1e-10 max 20; {n} "
                       f"particles x {timed_steps} timed steps")
    return out


def injected_leg(ctx, torch, peaks, rows=((65536, 1000), (1048576, 200)), warm_steps=50):
    """Injection mode (Wiener increments supplied by the caller and read from HBM every
    step, the parity mode): Neel Cartesian Heun, FP64 (24 B of dW per particle-step) and
    FP32 (12 B), at the bench's 65536 particles and at 1048576 particles, which fill the
    GPU's resident warps.  The dW arrays (steps x 3 x particles) are far larger than L2,
    so each increment comes from HBM once.  Device-resident, CUDA-event timed after a
    warm-up chunk; reports particle-steps/s, the dW read rate against the measured HBM
    copy bandwidth, and the ceiling the step's arithmetic puts on that fraction: with F
    flops per particle-step (FMA = 2) and B bytes of dW, a kernel running at the
    measured FMA peak P reads at most P B / F bytes/s."""
    from stochasticphysics_b200 import provider
    from stochasticphysics_b200._abi import Precision

    hbm, hbm_src = None, "MEASURED_PEAKS.json hbm_gbs (measured copy bandwidth)"
    try:
        hbm = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()).get("hbm_gbs")
    except (OSError, ValueError):
        pass
    if not hbm:  # no measured peaks file: an earlier copy-bandwidth measurement on B200
        hbm, hbm_src = 6650.0, "fallback: 6.65 TB/s, an earlier copy-bandwidth measurement on B200"
    flops = json.loads((ROOT / "stochasticphysics_b200" / "flops_table.json").read_text())["table"][
        "Neel/Uniaxial/Heun_Strong"]["flops"]
    st = torch.cuda.Stream()
    out = {"hbm_peak_gbs": hbm, "hbm_peak_source": hbm_src, "flops_per_particle_step": flops, "rows": []}
    for n, timed_steps in rows:
        base = provider.neel_relaxation(n=n, steps=timed_steps + warm_steps + 100, oversampling=100)
        base = provider.with_injected_noise(base, seed=7)
        row = {"particles": n, "timed_steps": timed_steps,
               "fp64_dw_gb": 3 * n * base.integrated_steps * 8 / 1e9}
        for prec in (Precision.FP64, Precision.FP32):
            with ctx.ensemble(dataclasses.replace(base, precision=prec)) as e:
                e.advance(warm_steps, st.cuda_stream)
                torch.cuda.synchronize()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(st)
                e.advance(timed_steps, st.cuda_stream)
                b.record(st)
                torch.cuda.synchronize()
            sec = a.elapsed_time(b) / 1e3
            ps = n * timed_steps / sec
            dw_bytes = 3 * (8 if prec == Precision.FP64 else 4)
            gbs = ps * dw_bytes / 1e9
            peak = peaks[prec.name]
            ceiling = peak * 1e12 * dw_bytes / flops / 1e9
            row[prec.name] = {"value": ps, "unit": UNIT, "dw_bytes_per_particle_step": dw_bytes,
                              "dw_read_gbs": gbs, "hbm_frac": gbs / hbm,
                              "fma_frac": ps * flops / (peak * 1e12),
                              "hbm_frac_ceiling_at_fma_peak": min(1.0, ceiling / hbm)}
        out["rows"].append(row)
        del base
    first = out["rows"][0]
    out["FP64"], out["FP32"] = first["FP64"], first["FP32"]  # the bench workload's size
    out["workload"] = ("neel_relaxation with injected dW: Neel, Heun, uniaxial; rows at 65536 and 1048576 "
                       "particles (the first is the FP64/FP32 entry above)")
    return out


def sizes_leg(ctx, torch, sizes=(16384, 65536, 262144, 1048576)):
    """The Brown+Neel workload one ensemble at a time at several sizes, FP32 and FP64,
    Millstein and Heun, with the launch shapes tuned for the bench workload: a 65536-
    particle ensemble (2048 warps) does not fill the GPU's resident warps by itself, so
    larger ensembles show the kernels' own rate.  Device-resident, CUDA-event timed after
    a warm-up window."""
    from stochasticphysics_b200 import provider
    from stochasticphysics_b200._abi import Precision, Solver

    st = torch.cuda.Stream()
    rows = []
    for n in sizes:
        for solver in (Solver.Millstein, Solver.Heun_Strong):
            row = {"particles": n, "solver": solver.name}
            for prec, steps in ((Precision.FP32, 4000), (Precision.FP64, 2000)):
                spec = provider.brown_neel_relaxation(n=n, steps=steps + 2000, oversampling=1000, solver=solver,
                                                      precision=prec)
                with ctx.ensemble(spec) as e:
                    e.advance(1000, st.cuda_stream)
                    torch.cuda.synchronize()
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(st)
                    e.advance(steps, st.cuda_stream)
                    b.record(st)
                    torch.cuda.synchronize()
                row[prec.name.lower()] = n * steps / (a.elapsed_time(b) / 1e3)
            row["fp32_over_fp64"] = row["fp32"] / row["fp64"]
            rows.append(row)
    return {"unit": UNIT, "rows": rows}


def fp32_accuracy(ctx, shards=16, n_shard=65536, steps=101000, oversampling=1000):
    """FP32 form against the plain FP64 kernel on the headline workload's particle model
    (Brown+Neel Euler/spherical, Milstein and Heun, the same Philox increments), on an
    ensemble of shards x n_shard particles large enough for the comparison's standard error
    to sit well below 1e-3.  Each shard keeps its global particle ids; the shards of one
    precision are submitted together to the server and merged with sp_merge_shards
    (MeanSimulationResult::operator+=).  Relative error: |M32 - M64| of the moment-weighted
    mean magnetisation (outputs 7-9), whose saturation value is 1 (|m| = 1 per particle), per
    window and component.  Its standard error comes from the spread of the per-shard
    differences (batch means over `shards` independent shards)."""
    import numpy as np

    import stochasticphysics_b200 as sp
    from stochasticphysics_b200 import merge_shards, provider
    from stochasticphysics_b200._abi import Precision, Solver

    out = {}
    for solver in (Solver.Millstein, Solver.Heun_Strong):
        whole = provider.brown_neel_relaxation(n=shards * n_shard, steps=steps, oversampling=oversampling,
                                               solver=solver)
        parts = [whole.subset(i * n_shard, (i + 1) * n_shard) for i in range(shards)]
        res = {}
        for prec in (Precision.FP64, Precision.FP32):
            specs = [dataclasses.replace(s, precision=prec) for s in parts]
            with sp.Server(ctx) as srv:
                ids = srv.submit_many(specs)
                res[prec] = [srv.wait(i)[0] for i in ids]
        merged = {prec: merge_shards([r.weighted_sum for r in rs], [r.weight for r in rs])[0]
                  for prec, rs in res.items()}
        d = (merged[Precision.FP32] - merged[Precision.FP64])[1:, 6:9]  # windows k >= 1, magnetisation
        per_shard = np.stack([(a.mean - b.mean)[1:, 6:9] for a, b in zip(res[Precision.FP32], res[Precision.FP64])])
        wts = np.array([r.weight[6] for r in res[Precision.FP64]])
        wts = wts / wts.sum()
        # weighted batch-means standard error of the merged difference
        dev = per_shard - np.tensordot(wts, per_shard, axes=1)[None]
        se = np.sqrt(np.tensordot(wts ** 2, dev ** 2, axes=1) * shards / (shards - 1))
        bias = d.mean(axis=0)  # signed difference averaged over the windows, per component
        bias_se = np.sqrt(np.tensordot(wts ** 2, (per_shard.mean(axis=1) - bias[None]) ** 2, axes=1)
                          * shards / (shards - 1))
        amp = float(np.abs(merged[Precision.FP64][1:, 6:9]).max())
        out[solver.name] = {
            "max_rel_error": float(np.abs(d).max()), "mean_rel_error": float(np.abs(d).mean()),
            "first_window_rel_error": float(np.abs(d[0]).max()),
            "max_se": float(se.max()), "mean_se": float(se.mean()), "max_z": float((np.abs(d) / se).max()),
            "window_mean_bias": [float(x) for x in bias], "window_mean_bias_se": [float(x) for x in bias_se],
            "max_abs_mean_m_fp64": amp, "max_error_over_response": float(np.abs(d).max()) / amp}
    out["workload"] = (f"brown_neel_relaxation, {shards} shards x {n_shard} particles = {shards * n_shard}, "
                       f"{(steps // oversampling - 1) * oversampling} integrated steps ({steps // oversampling - 1} "
                       f"windows of {oversampling}), same Philox stream in both precisions")
    out["definition"] = ("relative error = |M32 - M64| of the moment-weighted mean magnetisation per window and "
                         "component (saturation value 1); se = batch-means standard error over the shards")
    return out


def merged_shards_check(ctx, torch, dist, world, rank, steps=3000):
    """Multi-GPU: every rank runs its shard (global particle ids) of one verification
    ensemble of world x N_PER_GPU particles, the shards' FP64 window sums and weights are
    all-gathered over NCCL (the path's only exchange) and rank 0 merges them with
    sp_merge_shards and compares the merged mean with its own run of the whole union."""
    import numpy as np

    from stochasticphysics_b200 import merge_shards, provider
    from stochasticphysics_b200._abi import Precision

    whole = provider.brown_neel_relaxation(n=N_PER_GPU * world, steps=steps, oversampling=1000,
                                           precision=Precision.FP64)
    r = ctx.simulate(whole.subset(N_PER_GPU * rank, N_PER_GPU * (rank + 1)))
    k, od = r.weighted_sum.shape
    mine = torch.from_numpy(np.concatenate([r.weighted_sum.ravel(), r.weight])).cuda()
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine)
    if rank != 0:
        return None
    host = [q.cpu().numpy() for q in parts]
    mean, _, weight = merge_shards([h[:k * od].reshape(k, od) for h in host], [h[k * od:] for h in host])
    ref = ctx.simulate(whole)
    return {"ranks": world, "particles": whole.n, "integrated_steps": whole.integrated_steps,
            "max_abs_diff_vs_whole": float(np.abs(mean - ref.mean).max()),
            "weight_rel_diff": float(np.abs(weight / ref.weight - 1).max()),
            "exchange_bytes_per_rank": int(mine.numel() * 8)}


def cpu_baseline(steps_sample=2000, n=None):
    """The CPU oracle on all host cores for a bounded sample of the workload."""
    import oracle
    from stochasticphysics_b200 import provider
    from stochasticphysics_b200._abi import Solver
    n = n or N_PER_GPU
    cores = os.cpu_count() or 1
    # sample 0 is the initial state and only whole windows are integrated, so the sample
    # runs steps_sample + W steps with W = min(1000, steps_sample): steps_sample integrated
    w = min(1000, steps_sample)
    total_ps, total_s = 0, 0.0
    for solver in (Solver.Millstein, Solver.Heun_Strong):
        spec = provider.brown_neel_relaxation(n=n, steps=steps_sample + w, oversampling=w, solver=solver)
        assert spec.integrated_steps == steps_sample, (spec.integrated_steps, steps_sample)
        t = time.perf_counter()
        oracle.simulate(spec, threads=cores)
        total_s += time.perf_counter() - t
        total_ps += n * spec.integrated_steps
    return {"value": total_ps / total_s, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n} particles x {steps_sample} integrated steps (window {w}), Milstein + Heun, FP64 C++ "
                      f"restatement ({total_s:.1f} s on {cores} threads)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle  # noqa: F401  (the reference arm is the CPU restatement; the C++ reference cannot be built)
    n, steps_sample = N_PER_GPU, 300
    times = []
    for i in range(args.warmup + args.steps):
        base = cpu_baseline(steps_sample=steps_sample, n=n)
        if i >= args.warmup:
            times.append(2 * n * steps_sample / base["value"])
    ps = 2 * n * steps_sample * len(times)
    value = ps / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(args),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                             "sample": f"{n} particles x {steps_sample} steps per step, Milstein + Heun"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference C++ is not buildable here (Eigen/MyCEL/SerAr/Boost absent); this arm runs the "
                    "FP64 C++ restatement of its formulas (oracle/) on all host cores"}
    print(json.dumps(line), flush=True)


def config_dict(args):
    return {"workload": "brown_neel_relaxation: BrownAndNeelEulerSpherical, Milstein + Heun, "
                        f"{N_PER_GPU} particles/GPU, dt=1e-11 s, W=1000, {CHUNK} steps per bench step",
            "global_batch": N_PER_GPU * args.gpus, "seq_len": CHUNK, "parallelism": f"shards{args.gpus}",
            "l2": "flushed between timed steps (256 MiB write); state of 65536 particles is ~6 MiB"}


def time_ensembles(ensembles, steps, warmup, streams, flush, torch, concurrent):
    """Per step: L2 flush, then one chunk of every ensemble.

    concurrent=True: the ensembles advance on their own streams at the same time (as the
    server co-schedules them); one pair of events on streams[0] brackets the step.
    concurrent=False: one after another on streams[0], each chunk bracketed by its own
    events (per-launch durations for the roofline)."""
    from stochasticphysics_b200 import kernel_launch_count
    s0 = streams[0]
    evs, launches0 = [], None
    for i in range(warmup + steps):
        flush.zero_()
        torch.cuda.synchronize()
        if i == warmup:
            launches0 = kernel_launch_count()
        if concurrent:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s0)
            ends = []
            for e, st in zip(ensembles, streams):
                st.wait_event(a)
                e.advance(CHUNK, st.cuda_stream)
                ev = torch.cuda.Event()
                ev.record(st)
                ends.append(ev)
            for ev in ends:
                s0.wait_event(ev)
            b.record(s0)
            pair = [(a, b)]
        else:
            pair = []
            for e in ensembles:
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(s0)
                e.advance(CHUNK, s0.cuda_stream)
                b.record(s0)
                pair.append((a, b))
        if i >= warmup:
            evs.append(pair)
    torch.cuda.synchronize()
    per_launch = [[a.elapsed_time(b) for a, b in pair] for pair in evs]
    return per_launch, kernel_launch_count() - launches0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--n-particles", type=int, default=N_PER_GPU, help="smaller case for profiling")
    ap.add_argument("--chunk", type=int, default=CHUNK, help="SDE steps per bench step")
    ap.add_argument("--no-autotune", action="store_true", help="use the default launch shapes")
    ap.add_argument("--serving-seconds", type=float, default=8.0, help="arrival window of the serving leg (0: skip)")
    ap.add_argument("--serving-rate", type=float, default=50.0, help="mean Poisson arrival rate (requests/s)")
    ap.add_argument("--serving-step-scale", type=float, default=0.006,
                    help="scale of the request step counts (S ~ logU[1e5, 1e7] x scale)")
    ap.add_argument("--batched-sets", type=int, default=256, help="parameter sets of the batched leg (0: skip)")
    ap.add_argument("--no-stiff", action="store_true", help="skip the stiff ImplicitMidpoint leg")
    ap.add_argument("--no-injected", action="store_true", help="skip the injected-noise (HBM) leg")
    ap.add_argument("--no-sizes", action="store_true", help="skip the ensemble-size sweep")
    ap.add_argument("--batched-step-scale", type=float, default=1.0,
                    help="scale of the batched sets' step counts (S ~ logU[1e5, 1e7] x scale)")
    ap.add_argument("--overload-seconds", type=float, default=30.0,
                    help="observation window of the full-size serving overload leg (0: skip)")
    ap.add_argument("--accuracy-shards", type=int, default=16,
                    help="65536-particle shards of the FP32-vs-FP64 accuracy leg (0: skip)")
    ap.add_argument("--accuracy-steps", type=int, default=101000, help="steps of the accuracy leg")
    args = ap.parse_args()
    globals()["N_PER_GPU"], globals()["CHUNK"] = args.n_particles, args.chunk
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import numpy as np
    import torch
    import torch.distributed as dist

    import stochasticphysics_b200 as sp
    from stochasticphysics_b200._abi import Precision

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    total_steps = (args.warmup + args.steps) * CHUNK + 2000
    flops_table = json.loads((ROOT / "stochasticphysics_b200" / "flops_table.json").read_text())["table"]
    flops_step = [flops_table["BrownAndNeelEulerSpherical/Uniaxial/Millstein"]["flops"],
                  flops_table["BrownAndNeelEulerSpherical/Uniaxial/Heun_Strong"]["flops"]]

    def barrier_max(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    with sp.Context(local) as ctx:
        peak32 = ctx.fma_peak_tflops(1)
        peak64 = ctx.fma_peak_tflops(0)
        results, shapes = {}, {}
        for prec in (Precision.FP32, Precision.FP64):
            for s in workload_specs(N_PER_GPU, total_steps, prec, rank):
                if not args.no_autotune:
                    ctx.autotune(s, probe_particles=N_PER_GPU)
                shapes[f"{prec.name}/{s.solver.name}"] = ctx.launch_config(s)
        for prec in (Precision.FP32, Precision.FP64):
            wspecs = workload_specs(N_PER_GPU, total_steps, prec, rank)
            # the co-scheduled pair: tuned CTA shape, CO_CHUNK-step chunks; the per-launch
            # (roofline) timings use separate ensembles with the tuned shape as it is
            ens = [ctx.ensemble(s, shape=dict(ctx.launch_config(s), chunk_steps=CO_CHUNK)) for s in wspecs]
            solo = [ctx.ensemble(s) for s in wspecs]
            # co-scheduled launches go longest first (the lower tuned rate): the shorter
            # ensemble's CTAs then fill the SMs the longer one leaves free, instead of the
            # longer one running alone at the end
            rate = [ctx.launch_config(s)["particle_steps_per_s"] for s in wspecs]
            lpt = [e for _, e in sorted(zip(rate, ens), key=lambda t: t[0])]
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            with ClockSampler(local) as clk:
                conc, launches = time_ensembles(lpt, args.steps, args.warmup, streams, flush, torch, True)
            seq, _ = time_ensembles(solo, args.steps, args.warmup, streams, flush, torch, False)
            total_ms = barrier_max(sum(sum(p) for p in conc))
            reads = [e.read() for e in ens]
            for e in ens + solo:
                e.close()
            results[prec.name] = {"per_launch": seq, "total_ms": total_ms, "launches": launches,
                                  "seq_ms": barrier_max(sum(sum(p) for p in seq)),
                                  "clocks": clk.summary(), "means": [r.mean for r in reads],
                                  "nonfinite": sum(r.stats["nonfinite_particles"] for r in reads)}

        ps_per_step = 2 * N_PER_GPU * CHUNK
        v32 = world * ps_per_step * args.steps / (results["FP32"]["total_ms"] / 1e3)
        v64 = world * ps_per_step * args.steps / (results["FP64"]["total_ms"] / 1e3)
        # roofline of the dominant kernel (the step kernel; >99% of each chunk graph)
        pl = np.array(results["FP32"]["per_launch"])  # [steps][2 ensembles]
        ach = [flops_step[j] * N_PER_GPU * CHUNK / (pl[:, j].mean() / 1e3) / 1e12 for j in range(2)]
        pl64 = np.array(results["FP64"]["per_launch"])
        ach64 = [flops_step[j] * N_PER_GPU * CHUNK / (pl64[:, j].mean() / 1e3) / 1e12 for j in range(2)]

        # FP32 vs FP64 ensemble mean (same Philox stream): windows covered by the run
        m32, m64 = results["FP32"]["means"], results["FP64"]["means"]
        kdone = (args.warmup + args.steps) * CHUNK // 1000
        diffs = [np.abs(a[1:kdone + 1, 6:9] - b[1:kdone + 1, 6:9]) for a, b in zip(m32, m64)]
        se_indep = math.sqrt(2.0 / (3.0 * N_PER_GPU))

        # e2e through the public C ABI with host buffers: per bench step, the two ensembles
        # submitted together to the server (sp_server_submit_many: host arrays in) and
        # waited for (results out); sp_simulate of the two one after the other beside it
        e2e_specs = workload_specs(N_PER_GPU, CHUNK + 1000, Precision.FP32, rank)
        # submitted longest first (the lower tuned rate), as the co-scheduled leg launches
        e2e_specs.sort(key=lambda s: ctx.launch_config(s)["particle_steps_per_s"])
        for s in e2e_specs:
            ctx.simulate(s)  # warm the path
        e2e_times, seq_times, phases = [], [], []
        with sp.Server(ctx) as srv:
            ids = srv.submit_many(e2e_specs)
            for i in ids:
                srv.wait(i)
            for _ in range(args.steps):
                if world > 1:
                    dist.barrier()
                t = time.perf_counter()
                ids = srv.submit_many(e2e_specs)
                outs = [srv.wait(i)[0] for i in ids]
                e2e_times.append(time.perf_counter() - t)
                phases.append([[o.stats[k] for k in ("queue_ms", "setup_ms", "run_ms", "readback_ms")] for o in outs])
        # continuous batching: step k + 1's pair is submitted before step k's results are
        # awaited, so its upload and set-up overlap the rounds still running (every step
        # still uploads its inputs from host memory and reads its results back)
        with sp.Server(ctx) as srv:
            # warm-up in the timed pattern (two pairs in flight), so the server's groups
            # and their streams exist before the clock starts
            first = srv.submit_many(e2e_specs)
            second = srv.submit_many(e2e_specs)
            for i in first + second:
                srv.wait(i)
            if world > 1:
                dist.barrier()
            t = time.perf_counter()
            pending = srv.submit_many(e2e_specs)
            for k in range(args.steps):
                nxt = srv.submit_many(e2e_specs) if k + 1 < args.steps else None
                outs = [srv.wait(i)[0] for i in pending]
                pending = nxt
            pipelined_s = time.perf_counter() - t
        for _ in range(args.steps):
            if world > 1:
                dist.barrier()
            t = time.perf_counter()
            for s in e2e_specs:
                ctx.simulate(s)
            seq_times.append(time.perf_counter() - t)
        e2e_sync_value = world * ps_per_step * args.steps / barrier_max(sum(e2e_times))
        e2e_value = world * ps_per_step * args.steps / barrier_max(pipelined_s)
        e2e_simulate_value = world * ps_per_step * args.steps / barrier_max(sum(seq_times))
        h2d = sum(s.n * 13 * 8 for s in e2e_specs)
        ph = np.array(phases)  # [steps][requests][phase]
        e2e_breakdown = {
            "step_ms": 1e3 * statistics.mean(e2e_times),
            "per_request_ms": {name: [float(x) for x in ph[:, :, j].mean(axis=0)]
                               for j, name in enumerate(("queue", "setup", "run", "readback"))},
            "note": "server host clock per request (submit -> admission -> set-up -> rounds -> read-back); "
                    "requests in submission order"}
        d2h = sum(o.mean.nbytes + o.weight.nbytes + o.time.nbytes + o.field.nbytes for o in outs)
        serving = batched = None
        if world == 1 and args.serving_seconds > 0:
            serving = serving_leg(ctx, args.serving_seconds, args.serving_rate, args.serving_step_scale)
        overload = None
        if world == 1 and args.overload_seconds > 0:
            overload = overload_leg(ctx, observe_s=args.overload_seconds, rate=args.serving_rate)
        if world == 1 and args.batched_sets > 0:
            batched = batched_leg(ctx, args.batched_sets, args.batched_step_scale)
        accuracy = None if (world > 1 or args.accuracy_shards <= 0) else fp32_accuracy(
            ctx, shards=args.accuracy_shards, steps=args.accuracy_steps)
        merged = merged_shards_check(ctx, torch, dist, world, rank) if world > 1 else None
        stiff = None if (world > 1 or args.no_stiff) else stiff_leg(ctx, torch)
        injected = None if (world > 1 or args.no_injected) else injected_leg(ctx, torch, {"FP64": peak64, "FP32": peak32})
        sizes = None if (world > 1 or args.no_sizes) else sizes_leg(ctx, torch)
        plain_neel = None if (world > 1 or args.no_cpu_baseline) else plain_neel_leg(ctx, torch)

    if rank == 0:
        tpp, tsrc = profiled_traffic_per_particle()
        ipp, isrc = profiled_instructions()
        issue = None
        if ipp is not None:
            # peak issue: 4 schedulers per SM, one warp-instruction per cycle each, at the
            # median SM clock sampled during the timed region
            sms = torch.cuda.get_device_properties(local).multi_processor_count
            clk = results["FP32"]["clocks"].get("sm_mhz") or 1965.0
            peak_ti = sms * 4 * 32 * clk * 1e6 / 1e12  # tera thread-instructions/s
            ach_ti = v32 / world * (ipp[0] + ipp[1]) / 2 / 1e12
            issue = {"achieved": ach_ti, "peak": peak_ti, "unit": "T thread-instructions/s", "frac": ach_ti / peak_ti,
                     "instructions_per_particle_step": {"Millstein": ipp[0], "Heun": ipp[1]},
                     "source": f"profiles/{isrc}: ncu smsp__inst_executed per particle-step x measured FP32 rate; "
                               "peak = SMs x 4 schedulers x 32 lanes x median SM clock"}
            ipp64, _ = profiled_instructions("fp64_")
            if ipp64 is not None:
                clk64 = results["FP64"]["clocks"].get("sm_mhz") or 1965.0
                peak64_ti = sms * 4 * 32 * clk64 * 1e6 / 1e12
                ach64_ti = v64 / world * (ipp64[0] + ipp64[1]) / 2 / 1e12
                issue["fp64"] = {"achieved": ach64_ti, "peak": peak64_ti, "frac": ach64_ti / peak64_ti,
                                 "instructions_per_particle_step": {"Millstein": ipp64[0], "Heun": ipp64[1]}}
        cpu = None if (args.no_cpu_baseline or world > 1) else cpu_baseline()  # rank 0 at N = 1 only
        c32 = results["FP32"]["clocks"]
        line = {
            "metric": METRIC, "value": v32, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": results["FP32"]["total_ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, the stated distributions of each workload)",
            "config": config_dict(args),
            "fp64_plain": {"value": v64, "unit": UNIT, "ms_per_step": results["FP64"]["total_ms"] / args.steps,
                           "clocks": results["FP64"]["clocks"]},
            "fp32_over_fp64": v32 / v64,
            "fp32_served_over_fp64_plain": {
                "co_scheduled_pair": v32 / v64,
                "batched_sets": None if not batched else batched["batched_over_plain_fp64"],
                "serving_overload": None if not overload else overload["served_over_plain_fp64"],
                "note": "co_scheduled_pair: both forms on the timed workload, launched the same way; "
                        "batched_sets / serving_overload: the FP32 batched or served run against the same "
                        "requests one at a time through the plain FP64 kernel"},
            "sequential_ensembles": {"fp32": world * ps_per_step * args.steps / (results["FP32"]["seq_ms"] / 1e3),
                                     "fp64": world * ps_per_step * args.steps / (results["FP64"]["seq_ms"] / 1e3)},
            "fp32_vs_fp64_mean_m": {
                "ensemble": accuracy,
                "bench_run_65536": {"max_abs_diff": float(max(d.max() for d in diffs)),
                                    "first_window_abs_diff": float(max(d[0].max() for d in diffs)),
                                    "two_sample_se": se_indep,
                                    "note": "the timed 65536-particle ensembles themselves: their difference "
                                            "after the first windows is Monte-Carlo, of the order of the SE"}},
            "merged_shards": merged,
            "nonfinite_particles": {"fp32": results["FP32"]["nonfinite"], "fp64": results["FP64"]["nonfinite"]},
            "roofline": {"bound": "fp32-fma", "achieved": sum(ach) / 2, "peak": peak32, "unit": "TFLOP/s",
                         "frac": (sum(ach) / 2) / peak32,
                         "traffic": None if tpp is None else tpp * N_PER_GPU,
                         "traffic_source": None if tpp is None else
                         f"profiles/{tsrc}: DRAM bytes per particle per launch x {N_PER_GPU} particles",
                         "peak_source": "measured in bench.py: FMA-chain kernel on this GPU",
                         "flops_per_particle_step": {"Millstein": flops_step[0], "Heun": flops_step[1]},
                         "fp64": {"achieved": sum(ach64) / 2, "peak": peak64, "frac": (sum(ach64) / 2) / peak64},
                         "pipe_utilisation_pct": profiled_pipes(),
                         "issue": issue},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "api": "sp_server_submit_many / sp_server_wait: each step's pair submitted (host arrays in) "
                           "while the previous pair runs, results read back per step",
                    "one_step_at_a_time": e2e_sync_value,
                    "breakdown": e2e_breakdown,
                    "sp_simulate_one_after_the_other": e2e_simulate_value},
            "gpu_launches": results["FP32"]["launches"],
            "clocks": c32,
            "cpu_baseline": cpu,
            "launch_shapes": shapes,
            "co_scheduled_chunk_steps": CO_CHUNK,
            "serving": serving,
            "serving_overload": overload,
            "batched": batched,
            "stiff": stiff,
            "injected": injected,
            "ensemble_sizes": sizes,
            "plain_neel_1024": plain_neel,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
