#!/usr/bin/env python
"""Benchmark of the B200 FDTD engine on the plain large solve.

Workload (one GPU): uniform 512^3 lines, 0.5 mm, 40 seeded boxes (20 PEC,
20 dielectric eps_r ~ U[2,10]), Mur ABC on +-x/+-y, 8-cell UPML on +-z, TFSF
Gaussian plane wave f0 = 10 GHz fc = 5 GHz at normal incidence, NF2FF box 10
cells inside with 3 frequencies (workloads.large_plain).  Synthetic, seeded.

A step is one pass of the reference orchestrator's loop body
(scripts/lib/sim-engine.mjs:648-681): iterate(100) timesteps, then the lagged
energy readback.  Metric: MCells/s = cells x timesteps / device time.

Multi-GPU: replicas only (independent solves, no collective); value is the
sum over ranks of cells x timesteps over the max-over-ranks device time.

--impl reference times the reference's CPU algorithm (the oracle port of
CPUFDTDEngine, js arithmetic, all host threads) on a bounded sample of the
same workload.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BATCH = 100          # timesteps per step (the orchestrator's readback interval)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--n", type=int, default=512, help="grid lines per axis")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--ref-timesteps", type=int, default=2, help="timesteps per reference-arm step")
    p.add_argument("--no-batched", action="store_true", help="skip the batched-sweep measurement")
    p.add_argument("--no-patch", action="store_true", help="skip the patch-antenna solve")
    p.add_argument("--cpu-timesteps", type=int, default=40, help="timesteps of the CPU-baseline sample")
    p.add_argument("--no-far-field", action="store_true", help="skip the 181 x 361 far-field measurement")
    p.add_argument("--no-dispersive", action="store_true", help="skip the 800 x 800 x 400 dispersive solve")
    p.add_argument("--dispersive-timesteps", type=int, default=200, help="timed timesteps of the dispersive solve")
    p.add_argument("--dispersive-batch", type=int, default=16,
                   help="dispersive 200x200x100 solves of the batched dispersive form (0: skip)")
    p.add_argument("--no-served", action="store_true", help="skip the served request stream")
    p.add_argument("--served-arrivals-s", type=float, default=10.0, help="seconds of 20 req/s arrivals (saturated legs)")
    p.add_argument("--served-horizon-s", type=float, default=40.0, help="serving time of the saturated legs")
    p.add_argument("--served-capacity-rate", type=float, default=0.5, help="req/s of the capacity-matched leg")
    p.add_argument("--served-capacity-s", type=float, default=40.0, help="seconds of capacity-matched arrivals")
    p.add_argument("--batch-count", type=int, default=64, help="instances of the batched sweep")
    return p.parse_args()


from efs_b200.replicas import barrier_fn, dist_env, init_group, max_over_ranks, share, whole_job_rate


def build_job(n, rank, world, barrier):
    """Rank 0 builds the seeded job; other ranks load rank 0's copy."""
    from efs_b200 import workloads
    return share(lambda: workloads.large_plain(n), "bench_job_%d" % n, rank, world, barrier)


class Clocks:
    """nvidia-smi sampler running across the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of the core kernels from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "core_traffic.txt")
    if not os.path.exists(p):
        return None
    out = {}
    for line in open(p):
        f = line.split()
        if len(f) == 3 and not line.startswith("#"):
            out[f[0]] = (float(f[1]), int(f[2]))   # kernel -> (bytes per launch, cells of the captured grid)
    return out


def cpu_sample(job, mode, timesteps):
    """Time the CPU oracle on `timesteps` steps of `job` (all host threads)."""
    from oracle import oracle
    from efs_b200 import workloads
    threads = oracle.set_threads(os.cpu_count() or 1)
    e = oracle.OracleEngine(mode=mode)
    workloads.configure(e, dict(job, probes=[]))
    e.iterate(1)   # first-touch / page-in outside the sample
    t = time.perf_counter()
    e.iterate(timesteps)
    dt = time.perf_counter() - t
    N = job["grid"][0] * job["grid"][1] * job["grid"][2]
    return N * timesteps / dt / 1e6, threads, dt


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    from efs_b200 import workloads
    job = workloads.large_plain(args.n)
    from oracle import oracle
    from efs_b200 import workloads as wl
    threads = oracle.set_threads(os.cpu_count() or 1)
    e = oracle.OracleEngine(mode="js")
    wl.configure(e, dict(job, probes=[]))
    N = job["grid"][0] * job["grid"][1] * job["grid"][2]
    for _ in range(args.warmup):
        e.iterate(args.ref_timesteps)
    t = time.perf_counter()
    for _ in range(args.steps):
        e.iterate(args.ref_timesteps)
    dt = time.perf_counter() - t
    value = N * args.ref_timesteps * args.steps / dt / 1e6
    sample = "%d timesteps of the %d^3 workload per step (CPUFDTDEngine arithmetic, %d threads)" % (
        args.ref_timesteps, args.n, threads)
    print(json.dumps({
        "impl": "reference", "metric": "MCells/s", "value": round(value, 3), "unit": "MCells/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1000 * dt / args.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": "large_plain %d^3: 40 boxes, Mur +-x/+-y, UPML8 +-z, TFSF, NF2FF F=3" % args.n,
                   "cells": N, "timesteps_per_step": args.ref_timesteps},
        "cpu_baseline": {"value": round(value, 3), "unit": "MCells/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "MCells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def batch_vs_sequential(jobs, T, local):
    """Configure one engine per job, autotune the batch, then time T timesteps
    per member batched and the same engines stepped one after another (each
    leg after an identical untimed leg that captures its graphs).  Returns
    (cells, batched MCells/s, sequential MCells/s, autotuned shape)."""
    from efs_b200 import workloads
    from efs_b200.engine import CudaBatch, CudaEngine
    engines = []
    for j in jobs:
        e = CudaEngine(device=local)
        e.initGPU()
        workloads.configure(e, dict(j, probes=j.get("probes") or []))
        engines.append(e)
    cells = sum(j["grid"][0] * j["grid"][1] * j["grid"][2] for j in jobs)
    b = CudaBatch(engines)
    tuned = b.autotune(steps=8)                  # real timesteps, identical results under every shape
    tuned["phases_ms"] = b.timePhases(32)        # per-phase device ms per batched timestep
    b.iterate(T)
    b.sync()
    t0 = time.perf_counter()
    b.iterate(T)
    b.sync()
    t_batch = time.perf_counter() - t0
    for e in engines:                            # sequential: one engine after another, each its own graphs
        e.iterate(T)
    for e in engines:
        e.sync()
    t0 = time.perf_counter()
    for e in engines:
        e.iterate(T)
        e.sync()
    t_seq = time.perf_counter() - t0
    b.destroy()
    for e in engines:
        e.destroy()
    return cells, cells * T / t_batch / 1e6, cells * T / t_seq / 1e6, tuned


def batched_sweep(args, local):
    """Batched form on the stub-filter sweep (64 microstrip filters, uneven
    grids): every member advanced by one persistent fused launch per timestep
    (efs_batch_*), against the same engines stepped one after another.  Both
    legs run the same number of timesteps per member (graphs captured in an
    identical warm-up leg) and are timed by the wall clock around
    device-synchronised runs."""
    from efs_b200 import workloads
    jobs = workloads.stub_filters(count=args.batch_count)
    T = 1024                                     # timesteps per member in each timed leg (16 graphs of 64)
    cells, v_b, v_s, tuned = batch_vs_sequential(jobs, T, local)
    return {"workload": "stub_filters x%d: per-axis U[60,180] lines, 0.2 mm, Mur, two 50-ohm ports" % len(jobs),
            "instances": len(jobs), "cells": cells, "timesteps_per_member": T,
            "batched_mcells_s": round(v_b, 1), "sequential_mcells_s": round(v_s, 1), "speedup": round(v_b / v_s, 3),
            "batched_solves_per_s_15000_steps": round(v_b * 1e6 / (cells / len(jobs)) / 15000, 3),
            "sequential_solves_per_s_15000_steps": round(v_s * 1e6 / (cells / len(jobs)) / 15000, 3),
            "autotuned": tuned, "timing": "wall clock around device-synchronised runs of %d timesteps" % T}


def patch_solve(local):
    """The plain single solve of the reference's published benchmark: the
    86 x 87 x 71 patch antenna (graded mesh, UPML 8, 50-ohm port, probes every
    step), 30 000 timesteps through the orchestrator's loop (iterate(100) +
    lagged energy, sim-engine.mjs:648-681).  Device time by CUDA events on the
    engine stream; the published figures are for the same grid and step count
    (README.md:137-140 of the reference; the WebGPU figure recomputed from its
    6.2 s)."""
    import torch
    from efs_b200 import workloads
    from efs_b200.engine import CudaEngine
    job = workloads.patch_antenna()
    N = job["grid"][0] * job["grid"][1] * job["grid"][2]
    g = CudaEngine(device=local)
    g.initGPU()
    workloads.configure(g, job)
    stream = torch.cuda.ExternalStream(g.stream)
    for _ in range(5):
        g.iterate(100)
        g.computeEnergy()
    g.sync()
    T = job["maxTS"]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    ev0.record(stream)
    for _ in range(T // 100):
        g.iterate(100)
        g.computeEnergy()
    ev1.record(stream)
    ev1.synchronize()
    wall = time.perf_counter() - t0
    ms = ev0.elapsed_time(ev1)
    g.destroy()
    return {"workload": "patch antenna 86x87x71 graded mesh, UPML 8, 50-ohm port, probes every step",
            "cells": N, "timesteps": T, "mcells_s": round(N * T / (ms / 1e3) / 1e6, 1), "seconds": round(ms / 1e3, 3),
            "wall_s": round(wall, 3),
            "published_30000_steps": {"openems_multithreaded_mcells_s": 444, "openems_multithreaded_s": 36,
                                      "webgpu_mcells_s": 2570, "webgpu_s": 6.2,
                                      "note": "reference README.md:137-140 (their hardware, Mur boundaries)"}}


FF_FLOPS_PER_PAIR = 40     # per (angle, point): 3 FMA phase + 2 phase reduction + 16 FMA (4 complex MACs)


def fp32_peak_tflops(device):
    """Nominal FP32 (non-tensor) peak: SMs x 128 lanes x 2 flops x max SM clock."""
    import torch
    props = torch.cuda.get_device_properties(device)
    try:
        out = subprocess.run(["nvidia-smi", "-i", str(device), "--query-gpu=clocks.max.sm", "--format=csv,noheader,nounits"],
                             capture_output=True, text=True, timeout=20)
        mhz = float(out.stdout.strip().splitlines()[0])
    except Exception:
        mhz = 1965.0
    return props.multi_processor_count * 128 * 2 * mhz * 1e6 / 1e12


def far_field_leg(eng, job, local):
    """The NF2FF far field of the headline job at its configured size: a
    181 x 361 theta/phi grid (1-degree steps) at each of the 3 frequencies,
    on the accumulators of the timed run (computeNF2FFfarField through the
    public API).  GFLOP/s counts FF_FLOPS_PER_PAIR per (angle, point) pair
    over the angle kernel's device time; e2e is the call's wall time (point
    metadata upload, both kernels, result readback)."""
    theta = np.deg2rad(np.arange(181, dtype=np.float64)).astype(np.float32)
    phi = np.deg2rad(np.arange(361, dtype=np.float64)).astype(np.float32)
    A = theta.size * phi.size
    npts = job["nf2ff"]["numPoints"]
    per = []
    for fi, fr in enumerate(job["nf2ff_freqs"]):
        cfg = dict(pointMeta=job["nf2ff_meta"], theta=theta, phi=phi, center=[0.0, 0.0, 0.0], frequency=fr, radius=1.0,
                   numPoints=npts, freqIndex=fi)
        eng.computeNF2FFfarField(cfg)                  # warm-up
        t0 = time.perf_counter()
        out = eng.computeNF2FFfarField(cfg)
        wall = time.perf_counter() - t0
        prep_ms, ang_ms = eng.farFieldTime()
        per.append({"freq_GHz": round(fr / 1e9, 3), "angles_ms": round(ang_ms, 3), "prep_ms": round(prep_ms, 3),
                    "call_wall_ms": round(1e3 * wall, 2), "P_max": float(np.asarray(out).reshape(-1, 5)[:, 0].max())})
    pairs = float(A) * npts
    ang = sum(p["angles_ms"] for p in per) / len(per)
    gflops = pairs * FF_FLOPS_PER_PAIR / (ang / 1e3) / 1e9
    peak = fp32_peak_tflops(local)
    return {"angles": A, "grid": "181 x 361 (1 degree)", "points": npts, "frequencies": len(per),
            "pairs_per_frequency": int(pairs), "flops_per_pair": FF_FLOPS_PER_PAIR,
            "gflops": round(gflops, 1), "fp32_peak_tflops_nominal": round(peak, 1),
            "frac_of_nominal_fp32": round(gflops / 1e3 / peak, 4),
            "e2e_ms_per_frequency": round(sum(p["call_wall_ms"] for p in per) / len(per), 2), "per_frequency": per}


def dispersive_leg(args, local):
    """The plain dispersive solve of the configuration list at its full size:
    800 x 800 x 400 lines, 0.25 mm, UPML 8 on all faces, Drude (stiff) and
    Lorentz spheres over 30% of the cells, TFSF at 30 degrees, NF2FF with 5
    frequencies (workloads.dispersive).  Run twice on the same job: as the
    reference's engine runs it (ADE state updated, not applied to the fields)
    and with the ADE apply step on.  Each is timed with CUDA events on the
    engine stream over `--dispersive-timesteps` timesteps after 2 x 100
    warm-up timesteps."""
    import torch
    from efs_b200 import workloads
    from efs_b200.engine import CudaEngine
    t0 = time.perf_counter()
    job = workloads.dispersive()
    t_gen = time.perf_counter() - t0
    N = job["grid"][0] * job["grid"][1] * job["grid"][2]

    def run(apply):
        g = CudaEngine(device=local)
        g.initGPU()
        t0 = time.perf_counter()
        workloads.configure(g, dict(job, probes=[], ade=dict(job["ade"], apply=apply)))
        g.iterate(1)
        g.sync()
        t_cfg = time.perf_counter() - t0
        stream = torch.cuda.ExternalStream(g.stream)
        for _ in range(2):
            g.iterate(100)
            g.computeEnergy()
        g.sync()
        T = max(1, args.dispersive_timesteps // 100) * 100
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(T // 100):
            g.iterate(100)
            g.computeEnergy()
        ev1.record(stream)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1)
        out = {"timesteps": T, "ms_per_timestep": round(ms / T, 4), "mcells_s": round(N * T / (ms / 1e3) / 1e6, 1),
               "kernels_per_timestep": g.kernelsPerStep(), "device_gb": round(g.deviceBytes() / 1e9, 2),
               "host_configure_s": round(t_cfg, 1), "phases_ms": g.timePhases(16)}
        g.destroy()
        return out

    out = {"workload": "dispersive 800x800x400, UPML8 all faces, Drude/Lorentz spheres 30%, TFSF 30 deg, NF2FF F=5",
           "cells": N, "dispersive_cells": int(job["dispersive_cells"]), "host_generate_s": round(t_gen, 1)}
    out.update(run(False))
    out["ade_applied"] = run(True)
    # batched form: 16 seeded dispersive solves of 200 x 200 x 100 lines (same
    # media, UPML, TFSF and NF2FF layout), as the reference's engine runs them
    if args.dispersive_batch:
        small = [workloads.dispersive(grid=(200, 200, 100), seed=100 + i, apply=False) for i in range(args.dispersive_batch)]
        T = 256
        cells, v_b, v_s, tuned = batch_vs_sequential(small, T, local)
        out["batched"] = {"workload": "%d dispersive solves 200x200x100" % len(small), "cells": cells,
                          "timesteps_per_member": T, "batched_mcells_s": round(v_b, 1),
                          "sequential_mcells_s": round(v_s, 1), "speedup": round(v_b / v_s, 3), "autotuned": tuned}
    return out


def _served_template(a):
    from efs_b200 import workloads
    kind, side, steps = a
    return workloads.served_template(kind, side, steps=steps)


def served_leg(args, local):
    """The served request stream of the configuration list (Poisson arrivals,
    cubic-ish grids with sides log-uniform in [40, 300], 70% lumped-port/Mur
    jobs and 30% TFSF+NF2FF jobs with 2 frequencies, 5000-25000 steps, 150 GB
    HBM budget; serve.request_stream, numpy default_rng(4)), in shortened
    windows (the configuration's run is 10 minutes):
      saturated:  20 req/s for --served-arrivals-s, served for --served-horizon-s,
                  with continuous batching (64 member slots) and as a plain
                  one-slot queue (the plain engine's sequential solves) on the
                  same stream; throughput = cell-steps/s of each, solves/s =
                  completions / horizon;
      capacity:   --served-capacity-rate req/s for --served-capacity-s, drained:
                  p50/p95/p99 latency near the device's capacity.
    Request inputs are prepared before the clock starts."""
    from efs_b200 import serve, workloads
    sat = serve.request_stream(20.0, args.served_arrivals_s)
    cap = serve.request_stream(args.served_capacity_rate, args.served_capacity_s, seed=5)
    keys = sorted({(k, sd) for _, k, sd, _ in sat + cap})
    t0 = time.perf_counter()
    made = workloads._parallel_map(_served_template, [(k, sd, 25000) for k, sd in keys], min(len(keys), 8))
    templates = dict(zip(keys, made))
    prep = time.perf_counter() - t0

    def work(stream):                 # mean cell-steps of one request of the stream
        return float(np.mean([np.prod(templates[(k, sd)]["grid"]) * steps for _, k, sd, steps in stream]))

    def one(stream, members, horizon):
        srv = serve.Server(hbm_budget=150e9, max_members=members, chunk=256, device=local)
        serve.run_stream(stream, templates, srv, horizon=horizon)
        wall = srv.now()
        srv.close()
        done = srv.finished
        rate = srv.cell_steps / wall
        return {"arrivals": len(stream), "completed": len(done), "wall_s": round(wall, 2),
                "solves_per_s": round(len(done) / wall, 4), "mcells_s": round(rate / 1e6, 1),
                # completions in a window cut short favour one-at-a-time service; the
                # steady-state rate is the throughput over the mean request's work
                "work_equivalent_solves_per_s": round(rate / work(stream), 4),
                "latency": serve.latency_stats(done), "member_slots": members}
    batched = one(sat, 64, args.served_horizon_s)
    plain = one(sat, 1, args.served_horizon_s)
    capacity = one(cap, 64, None)
    return {"window": "shortened: %.0f s of 20 req/s arrivals served for %.0f s; %.2f req/s for %.0f s drained" % (
                args.served_arrivals_s, args.served_horizon_s, args.served_capacity_rate, args.served_capacity_s),
            "template_prep_s": round(prep, 1), "saturated_continuous": batched, "saturated_plain_queue": plain,
            "throughput_ratio_vs_plain": round(batched["mcells_s"] / max(plain["mcells_s"], 1e-9), 3),
            "capacity_matched": capacity}


def run_b200(args):
    import torch
    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        init_group("nccl", timeout_s=600)
    barrier = barrier_fn(world)
    from efs_b200.build import build
    if rank == 0:
        build()
    barrier()
    from efs_b200.engine import CudaEngine
    from efs_b200 import workloads

    job = build_job(args.n, rank, world, barrier)
    N = job["grid"][0] * job["grid"][1] * job["grid"][2]
    eng = CudaEngine(device=local)
    assert eng.initGPU(), "no CUDA device"
    workloads.configure(eng, dict(job, probes=[]))
    stream = torch.cuda.ExternalStream(eng.stream)

    def step():
        eng.iterate(BATCH)
        eng.computeEnergy()          # lagged readback, as the orchestrator does every 100 steps

    for _ in range(args.warmup):
        step()
    eng.sync()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    eng.sync()
    barrier()
    torch.cuda.synchronize()
    ms_max = max_over_ranks(ms, world, device="cuda")
    steps_total = args.steps * BATCH
    value = whole_job_rate(N, steps_total, ms_max, world)

    # dominant kernel (the fused E+H update) timed alone with CUDA events on the engine stream
    core_ms = eng.timeCore(20)               # [fused kernel, UPML-cell passes around it]
    bytes_core = 52.0 * N                    # fused-step algorithmic minimum: 48 B fields + 4 B material index
    t_core = core_ms[0] / 1e3
    peak, peak_kind = peaks()
    achieved = bytes_core / t_core / 1e9
    traffic = None
    tr = profiled_traffic()
    if tr and "k_fused_tma" in tr:
        b, cells = tr["k_fused_tma"]
        traffic = int(b * N / cells)         # DRAM bytes per launch, scaled from the profiled grid
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": traffic,
            "kernel": "k_fused_tma (TMA-fed fused E+H update), 52 B/cell algorithmic",
            "ms_per_launch": round(core_ms[0], 4), "upml_passes_ms": round(core_ms[1], 4),
            "peak_kind": "of " + peak_kind}
    step_bytes = workloads.job_bytes_per_step(job)
    # our kernels in the timed region: per timestep plan + per captured graph (64
    # steps each) one counter update and ceil(m/16) NF2FF accumulator passes +
    # the two energy-reduction kernels per step
    chunks = [64] * (BATCH // 64) + ([BATCH % 64] if BATCH % 64 else [])
    nf_passes = sum(math.ceil(m / 16) for m in chunks) if job.get("nf2ff") else 0
    launches = args.steps * (BATCH * eng.kernelsPerStep() + len(chunks) + nf_passes + 2)
    phases = eng.timePhases(32)              # per-phase device ms per timestep, launched kernel by kernel
    tfsf_faces = [int(v) for v in eng.debugRead("tfsf_faces")]
    far = None
    if rank == 0 and world == 1 and not args.no_far_field and job.get("nf2ff"):
        far = far_field_leg(eng, job, local)
    eng.destroy()

    # end to end through the public API from host buffers
    e2e = None
    if rank == 0 or world > 1:
        torch.cuda.synchronize()
        h2d = 0
        for k, v in job["coefficients"].items():
            h2d += np.asarray(v).nbytes
        for r in job.get("pml") or []:
            h2d += sum(np.asarray(r[k]).nbytes for k in ("vv", "vvfo", "vvfn", "ii", "iifo", "iifn"))
        t0 = time.perf_counter()
        g = CudaEngine(device=local)
        g.initGPU()
        workloads.configure(g, dict(job, probes=[]))
        g.sync()
        t1 = time.perf_counter()
        for _ in range(args.steps):
            g.iterate(BATCH)
            g.computeEnergy()
        g.sync()
        t2 = time.perf_counter()
        acc = g.readNF2FFAccumulation(True)
        en = g.flushEnergy()
        g.destroy()
        dt = time.perf_counter() - t0
        d2h = (acc["accumE"].nbytes + acc["accumH"].nbytes + 8 * (args.steps + 1)) if acc else 8 * args.steps
        e2e = {"value": round(N * steps_total / dt / 1e6, 3), "unit": "MCells/s",
               "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
               "wall_s": round(dt, 3), "setup_s": round(t1 - t0, 3), "run_s": round(t2 - t1, 3),
               "readback_s": round(dt - (t2 - t0), 3)}
        del en
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, threads, dt = cpu_sample(job, "js", args.cpu_timesteps)
        cpu = {"value": round(v, 3), "unit": "MCells/s", "cores": threads, "kind": "port",
               "sample": "%d timesteps of the same %d^3 job on the CPU oracle (CPUFDTDEngine arithmetic), %.1f s" % (
                   args.cpu_timesteps, args.n, dt)}
    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        batched = batched_sweep(args, local)
    patch = None
    if rank == 0 and world == 1 and not args.no_patch:
        patch = patch_solve(local)
    disp = None
    if rank == 0 and world == 1 and not args.no_dispersive:
        disp = dispersive_leg(args, local)
    served = None
    if rank == 0 and world == 1 and not args.no_served:
        served = served_leg(args, local)
    if rank == 0:
        print(json.dumps({
            "metric": "MCells/s", "value": round(value, 3), "unit": "MCells/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded numpy default_rng(2))",
            "config": {"workload": "large_plain %d^3: 40 boxes, Mur +-x/+-y, UPML8 +-z, TFSF, NF2FF F=3" % args.n,
                       "cells": N, "timesteps_per_step": BATCH, "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs larger than L2 (%.1f GB of fields)" % (24 * N / 1e9),
                       "bytes_per_timestep_algorithmic": step_bytes},
            "step_roofline": {"achieved": round(step_bytes / (ms_max / steps_total / 1e3) / 1e9, 1), "peak": peak,
                              "unit": "GB/s", "frac": round(step_bytes / (ms_max / steps_total / 1e3) / 1e9 / peak, 4),
                              "what": "whole timestep (all kernels) against its algorithmic bytes"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "phases_ms": phases, "tfsf_faces_in_core": tfsf_faces,
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "batched": batched,
            "patch": patch,
            "far_field": far,
            "dispersive": disp,
            "served": served,
        }))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
