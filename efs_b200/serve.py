"""Served form: a request loop with continuous batching on one GPU.

Requests (a job's inputs + its step count) arrive over time.  The loop keeps
a batch (efs_batch_*) of resident solves: between chunks it retires the
members that finished, then admits waiting requests in arrival order while a
member slot is free and their device memory fits the HBM budget, so requests
that arrive while others run join the work already on the device.  Each chunk
advances every member by the same number of timesteps (at most `chunk`, and
never past the nearest member's end), as one persistent launch per timestep
inside CUDA graphs.  New members are configured on their own streams while
the previous chunk is still running.  Every request's result is what the
same engine computes alone (the batch runs the single engine's kernels per
member), which tests/test_gpu_serve.py checks.

    python -m efs_b200.serve --rate 20 --duration 60        # 20 req/s Poisson arrivals for 60 s
"""
import argparse
import json
import math
import time
from collections import deque

import numpy as np

from . import workloads
from .engine import CudaBatch, CudaEngine, EfsError


class Request:
    __slots__ = ("rid", "job", "steps", "arrival", "admitted", "done", "engine", "remaining", "slices", "result", "cells",
                 "saved", "evictions", "retry_below")

    def __init__(self, rid, job, steps, arrival):
        self.rid, self.job, self.steps, self.arrival = rid, job, int(steps), arrival
        self.admitted = self.done = None
        self.saved = None                          # host copy of an evicted solve's state (efs_get_state)
        self.evictions = 0
        self.retry_below = None                    # device bytes in use when its admission last failed
        self.engine = None
        self.remaining = int(steps)
        self.slices = None
        self.result = None
        g = job["grid"]
        self.cells = g[0] * g[1] * g[2]


def estimate_bytes(job):
    """Device bytes a job will hold once configured (upper estimate for admission)."""
    g = job["grid"]
    n = g[0] * g[1] * ((g[2] + 3) // 4 * 4)                     # device cells: z rows padded to 4 floats
    b = n * (4 * 3 * 4 + 4)                                     # E, H in two parities + material index
    if job.get("mur"):
        b += len(job["mur"]["coeff_nyP"]) * 2 * 48
    if job.get("tfsf"):
        t = job["tfsf"]
        b += 40 * (len(t["voltagePoints"]["field_idx"]) + len(t["currentPoints"]["field_idx"]))
    if job.get("nf2ff"):
        nf = job["nf2ff"]
        b += nf["numPoints"] * (len(nf["omegas"]) * 48 + 16 * 24 + 32)
    b += n // 8                                                 # deferred-H cell list
    return b + (8 << 20)


class Server:
    """Continuous-batching request loop.  hbm_budget: bytes the resident
    solves may hold; max_members: member slots of the batch; chunk: most
    timesteps per scheduling round.

    evict_ratio: when set, a waiting request that cannot be admitted (no slot
    or no memory) and whose step count is at most 1/evict_ratio of the
    largest remaining step count among the resident solves has that solve
    evicted: its whole device state is copied to the host (efs_get_state),
    its engine is freed, and it waits right behind the newcomer; it resumes
    later on a fresh engine from that copy (efs_set_state), with the same
    result as if it had never left.  A solve is evicted at most
    `max_evictions` times."""

    def __init__(self, hbm_budget=150e9, max_members=64, chunk=256, device=0, evict_ratio=None, max_evictions=1):
        self.budget = float(hbm_budget)
        self.max_members = int(max_members)
        self.chunk = int(chunk)
        self.device = device
        self.waiting = deque()
        self.active = []
        self.finished = []
        self.failed = []                           # requests whose engine could not be set up alone
        self.used = 0
        self.batch = None
        self.next_id = 0
        self.t0 = time.perf_counter()
        self.cell_steps = 0
        self.evict_ratio = evict_ratio
        self.max_evictions = int(max_evictions)
        self.evicted = 0

    def now(self):
        return time.perf_counter() - self.t0

    def submit(self, job, steps, arrival=None):
        r = Request(self.next_id, job, steps, self.now() if arrival is None else arrival)
        self.next_id += 1
        self.waiting.append(r)
        return r.rid

    def _admit(self):
        added = False
        while self.waiting and len(self.active) < self.max_members:
            r = self.waiting[0]
            need = estimate_bytes(r.job)
            if self.used + need > self.budget and self.active:
                break                                           # wait for memory to free up
            if r.retry_below is not None and self.used >= r.retry_below and self.active:
                break                                           # failed beside the same residents: wait
            self.waiting.popleft()
            e = CudaEngine(device=self.device)
            try:
                if not e.initGPU():
                    raise EfsError(3, "no usable CUDA device %r" % (self.device,))
                r.slices = workloads.configure(e, r.job)
                if r.saved is not None:                         # an evicted solve resumes where it stopped
                    e.setState(r.saved)
            except (EfsError, MemoryError) as exc:
                # The engine's allocations (cudaMalloc inside configure, or
                # the state upload) failed: free what it holds.  Beside other
                # resident solves the request waits at the head of the queue
                # until they have released memory; alone on the device it can
                # never run, and is reported as failed.
                e.destroy()
                if self.active:
                    r.retry_below = self.used
                    self.waiting.appendleft(r)
                    break
                r.result = {"error": str(exc)}
                r.done = self.now()
                r.saved = None
                self.failed.append(r)
                continue
            r.saved = None
            r.retry_below = None
            r.engine = e
            if r.admitted is None:
                r.admitted = self.now()
            self.used += e.deviceBytes()
            self.active.append(r)
            added = True
        return added

    def _retire(self, r):
        e = r.engine
        out = {}
        if r.job.get("probes"):
            out["probes"] = workloads.probe_series(e, r.job, r.slices)
        if r.job.get("nf2ff"):
            acc = e.readNF2FFAccumulation(True)
            out["nf2ff"] = (acc["accumE"], acc["accumH"])
        # The allocation-free reduction keeps the retirement inside the HBM
        # budget the loop accounts for; grids beyond its fixed scratch
        # (2^30 interior cells) take the allocating one.
        nx, ny, nz = e.numLines
        if (nx - 1) * (ny - 1) * (nz - 1) <= 1 << 30:
            out["energy"] = e.energyNoAlloc()
        else:
            out["energy"] = e.computeEnergy(lagged=False)
        r.result = out
        r.done = self.now()
        self.used -= e.deviceBytes()
        e.destroy()
        r.engine = None
        self.finished.append(r)

    def _evict(self):
        """Evict one resident solve for the head of the queue (see evict_ratio);
        the batch must be idle.  Returns True when one was evicted."""
        if not self.evict_ratio or not self.waiting or not self.active:
            return False
        head = self.waiting[0]
        fits = len(self.active) < self.max_members and (self.used + estimate_bytes(head.job) <= self.budget)
        if fits:
            return False
        cand = [r for r in self.active if r.evictions < self.max_evictions and r.remaining >= self.evict_ratio * head.steps]
        if not cand:
            return False
        victim = max(cand, key=lambda r: r.remaining)
        if self.batch is not None:
            self.batch.destroy()
            self.batch = None
        e = victim.engine
        victim.saved = e.getState()
        self.used -= e.deviceBytes()
        e.destroy()
        victim.engine = None
        victim.evictions += 1
        self.evicted += 1
        self.active = [r for r in self.active if r is not victim]
        self.waiting.insert(1, victim)                          # right behind the newcomer
        return True

    def _rebatch(self):
        if self.batch is not None:
            self.batch.destroy()
            self.batch = None
        if self.active:
            self.batch = CudaBatch([r.engine for r in self.active])

    def round(self):
        """One scheduling round: start a chunk for the resident solves, admit
        newcomers while it runs, then retire the solves that finished.
        Returns False when there is nothing to run."""
        running = list(self.active)
        n = 0
        if running:
            if self.batch is None:
                self._rebatch()
            n = min(self.chunk, min(r.remaining for r in running))
            self.batch.iterate(n)                          # asynchronous
        admitted = self._admit()                           # configured on their own streams meanwhile
        if not running:
            if admitted:
                self._rebatch()
            return admitted
        self.batch.sync()
        self.cell_steps += n * sum(r.cells for r in running)
        done = []
        for r in running:
            r.remaining -= n
            if r.remaining == 0:
                done.append(r)
        if done:
            self.active = [r for r in self.active if r.remaining > 0]
            if self.batch is not None:
                self.batch.destroy()
                self.batch = None
            for r in done:
                self._retire(r)
        evicted = self._evict()
        if done or admitted or evicted:
            self._rebatch()
        return True

    def close(self):
        if self.batch is not None:
            self.batch.destroy()
            self.batch = None
        for r in self.active:
            r.engine.destroy()
        self.active = []


def latency_stats(reqs):
    lat = np.array([r.done - r.arrival for r in reqs]) if reqs else np.zeros(0)
    if lat.size == 0:
        return {"completed": 0}
    return {"completed": int(lat.size), "p50_s": round(float(np.percentile(lat, 50)), 3),
            "p95_s": round(float(np.percentile(lat, 95)), 3), "p99_s": round(float(np.percentile(lat, 99)), 3),
            "mean_s": round(float(lat.mean()), 3)}


def request_stream(rate, duration, seed=4, side_range=(40, 300), steps_range=(5000, 25000), tfsf_frac=0.3):
    """Poisson arrivals at `rate` per second: (arrival time, kind, side, steps)
    with sides log-uniform over side_range (rounded to a multiple of 8, so
    request inputs come from a bounded set of templates)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return out
        side = int(round(math.exp(rng.uniform(math.log(side_range[0]), math.log(side_range[1]))) / 8.0)) * 8
        side = max(side_range[0], min(side_range[1], side))
        kind = "tfsf" if rng.random() < tfsf_frac else "port"
        out.append((t, kind, side, int(rng.integers(steps_range[0], steps_range[1] + 1))))


def run_stream(stream, templates, server, drain=True, horizon=None):
    """Feed `stream` (arrival, kind, side, steps) into `server` in real time."""
    pending = deque(stream)
    server.t0 = time.perf_counter()
    while pending or server.waiting or server.active:
        now = server.now()
        if horizon is not None and now > horizon:
            break
        while pending and pending[0][0] <= now:
            t, kind, side, steps = pending.popleft()
            server.submit(templates[(kind, side)], steps, arrival=t)
        if not server.round():
            if not pending:
                break
            time.sleep(max(0.0, min(0.05, pending[0][0] - server.now())))
        if not drain and not pending:
            break
    return server


def _template(args):
    kind, side, steps = args
    return workloads.served_template(kind, side, steps=steps)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=20.0, help="arrivals per second")
    ap.add_argument("--duration", type=float, default=60.0, help="seconds of arrivals")
    ap.add_argument("--horizon", type=float, default=None, help="stop serving at this time (s)")
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--chunk", type=int, default=256)
    ap.add_argument("--steps-min", type=int, default=5000)
    ap.add_argument("--steps-max", type=int, default=25000)
    ap.add_argument("--side-min", type=int, default=40)
    ap.add_argument("--side-max", type=int, default=300)
    args = ap.parse_args()
    stream = request_stream(args.rate, args.duration, side_range=(args.side_min, args.side_max),
                            steps_range=(args.steps_min, args.steps_max))
    keys = sorted({(k, s) for _, k, s, _ in stream})
    t = time.perf_counter()                      # request inputs, prepared before the clock starts
    made = workloads._parallel_map(_template, [(k, s, args.steps_max) for k, s in keys],
                                   min(len(keys), 16) if len(keys) > 1 else 1)
    templates = dict(zip(keys, made))
    prep = time.perf_counter() - t
    srv = Server(hbm_budget=args.budget_gb * 1e9, max_members=args.members, chunk=args.chunk)
    run_stream(stream, templates, srv, horizon=args.horizon)
    wall = srv.now()
    srv.close()
    done = srv.finished
    print(json.dumps({"arrivals": len(stream), "rate": args.rate, "duration_s": args.duration, "wall_s": round(wall, 2),
                      "template_prep_s": round(prep, 1), "latency": latency_stats(done),
                      "solves_per_s": round(len(done) / wall, 3), "mcells_s": round(srv.cell_steps / wall / 1e6, 1),
                      "unserved": len(stream) - len(done) - len(srv.failed), "failed": len(srv.failed), "members": args.members, "budget_gb": args.budget_gb}))


if __name__ == "__main__":
    main()
