"""Small, self-terminating runs of the benchmark workloads for profilers.

    python -m efs_b200.profile_case --n 256 --steps 4
    python -m efs_b200.profile_case --batch 64 --steps 4
    python -m efs_b200.profile_case --dispersive --steps 4
    python -m efs_b200.profile_case --dispersive-batch 16 --steps 64

The first builds workloads.large_plain(n) (n^3 lines: same features as the
headline benchmark), configures the CUDA engine and runs `steps` timesteps,
printing the mean device time per timestep.  --batch N instead builds the
first N stub filters of the batched sweep (workloads.stub_filters) and runs
them as one batch; --dispersive runs workloads.dispersive() (800 x 800 x 400,
or --grid); --dispersive-batch N runs N seeded dispersive solves of
--member-grid lines batched, then the same solves one after another.
Sized by --n / --batch so a profiler capture stays small.
"""
import argparse
import time


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--batch", type=int, default=0, help="run N stub filters as one batch instead")
    ap.add_argument("--dispersive", action="store_true", help="run the 800 x 800 x 400 dispersive solve instead")
    ap.add_argument("--grid", type=int, nargs=3, default=[800, 800, 400], help="grid of the dispersive solve")
    ap.add_argument("--dispersive-batch", type=int, default=0, help="run N dispersive solves as one batch and in sequence")
    ap.add_argument("--member-grid", type=int, nargs=3, default=[200, 200, 100], help="grid of each batched dispersive solve")
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--time-core", type=int, default=0, help="also time N launches of the core kernel(s) alone")
    args = ap.parse_args()
    from efs_b200.build import build
    build()
    from efs_b200 import workloads
    from efs_b200.engine import CudaBatch, CudaEngine
    if args.dispersive_batch:
        jobs = [workloads.dispersive(grid=tuple(args.member_grid), seed=5 + i, tfsf_inset=12, nf2ff_inset=10)
                for i in range(args.dispersive_batch)]
        engines = []
        for j in jobs:
            e = CudaEngine()
            e.initGPU()
            workloads.configure(e, j)
            engines.append(e)
        cells = sum(j["grid"][0] * j["grid"][1] * j["grid"][2] for j in jobs)
        b = CudaBatch(engines)
        b.iterate(args.warmup)
        b.sync()
        t = time.perf_counter()
        b.iterate(args.steps)
        b.sync()
        tb = (time.perf_counter() - t) / max(1, args.steps)
        b.destroy()
        for e in engines:
            e.iterate(args.warmup)
            e.sync()
        t = time.perf_counter()
        for e in engines:
            e.iterate(args.steps)
            e.sync()
        ts = (time.perf_counter() - t) / max(1, args.steps)
        print("dispersive batch=%d grid=%s cells=%d steps=%d  batched %.3f ms/timestep %.1f MCells/s  "
              "sequential %.3f ms/timestep %.1f MCells/s  (%.2fx)" % (
                  args.dispersive_batch, "x".join(map(str, args.member_grid)), cells, args.steps, tb * 1e3,
                  cells / tb / 1e6, ts * 1e3, cells / ts / 1e6, ts / tb))
        for e in engines:
            e.destroy()
        return
    if args.batch:
        jobs = workloads.stub_filters(count=args.batch)
        engines = []
        for j in jobs:
            e = CudaEngine()
            e.initGPU()
            workloads.configure(e, j)
            engines.append(e)
        b = CudaBatch(engines)
        b.iterate(args.warmup)
        b.sync()
        t = time.perf_counter()
        b.iterate(args.steps)
        b.sync()
        dt = (time.perf_counter() - t) / max(1, args.steps)
        N = sum(j["grid"][0] * j["grid"][1] * j["grid"][2] for j in jobs)
        print("batch=%d cells=%d steps=%d  %.3f ms/timestep  %.1f MCells/s" % (args.batch, N, args.steps, dt * 1e3,
                                                                             N / dt / 1e6))
        b.destroy()
        for e in engines:
            e.destroy()
        return
    if args.dispersive:
        t = time.perf_counter()
        job = workloads.dispersive(grid=tuple(args.grid))
        print("dispersive job built in %.1f s: %d dispersive cells" % (time.perf_counter() - t, job["dispersive_cells"]),
              flush=True)
    else:
        job = workloads.large_plain(args.n)
    eng = CudaEngine()
    if not eng.initGPU():
        raise SystemExit("no CUDA device")
    workloads.configure(eng, dict(job, probes=[]))
    eng.iterate(args.warmup)
    eng.sync()
    t = time.perf_counter()
    eng.iterate(args.steps)
    eng.sync()
    dt = (time.perf_counter() - t) / max(1, args.steps)
    N = job["grid"][0] * job["grid"][1] * job["grid"][2]
    line = "grid=%s steps=%d  %.3f ms/timestep  %.1f MCells/s  kernels/step=%d  device %.1f GB" % (
        "x".join(map(str, job["grid"])), args.steps, dt * 1e3, N / dt / 1e6, eng.kernelsPerStep(), eng.deviceBytes() / 1e9)
    if args.time_core:
        ms = eng.timeCore(args.time_core)
        core = ms[0] + ms[1]
        line += "  core %.3f ms (%.0f GB/s at 52 B/cell)" % (core, 52.0 * N / (core / 1e3) / 1e9)
    print(line)
    eng.destroy()


if __name__ == "__main__":
    main()
