"""Small, self-terminating runs of the benchmark workloads for profilers.

    python -m efs_b200.profile_case --n 256 --steps 4
    python -m efs_b200.profile_case --batch 64 --steps 4
    python -m efs_b200.profile_case --dispersive --steps 4

The first builds workloads.large_plain(n) (n^3 lines: same features as the
headline benchmark), configures the CUDA engine and runs `steps` timesteps,
printing the mean device time per timestep.  --batch N instead builds the
first N stub filters of the batched sweep (workloads.stub_filters) and runs
them as one batch; --dispersive runs workloads.dispersive() (800 x 800 x 400,
or --grid).
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
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--time-core", type=int, default=0, help="also time N launches of the core kernel(s) alone")
    args = ap.parse_args()
    from efs_b200.build import build
    build()
    from efs_b200 import workloads
    from efs_b200.engine import CudaBatch, CudaEngine
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
