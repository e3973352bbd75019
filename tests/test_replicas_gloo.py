"""Multi-rank plumbing of replica runs (efs_b200.replicas) with world_size 2
over gloo on the CPU: the job built once on rank 0 and loaded by rank 1, the
slowest rank's time as the job's time, the whole-job rate over both ranks,
identical replicas, and a rank that leaves before a collective turning into
an error on the other rank instead of a hang.  Each rank steps its replica
on the CPU oracle (no GPU)."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _small_job():
    from efs_b200 import workloads
    return workloads.stub_filters(count=1, steps=60, workers=1)[0]


def _replica_rank(rank, world, port, outdir, tag):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import time
    import torch
    from efs_b200 import replicas, workloads
    from oracle.oracle import OracleEngine
    dist = replicas.init_group("gloo", timeout_s=60)
    barrier = replicas.barrier_fn(world)
    job = replicas.share(_small_job, tag, rank, world, barrier)
    o = OracleEngine(mode="f32")
    workloads.configure(o, job)
    barrier()
    t = time.perf_counter()
    o.iterate(3)
    ms = (time.perf_counter() - t) * 1e3
    ms_max = replicas.max_over_ranks(ms, world)
    cells = job["grid"][0] * job["grid"][1] * job["grid"][2]
    rate = replicas.whole_job_rate(cells, 3, ms_max, world)
    check = torch.tensor([float(np.asarray(o.volt, np.float64).sum()), float(cells)], dtype=torch.float64)
    got = [torch.zeros(2, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(got, check)
    np.save(os.path.join(outdir, "rank%d.npy" % rank),
            np.array([ms, ms_max, rate] + [float(g[1]) for g in got] + [float(g[0]) for g in got]))
    dist.destroy_process_group()


def _leaving_rank(rank, world, port, outdir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from efs_b200 import replicas
    dist = replicas.init_group("gloo", timeout_s=5)
    dist.barrier()
    if rank == 1:
        return                                    # leaves between steps, before the next collective
    try:
        replicas.max_over_ranks(1.0, world)
        outcome = "completed"
    except Exception as e:                        # the peer is gone: an error, not a hang
        outcome = "error: " + type(e).__name__
    with open(os.path.join(outdir, "rank0.txt"), "w") as f:
        f.write(outcome)


def test_two_replicas_over_gloo():
    out = tempfile.mkdtemp()
    mp.start_processes(_replica_rank, args=(2, _free_port(), out, "gloo_test_%d" % os.getpid()), nprocs=2,
                       start_method="spawn", join=True)
    r0, r1 = np.load(os.path.join(out, "rank0.npy")), np.load(os.path.join(out, "rank1.npy"))
    assert r0[1] == r1[1] == max(r0[0], r1[0])      # the job's time is the slowest rank's
    assert r0[2] == pytest.approx(2 * r0[3] * 3 / (r0[1] / 1e3) / 1e6)
    assert r0[3] == r0[4] == r1[3]                  # both ranks loaded the same job
    assert r0[5] == r0[6] and np.isfinite(r0[5])    # identical replicas: identical fields


def test_rank_leaving_before_a_collective_is_an_error():
    out = tempfile.mkdtemp()
    mp.start_processes(_leaving_rank, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    with open(os.path.join(out, "rank0.txt")) as f:
        assert f.read().startswith("error")
