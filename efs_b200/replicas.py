"""Replica runs across ranks: one process per GPU, each advancing its own
independent solve, with no collective on the data path.

The plain, batched and served forms do not shard (their solves are
independent), so N GPUs run N replicas.  The only cross-rank steps are host
plumbing: rank 0 builds the seeded job once and the other ranks load its copy,
barriers bracket the timed region, and the timed region's length is reduced as
the maximum over ranks.  The whole-job rate counts every rank's cells.
torch.distributed carries these steps (nccl on GPUs, gloo in the CPU tests).
"""
import datetime
import os
import pickle
import tempfile


def dist_env():
    """(rank, local rank, world size) from the launcher's environment."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def init_group(backend, timeout_s=600):
    """Join the process group; a collective whose peers are gone fails after timeout_s."""
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def barrier_fn(world):
    if world == 1:
        return lambda: None
    import torch.distributed as dist
    return lambda: dist.barrier()


def share(build, tag, rank, world, barrier):
    """The object `build()` makes, built once on rank 0 and loaded by the others."""
    if world == 1:
        return build()
    path = os.path.join(tempfile.gettempdir(), "efs_replica_%s.pkl" % tag)
    if rank == 0:
        obj = build()
        with open(path + ".tmp", "wb") as f:
            pickle.dump(obj, f, protocol=4)
        os.replace(path + ".tmp", path)
    barrier()
    if rank != 0:
        with open(path, "rb") as f:
            obj = pickle.load(f)
    return obj


def max_over_ranks(value, world, device="cpu"):
    """Maximum of `value` over all ranks (the job's time is its slowest rank's)."""
    if world == 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(cells_per_rank, timesteps, ms_max, world):
    """MCells/s of the whole job: every rank's cells x timesteps over the slowest rank's time."""
    return world * cells_per_rank * timesteps / (ms_max / 1e3) / 1e6
