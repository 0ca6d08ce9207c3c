"""Independent replicas on several GPUs (one process per GPU).

The large step of one domain does not shard here (the reference's MPI
decomposition is not built), so N GPUs run N independent replicas: each rank
advances its own seeded copy of the workload, no collective touches the data
path, and a job's throughput is the cells of all ranks over the slowest rank's
time (weak scaling).  These helpers hold that arithmetic and the one
collective (the max of the ranks' times), so that the same code runs with
NCCL on the GPUs and with gloo in the CPU tests.
"""
import os


def rank_env():
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(rank, base=1234):
    """Seed of a rank's replica: every rank advances a different realisation."""
    return base + rank


def max_over_ranks(value, dist=None, device="cpu"):
    """The largest of the ranks' values (a time in ms); `dist` is
    torch.distributed with an initialised process group, or None for one rank."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world, cells_per_rank, steps, ms_max):
    """Cell updates per second of the whole job: all ranks' cells over the
    slowest rank's time."""
    if ms_max <= 0:
        raise ValueError("time must be positive")
    return world * cells_per_rank * steps / (ms_max * 1e-3)
