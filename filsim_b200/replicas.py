"""Replica runs: one independent box per rank (one process per GPU), no
collective on the data path. torch.distributed is plumbing only: a barrier
around the timed region and the maximum of the per-rank device times."""
import torch


def replica_seed(base, rank):
    """Each rank simulates its own seeded suspension."""
    return base + rank


def barrier(dist, cuda=True):
    if cuda:
        torch.cuda.synchronize()
    if dist is not None and dist.is_initialized():
        dist.barrier()
    if cuda:
        torch.cuda.synchronize()


def max_over_ranks(x, dist=None, device="cpu"):
    """The slowest rank's value (every rank gets it)."""
    if dist is None or not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank, steps, ms_max, world):
    """Whole-job units per second: every rank processed units_per_rank per step."""
    return world * units_per_rank * steps / (ms_max / 1e3)
