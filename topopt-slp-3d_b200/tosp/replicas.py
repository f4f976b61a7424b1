"""Replica bookkeeping for runs on several GPUs of one node.

The solve path does not shard (one problem per GPU); N ranks run independent
replicas.  The whole-job rate is the units all ranks processed divided by the
slowest rank's device time, so every rank takes the same collective steps:
a barrier before and after the timed region and one MAX all-reduce of the
elapsed time.
"""
import torch
import torch.distributed as dist


def world():
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def barrier():
    if world()[0] > 1:
        dist.barrier()


def max_over_ranks(value, device=None):
    """Maximum of a float over all ranks (identity for one rank)."""
    n, _ = world()
    if n == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(local_units, local_seconds, device=None):
    """Whole-job rate: total units over all ranks / slowest rank's time."""
    n, _ = world()
    t = max_over_ranks(local_seconds, device)
    return n * local_units / t if t > 0 else float("nan"), t
