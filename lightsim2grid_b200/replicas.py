"""Multi-GPU plumbing: one process per GPU, independent cases, no data-path collective.

The batched power flows are independent (contingencies, snapshots), so a multi-GPU job
either runs the same batch on every GPU (replicas, what ``bench.py --gpus N`` measures) or
gives every rank a contiguous slice of the cases.  ``torch.distributed`` is only used to
agree on timings (max over ranks) and, optionally, to gather results for the caller.
"""
import numpy as np


def shard_bounds(ncases, rank, world):
    """Contiguous slice ``[a, b)`` of ``ncases`` for ``rank`` (sizes differ by at most one)."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("invalid rank / world size")
    a = (ncases * rank) // world
    b = (ncases * (rank + 1)) // world
    return a, b


def max_over_ranks(value, group=None):
    """Max of a float over all ranks (the job's device time is that of its slowest rank)."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def aggregate_rate(units_per_rank, seconds_per_rank_max, world):
    """Whole-job throughput: units processed by all ranks over the slowest rank's time."""
    return float(units_per_rank) * world / float(seconds_per_rank_max)


def gather_rows(local_rows, ncases, group=None):
    """Gathers every rank's contiguous slice of a ``(cases, ...)`` array on all ranks."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    out = [None] * world
    dist.all_gather_object(out, np.asarray(local_rows), group=group)
    full = np.concatenate(out, axis=0)
    if full.shape[0] != ncases:
        raise RuntimeError("gathered {} rows, expected {}".format(full.shape[0], ncases))
    return full
