"""Rank logic of the multi-GPU runs (one process per GPU, torch.distributed).

A single world does not shard: N ranks run N replicas. Batched worlds
partition by world id: rank r steps worlds [r*W/N, (r+1)*W/N) in its own
context, renumbered from 0, with no data-path collective. The only
collectives are the barrier and the maximum of the ranks' device times (the
job takes as long as its slowest rank)."""
import numpy as np


def world_range(nworlds, rank, ranks):
    """[lo, hi): the worlds of `rank` among `ranks`. The ranges are contiguous,
    differ in size by at most one and cover [0, nworlds) once."""
    if ranks < 1 or not 0 <= rank < ranks:
        raise ValueError(f"rank {rank} of {ranks}")
    return nworlds * rank // ranks, nworlds * (rank + 1) // ranks


def shard_specs(specs, nworlds, rank, ranks):
    """(specs of this rank's worlds with world ids renumbered from 0, lo, hi).
    Spec order within the shard is the input order, so a world's bodies come
    out of `bodies_from_specs` as they would from the whole batch."""
    lo, hi = world_range(nworlds, rank, ranks)
    mine = specs[(specs["world"] >= lo) & (specs["world"] < hi)].copy()
    mine["world"] -= np.asarray(lo, dtype=mine.dtype["world"])
    return mine, lo, hi


def max_over_ranks(value, dist=None, device="cpu"):
    """The largest `value` over all ranks of the default process group (`dist`
    is torch.distributed); `value` itself when there is no group."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
