"""Host-side scheduling for more than one GPU (one process per GPU).

The unwrapping path has no exchange between independent scenes, so N GPUs
run N replicas of the single-GPU pipeline: a batch of interferograms is
split by scene (no data-path collective), and timings are combined as the
maximum over ranks.  Both helpers work with any torch.distributed backend
(nccl on GPUs, gloo on CPU).
"""
from __future__ import annotations

__all__ = ["shard_scenes", "max_over_ranks"]


def shard_scenes(sizes, rank: int, world: int):
    """Indices of the scenes rank ``rank`` of ``world`` processes solves:
    largest scenes first, each to the rank with the least total pixels so
    far (ties to the lower rank), so every rank computes the same partition
    without communicating.  ``sizes`` are the scenes' pixel counts."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("need 0 <= rank < world")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    loads = [0] * world
    owner = [0] * len(sizes)
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        owner[i] = r
        loads[r] += int(sizes[i])
    return [i for i in range(len(sizes)) if owner[i] == rank]


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of ``value`` over the ranks of the default process group (the
    value itself without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    if device is None:
        device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
