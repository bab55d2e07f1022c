"""Shot sharding across GPUs (one process per GPU) and the single image reduction.

The operators are independent per shot; the only exchange is one sum of the
images (Born / tomo / WEMVA adjoint, WEMVA forward) or none (forward data is
per shot). Each rank takes a contiguous range of shots — the same split the C++
shot-loop classes use across the GPUs of one process — and the images are
summed with one all-reduce (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations


def shard(n_shots: int, rank: int, world: int) -> range:
    """Contiguous shot range of `rank`: ceil(n/world) shots per rank, the last ranks may get fewer."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    per = (n_shots + world - 1) // world
    return range(min(n_shots, rank * per), min(n_shots, (rank + 1) * per))


def reduce_image(image, group=None):
    """Sum a per-rank image tensor over all ranks in place (torch.distributed all-reduce)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(image, op=dist.ReduceOp.SUM, group=group)
    return image


def max_over_ranks(value: float, device=None, group=None) -> float:
    """Largest value over ranks (timings are reported as the slowest rank)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
