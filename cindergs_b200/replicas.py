"""Multi-GPU replicas: views shard across ranks with no data exchange.

Every frame needs the whole scene and the whole tile list, so a frame does
not split across GPUs; independent views do. Rank r of N renders frames
r, r+N, r+2N, ...; the only communication is a barrier around the timed
region and a max over ranks of the elapsed device time (one process per GPU,
torch.distributed over NCCL on GPUs, gloo in CPU tests).
"""
from __future__ import annotations


def view_frames(rank: int, world: int, steps: int, start: int = 0) -> list[int]:
    """Frame indices rank `rank` renders in `steps` steps."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    return [start + rank + k * world for k in range(steps)]


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of `value` over all ranks of the default process group (the
    value itself when torch.distributed is not initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
