"""Replica bookkeeping for runs with one process per GPU.

Every rank renders its own frames (pixels, samples and scenes are
independent, so no data crosses between ranks); the only exchange is the
reduction of the timing and the work counts at the end of a run: the
slowest rank's time and the sum of all ranks' rays.  Works with any
torch.distributed backend (nccl on the GPUs, gloo on the CPU)."""
from __future__ import annotations

from typing import Tuple


def combine(elapsed: float, units: float, device: str = "cpu") -> Tuple[float, float]:
    """(max over ranks of `elapsed`, sum over ranks of `units`).  Without an
    initialised process group the values are returned unchanged."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(elapsed), float(units)
    t = torch.tensor([float(elapsed)], dtype=torch.float64, device=device)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())


def shard(n: int, rank: int, world: int) -> range:
    """Contiguous share of `n` independent units (scenes, tiles) for `rank`;
    the shares cover 0..n-1 once and differ in size by at most one."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return range(lo, lo + base + (1 if rank < extra else 0))
