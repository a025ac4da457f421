"""Replica sharding across ranks (one process per GPU): the reference's only multi-GPU use is
independent lattices per MPI rank (kpz/kpzFrontendCuda.cu:31-48), so the path has no data
exchange -- ranks split the replicas, run them independently, and only the measurements are
combined (max of the timings, gather of the per-replica results).  Works with any
torch.distributed backend (NCCL on GPUs, gloo on CPU for tests).
"""
from __future__ import annotations

from typing import List, Sequence


def shard(n: int, world: int, rank: int) -> List[int]:
    """Replica indices run by `rank`: round robin, so uneven sizes spread evenly."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    return list(range(rank, n, world))


def stream_id(replica: int) -> int:
    """Counter-stream id of a replica: its global index, so results do not depend on world."""
    return replica


def max_over_ranks(x: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(n: int, mine: Sequence[int], values: Sequence[float], device=None) -> List[float]:
    """Every rank's (replica -> value) pairs into one list indexed by replica."""
    import torch
    import torch.distributed as dist
    out = torch.zeros(n, dtype=torch.float64, device=device)
    for i, v in zip(mine, values):
        out[i] = float(v)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(out, op=dist.ReduceOp.SUM)
    return [float(v) for v in out.tolist()]
