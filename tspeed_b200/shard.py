"""Multi-GPU sharding of independent shots (replicas with disjoint shots).

Shots are independent (no per-step exchange), so N GPUs take contiguous
slices of one global shot list, run with no collective in the data path, and
meet only to time the run (barrier, max over ranks) and to gather
seismograms at the end.
"""
from __future__ import annotations

import numpy as np


def shots_for_rank(total: int, rank: int, world: int) -> range:
    """Contiguous, balanced slice of `total` shots for `rank` of `world`."""
    if not (0 <= rank < world) or total < 0:
        raise ValueError("bad rank/world/total")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(value: float, dist, device=None) -> float:
    """Max of a per-rank timing over all ranks (dist = torch.distributed or None)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_seismograms(local: np.ndarray, total: int, dist, device=None):
    """Gathers per-rank seismograms [nshots_local, nk, nrcv, 2] into the
    global shot order on rank 0 (None on the other ranks)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return local
    import torch
    world, rank = dist.get_world_size(), dist.get_rank()
    counts = [len(shots_for_rank(total, r, world)) for r in range(world)]
    tail = local.shape[1:]
    pad = max(counts)
    buf = np.zeros((pad,) + tail)
    buf[:local.shape[0]] = local
    t = torch.from_numpy(buf).to(device if device is not None else "cpu")
    parts = [torch.zeros_like(t) for _ in range(world)] if rank == 0 else None
    dist.gather(t, parts, dst=0)
    if rank != 0:
        return None
    return np.concatenate([p.cpu().numpy()[:c] for p, c in zip(parts, counts)], 0)
