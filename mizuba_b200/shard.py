"""Time-axis sharding of a conjunction screen across ranks.

Conjunction steps are independent (mizuba/detect_conjunctions.cpp:338-417
shares no state between steps), so a multi-GPU screen gives each rank a
contiguous range of steps and needs no collective on the data path: the
only cross-rank operation is the max-reduction of the per-rank times.
"""

from __future__ import annotations


def step_range(rank: int, world: int, n_steps: int):
    """Contiguous, balanced step range [begin, end) of `rank` out of `world`."""
    if not (0 <= rank < world):
        raise ValueError(f"invalid rank {rank} for a world of size {world}")
    base, extra = divmod(n_steps, world)
    begin = rank * base + min(rank, extra)
    end = begin + base + (1 if rank < extra else 0)
    return begin, end


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar over the default process group (identity
    without one).  Used for the benchmark's times."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
