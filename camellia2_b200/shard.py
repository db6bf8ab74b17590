"""Multi-rank plumbing for the per-cell assembly: one process per GPU.

Cells are independent units (a cell's K, l, S, s depend only on its own vertices,
side parities and coefficients), so ranks take disjoint cell ranges and the data
path has no collective; torch.distributed carries only the barrier and the
max-over-ranks step time of a measurement."""
from __future__ import annotations


def shard_range(C: int, rank: int, world: int):
    """Contiguous cell range [lo, hi) of `rank` among `world` ranks (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    base, extra = divmod(C, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def max_over_ranks(x: float, device=None) -> float:
    """Maximum of a per-rank scalar over the process group (the step time every
    rank waits for); the identity without an initialised group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
