"""Ciphertext-level sharding across ranks (one process per GPU).

Bootstrapping and serving units are independent ciphertexts (or shared-a groups), so a
batch splits by contiguous ranges with no collective on the data path; the only
collectives are the max-over-ranks of the step time and the final gather of results
to rank 0.  Works with any torch.distributed backend (NCCL on the B200s, gloo on CPU).
"""
from __future__ import annotations


def shard(total: int, rank: int, world: int, unit: int = 1) -> tuple[int, int]:
    """(start, count) of rank's contiguous share of `total` items, in multiples of `unit`
    (a shared-a group size) except for the remainder on the last ranks."""
    if total % unit:
        raise ValueError("total is not a multiple of the unit")
    groups = total // unit
    base, extra = divmod(groups, world)
    start = (rank * base + min(rank, extra)) * unit
    count = (base + (1 if rank < extra else 0)) * unit
    return start, count


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest `value` over all ranks (a step time); identity without a process group."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_rank0(obj, dist=None):
    """List of every rank's `obj` on rank 0 (None elsewhere); [obj] without a process group."""
    if dist is None:
        return [obj]
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out
