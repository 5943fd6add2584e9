"""Host-side plumbing of multi-GPU runs: one process per GPU, independent
units (ensemble scenarios, training runs, held-out inversions, grid
replicas) split across ranks with no data-path collective, and the run's
figures combined once at the end (timings: max over ranks; work: sum).
"""
from __future__ import annotations

from typing import List, Sequence

import torch


def shard_indices(count: int, world: int, rank: int) -> List[int]:
    """Round-robin share of `count` units for `rank` of `world`."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return list(range(rank, count, world))


def reduce_over_ranks(values: Sequence[float], op: str, device=None) -> List[float]:
    """All-reduce a few floats (float64) with op "max" or "sum"; identity
    when torch.distributed is not initialised."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    ops = {"max": dist.ReduceOp.MAX, "sum": dist.ReduceOp.SUM}
    if op not in ops:
        raise ValueError(f"op must be max or sum, got {op!r}")
    t = torch.tensor([float(v) for v in values], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=ops[op])
    return [float(v) for v in t.cpu()]


def gather_rows(count: int, mine: Sequence[int], tensors: Sequence, world: int) -> List:
    """Each rank holds rows `mine` (indices into `count` units) of some
    tensors; returns on every rank the full tensors [count, ...] in unit
    order (one all_gather of the host copies, once, at the end of a run)."""
    import torch.distributed as dist
    local = [None if t is None else t.detach().cpu() for t in tensors]
    parts = [None] * world
    dist.all_gather_object(parts, (list(mine), local))
    device = next((t.device for t in tensors if t is not None), torch.device("cpu"))
    out = []
    for j in range(len(tensors)):
        rows = {}
        for idx, ts in parts:
            if ts[j] is None:
                continue
            for r, i in enumerate(idx):
                rows[i] = ts[j][r]
        if len(rows) != count:
            raise RuntimeError(f"gathered {len(rows)} of {count} units")
        out.append(torch.stack([rows[i] for i in range(count)]).to(device))
    return out


__all__ = ["shard_indices", "reduce_over_ranks", "gather_rows"]
