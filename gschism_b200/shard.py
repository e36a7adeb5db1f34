"""Ensemble members across GPUs: one process per GPU, members assigned by HBM footprint.

The step has no data exchange between members, so multi-GPU work is member sharding: every rank
builds one batch context from its share of the members and steps it; the only collectives are the
max-over-ranks of the device time (for the job's throughput) and, if wanted, a gather of results.
"""
from __future__ import annotations

from typing import Callable, List, Sequence


def shard_members(weights: Sequence[float], world: int) -> List[List[int]]:
    """Greedy largest-first bin packing of members (by weight, e.g. device bytes) onto `world`
    ranks: each member goes to the currently lightest rank, ties to the lowest rank.  The result
    depends only on the weights, so every rank computes the same assignment without talking.
    Members keep their input order within a rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += float(weights[i])
    return [sorted(s) for s in out]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of a per-rank scalar (device time of the timed region) over all ranks."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(obj, dist=None) -> list:
    """Every rank's object, in rank order (all ranks receive the list)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out


def run_shard(cases, rank: int, world: int, steps: int, build: Callable, weights=None, dist=None):
    """Build this rank's members with `build(list_of_cases)` (a context with step(n) and
    elapsed timing) and step them; returns (member indices, context)."""
    from .model import footprint_bytes
    w = weights if weights is not None else [footprint_bytes([c]) for c in cases]
    mine = shard_members(w, world)[rank]
    ctx = build([cases[i] for i in mine]) if mine else None
    if ctx is not None and steps > 0:
        ctx.step(steps)
    return mine, ctx
