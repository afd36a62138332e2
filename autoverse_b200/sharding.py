"""Independent worlds across ranks (one process per GPU).

Worlds never interact, so a batch shards with no data-path collective: every
rank computes the same cost-balanced partition of the world list, runs its
share through its own BatchedPropagator, and per-world scalars (mass, metrics)
are gathered once at the end.  The reference runs such populations one
CpuPropagator per candidate over a rayon pool (src/evolution/search.rs:152-172).
"""
from __future__ import annotations

import heapq
import math
from typing import Any, Callable, Sequence

from .propagator import SimulationConfig


def world_cost(config: Any) -> float:
    """Relative cost of one step of one world: the FFT passes (one forward per
    source channel, one inverse per kernel, N log2 N each) plus the per-cell
    stencil and gather work of every channel."""
    c = SimulationConfig.load(config)
    n = c.width * c.height * c.depth
    kernels = c.get("kernels", [])
    n_src = len({k["source_channel"] for k in kernels})
    return n * (math.log2(max(n, 2)) * (n_src + len(kernels)) + 24.0 * c.channels)


def lpt_partition(costs: Sequence[float], n_ranks: int) -> list[list[int]]:
    """Longest-processing-time-first: worlds in decreasing cost, each to the
    currently least-loaded rank (ties to the lower rank).  Deterministic, so
    every rank derives the same partition without communicating; the largest
    load is at most 4/3 of the optimum.  Each rank's list is in world order."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(n_ranks)]
    parts: list[list[int]] = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def batched_runner(worlds: Sequence[tuple[Any, Any]], steps: int) -> list[float]:
    """Runs worlds (config, seed) for `steps` steps in one BatchedPropagator on
    the current device; returns each world's FP64 total mass."""
    from .batch import BatchedPropagator
    if not worlds:
        return []
    with BatchedPropagator([c for c, _ in worlds]) as b:
        for i, (_, seed) in enumerate(worlds):
            b.load_seed(i, seed)
        b.run(steps)
        b.synchronize()
        return [float(m) for m in b.total_mass()]


def run_sharded(worlds: Sequence[tuple[Any, Any]], steps: int, rank: int = 0, world_size: int = 1,
                group: Any = None, runner: Callable[[Sequence[tuple[Any, Any]], int], list] = batched_runner) -> list:
    """Runs this rank's LPT share of `worlds` and returns every world's result
    in world order on every rank (one all_gather_object at the end; none when
    world_size is 1)."""
    parts = lpt_partition([world_cost(c) for c, _ in worlds], world_size)
    mine = parts[rank]
    local = runner([worlds[i] for i in mine], steps)
    if world_size == 1:
        return list(local)
    import torch.distributed as dist
    gathered: list = [None] * world_size
    dist.all_gather_object(gathered, (mine, list(local)), group=group)
    out: list = [None] * len(worlds)
    for idx, vals in gathered:
        for i, v in zip(idx, vals):
            out[i] = v
    return out
