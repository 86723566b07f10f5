"""Region sharding across GPUs (one process per GPU).

Regions are independent and nothing is exchanged between them (fgkl docs/design.md:37-39), so a
batch splits across ranks with no data-path collective: each rank plans, uploads and runs its own
regions on its own GPU. `partition_regions` balances ranks greedily by estimated cost (longest
first onto the least-loaded rank); `assemble` puts each rank's outputs back in the caller's region
order. Timing is the max over ranks; the only collectives are that max and the optional gather of
results, neither on the hot path.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np


def region_costs(workload) -> np.ndarray:
    """Per-region cost estimate: nominal cells (Σ read lengths x Σ haplotype lengths)."""
    return workload.region_nominal_cells().astype(np.float64)


def partition_regions(costs: Sequence[float], world: int) -> list[list[int]]:
    """Assigns regions to `world` ranks: costliest first, each to the least-loaded rank (ties to the
    lowest rank); each rank's regions in ascending order."""
    if world < 1:
        raise ValueError("world must be at least 1")
    costs = np.asarray(costs, np.float64)
    order = sorted(range(costs.size), key=lambda g: (-costs[g], g))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for g in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(g)
        load[r] += float(costs[g])
    return [sorted(p) for p in parts]


def rank_workload(workload, regions: Sequence[int]):
    """The sub-batch of `regions` (a Workload with the same layout)."""
    return workload.subset(list(regions))


def assemble(workload, partition: list[list[int]], outputs: list[np.ndarray]) -> np.ndarray:
    """The whole batch's likelihoods from each rank's outputs (its regions' blocks in its order)."""
    offs = workload.output_offsets()
    full = np.empty(int(offs[-1]), np.float64)
    for regions, out in zip(partition, outputs):
        pos = 0
        for g in regions:
            n = int(offs[g + 1] - offs[g])
            full[offs[g]:offs[g + 1]] = out[pos:pos + n]
            pos += n
        if pos != out.size:
            raise ValueError("a rank's output does not match its regions")
    return full


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """The max of `value` over the process group (`dist` = torch.distributed, or None for one rank)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
