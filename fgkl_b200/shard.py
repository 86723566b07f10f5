"""Region sharding across GPUs: one batch split over several devices.

Regions are independent and nothing is exchanged between them (fgkl docs/design.md:37-39), so a
batch splits across devices with no data-path collective: each device plans, uploads and runs its
own regions. `region_costs` asks the planner for the DP cells each region's batched run computes
(prefix and suffix sharing included); `partition_regions` balances devices greedily by that cost
(longest first onto the least-loaded device); `assemble` puts each device's outputs back in the
caller's region order. Two ways to use it:

- `MultiDeviceContext`: one process drives several devices (one batch context each).
- one process per GPU (torchrun): every rank partitions the same batch and runs its own part;
  timing is the max over ranks, and the only collectives are that max and the optional gather of
  results, neither on the hot path.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np


def region_costs(workload, config=None) -> np.ndarray:
    """Per region, the DP cells a batched run computes (fgkl_plan_region_cells; host only)."""
    from . import _lib
    from .pairhmm import Config, _check

    cells = np.zeros(workload.num_regions, np.uint64)
    if workload.num_regions == 0:
        return cells.astype(np.float64)
    b = workload.as_batch()
    cfg = (config or Config())._c()
    _check(_lib.lib().fgkl_plan_region_cells(C.byref(b), C.byref(cfg), cells.ctypes.data_as(C.POINTER(C.c_uint64))))
    return cells.astype(np.float64)


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


class MultiDeviceContext:
    """One batch over several devices from one process: regions partitioned by planned cells, one
    batch context (engine, streams, CUDA graph) per device, each part planned and launched before the
    next is planned, results reassembled in the caller's order. `devices` may repeat a device (two
    contexts sharing it)."""

    def __init__(self, devices: Sequence[int]):
        from .pairhmm import BatchContext

        if not devices:
            raise ValueError("at least one device")
        self.devices = list(devices)
        self.contexts = [BatchContext(d) for d in self.devices]
        self.partition: list[list[int]] = []

    def compute(self, workload, config=None) -> np.ndarray:
        self.partition = partition_regions(region_costs(workload, config), len(self.contexts))
        parts = [rank_workload(workload, p) for p in self.partition]
        for ctx, w in zip(self.contexts, parts):
            if w.num_regions:
                ctx.prepare(w, config)
                ctx.run()
        outputs = [ctx.fetch()[0] if w.num_regions else np.zeros(0) for ctx, w in zip(self.contexts, parts)]
        return assemble(workload, self.partition, outputs)

    def close(self) -> None:
        for ctx in self.contexts:
            ctx.close()
