"""Region sharding for N > 1 GPUs, on the CPU: the partition, the reassembly of outputs and the
max-over-ranks timing, with world_size 2 `gloo` process groups (no GPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from fgkl_b200 import synthetic
from fgkl_b200.shard import assemble, max_over_ranks, partition_regions, region_costs


def test_partition_covers_every_region_once_and_balances_cost():
    rng = np.random.default_rng(3)
    costs = rng.integers(1, 1000, size=257).astype(float)
    for world in (1, 2, 3, 8):
        parts = partition_regions(costs, world)
        flat = sorted(g for p in parts for g in p)
        assert flat == list(range(costs.size))
        loads = [costs[p].sum() for p in parts]
        # Greedy longest-first: no rank exceeds the average by more than the largest single cost.
        assert max(loads) <= costs.sum() / world + costs.max()


def test_partition_is_deterministic_and_handles_more_ranks_than_regions():
    assert partition_regions([5, 5, 5], 2) == partition_regions([5, 5, 5], 2)
    parts = partition_regions([1.0, 2.0], 4)
    assert sorted(len(p) for p in parts) == [0, 0, 1, 1]


def test_assemble_restores_the_caller_region_order():
    parts_in = [synthetic.reference_region(s, 3 + s, 20, 2 + s % 3, 40).region(0) for s in range(6)]
    w = synthetic.from_regions(parts_in)
    offs = w.output_offsets()
    expected = np.arange(offs[-1], dtype=np.float64)
    partition = partition_regions(region_costs(w), 3)
    outputs = [np.concatenate([expected[offs[g]:offs[g + 1]] for g in p]) if p else np.zeros(0) for p in partition]
    assert np.array_equal(assemble(w, partition, outputs), expected)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        parts_in = [synthetic.reference_region(10 + s, 4, 30, 3, 50).region(0) for s in range(5)]
        w = synthetic.from_regions(parts_in)
        partition = partition_regions(region_costs(w), world)
        offs = w.output_offsets()
        # Stand-in for the rank's GPU results: each pair's global output index.
        mine = np.concatenate([np.arange(offs[g], offs[g + 1], dtype=np.float64) for g in partition[rank]]) \
            if partition[rank] else np.zeros(0)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        step_max = max_over_ranks(0.5 + rank, dist)
        if rank == 0:
            full = assemble(w, partition, gathered)
            q.put((bool(np.array_equal(full, np.arange(offs[-1], dtype=np.float64))), step_max))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_shard_gather_and_take_the_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(100)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    ok, step_max = q.get(timeout=5)
    assert ok
    assert step_max == 1.5
