"""Region sharding for N > 1 GPUs, on the CPU: the planner's per-region cells, the partition, the
per-rank sub-batches, the reassembly of outputs and the max-over-ranks timing, with world_size 2
`gloo` process groups (no GPU). tests/test_gpu_shard.py runs the same path on a device."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from fgkl_b200 import Read, synthetic
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


def test_planned_cells_reflect_sharing():
    """Regions of shared haplotypes cost less than their nominal cells; reads beyond one block and
    unshared runs cost their full cells."""
    w = synthetic.workload(2, seed=4, regions=3, threads=4)
    planned = region_costs(w)
    nominal = w.region_nominal_cells()
    assert np.all(planned > 0) and np.all(planned < 0.6 * nominal)
    hap = bytes(b"ACGT"[(7 * i + i // 5) % 4] for i in range(800))
    reads = [Read(hap[s:s + 700], bytes([30] * 700), bytes([45] * 700), bytes([45] * 700), bytes([10] * 700)) for s in (0, 50)]
    one = synthetic.from_regions([(reads, [hap, hap])])
    assert region_costs(one)[0] == 2 * 700 * 800  # the duplicate haplotype runs once


def test_subset_keeps_each_region_and_its_order():
    w = synthetic.workload(1, seed=9, regions=12, threads=4)
    pick = [7, 0, 11, 3]
    sub = w.subset(pick)
    assert sub.num_regions == 4
    for i, g in enumerate(pick):
        assert sub.region(i) == w.region(g)


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
        # The bench's sharding: every rank draws the same batch, partitions it by planned cells and
        # takes its part as a sub-batch.
        w = synthetic.workload(1, seed=5, regions=9, threads=2)
        partition = partition_regions(region_costs(w), world)
        part = w.subset(partition[rank])
        offs = w.output_offsets()
        assert part.output_len() == sum(int(offs[g + 1] - offs[g]) for g in partition[rank])
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
