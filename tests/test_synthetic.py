"""Synthetic generators: fgkl's Region/PdRegion restated draw for draw, and the workload shapes."""
import numpy as np

from fgkl_b200 import synthetic
from refgen import Rng


def test_rng_matches_splitmix64_reference_values():
    # SplitMix64 from seed 0: the first outputs of the published algorithm.
    r = Rng(0)
    assert [r.next_u64() for _ in range(3)] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_same_seed_gives_the_same_region():
    a = synthetic.reference_region(5, 20, 50, 4, 80)
    b = synthetic.reference_region(5, 20, 50, 4, 80)
    assert a.hap_bases.tobytes() == b.hap_bases.tobytes()
    assert a.bases.tobytes() == b.bases.tobytes() and a.quals.tobytes() == b.quals.tobytes()


def test_reference_region_shapes_follow_the_generator():
    w = synthetic.reference_region(11, 70, 120, 24, 300)
    reads, haps = w.region(0)
    assert len(reads) == 70 and len(haps) == 24
    assert haps[0] == bytes(Rng_bases(11, 300))
    assert all(1 <= len(r.bases) <= 120 for r in reads)
    assert all(set(r.gcp) == {10} for r in reads)


def Rng_bases(seed, n):
    r = Rng(seed)
    return [r.base() for _ in range(n)]


def test_pd_region_reads_are_valid_and_haplotypes_carry_flags():
    w = synthetic.reference_pd_region(31, 70, 120, 24, 300)
    reads, haps = w.region(0)
    assert all(len(r.bases) > 0 for r in reads)
    assert any(any(f != 0 for f in h.flags) for h in haps)
    assert w.nominal_cells() > 0


def test_workload_shapes():
    w0 = synthetic.workload(0, seed=0)
    assert w0.num_regions == 1
    reads, haps = w0.region(0)
    assert len(reads) == 32 and all(len(r.bases) == 151 for r in reads)
    assert len(haps) == 4 and all(280 <= len(h) <= 320 for h in haps)
    w1 = synthetic.workload(1, seed=1, regions=64)
    assert w1.num_regions == 64
    assert (w1.region_reads >= 8).all() and (w1.region_reads <= 256).all()
    assert (w1.region_haps >= 2).all() and (w1.region_haps <= 32).all()
    lens = np.diff(w1.read_offsets)
    assert 0.6 < np.mean(lens == 151) < 0.9 and lens.min() >= 50 and lens.max() <= 250
    w2 = synthetic.workload(2, seed=2, regions=2)
    reads, haps = w2.region(0)
    assert len(reads) == 200 and len(haps) == 128 and all(len(h) == 400 for h in haps)
    assert all(h[340:] == haps[0][340:] and h[:200] == haps[0][:200] for h in haps)
    w3 = synthetic.workload(3, seed=3, regions=2)
    reads, haps = w3.region(0)
    assert len(reads) == 64 and len(haps) == 16 and w3.hap_flags is not None
    flags = np.frombuffer(b"".join(h.flags for h in haps), np.uint8)
    assert 0.03 < np.mean(flags & 1) < 0.08
    w4 = synthetic.workload(4, seed=4, regions=3)
    assert w4.num_regions == 3 and set(w4.region_haps) == {8} and set(w4.region_reads) == {64}


def test_workloads_are_deterministic_across_thread_counts():
    a = synthetic.workload(1, seed=9, regions=16, threads=1)
    b = synthetic.workload(1, seed=9, regions=16, threads=8)
    assert a.bases.tobytes() == b.bases.tobytes() and a.hap_bases.tobytes() == b.hap_bases.tobytes()
