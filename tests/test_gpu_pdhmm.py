"""GPU parity of the PD-HMM against the FP64 PD oracle, through the C ABI.

Restates the reference's own PD tests (crates/pairhmm/src/pd.rs:132-465) with its regions (rebuilt
draw for draw from their seeds), tolerances (1e-9 log10 in double, 1e-4 in float) and invariants.
The "every backend" loops collapse to the one sm_100a backend.
"""
import numpy as np
import pytest

from fgkl_b200 import (ALT_C, ALT_G, ALT_T, DEL_END, DEL_START, SNP, BatchContext, Config, PairHmm, PdHaplotype, PdPairHmm,
                       Precision, Read, synthetic)
from oracle import oracle as O
from refgen import Rng

pytestmark = pytest.mark.gpu

FLOAT = Config(precision=Precision.FLOAT)
DOUBLE = Config(precision=Precision.DOUBLE)


def pd_region(seed, num_reads, read_len, num_haps, hap_len):
    return synthetic.reference_pd_region(seed, num_reads, read_len, num_haps, hap_len).region(0)


def reference_all(reads, haps):
    return O.compute_matrix(reads, haps)


def compute_counting(config, reads, haps):
    hmm = PdPairHmm(config)
    out = hmm.compute_log10_likelihoods(reads, haps)
    return out, hmm.fallback_pairs()


def compute(config, reads, haps):
    return compute_counting(config, reads, haps)[0]


def assert_close(actual, expected, tol, what=""):
    assert actual.shape == expected.shape
    d = np.abs(actual - expected)
    worst = int(np.argmax(d))
    assert np.all(d <= tol), f"{what}: pair {worst}: got {actual[worst]}, expected {expected[worst]} (diff {d[worst]})"
    assert np.isfinite(d).all()


def read(bases: bytes):
    n = len(bases)
    return Read(bases, bytes([30] * n), bytes([45] * n), bytes([45] * n), bytes([10] * n))


def region():
    return pd_region(31, 70, 120, 24, 300)


def test_double_precision_matches_the_pd_reference(gpu):
    reads, haps = region()
    assert_close(compute(DOUBLE, reads, haps), reference_all(reads, haps), 1e-9, "double")


def test_single_precision_matches_the_pd_reference_within_float_tolerance(gpu):
    reads, haps = region()
    assert_close(compute(FLOAT, reads, haps), reference_all(reads, haps), 1e-4, "float")


def test_flagged_alternates_and_deletions_change_the_result(gpu):
    reads, haps = region()
    unflagged = [PdHaplotype(h.bases, bytes(len(h.bases))) for h in haps]
    with_flags = compute(DOUBLE, reads, haps)
    without = compute(DOUBLE, reads, unflagged)
    changed = int(np.sum(np.abs(with_flags - without) > 1.0))
    assert changed >= 20, f"{changed} of {with_flags.size} pairs changed"
    # fgkl asserts this exactly (pd.rs:201), its FP64 arithmetic being the oracle's own. Here a pair
    # the flags do not affect is computed through other sharing chains (the PD sort key includes the
    # flags, and each resume rescales the state), so the two sides agree only to FP64 rounding:
    # 5.7e-14 in log10 at most on this region, each within that of the oracle.
    assert np.all(with_flags >= without - 1e-12), "flags never lower a likelihood"


def test_haplotypes_without_flags_agree_with_the_plain_kernel(gpu):
    reads, plain = synthetic.reference_region(5, 40, 100, 8, 200).region(0)
    pd = [PdHaplotype(h, bytes(len(h))) for h in plain]
    for precision, tol in ((Precision.DOUBLE, 1e-9), (Precision.FLOAT, 1e-4)):
        c = Config(precision=precision)
        assert_close(compute(c, reads, pd), PairHmm(c).compute_log10_likelihoods(reads, plain), tol, str(precision))


def test_flags_on_the_last_columns_carry_their_state_into_the_next_row(gpu):
    hap = b"ACGTTGCAAGGCTTAGGCTTACG"
    n = len(hap)
    ends_del = bytearray(n)
    ends_del[n - 3] = DEL_START
    ends_del[n - 1] = DEL_END
    starts_del = bytearray(n)
    starts_del[n - 1] = DEL_START
    single_del = bytearray(n)
    single_del[n - 1] = DEL_START | DEL_END
    first_del = bytearray(n)
    first_del[0] = DEL_START | DEL_END
    first_del[1] = SNP | ALT_G
    snp = bytearray(n)
    snp[n - 1] = SNP | ALT_C | ALT_T
    haps = [PdHaplotype(hap, bytes(f)) for f in (ends_del, starts_del, single_del, first_del, snp)]
    reads = [read(b"GTTGCAAGGCTTAG"), read(b"GGCTTAGGCTTACG"), read(b"GGCTTAGGCTTC"), read(b"GGCTTAGGCTTA"),
             read(b"CGTTGCAAGG"), read(hap)]
    expected = reference_all(reads, haps)
    assert_close(compute(DOUBLE, reads, haps), expected, 1e-9, "double")
    assert_close(compute(FLOAT, reads, haps), expected, 1e-4, "float")


def test_adjacent_and_single_base_deletions_match_the_reference(gpu):
    hap = b"ACGTTGCAAGGCTTAGGCTTACGATCGATTACA"
    n = len(hap)
    back_to_back = bytearray(n)
    back_to_back[5] = DEL_START
    back_to_back[7] = DEL_END
    back_to_back[8] = DEL_START | DEL_END
    back_to_back[9] = DEL_START
    back_to_back[12] = DEL_END
    singles = bytearray(n)
    for j in range(3, n, 4):
        singles[j] = DEL_START | DEL_END
    snp_in_del = bytearray(n)
    snp_in_del[10] = DEL_START
    snp_in_del[11] = SNP | ALT_T
    snp_in_del[13] = DEL_END | SNP | ALT_G
    haps = [PdHaplotype(hap, bytes(f)) for f in (back_to_back, singles, snp_in_del)]
    reads, _ = pd_region(9, 30, 25, 1, 33)
    assert_close(compute(DOUBLE, reads, haps), reference_all(reads, haps), 1e-9, "double")


def test_prefix_sharing_handles_nested_prefixes_lengths_and_flag_splits(gpu):
    base = b"ACGTTGCAAGGCTTAGGCTTACGATCGATTACAGGT"
    n = len(base)
    plain = bytes(n)
    snp_early = bytearray(n)
    snp_early[5] = SNP | ALT_T
    snp_late = bytearray(n)
    snp_late[30] = SNP | ALT_C
    del_mid = bytearray(n)
    del_mid[12] = DEL_START
    del_mid[15] = DEL_END
    del_mid_and_snp = bytearray(del_mid)
    del_mid_and_snp[25] = SNP | ALT_G
    del_last = bytearray(n)
    del_last[n - 2] = DEL_START
    del_last[n - 1] = DEL_END
    short = base[:20]
    short_del = bytearray(20)
    short_del[12] = DEL_START
    short_del[15] = DEL_END
    longer = base + b"ACGTAC"
    longer_flags = bytearray(len(longer))
    longer_flags[12] = DEL_START
    longer_flags[15] = DEL_END
    haps = [PdHaplotype(base, bytes(del_last)), PdHaplotype(base, bytes(snp_late)), PdHaplotype(short, bytes(short_del)),
            PdHaplotype(base, plain), PdHaplotype(base, bytes(del_mid_and_snp)), PdHaplotype(longer, bytes(longer_flags)),
            PdHaplotype(base, bytes(del_mid)), PdHaplotype(base, bytes(snp_early)), PdHaplotype(base, plain)]
    reads, _ = pd_region(13, 40, 30, 1, 36)
    expected = reference_all(reads, haps)
    assert_close(compute(DOUBLE, reads, haps), expected, 1e-9, "double")
    assert_close(compute(FLOAT, reads, haps), expected, 1e-4, "float")


def test_haplotype_order_does_not_change_results(gpu):
    reads, haps = region()
    fwd = compute(DOUBLE, reads, haps)
    rev = compute(DOUBLE, reads, haps[::-1])
    n = len(haps)
    for r in range(len(reads)):
        for h in range(n):
            assert abs(fwd[r * n + h] - rev[r * n + (n - 1 - h)]) < 1e-11, (r, h)


def test_float_underflow_falls_back_to_double(gpu):
    r = Read(b"A" * 80, bytes([40] * 80), bytes([45] * 80), bytes([45] * 80), bytes([10] * 80))
    flags = bytearray(80)
    flags[10] = DEL_START
    flags[20] = DEL_END
    haps = [PdHaplotype(b"C" * 80, bytes(flags))]
    expected = reference_all([r], haps)
    assert np.isfinite(expected[0]) and expected[0] < -50.0
    out, fallbacks = compute_counting(FLOAT, [r], haps)
    assert_close(out, expected, 1e-9)
    assert fallbacks == 1


def test_a_read_gets_the_same_bits_whatever_shares_its_batch(gpu):
    reads, haps = region()
    alone = reads[:3]
    rng = Rng(77)
    batched = list(alone) + [Read(bytes(rng.base() for _ in range(120)), bytes([30] * 120), bytes([45] * 120),
                                  bytes([45] * 120), bytes([10] * 120)) for _ in range(29)]
    for precision in (Precision.FLOAT, Precision.DOUBLE):
        c = Config(precision=precision)
        solo = compute(c, alone, haps)
        with_others, fallbacks = compute_counting(c, batched, haps)
        assert solo.tobytes() == with_others[:solo.size].tobytes(), precision
        if precision is Precision.FLOAT:
            assert fallbacks > 0, "the random reads must underflow"


@pytest.mark.parametrize("seed,n_reads", [(41, 1), (42, 37), (43, 65)])
def test_more_reads_than_lanes_and_single_read_both_work(gpu, seed, n_reads):
    reads, haps = pd_region(seed, n_reads, 50, 3, 60)
    assert_close(compute(Config(), reads, haps), reference_all(reads, haps), 1e-4, f"{n_reads} reads")


def test_pd_batch_of_regions_matches_the_oracle(gpu):
    parts = [pd_region(100 + i, 20, 90 + 30 * i, 6, 200 + 40 * i) for i in range(4)]
    w = synthetic.from_regions(parts)
    ctx = BatchContext()
    ctx.prepare(w, FLOAT)
    ctx.run()
    out, _ = ctx.fetch()
    expected = np.concatenate([reference_all(r, h) for r, h in parts])
    assert_close(out, expected, 1e-4, "batched PD")


def test_one_or_two_reads_per_warp_give_the_same_bits_and_the_autotuner_tries_both(gpu):
    # Two reads per warp run the FP32 recurrence in FP32x2 lanes, one read per warp in scalar FP32:
    # the same round-to-nearest operations in the same order, so every pair keeps its bits.
    parts = [pd_region(200 + i, 21, 100 + 20 * i, 5, 220) for i in range(3)]
    w = synthetic.from_regions(parts)
    pairs = BatchContext()
    two, _ = pairs.compute(w, FLOAT)
    single = BatchContext()
    single.set_tuning(8, 100, 1)
    one, _ = single.compute(w, FLOAT)
    assert one.tobytes() == two.tobytes()
    expected = np.concatenate([reference_all(r, h) for r, h in parts])
    assert_close(one, expected, 1e-4, "one read per warp")
    for warps in (1, 2):
        shaped = BatchContext()
        shaped.set_tuning(8, 100, 2, 0, warps)
        assert shaped.compute(w, FLOAT)[0].tobytes() == two.tobytes(), warps
    chosen, tried = BatchContext().autotune(w, FLOAT, repeats=1)
    assert len(tried) == 20  # 16 launch configurations, 2 with one read per warp, 2 tile shapes (warps)
    assert sorted({t["reads_per_warp"] for t in tried}) == [1, 2]
    assert sorted({t["warps_per_block"] for t in tried}) == [1, 2, 4]
    assert all(t["rows_extra"] == 0 for t in tried)
    assert chosen["ms"] == min(t["ms"] for t in tried)


def test_dense_reads_are_recomputed_with_their_shared_program(gpu):
    """fgkl lib.rs:495-520 for PD haplotypes: a read lost in FP32 against at least a third of them is
    recomputed in FP64 with its region's shared program (its lost pairs get the double-precision
    pass's bits), a read lost against fewer pair by pair; the pairs kept keep their FP32 bits."""
    rng = Rng(29)
    hap_len, read_len = 260, 120
    fam = [bytes(rng.base() for _ in range(hap_len)) for _ in range(2)]
    haps, fam_of_hap = [], []
    for f, count in ((0, 5), (1, 2)):
        for i in range(count):
            flags = bytearray(hap_len)
            for j in range(10, hap_len - 10, 53):
                flags[j] = SNP | ALT_G
            flags[100] |= DEL_START
            flags[103] |= DEL_END
            if i < 3:  # near the end (long shared prefixes); the family's last two are duplicates
                flags[hap_len - 40 + rng.below(30)] |= SNP | ALT_T
            haps.append(PdHaplotype(fam[f], bytes(flags)))
            fam_of_hap.append(f)
    reads, owner = [], []
    for i in range(12):
        f = int(i % 3 == 2)
        start = rng.below(hap_len - read_len)
        reads.append(Read(fam[f][start:start + read_len], bytes(20 + rng.below(21) for _ in range(read_len)),
                          bytes([45] * read_len), bytes([45] * read_len), bytes([10] * read_len)))
        owner.append(f)
    expected = reference_all(reads, haps).reshape(len(reads), len(haps))
    lost_mask = np.array([[owner[r] != fam_of_hap[h] for h in range(len(haps))] for r in range(len(reads))])
    assert (expected[lost_mask] < -70.0).all() and (expected[~lost_mask] > -60.0).all()
    out, fallbacks = compute_counting(FLOAT, reads, haps)
    out = out.reshape(len(reads), len(haps))
    assert fallbacks == int(lost_mask.sum())
    assert_close(out[lost_mask], expected[lost_mask], 1e-9, "lost pairs")
    assert_close(out[~lost_mask], expected[~lost_mask], 1e-4, "kept pairs")
    double = compute(DOUBLE, reads, haps).reshape(len(reads), len(haps))
    for r in range(len(reads)):
        if owner[r] == 1:
            assert out[r][lost_mask[r]].tobytes() == double[r][lost_mask[r]].tobytes(), r


def test_a_long_pd_haplotype_resumed_from_a_one_base_prefix_keeps_its_own_scale(gpu):
    # As in the plain kernel: the resumed segment, branch values included, is rescaled to its own
    # initial constant, so a short read's likelihood near 1 does not overflow.
    rng = Rng(78)
    bases = b"C" + bytes(rng.base() for _ in range(1999))
    flags = bytearray(len(bases))
    flags[40] = DEL_START
    flags[43] = DEL_END
    flags[900] = SNP | ALT_G
    haps = [PdHaplotype(bases, bytes(flags)), PdHaplotype(b"C", b"\x00"), PdHaplotype(bases[:700], bytes(flags[:700]))]
    reads = [read(b"A"), read(b"CT"), read(b"GCA"), read(bases[30:60])]
    expected = reference_all(reads, haps)
    assert_close(compute(DOUBLE, reads, haps), expected, 1e-9, "double")
    assert_close(compute(Config(precision=Precision.FLOAT, double_fallback=True), reads, haps), expected, 1e-4, "float")
