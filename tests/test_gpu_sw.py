"""GPU Smith-Waterman against the oracle (oracle/sw_oracle.c, GATK's SmithWatermanJavaAligner as fgkl
restates it in crates/smithwaterman/src/reference.rs), through the C ABI.

Restates fgkl's own Smith-Waterman tests (crates/smithwaterman/src/lib.rs:854-1065): the known
answers, random related and unrelated pairs under the three parameter sets and four overhang
strategies, odd scores, and pairs whose reference spans several 256-row blocks. Alignments are
integers, so CIGAR and offset must be identical.
"""
import pytest

from fgkl_b200 import _lib
from fgkl_b200.pairhmm import DeviceError
from fgkl_b200.sw import (ALIGNMENT_TO_BEST_HAPLOTYPE, HAPLOTYPE_TO_REFERENCE, ORIGINAL_DEFAULT, Alignment, OverhangStrategy,
                          SwParameters, align, align_batch)
from oracle import oracle as O
from refgen import Rng, related_pair

pytestmark = pytest.mark.gpu

HAP_TO_REF, READ_TO_HAP, ORIGINAL = HAPLOTYPE_TO_REFERENCE, ALIGNMENT_TO_BEST_HAPLOTYPE, ORIGINAL_DEFAULT
STRATEGIES = list(OverhangStrategy)


def expected(ref, alt, params, strategy):
    cigar, offset = O.sw_align(ref, alt, (params.match_value, params.mismatch_penalty, params.gap_open_penalty,
                                          params.gap_extend_penalty), int(strategy))
    return Alignment(cigar, offset)


def check_batch(pairs, params, strategy):
    got = align_batch(pairs, params, strategy)
    for k, ((r, a), g) in enumerate(zip(pairs, got)):
        assert g == expected(r, a, params, strategy), (k, len(r), len(a), strategy, params)


def test_exact_substring_short_circuits_for_softclip_and_ignore(gpu):
    assert align(b"AAACGTACGTAAA", b"ACGTACGT", HAP_TO_REF, OverhangStrategy.SOFTCLIP) == Alignment("8M", 2)
    assert align(b"ACGTACGTACGT", b"ACGT", HAP_TO_REF, OverhangStrategy.IGNORE).offset == 8


def test_simple_indels_are_reported_with_gatk_conventions(gpu):
    reference = b"NNNNNNNNNNACGTTTGCAAGGCTTAGGCTNNNNNNNNNN"
    assert align(reference, b"NNNNNNNNNNACGTTTGCGGCTTAGGCTNNNNNNNNNN", HAP_TO_REF, OverhangStrategy.INDEL) == \
        Alignment("18M2D20M", 0)
    assert align(reference, b"NNNNNNNNNNACGTTTGCAAGGCTTTTAGGCTNNNNNNNNNN", HAP_TO_REF, OverhangStrategy.INDEL) == \
        Alignment("23M2I17M", 0)


def test_soft_clips_read_bases_beyond_the_reference_ends(gpu):
    read = b"GGGGACGTACGTAGGCCTTAGCAGGGG"
    assert align(b"ACGTACGTAGGCCTTAGCA", read, READ_TO_HAP, OverhangStrategy.SOFTCLIP) == Alignment("4S19M4S", 0)
    padded = b"TTTTTTTTTTACGTACGTAGGCCTTAGCATTTTTTTTTT"
    assert align(padded, read, READ_TO_HAP, OverhangStrategy.SOFTCLIP).cigar == "4I19M4I"


def test_empty_sequences_and_unknown_strategies_are_rejected(gpu):
    with pytest.raises(DeviceError) as e:
        align(b"", b"A", HAP_TO_REF, OverhangStrategy.SOFTCLIP)
    assert e.value.code == _lib.FGKL_E_EMPTY_SEQUENCE
    with pytest.raises(DeviceError) as e:
        align(b"A", b"", HAP_TO_REF, OverhangStrategy.INDEL)
    assert e.value.code == _lib.FGKL_E_EMPTY_SEQUENCE
    with pytest.raises(DeviceError) as e:
        align(b"ACGT", b"ACG", HAP_TO_REF, 7)
    assert e.value.code == _lib.FGKL_E_INVALID_ARGUMENT


@pytest.mark.parametrize("strategy", STRATEGIES)
@pytest.mark.parametrize("params", [HAP_TO_REF, READ_TO_HAP, ORIGINAL], ids=["hap_to_ref", "read_to_hap", "original"])
def test_matches_the_oracle_on_random_related_sequences(gpu, params, strategy):
    rng = Rng(7)
    pairs = []
    for case in range(200):
        ref_len, alt_len = (40 + rng.below(300), 20 + rng.below(200)) if case % 2 == 0 else (5 + rng.below(30), 3 + rng.below(30))
        pairs.append(related_pair(rng, ref_len, alt_len))
    check_batch(pairs, params, strategy)


@pytest.mark.parametrize("strategy", STRATEGIES)
def test_matches_the_oracle_on_unrelated_sequences(gpu, strategy):
    rng = Rng(11)
    pairs = [(bytes(rng.base() for _ in range(5 + rng.below(80))), bytes(rng.base() for _ in range(5 + rng.below(80))))
             for _ in range(100)]
    check_batch(pairs, HAP_TO_REF, strategy)
    check_batch(pairs, READ_TO_HAP, strategy)


@pytest.mark.parametrize("strategy", STRATEGIES)
def test_odd_scores(gpu, strategy):
    rng = Rng(31)
    dangling = SwParameters(25, -50, -110, -6)
    pairs = [related_pair(rng, 40 + rng.below(200), 20 + rng.below(150)) for _ in range(50)]
    check_batch(pairs, dangling, strategy)


@pytest.mark.parametrize("strategy", STRATEGIES)
def test_references_spanning_several_row_blocks(gpu, strategy):
    """References of 257 to 1,500 bases run over consecutive 256-row blocks."""
    rng = Rng(13)
    pairs = [related_pair(rng, 600, 520), related_pair(rng, 257, 200), related_pair(rng, 1500, 900), related_pair(rng, 513, 40)]
    r = bytes(rng.base() for _ in range(700))
    pairs.append((r, bytes(rng.base() for _ in range(700))))  # unrelated: short local alignments deep in the matrix
    check_batch(pairs, HAP_TO_REF, strategy)
    check_batch(pairs, READ_TO_HAP, strategy)


def test_batch_and_per_call_agree(gpu):
    rng = Rng(23)
    pairs = [related_pair(rng, 30 + rng.below(400), 10 + rng.below(300)) for _ in range(40)]
    batch = align_batch(pairs, READ_TO_HAP, OverhangStrategy.SOFTCLIP)
    assert batch == [align(r, a, READ_TO_HAP, OverhangStrategy.SOFTCLIP) for r, a in pairs]


def test_the_batch_kernel_time_is_reported_for_the_last_call(gpu):
    import ctypes as C
    import time

    from fgkl_b200 import BatchContext

    ctx = BatchContext()
    try:
        ms = C.c_float()
        # No batch yet on this context: an error, not a stale number.
        assert _lib.lib().fgkl_sw_last_kernel_ms(ctx._ctx, C.byref(ms)) != 0
        rng = Rng(41)
        pairs = [related_pair(rng, 300, 280) for _ in range(64)]
        t0 = time.perf_counter()
        check_batch_on(ctx, pairs)
        wall_ms = 1e3 * (time.perf_counter() - t0)
        assert _lib.lib().fgkl_sw_last_kernel_ms(ctx._ctx, C.byref(ms)) == 0
        assert 0.0 < ms.value < wall_ms
    finally:
        ctx.close()


def check_batch_on(ctx, pairs):
    got = align_batch(pairs, HAP_TO_REF, OverhangStrategy.INDEL, ctx)
    for (r, a), g in zip(pairs, got):
        assert g == expected(r, a, HAP_TO_REF, OverhangStrategy.INDEL)


def test_the_integer_alu_probe_measures_a_plausible_rate(gpu):
    import ctypes as C

    gops = C.c_double()
    assert _lib.lib().fgkl_probe_int32_alu_gops(0, C.byref(gops)) == 0
    # 148 SMs at up to 64 ALU operations a cycle near 2 GHz: some thousands of Gop/s, never above the
    # 128-lane FP32 rate.
    assert 1000.0 < gops.value < 148 * 128 * 2.1


def test_weak_alignments_of_unrelated_700_mers(gpu):
    # fgkl's weak_alignments_saturate_the_narrow_lanes_and_fall_back_exactly (lib.rs:855-866): its
    # 16-bit lanes saturate here; the 32-bit scores here have no narrow form, but the case stands.
    rng = Rng(23)
    r = bytes(rng.base() for _ in range(700))
    a = bytes(rng.base() for _ in range(700))
    want = expected(r, a, HAP_TO_REF, OverhangStrategy.SOFTCLIP)
    assert align(r, a, HAP_TO_REF, OverhangStrategy.SOFTCLIP) == want
    assert align_batch([(r, a)], HAP_TO_REF, OverhangStrategy.SOFTCLIP) == [want]


def test_a_haplotype_matching_the_far_end_of_the_reference(gpu):
    # fgkl's a_haplotype_matching_the_far_end_of_the_reference_stays_in_narrow_lanes (lib.rs:869-881).
    rng = Rng(29)
    r = bytes(rng.base() for _ in range(600))
    a = bytearray(r[380:])
    a[100] = ord("C") if a[100] == ord("A") else ord("A")
    a = bytes(a)
    want = expected(r, a, HAP_TO_REF, OverhangStrategy.SOFTCLIP)
    assert align(r, a, HAP_TO_REF, OverhangStrategy.SOFTCLIP) == want
    assert align_batch([(r, a)], HAP_TO_REF, OverhangStrategy.SOFTCLIP) == [want]


def test_a_reused_context_matches_the_oracle_as_pair_sizes_shrink_and_grow(gpu):
    # fgkl's a_reused_aligner_matches_the_reference_as_pair_sizes_shrink_and_grow (lib.rs:1023-1065):
    # the first pair is unrelated, and the scratch each later pair finds is what the earlier ones left.
    from fgkl_b200 import BatchContext

    rng = Rng(11)
    sizes = [(600, 520), (500, 150), (40, 30), (320, 310), (8, 5), (590, 600), (60, 200)]
    pairs = []
    for k, (n, m) in enumerate(sizes):
        if k == 0:
            pairs.append((bytes(rng.base() for _ in range(n)), bytes(rng.base() for _ in range(m))))
        else:
            pairs.append(related_pair(rng, n, m))
    ctx = BatchContext()
    try:
        for r, a in pairs:
            for params in (HAP_TO_REF, READ_TO_HAP):
                for strategy in STRATEGIES:
                    want = expected(r, a, params, strategy)
                    assert align(r, a, params, strategy) == want, (len(r), len(a), strategy)
                    assert align_batch([(r, a)], params, strategy, ctx) == [want], (len(r), len(a), strategy)
    finally:
        ctx.close()
