"""The Smith-Waterman oracle (oracle/sw_oracle.c) against the known answers of fgkl's own tests
(crates/smithwaterman/src/lib.rs:927-981), which pin GATK's conventions: the exact-substring
shortcut (last occurrence wins), indel placement, soft clips, and rejection of empty sequences."""
import pytest

from oracle import oracle as O

HAP_TO_REF = (200, -150, -260, -11)   # lib.rs:741
READ_TO_HAP = (10, -15, -30, -5)      # lib.rs:742
SOFTCLIP, INDEL, LEADING_INDEL, IGNORE = 0, 1, 2, 3


def test_exact_substring_short_circuits_for_softclip_and_ignore():
    assert O.sw_align(b"AAACGTACGTAAA", b"ACGTACGT", HAP_TO_REF, SOFTCLIP) == ("8M", 2)
    cigar, offset = O.sw_align(b"ACGTACGTACGT", b"ACGT", HAP_TO_REF, IGNORE)
    assert offset == 8, "last occurrence wins"


def test_simple_indels_are_reported_with_gatk_conventions():
    reference = b"NNNNNNNNNNACGTTTGCAAGGCTTAGGCTNNNNNNNNNN"
    deletion = b"NNNNNNNNNNACGTTTGCGGCTTAGGCTNNNNNNNNNN"
    assert O.sw_align(reference, deletion, HAP_TO_REF, INDEL) == ("18M2D20M", 0)
    insertion = b"NNNNNNNNNNACGTTTGCAAGGCTTTTAGGCTNNNNNNNNNN"
    # The extra TT lands at the left of the run of Ts because ties prefer the diagonal.
    assert O.sw_align(reference, insertion, HAP_TO_REF, INDEL) == ("23M2I17M", 0)


def test_soft_clips_read_bases_beyond_the_reference_ends():
    hap = b"ACGTACGTAGGCCTTAGCA"
    read = b"GGGGACGTACGTAGGCCTTAGCAGGGG"
    assert O.sw_align(hap, read, READ_TO_HAP, SOFTCLIP) == ("4S19M4S", 0)
    padded = b"TTTTTTTTTTACGTACGTAGGCCTTAGCATTTTTTTTTT"
    assert O.sw_align(padded, read, READ_TO_HAP, SOFTCLIP)[0] == "4I19M4I"


def test_empty_sequences_are_rejected():
    with pytest.raises(ValueError):
        O.sw_align(b"", b"A", HAP_TO_REF, SOFTCLIP)
    with pytest.raises(ValueError):
        O.sw_align(b"A", b"", HAP_TO_REF, INDEL)


@pytest.mark.parametrize("strategy", [SOFTCLIP, INDEL, LEADING_INDEL, IGNORE])
def test_every_cigar_spans_the_alternate(strategy):
    """Whatever the strategy, M, I and S elements cover the alternate exactly once."""
    import random

    rng = random.Random(5)
    for _ in range(50):
        ref = bytes(rng.choice(b"ACGT") for _ in range(rng.randint(5, 120)))
        alt = bytes(rng.choice(b"ACGT") for _ in range(rng.randint(3, 90)))
        cigar, _ = O.sw_align(ref, alt, READ_TO_HAP, strategy)
        import re

        used = sum(int(n) for n, op in re.findall(r"(\d+)([MIDS])", cigar) if op in "MIS")
        assert used == len(alt), (cigar, len(alt))
