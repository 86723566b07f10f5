"""GPU parity of reads longer than one 32 x 20-row block (620 bases), and of PD regions whose reads
hold more distinct bytes than the class bits describe, against the FP64 oracles, through the C ABI.

fgkl sizes its row tables by the batch's longest read (crates/pairhmm/src/kernel.rs:485-577) and
its PD match sets have no limit (pd_kernel.rs:196-214), so both inputs are part of the drop-in
contract. Tolerances are fgkl's own (lib.rs:621-660): 1e-9 log10 in double, 1e-4 in float.
"""
import numpy as np
import pytest

from fgkl_b200 import (ALT_A, ALT_C, ALT_G, ALT_T, DEL_END, DEL_START, SNP, BatchContext, Config, PairHmm, PdHaplotype,
                       PdPairHmm, Precision, Read, synthetic)
from oracle import oracle as O
from refgen import Rng, reference_like

pytestmark = pytest.mark.gpu

FLOAT = Config(precision=Precision.FLOAT)
DOUBLE = Config(precision=Precision.DOUBLE)


def assert_close(actual, expected, tol, what=""):
    assert actual.shape == expected.shape
    same = actual == expected  # equal infinities: a likelihood of zero on both sides
    d = np.where(same, 0.0, np.abs(actual - expected))
    worst = int(np.argmax(d))
    assert np.all(d <= tol), f"{what}: pair {worst}: got {actual[worst]}, expected {expected[worst]} (diff {d[worst]})"
    assert np.isfinite(d).all()


def region(seed, num_reads, read_len, num_haps, hap_len):
    return synthetic.reference_region(seed, num_reads, read_len, num_haps, hap_len).region(0)


def pd_region(seed, num_reads, read_len, num_haps, hap_len):
    return synthetic.reference_pd_region(seed, num_reads, read_len, num_haps, hap_len).region(0)


def computed(hmm_class, config, reads, haps):
    hmm = hmm_class(config)
    return hmm.compute_log10_likelihoods(reads, haps), hmm.fallback_pairs()


@pytest.mark.parametrize("read_len", [621, 1000, 2500])
def test_long_reads_match_the_oracle_in_double(gpu, read_len):
    reads, haps = region(41 + read_len, 3, read_len, 3, read_len + 150)
    got, _ = computed(PairHmm, DOUBLE, reads, haps)
    assert_close(got, O.compute_matrix(reads, haps), 1e-9, f"double {read_len}")


@pytest.mark.parametrize("read_len", [621, 1000, 2500])
def test_long_reads_match_the_oracle_in_float(gpu, read_len):
    reads, haps = region(43 + read_len, 3, read_len, 3, read_len + 150)
    got, _ = computed(PairHmm, FLOAT, reads, haps)
    assert_close(got, O.compute_matrix(reads, haps), 1e-4, f"float {read_len}")


@pytest.mark.parametrize("read_len", [621, 1000, 2500])
def test_long_pd_reads_match_the_pd_oracle(gpu, read_len):
    reads, haps = pd_region(47 + read_len, 3, read_len, 3, read_len + 150)
    expected = O.compute_matrix(reads, haps)
    got64, _ = computed(PdPairHmm, DOUBLE, reads, haps)
    assert_close(got64, expected, 1e-9, f"pd double {read_len}")
    got32, _ = computed(PdPairHmm, FLOAT, reads, haps)
    assert_close(got32, expected, 1e-4, f"pd float {read_len}")


def sampled_reads(seed, haps, count, length, subst=0.0, quals=(10, 40)):
    """Reads copied from random haplotypes at random offsets, a fraction `subst` of bases replaced."""
    rng = Rng(seed)
    out = []
    for _ in range(count):
        h = haps[rng.below(len(haps))]
        start = rng.below(len(h) - length + 1)
        b = bytearray(h[start:start + length])
        for i in range(length):
            if subst and rng.chance(subst):
                b[i] = b"ACGT"[rng.below(4)]
        q = bytes(quals[0] + rng.below(quals[1] - quals[0] + 1) for _ in range(length))
        out.append(Read(bytes(b), q, bytes([45] * length), bytes([45] * length), bytes([10] * length)))
    return out


def test_short_and_long_reads_in_one_region(gpu):
    """Long reads take the strip-mined path beside the region's shared program; the short reads'
    results keep the bits they have without the long reads."""
    short, haps = region(5, 12, 151, 6, 900)
    long_ = sampled_reads(6, haps, 4, 800)
    reads = short[:6] + long_ + short[6:]
    for config, tol in ((DOUBLE, 1e-9), (FLOAT, 1e-4)):
        got, _ = computed(PairHmm, config, reads, haps)
        assert_close(got, O.compute_matrix(reads, haps), tol)
        alone, _ = computed(PairHmm, config, short, haps)
        n = len(haps)
        mixed = got.reshape(len(reads), n)
        assert mixed[:6].tobytes() == alone.reshape(len(short), n)[:6].tobytes()
        assert mixed[10:].tobytes() == alone.reshape(len(short), n)[6:].tobytes()


def test_duplicate_haplotypes_share_a_long_read_result(gpu):
    reads, haps = region(9, 2, 700, 3, 820)
    haps = [haps[0], haps[1], haps[0], haps[2], haps[1]]
    got, _ = computed(PairHmm, FLOAT, reads, haps)
    m = got.reshape(len(reads), len(haps))
    assert m[:, 0].tobytes() == m[:, 2].tobytes() and m[:, 1].tobytes() == m[:, 4].tobytes()
    assert_close(got, O.compute_matrix(reads, haps), 1e-4)


def test_long_reads_unrelated_to_the_haplotypes_are_recomputed_in_double(gpu):
    """A long read that matches nothing underflows the FP32 range; its pairs go to the FP64
    recomputation (fgkl lib.rs:461-487) and come back at double precision."""
    rng = Rng(77)
    base = bytearray(reference_like(rng, b"ACGT", 1100))
    haps = []
    for _ in range(3):
        h = bytearray(base)
        for _ in range(4):
            h[rng.below(len(h))] = b"ACGT"[rng.below(4)]
        haps.append(bytes(h))
    # 40% of bases replaced at quality 20: about 1e-520 per pair, inside the FP64 range only.
    reads = sampled_reads(78, haps, 2, 700, subst=0.4, quals=(20, 20))
    got, fallback = computed(PairHmm, FLOAT, reads, haps)
    assert fallback == len(reads) * len(haps)
    assert_close(got, O.compute_matrix(reads, haps), 1e-9)


def test_batched_long_reads_have_the_per_call_bits(gpu):
    parts = [region(61, 3, 700, 4, 850), region(62, 5, 151, 3, 400), region(63, 2, 1300, 2, 1400)]
    w = synthetic.from_regions(parts)
    ctx = BatchContext()
    out, _ = ctx.compute(w, FLOAT)
    per_call = np.concatenate([computed(PairHmm, FLOAT, r, h)[0] for r, h in parts])
    assert out.tobytes() == per_call.tobytes()
    ctx.close()


def many_byte_reads(seed, reads, classes, every=0):
    """Reads whose bases are drawn from `classes` distinct bytes (more than 31), with ACGT among them:
    a random quarter of the bases replaced, or with `every` > 0 every `every`-th base, the alphabet's
    bytes taken in turn (few enough substitutions that long reads keep a finite likelihood)."""
    rng = Rng(seed)
    alphabet = b"ACGTNacgtn" + bytes(range(ord("!"), ord("!") + classes - 10))  # punctuation and digits
    assert len(set(alphabet)) == classes
    out, turn = [], 0
    for r in reads:
        b = bytearray(r.bases)
        for i in range(len(b)):
            if every > 0:
                if i % every == every // 2:
                    b[i] = alphabet[turn % len(alphabet)]
                    turn += 1
            elif rng.below(4) == 0:
                b[i] = alphabet[rng.below(len(alphabet))]
        out.append(Read(bytes(b), r.quals, r.ins_gop, r.del_gop, r.gcp))
    return out


def test_pd_region_with_40_distinct_read_bytes(gpu):
    reads, haps = pd_region(31, 24, 120, 8, 300)
    reads = many_byte_reads(5, reads, 40)
    assert len({b for r in reads for b in r.bases}) == 40
    expected = O.compute_matrix(reads, haps)
    got64, _ = computed(PdPairHmm, DOUBLE, reads, haps)
    assert_close(got64, expected, 1e-9, "double")
    got32, _ = computed(PdPairHmm, FLOAT, reads, haps)
    assert_close(got32, expected, 1e-4, "float")


def test_pd_region_with_40_read_bytes_and_long_reads(gpu):
    reads, haps = pd_region(33, 3, 900, 3, 1000)
    reads = many_byte_reads(6, reads, 40, every=60)
    assert len({b for r in reads for b in r.bases}) >= 40
    expected = O.compute_matrix(reads, haps)
    assert np.isfinite(expected).all()
    got, _ = computed(PdPairHmm, FLOAT, reads, haps)
    assert_close(got, expected, 1e-4)


def test_pd_region_with_more_than_256_match_sets(gpu):
    """Haplotype bytes x flagged alternates beyond the 256 codes a stream entry holds."""
    rng = Rng(12)
    alts = [ALT_A, ALT_C, ALT_G, ALT_T]
    hap_bytes = b"ACGT" + bytes(range(ord("a"), ord("a") + 20))
    haps = []
    for _ in range(6):
        n = 400
        bases = bytes(hap_bytes[rng.below(len(hap_bytes))] for _ in range(n))
        flags = bytearray(n)
        for j in range(n):
            mask = sum(a for a in alts if rng.below(2))
            if mask:
                flags[j] = SNP | mask
        for j in range(20, n - 20, 97):
            flags[j] |= DEL_START
            flags[j + 3] |= DEL_END
        haps.append(PdHaplotype(bases, bytes(flags)))
    sets = {(h.bases[j], h.flags[j] & 0x78 if h.flags[j] & SNP else 0) for h in haps for j in range(len(h.bases))}
    assert len(sets) > 256
    reads = []
    for _ in range(10):
        h = haps[rng.below(len(haps))].bases
        start = rng.below(len(h) - 150)
        b = h[start:start + 150]
        reads.append(Read(b, bytes([25] * 150), bytes([45] * 150), bytes([45] * 150), bytes([10] * 150)))
    expected = O.compute_matrix(reads, haps)
    got64, _ = computed(PdPairHmm, DOUBLE, reads, haps)
    assert_close(got64, expected, 1e-9, "double")
    got32, _ = computed(PdPairHmm, FLOAT, reads, haps)
    assert_close(got32, expected, 1e-4, "float")
