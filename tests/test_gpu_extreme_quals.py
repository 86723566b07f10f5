"""GPU parity against the FP64 oracle over the whole quality range (0-255) of every read array.

fgkl clamps qualities at 254 and sets the match-to-match probability to 0 when the two gap-open
probabilities sum to 1 or more (crates/pairhmm/src/model.rs:37-49, `match_to_match_at_zero_quals_is_zero`).
Low qualities therefore give rows with a match-to-match of 0, a base quality of 0 a match prior of 0,
and a gap continuation quality of 0 an indel-to-match of 0. The FP32 pass divides by the
match-to-match of each row, so such a row must come out NaN and go to the FP64 recomputation, never as
a finite wrong value; these tests hold every such case to the tolerances of the others (1e-9 log10 in
double, 1e-4 in float).
"""
import numpy as np
import pytest

from fgkl_b200 import DEL_START, Config, PairHmm, PdPairHmm, Precision, Read, synthetic
from oracle import oracle as O

pytestmark = pytest.mark.gpu

BASES = np.frombuffer(b"ACGT", np.uint8)


def cfg(precision, share=True):
    return Config(precision=precision, double_fallback=True, share_suffixes=share)


def quals(rng, n, typical):
    """A quality array mixing the extremes with typical values: the lowest qualities (0-3), the
    clamped ones (254, 255), uniform draws over 0-255, and the rest near `typical`."""
    kind = rng.random(n)
    q = np.clip(rng.normal(typical, 3, n).round(), 0, 60).astype(np.uint8)
    q[kind < 0.15] = rng.integers(0, 4, int((kind < 0.15).sum()))
    hi = (kind >= 0.15) & (kind < 0.25)
    q[hi] = rng.integers(254, 256, int(hi.sum()))
    un = (kind >= 0.25) & (kind < 0.35)
    q[un] = rng.integers(0, 256, int(un.sum()))
    return q.astype(np.uint8).tobytes()


def edited(rng, ref):
    h = bytearray(ref)
    for _ in range(int(rng.integers(0, 4))):
        h[int(rng.integers(0, len(h)))] = int(rng.choice(BASES))
    if rng.random() < 0.5:
        p = int(rng.integers(1, len(h) - 6))
        del h[p:p + int(rng.integers(1, 5))]
    if rng.random() < 0.5:
        p = int(rng.integers(1, len(h) - 1))
        h[p:p] = bytes(rng.choice(BASES, int(rng.integers(1, 5))))
    return bytes(h)


def extreme_region(seed, num_reads, read_len, num_haps, hap_len):
    rng = np.random.default_rng(seed)
    ref = bytes(rng.choice(BASES, hap_len))
    haps = [ref] + [edited(rng, ref) for _ in range(num_haps - 1)]
    reads = []
    for _ in range(num_reads):
        h = haps[int(rng.integers(0, len(haps)))]
        n = int(rng.integers(read_len // 2, read_len + 1))
        p = int(rng.integers(0, len(h) - n + 1))
        b = bytearray(h[p:p + n])
        for _ in range(int(rng.integers(0, 3))):
            b[int(rng.integers(0, n))] = int(rng.choice(BASES))
        if rng.random() < 0.2:
            b[int(rng.integers(0, n))] = ord("N")
        ins, dele = bytearray(quals(rng, n, 45)), bytearray(quals(rng, n, 45))
        if rng.random() < 0.5:
            # Half the reads keep a non-zero match-to-match in every row, so the FP32 pass computes them
            # at the other extremes instead of handing them to the FP64 recomputation.
            for i in range(n):
                if O.match_to_match(ins[i], dele[i]) == 0.0:
                    ins[i] = dele[i] = 45
        reads.append(Read(bytes(b), quals(rng, n, 30), bytes(ins), bytes(dele), quals(rng, n, 10)))
    return reads, haps


def assert_close(actual, expected, tol, what=""):
    """|actual - expected| <= tol, equal infinities (a likelihood of exactly 0) counting as equal."""
    assert actual.shape == expected.shape
    assert not np.isnan(actual).any(), f"{what}: NaN in the results"
    same = actual == expected
    with np.errstate(invalid="ignore"):  # -inf - -inf, where `same` already holds
        d = np.where(same, 0.0, np.abs(actual - expected))
    worst = int(np.argmax(d))
    assert np.all(d <= tol), f"{what}: pair {worst}: got {actual[worst]}, expected {expected[worst]} (diff {d[worst]})"


def zero_m2m_reads(reads):
    """Reads with at least one row whose match-to-match probability is 0."""
    return [i for i, r in enumerate(reads) if any(O.match_to_match(a, b) == 0.0 for a, b in zip(r.ins_gop, r.del_gop))]


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("share", [True, False])
def test_extreme_qualities_match_the_oracle_in_double(gpu, seed, share):
    reads, haps = extreme_region(seed, 48, 100, 12, 160)
    expected = O.compute_matrix(reads, haps)
    got = PairHmm(cfg(Precision.DOUBLE, share)).compute_log10_likelihoods(reads, haps)
    assert_close(got, expected, 1e-9, f"double, seed {seed}, share {share}")


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("share", [True, False])
def test_extreme_qualities_match_the_oracle_in_float(gpu, seed, share):
    reads, haps = extreme_region(seed, 48, 100, 12, 160)
    expected = O.compute_matrix(reads, haps)
    hmm = PairHmm(cfg(Precision.FLOAT, share))
    got = hmm.compute_log10_likelihoods(reads, haps)
    assert_close(got, expected, 1e-4, f"float, seed {seed}, share {share}")
    # Every pair of a read with a zero match-to-match row is NaN after the FP32 pass and recomputed.
    assert hmm.fallback_pairs() >= len(zero_m2m_reads(reads)) * len(haps)


def test_zero_likelihoods_come_back_as_minus_infinity(gpu):
    # A first row whose gap continuation quality is 0 has an indel-to-match of 0: no path reaches M,
    # and the likelihood is exactly 0, in the oracle as here.
    reads, haps = extreme_region(1, 48, 100, 12, 160)
    expected = O.compute_matrix(reads, haps)
    assert np.isneginf(expected).any()
    for precision in (Precision.FLOAT, Precision.DOUBLE):
        got = PairHmm(cfg(precision)).compute_log10_likelihoods(reads, haps)
        assert np.array_equal(np.isneginf(got), np.isneginf(expected))


def test_every_read_row_at_the_lowest_qualities(gpu):
    # Whole reads at qualities 0-3 in every array, next to reads at 254-255.
    rng = np.random.default_rng(7)
    ref = bytes(rng.choice(BASES, 120))
    haps = [ref, edited(rng, ref), edited(rng, ref)]
    reads = []
    for k in range(16):
        n = 40 + 3 * k
        p = int(rng.integers(0, len(ref) - n + 1))
        lo, hi = (0, 4) if k % 2 == 0 else (254, 256)
        q = [bytes(rng.integers(lo, hi, n).astype(np.uint8)) for _ in range(4)]
        reads.append(Read(ref[p:p + n], *q))
    expected = O.compute_matrix(reads, haps)
    for precision, tol in ((Precision.DOUBLE, 1e-9), (Precision.FLOAT, 1e-4)):
        for share in (True, False):
            got = PairHmm(cfg(precision, share)).compute_log10_likelihoods(reads, haps)
            assert_close(got, expected, tol, f"{precision}, share {share}")


def extreme_pd_region(seed):
    """fgkl's PD reference region (flags: SNPs, deletions) with its reads' qualities replaced by the
    extremes of `quals`, half the reads repaired to keep every match-to-match non-zero."""
    reads, haps = synthetic.reference_pd_region(seed, 40, 100, 10, 200).region(0)
    rng = np.random.default_rng(seed)
    out = []
    for r in reads:
        n = len(r.bases)
        ins, dele = bytearray(quals(rng, n, 45)), bytearray(quals(rng, n, 45))
        if rng.random() < 0.5:
            for i in range(n):
                if O.match_to_match(ins[i], dele[i]) == 0.0:
                    ins[i] = dele[i] = 45
        out.append(Read(r.bases, quals(rng, n, 30), bytes(ins), bytes(dele), quals(rng, n, 10)))
    return out, haps


@pytest.mark.parametrize("seed", [5, 6])
def test_pd_extreme_qualities_match_the_pd_oracle(gpu, seed):
    reads, haps = extreme_pd_region(seed)
    assert any(f & DEL_START for h in haps for f in h.flags)
    expected = O.compute_matrix(reads, haps)
    got = PdPairHmm(Config(precision=Precision.DOUBLE)).compute_log10_likelihoods(reads, haps)
    assert_close(got, expected, 1e-9, f"PD double, seed {seed}")
    hmm = PdPairHmm(Config(precision=Precision.FLOAT, double_fallback=True))
    got = hmm.compute_log10_likelihoods(reads, haps)
    assert_close(got, expected, 1e-4, f"PD float, seed {seed}")
    assert hmm.fallback_pairs() >= len(zero_m2m_reads(reads)) * len(haps)
