"""Pins the CPU oracle to the reference's own known-answer tests.

model.rs:112-154, reference.rs:81-114, pd_reference.rs:138-183 and the flag test of pd.rs are
restated here against oracle/pairhmm_oracle.c. The reference ships no numeric golden files; these
analytic answers (plus tests/golden/, generated from this pinned oracle) are the pins.
"""
import math

import pytest

from oracle import oracle as O
from fgkl_b200.pairhmm import ALT_A, ALT_C, ALT_G, ALT_T, DEL_END, DEL_START, SNP, Read


def read(bases: bytes, q=30, i=45, d=45, g=10) -> Read:
    n = len(bases)
    return Read(bases, bytes([q] * n), bytes([i] * n), bytes([d] * n), bytes([g] * n))


# ---- model.rs:112-154 ----

def test_error_prob_matches_phred_definition():
    assert abs(O.error_prob(0) - 1.0) < 1e-15
    assert abs(O.error_prob(10) - 0.1) < 1e-15
    assert abs(O.error_prob(30) - 0.001) < 1e-15


def test_quals_above_max_are_clamped():
    assert O.error_prob(255) == O.error_prob(254)
    assert O.match_to_match(255, 10) == O.match_to_match(254, 10)


def test_match_to_match_is_symmetric_and_close_to_one_minus_gap_opens():
    assert O.match_to_match(45, 30) == O.match_to_match(30, 45)
    expected = 1.0 - (O.error_prob(45) + O.error_prob(30))
    assert abs(O.match_to_match(45, 30) - expected) < 1e-6


def test_match_to_match_at_zero_quals_is_zero():
    assert O.match_to_match(0, 0) == 0.0


def test_transitions_use_gap_continuation_for_extension():
    t = O.transitions(45, 40, 10)  # [MM, IM, MI, II, MD, DD]
    assert abs(t[3] - 0.1) < 1e-15
    assert abs(t[5] - 0.1) < 1e-15
    assert abs(t[1] - 0.9) < 1e-15
    assert abs(t[2] - O.error_prob(45)) < 1e-15
    assert abs(t[4] - O.error_prob(40)) < 1e-15


def test_approximate_log10_sum_matches_exact_for_moderate_differences():
    a, b = -3.0, -2.5
    exact = math.log10(10 ** a + 10 ** b)
    assert abs(O.approximate_log10_sum_log10(a, b) - exact) < 1e-4
    assert O.approximate_log10_sum_log10(a, b) == O.approximate_log10_sum_log10(b, a)
    assert O.approximate_log10_sum_log10(-20.0, -2.0) == -2.0


def test_priors_are_one_minus_error_and_a_third_of_it():
    pm, px = O.priors(20)
    assert pm == 1.0 - O.error_prob(20) and px == O.error_prob(20) / 3.0


# ---- reference.rs:81-114 ----

def test_initial_condition_is_two_to_the_1020():
    assert O.initial_condition() == 2.0 ** 1020


def test_identical_single_base_has_likelihood_near_log10_of_match_probability():
    lk = O.log10_likelihood(b"A", read(b"A"))
    expected = math.log10((1.0 - 1e-3) * 0.9)
    assert abs(lk - expected) < 1e-12


def test_mismatch_is_less_likely_than_match():
    matched = O.log10_likelihood(b"ACGT", read(b"ACGT"))
    mismatched = O.log10_likelihood(b"ACGT", read(b"ACTT"))
    assert matched > mismatched
    assert matched <= 0.0


def test_n_matches_every_base_wherever_it_is_aligned():
    exact = O.log10_likelihood(b"ACGT", read(b"ACGT"))
    n_read = O.log10_likelihood(b"ACGT", read(b"NNNN"))
    assert n_read == O.log10_likelihood(b"TTTT", read(b"NNNN"))
    n_hap = O.log10_likelihood(b"NNNN", read(b"ACGT"))
    assert n_hap == O.log10_likelihood(b"NNNN", read(b"GGGG"))
    assert n_read >= exact and n_hap >= exact


# ---- pd_reference.rs:138-183 ----

HAP = b"ACGTTGCAAGGCTTAGGCTTACG"


def test_pd_without_flags_equals_the_plain_pairhmm():
    r = read(b"GTTGCAAGGCTTAG")
    pd = O.pd_log10_likelihood(HAP, bytes(len(HAP)), r)
    plain = O.log10_likelihood(HAP, r)
    assert abs(pd - plain) < 1e-12


def test_snp_alternate_makes_the_alternate_base_match():
    alt_read = read(b"GTTGCATGGCTTAG")
    flags = bytearray(len(HAP))
    flags[8] = SNP | ALT_T
    with_ = O.pd_log10_likelihood(HAP, bytes(flags), alt_read)
    without = O.pd_log10_likelihood(HAP, bytes(len(HAP)), alt_read)
    exact = O.pd_log10_likelihood(HAP, bytes(flags), read(b"GTTGCAAGGCTTAG"))
    assert with_ > without + 1.0
    assert abs(with_ - exact) < 0.2


def test_deletion_span_lets_the_read_skip_bases():
    r = read(b"GTTGCACTTAGGC")
    flags = bytearray(len(HAP))
    flags[7] = DEL_START
    flags[10] = DEL_END
    assert O.pd_log10_likelihood(HAP, bytes(flags), r) > O.pd_log10_likelihood(HAP, bytes(len(HAP)), r)


def test_base_matching_honours_only_flagged_alternates():
    assert O.base_matches_pd(ord("A"), SNP | ALT_A)
    assert O.base_matches_pd(ord("a"), SNP | ALT_A | ALT_G)
    assert not O.base_matches_pd(ord("C"), SNP | ALT_A)
    assert not O.base_matches_pd(ord("A"), ALT_A)
    assert not O.base_matches_pd(ord("N"), SNP | ALT_A | ALT_C | ALT_G | ALT_T)


# ---- adjoint oracle (no reference counterpart): FP64 forward-backward vs central differences ----

@pytest.mark.parametrize("seed", [1, 2, 3])
def test_adjoint_oracle_matches_central_differences(seed):
    import numpy as np

    rng = np.random.default_rng(seed)
    hap = bytes(rng.choice(list(b"ACGT"), 40))
    start = int(rng.integers(0, 10))
    rb = bytearray(hap[start:start + 25])
    rb[5] = ord("A") if rb[5] != ord("A") else ord("C")
    n = len(rb)
    d_ins = np.full(n, O.error_prob(45)) * rng.uniform(0.5, 2.0, n)
    d_del = np.full(n, O.error_prob(40)) * rng.uniform(0.5, 2.0, n)
    eps = np.full(n, 0.1)
    err = np.array([O.error_prob(int(q)) for q in rng.integers(10, 40, n)])
    ll, g_i, g_d, g_e, g_q = O.adj_gradient(hap, bytes(rb), d_ins, d_del, eps, err)
    assert abs(ll - O.adj_log10_likelihood(hap, bytes(rb), d_ins, d_del, eps, err)) < 1e-12
    # Directional derivative along a random per-position direction, relative step 1e-6.
    for grad, which in ((g_i, 0), (g_d, 1), (g_e, 2), (g_q, 3)):
        params = [d_ins.copy(), d_del.copy(), eps.copy(), err.copy()]
        direction = params[which] * rng.uniform(0.5, 1.5, n)
        h = 1e-6
        plus = [p.copy() for p in params]
        minus = [p.copy() for p in params]
        plus[which] += h * direction
        minus[which] -= h * direction
        fd = (O.adj_log10_likelihood(hap, bytes(rb), *plus) - O.adj_log10_likelihood(hap, bytes(rb), *minus)) / (2 * h)
        an = float(np.dot(grad, direction))
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (which, fd, an)
