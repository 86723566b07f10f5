"""Bit-exact planner parity with fgkl's SortedHaps / SuffixPlan (kernel.rs:53-81, plan.rs:61-235).

Restates the plan KATs of plan.rs:284-338 and the sorted-order example of lib.rs:666-669, and replays
every plan through the reference's own consistency check (plan.rs:248-278).
"""
from fgkl_b200 import plan
from refgen import Rng, edited, reference_like

MIN_SAVING = 4


def consistent_plan(haps):
    p = plan(haps, True)
    bases = [haps[i] for i in p.order]

    def suffix(k, depth):
        return bases[k][len(bases[k]) - depth:]

    written = {0: b""}
    for hap, resume, need, start, writes in p.sweeps:
        assert resume < need
        assert written.get(start) == suffix(hap, resume)
        for depth, node in writes:
            assert resume < depth <= need
            assert node not in written
            written[node] = suffix(hap, depth)
    assert len(written) == p.nodes
    for k, cut in enumerate(p.cuts):
        if cut is None:
            continue
        column, node = cut
        assert not p.dup[k]
        depth = len(bases[k]) - column
        assert depth >= MIN_SAVING
        assert written.get(node) == suffix(k, depth)
        nxt = next((j for j in range(k + 1, len(bases)) if not p.dup[j]), None)
        resumes_at = p.lcp[nxt] if nxt is not None else 0
        assert column > p.lcp[k] and column > resumes_at
    return p


def flip(b: int) -> int:
    return ord("C") if b == ord("A") else ord("A")


def test_a_substitution_cuts_both_haplotypes_right_after_their_shared_prefix():
    reference = reference_like(Rng(1), b"ACGT", 40)
    snp = bytearray(reference)
    snp[20] = flip(snp[20])
    p = consistent_plan([reference, bytes(snp)])
    assert p.cuts[0][0] == 21
    assert p.cuts[0] == p.cuts[1]
    assert len(p.sweeps) == 1


def test_a_haplotype_whose_suffix_is_its_own_runs_forward_to_its_end():
    reference = reference_like(Rng(2), b"ACGT", 40)
    late = bytearray(reference)
    late[38] = flip(late[38])
    p = consistent_plan([reference, bytes(late)])
    assert all(c is None for c in p.cuts)
    assert not p.sweeps


def test_duplicates_are_flagged_and_never_cut():
    reference = reference_like(Rng(3), b"ACGT", 30)
    snp = bytearray(reference)
    snp[10] = flip(snp[10])
    snp = bytes(snp)
    p = consistent_plan([snp, reference, snp, reference])
    assert p.dup == [False, True, False, True]
    assert p.cuts[0] is not None and p.cuts[2] is not None


def test_plans_of_random_haplotype_sets_are_consistent():
    rng = Rng(4)
    for case in range(400):
        alphabet = b"AC" if case % 2 == 0 else b"ACGT"
        n = 5 + rng.below(60)
        base = reference_like(rng, alphabet, n)
        haps = [base]
        for _ in range(rng.below(30)):
            if rng.chance(0.15):
                hap = haps[rng.below(len(haps))]
            else:
                hap = edited(rng, alphabet, haps[rng.below(len(haps))])
            haps.append(hap)
        consistent_plan(haps)


def test_sorted_order_puts_shorter_prefixes_first_and_keeps_input_order_for_ties():
    haps = [b"ABBC", b"AAAC", b"AC", b"AAAB", b"ABBB", b"AAAC", b"ABBCC"]
    p = plan(haps, False)
    assert [haps[i] for i in p.order] == [b"AAAB", b"AAAC", b"AAAC", b"ABBB", b"ABBC", b"ABBCC", b"AC"]
    assert p.order[1] == 1 and p.order[2] == 5  # stable: the first AAAC first
    assert p.lcp == [0, 3, 4, 1, 3, 4, 1]
    assert p.dup == [False, False, True, False, False, False, False]


def test_prefix_only_plan_has_no_cuts_and_columns_add_up():
    reference = reference_like(Rng(7), b"ACGT", 50)
    haps = [reference]
    rng = Rng(8)
    for _ in range(6):
        haps.append(edited(rng, b"ACGT", reference))
    shared = plan(haps, True)
    prefix = plan(haps, False)
    assert all(c is None for c in prefix.cuts) and not prefix.sweeps
    assert shared.columns.prefix_only == prefix.columns.prefix_only == prefix.columns.forward
    assert shared.columns.forward <= shared.columns.prefix_only
    assert shared.columns.backward == sum(need - resume for _, resume, need, _, _ in shared.sweeps)
