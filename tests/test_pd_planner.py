"""The PD planner on the CPU: deletion-state runs, match sets and the sorter, restating fgkl's own
unit tests (crates/pairhmm/src/pd_kernel.rs:928-985) and its sort key (pd_kernel.rs:61-136)."""
from fgkl_b200 import (AFTER_DEL, ALT_C, ALT_G, ALT_T, DEL_END, DEL_START, INSIDE_DEL, NORMAL, SNP, PdHaplotype, pd_match_accepts,
                       pd_plan, pd_row_states)


def runs(states, flags):
    """Collapse per-column states into fgkl's (lo, hi, state, del_end) runs."""
    out = []
    for j, (s, f) in enumerate(zip(states, flags)):
        de = bool(f & DEL_END)
        if out and out[-1][2] == s and out[-1][3] == de:
            out[-1] = (out[-1][0], j + 1, s, de)
        else:
            out.append((j, j + 1, s, de))
    return out


def test_unflagged_haplotype_is_one_normal_run_in_every_row():
    states, end = pd_row_states(bytes(5), NORMAL)
    assert runs(states, bytes(5)) == [(0, 5, NORMAL, False)]
    assert end == NORMAL


def test_a_deletion_splits_the_row_into_state_runs():
    flags = bytes([0, 0, DEL_START, 0, DEL_END, 0, 0, 0])
    states, end = pd_row_states(flags, NORMAL)
    assert runs(states, flags) == [(0, 3, NORMAL, False), (3, 4, INSIDE_DEL, False), (4, 5, INSIDE_DEL, True),
                                   (5, 6, AFTER_DEL, False), (6, 8, NORMAL, False)]
    assert end == NORMAL


def test_a_single_base_deletion_ends_in_the_state_it_started_in():
    flags = bytes([0, DEL_START | DEL_END, 0])
    states, end = pd_row_states(flags, NORMAL)
    assert runs(states, flags) == [(0, 1, NORMAL, False), (1, 2, NORMAL, True), (2, 3, AFTER_DEL, False)]
    assert end == NORMAL


def test_a_deletion_ending_on_the_last_column_carries_after_del_into_later_rows():
    flags = bytes([0, DEL_START, DEL_END])
    first, end = pd_row_states(flags, NORMAL)
    assert end == AFTER_DEL
    later, later_end = pd_row_states(flags, end)
    assert runs(later, flags)[0] == (0, 1, AFTER_DEL, False)
    assert later_end == AFTER_DEL
    assert runs(first, flags)[0] != runs(later, flags)[0]


def test_match_sets_accept_own_base_n_and_flagged_alternates():
    A, C, G, T, N = b"ACGTN"
    assert pd_match_accepts(A, 0, A) and pd_match_accepts(A, 0, N) and not pd_match_accepts(A, 0, C)
    snp = SNP | ALT_C | ALT_T
    assert pd_match_accepts(A, snp, C) and pd_match_accepts(A, snp, T) and not pd_match_accepts(A, snp, G)
    # Alternates need the SNP flag; deletion flags do not change the set.
    assert not pd_match_accepts(A, ALT_C, C)
    assert not pd_match_accepts(A, DEL_START | DEL_END, C)
    assert pd_match_accepts(N, 0, G)
    # Lower-case read bases match flagged alternates (pd.rs:99-110) but not the base itself.
    assert pd_match_accepts(A, SNP | ALT_C, ord("c")) and not pd_match_accepts(A, 0, ord("a"))


def test_sorter_orders_by_end_state_then_bases_and_flags():
    base = b"ACGTACGTAC"
    n = len(base)
    plain = bytes(n)
    snp = bytearray(n)
    snp[4] = SNP | ALT_G
    del_last = bytearray(n)
    del_last[n - 2] = DEL_START
    del_last[n - 1] = DEL_END
    haps = [PdHaplotype(base, bytes(del_last)), PdHaplotype(base, bytes(snp)), PdHaplotype(base, plain),
            PdHaplotype(base[:6], bytes(6)), PdHaplotype(base, plain)]
    p = pd_plan(haps)
    # End state NORMAL first (prefix before the longer, flags 0 before SNP), AFTER_DEL last.
    assert p.order == [3, 2, 4, 1, 0]
    assert p.end_state == [NORMAL, NORMAL, NORMAL, NORMAL, AFTER_DEL]
    assert p.lcp == [0, 6, n, 4, 0], "no sharing across end states; a flag difference splits"
    assert p.dup == [False, False, True, False, False]
    # Match sets: plain A, C, G, T and the SNP column's A-or-G.
    assert p.num_codes == 5
