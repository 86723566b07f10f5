"""GPU parity of the plain PairHMM against the FP64 oracle, through the C ABI.

Restates the reference's own tests (crates/pairhmm/src/lib.rs:583-1097) with its regions (rebuilt
draw for draw from their seeds), tolerances (1e-9 log10 in double, 1e-4 in float) and bit-identity
invariants. The "every backend" loops collapse to the one sm_100a backend.
"""
import numpy as np
import pytest

from fgkl_b200 import Config, PairHmm, Precision, Read, plan, synthetic
from oracle import oracle as O
from refgen import Rng, edited

pytestmark = pytest.mark.gpu

FLOAT = Config(precision=Precision.FLOAT)
DOUBLE = Config(precision=Precision.DOUBLE)


def region(seed, num_reads, read_len, num_haps, hap_len):
    return synthetic.reference_region(seed, num_reads, read_len, num_haps, hap_len).region(0)


def reference_all(reads, haps):
    return O.compute_matrix(reads, haps)


def compute(config, reads, haps):
    return PairHmm(config).compute_log10_likelihoods(reads, haps)


def compute_counting(config, reads, haps):
    hmm = PairHmm(config)
    out = hmm.compute_log10_likelihoods(reads, haps)
    return out, hmm.fallback_pairs()


def assert_close(actual, expected, tol, what=""):
    assert actual.shape == expected.shape
    d = np.abs(actual - expected)
    worst = int(np.argmax(d))
    assert np.all(d <= tol), f"{what}: pair {worst}: got {actual[worst]}, expected {expected[worst]} (diff {d[worst]})"
    assert np.isfinite(d).all()


def cfg(precision, share):
    return Config(precision=precision, double_fallback=True, share_suffixes=share)


def simple_read(bases: bytes, q=30):
    n = len(bases)
    return Read(bases, bytes([q] * n), bytes([45] * n), bytes([45] * n), bytes([10] * n))


def test_double_precision_matches_reference(gpu):
    reads, haps = region(11, 70, 120, 24, 300)
    assert_close(compute(DOUBLE, reads, haps), reference_all(reads, haps), 1e-9, "double")


def test_single_precision_matches_reference_within_float_tolerance(gpu):
    reads, haps = region(11, 70, 120, 24, 300)
    assert_close(compute(FLOAT, reads, haps), reference_all(reads, haps), 1e-4, "float")


def test_haplotype_order_does_not_change_results(gpu):
    reads, haps = region(11, 70, 120, 24, 300)
    fwd = compute(DOUBLE, reads, haps)
    rev = compute(DOUBLE, reads, haps[::-1])
    n = len(haps)
    for r in range(len(reads)):
        for h in range(n):
            assert abs(fwd[r * n + h] - rev[r * n + (n - 1 - h)]) < 1e-11


def test_prefix_sharing_handles_nested_and_repeated_prefixes(gpu):
    haps = [b"ABBC", b"AAAC", b"AC", b"AAAB", b"ABBB", b"AAAC", b"ABBCC"]
    reads, _ = region(3, 20, 6, 1, 8)
    assert_close(compute(DOUBLE, reads, haps), reference_all(reads, haps), 1e-9)


def test_haplotypes_of_different_lengths_share_prefixes_correctly(gpu):
    haps = [b"ACGTACGTAC", b"ACGTACGT", b"ACGTACGTACGTACGT", b"ACGT", b"A"]
    reads, _ = region(9, 40, 12, 1, 16)
    assert_close(compute(DOUBLE, reads, haps), reference_all(reads, haps), 1e-9)


def test_non_acgtn_bases_match_only_themselves(gpu):
    reads = [Read(b"ACRTN", bytes([30] * 5), bytes([45] * 5), bytes([45] * 5), bytes([10] * 5))]
    haps = [b"ACRTG", b"ACGTG", b"ACNTG", b"RRRRR"]
    expected = reference_all(reads, haps)
    assert_close(compute(DOUBLE, reads, haps), expected, 1e-9)
    assert expected[0] > expected[1]
    assert expected[2] >= expected[0]


def test_float_underflow_falls_back_to_double(gpu):
    reads = [Read(b"A" * 80, bytes([40] * 80), bytes([45] * 80), bytes([45] * 80), bytes([10] * 80))]
    haps = [b"C" * 80]
    expected = reference_all(reads, haps)
    assert np.isfinite(expected[0]) and expected[0] < -50.0
    assert_close(compute(FLOAT, reads, haps), expected, 1e-9)


def suffix_sharing_region():
    return region(21, 90, 150, 40, 260)


def test_suffix_sharing_matches_reference_in_double(gpu):
    reads, haps = suffix_sharing_region()
    assert sum(c is not None for c in plan(haps).cuts) > 20
    assert_close(compute(cfg(Precision.DOUBLE, True), reads, haps), reference_all(reads, haps), 1e-9)


def test_suffix_sharing_matches_reference_in_float_within_tolerance(gpu):
    reads, haps = suffix_sharing_region()
    assert_close(compute(cfg(Precision.FLOAT, True), reads, haps), reference_all(reads, haps), 1e-4)


def test_random_small_haplotype_sets_match_reference_with_suffix_sharing(gpu):
    rng = Rng(31)

    def letter():
        return ord("A") if rng.chance(0.5) else ord("C")

    for _ in range(60):
        haps = [bytes(letter() for _ in range(6 + rng.below(30)))]
        for _ in range(rng.below(12)):
            haps.append(edited(rng, b"AC", haps[rng.below(len(haps))]))
        reads = []
        for _ in range(1 + rng.below(20)):
            n = 1 + rng.below(25)
            reads.append(Read(bytes(letter() for _ in range(n)), bytes(10 + rng.below(31) for _ in range(n)),
                              bytes(20 + rng.below(26) for _ in range(n)), bytes(20 + rng.below(26) for _ in range(n)),
                              bytes(1 + rng.below(10) for _ in range(n))))
        assert_close(compute(cfg(Precision.DOUBLE, True), reads, haps), reference_all(reads, haps), 1e-9)


def test_haplotypes_without_a_cut_keep_their_prefix_only_bits(gpu):
    reads, haps = region(23, 20, 90, 24, 160)
    p = plan(haps)
    uncut = [p.order[k] for k in range(len(haps)) if p.cuts[k] is None and not p.dup[k]]
    assert uncut
    for precision in (Precision.FLOAT, Precision.DOUBLE):
        shared = compute(cfg(precision, True), reads, haps)
        prefix = compute(cfg(precision, False), reads, haps)
        for r in range(len(reads)):
            for h in uncut:
                i = r * len(haps) + h
                assert shared[i].tobytes() == prefix[i].tobytes(), (precision, r, h)


def test_deep_pairs_fall_back_to_double_with_suffix_sharing(gpu):
    base = bytearray(b"A" * 90)
    haps = [bytes(base)]
    for pos in (20, 45, 70):
        h = bytearray(base)
        h[pos] = ord("G")
        haps.append(bytes(h))
    assert any(c is not None for c in plan(haps).cuts)
    reads = [Read(b"C" * 70, bytes([40] * 70), bytes([45] * 70), bytes([45] * 70), bytes([10] * 70))]
    expected = reference_all(reads, haps)
    assert (expected < -50.0).all()
    out, fallbacks = compute_counting(cfg(Precision.FLOAT, True), reads, haps)
    assert fallbacks == len(haps)
    assert_close(out, expected, 1e-9)


def test_likelihoods_below_the_backward_range_are_recomputed_without_suffix_sharing(gpu):
    rng = Rng(99)
    reference = bytes(rng.base() for _ in range(700))
    haps = [reference]
    for pos in (20, 40, 60):
        h = bytearray(reference)
        h[pos] = ord("C") if h[pos] == ord("A") else ord("A")
        haps.append(bytes(h))
    assert any(c is not None for c in plan(haps).cuts)
    reads = []
    for n in (290, 360, 500):
        reads.append(Read(bytes(rng.base() for _ in range(n)), bytes([40] * n), bytes([45] * n), bytes([45] * n), bytes([10] * n)))
    expected = reference_all(reads, haps)
    assert (expected < -400.0).any()
    for precision in (Precision.DOUBLE, Precision.FLOAT):
        assert_close(compute(cfg(precision, True), reads, haps), expected, 1e-9, str(precision))


def foreign_reads(seed, n, length):
    rng = Rng(seed)
    out = []
    for _ in range(n):
        out.append(Read(bytes(rng.base() for _ in range(length)), bytes(20 + rng.below(21) for _ in range(length)),
                        bytes([45] * length), bytes([45] * length), bytes([10] * length)))
    return out


def test_reads_unrelated_to_every_haplotype_are_recomputed_in_double(gpu):
    _, haps = region(11, 70, 120, 24, 300)
    reads = foreign_reads(5, 40, 120)
    expected = reference_all(reads, haps)
    assert (expected < -64.0).all()
    out, fallbacks = compute_counting(FLOAT, reads, haps)
    assert_close(out, expected, 1e-9)
    assert fallbacks == expected.size


def test_matching_and_mismatching_reads_of_varied_lengths_share_a_batch(gpu):
    all_reads, haps = region(11, 70, 120, 24, 300)
    owned = all_reads[:20] + foreign_reads(6, 20, 120)
    reads = []
    for i, r in enumerate(owned):
        n = 30 + (i * 7) % 90
        reads.append(Read(r.bases[:n], r.quals[:n], r.ins_gop[:n], r.del_gop[:n], r.gcp[:n]))
    expected = reference_all(reads, haps)
    out, fallbacks = compute_counting(FLOAT, reads, haps)
    assert_close(out, expected, 1e-4)
    assert fallbacks > 0


def test_a_read_gets_the_same_bits_whatever_shares_its_batch(gpu):
    all_reads, haps = region(11, 70, 120, 24, 300)
    alone = all_reads[:3]
    batched = all_reads[:3] + foreign_reads(7, 29, 120)
    for precision in (Precision.FLOAT, Precision.DOUBLE):
        solo = compute(Config(precision=precision), alone, haps)
        with_others = compute(Config(precision=precision), batched, haps)
        assert solo.tobytes() == with_others[: solo.size].tobytes(), precision


def test_a_read_gets_the_same_bits_in_a_full_batch_and_in_a_remainder(gpu):
    reads, haps = region(5, 40, 60, 4, 100)
    for precision in (Precision.FLOAT, Precision.DOUBLE):
        config = Config(precision=precision)
        solo = [compute(config, [r], haps) for r in reads]
        for n in (1, 2, 3, 16, 17, 31, 33, 40):
            got = compute(config, reads[:n], haps)
            for r in range(n):
                assert got[r * len(haps):(r + 1) * len(haps)].tobytes() == solo[r].tobytes(), (precision, n, r)


def test_a_read_matching_only_the_previous_haplotype_is_recomputed_in_double(gpu):
    rng = Rng(8)
    reference = bytes(rng.base() for _ in range(300))
    tail = bytes(rng.base() for _ in range(150))
    h1 = reference
    h2 = reference[:150] + tail
    h3 = bytearray(reference)
    h3[200] = ord("C") if h3[200] == ord("A") else ord("A")
    haps = [h1, h2, bytes(h3)]
    reads = []
    for k in range(12):
        source = reference if k % 2 == 0 else h2
        start = 100 + (k * 13) % 80
        reads.append(Read(source[start:start + 100], bytes([35] * 100), bytes([45] * 100), bytes([45] * 100), bytes([10] * 100)))
    expected = reference_all(reads, haps)
    assert (expected < -64.0).any() and (expected > -10.0).any()
    out, fallbacks = compute_counting(FLOAT, reads, haps)
    assert_close(out, expected, 1e-4)
    assert 0 < fallbacks <= 24


def test_more_reads_than_lanes_and_single_read_both_work(gpu):
    reads, haps = region(21, 1, 50, 3, 60)
    assert_close(compute(Config(), reads, haps), reference_all(reads, haps), 1e-4, "single")
    reads, haps = region(22, 37, 50, 3, 60)
    assert_close(compute(Config(), reads, haps), reference_all(reads, haps), 1e-4, "many")


def test_empty_inputs_produce_no_output(gpu):
    _, haps = region(3, 5, 50, 4, 80)
    assert compute(FLOAT, [], haps).size == 0
    reads, _ = region(3, 5, 50, 4, 80)
    assert compute(FLOAT, reads, []).size == 0


# ---- the benchmark workloads at test size ----

def test_single_region_workload_double_and_float(gpu):
    w = synthetic.workload(0, seed=0)
    reads, haps = w.region(0)
    expected = reference_all(reads, haps)
    assert_close(compute(DOUBLE, reads, haps), expected, 1e-9, "double")
    assert_close(compute(FLOAT, reads, haps), expected, 1e-4, "float")


def test_batched_uneven_regions_match_oracle_and_per_call(gpu):
    from fgkl_b200 import BatchContext

    w = synthetic.workload(1, seed=3, regions=24)
    ctx = BatchContext()
    out, stats = ctx.compute(w, FLOAT)
    expected = O.workload_matrix(w)
    assert_close(out, expected, 1e-3, "batched float")
    assert stats.computed_cells < stats.nominal_cells
    # The batched form gives every pair the bits the per-call form gives it.
    offs = w.output_offsets()
    for g in (0, 5, 23):
        reads, haps = w.region(g)
        assert compute(FLOAT, reads, haps).tobytes() == out[offs[g]:offs[g + 1]].tobytes()


def test_shared_prefix_and_suffix_workload_against_unshared_oracle(gpu):
    from fgkl_b200 import BatchContext

    w = synthetic.workload(2, seed=5, regions=2)
    ctx = BatchContext()
    out, stats = ctx.compute(w, FLOAT)
    expected = O.workload_matrix(w)
    assert_close(out, expected, 1e-3, "c2 float")
    assert stats.backward_cells > 0
    assert stats.forward_cells < 0.5 * stats.prefix_only_cells + stats.forward_cells


def test_two_contexts_on_one_stream_stream_batches_with_unchanged_bits(gpu):
    # The streaming pattern of the C ABI: two contexts share a compute stream; batch k+1 is prepared
    # and run on one before batch k is fetched from the other. Every batch must come back with the
    # bits a lone, unoverlapped call gives it, including batches of other shapes (graph re-captured
    # and updated in place) and a PD batch between plain ones.
    import torch

    from fgkl_b200 import BatchContext

    batches = [synthetic.workload(1, seed=11, regions=16), synthetic.workload(1, seed=12, regions=9),
               synthetic.workload(3, seed=13, regions=3), synthetic.workload(1, seed=11, regions=16),
               synthetic.workload(2, seed=14, regions=1)]
    alone = [BatchContext().compute(w, FLOAT)[0] for w in batches]
    shared = torch.cuda.Stream()
    ctxs = [BatchContext(stream=shared.cuda_stream), BatchContext(stream=shared.cuda_stream)]
    got = [None] * len(batches)
    for k, w in enumerate(batches):
        ctxs[k % 2].prepare(w, FLOAT)
        ctxs[k % 2].run()
        if k > 0:
            got[k - 1] = ctxs[(k - 1) % 2].fetch()[0]
    got[-1] = ctxs[(len(batches) - 1) % 2].fetch()[0]
    for k in range(len(batches)):
        assert got[k].tobytes() == alone[k].tobytes(), k


def test_autotuner_times_every_launch_configuration_and_keeps_the_bits(gpu):
    from fgkl_b200 import BatchContext

    w = synthetic.workload(1, seed=21, regions=32)
    default, _ = BatchContext().compute(w, FLOAT)
    ctx = BatchContext()
    chosen, tried = ctx.autotune(w, FLOAT, repeats=2)
    assert len(tried) == 19
    launch = [t for t in tried if t["rows_extra"] == 0 and t["warps_per_block"] == 4]
    assert {(t["streams"], t["grid_percent"]) for t in launch[:16]} == {(s, g) for s in (1, 2, 4, 8) for g in (100, 90, 75, 60)}
    # The tile shapes are tried around the fastest launch configuration of the first 16.
    best16 = min(tried[:16], key=lambda t: t["ms"])
    shapes = [(t["streams"], t["grid_percent"], t["rows_extra"], t["warps_per_block"]) for t in tried[16:]]
    assert shapes == [(best16["streams"], best16["grid_percent"], 0, 1), (best16["streams"], best16["grid_percent"], 0, 2),
                      (best16["streams"], best16["grid_percent"], 1, 4)]
    assert all(t["ms"] > 0 for t in tried)
    assert chosen["ms"] == min(t["ms"] for t in tried)
    assert ctx.tuning() == {k: chosen[k] for k in ("streams", "grid_percent", "reads_per_warp", "rows_extra", "warps_per_block")}
    # The batch stays prepared with the chosen configuration; launch shapes never change a result.
    ctx.run()
    tuned, _ = ctx.fetch()
    assert tuned.tobytes() == default.tobytes()
    ctx.set_tuning(1, 10)
    narrow, _ = ctx.compute(w, FLOAT)
    assert narrow.tobytes() == default.tobytes()


@pytest.mark.parametrize("rows_extra,warps", [(1, 4), (0, 1), (0, 2), (1, 2)])
def test_tile_shapes_keep_the_bits(gpu, rows_extra, warps):
    """Rows per lane one step up (more padding rows) and 1 or 2 warps per block change no result bit:
    a cell's arithmetic does not depend on the rows beside it, and the joins sum in read-row order."""
    from fgkl_b200 import BatchContext

    parts = [region(11, 70, 120, 24, 300), region(12, 9, 260, 5, 400), region(13, 30, 60, 7, 200)]
    w = synthetic.from_regions(parts)
    base = BatchContext()
    base.set_profiling(True)
    default, _ = base.compute(w, FLOAT)
    ctx = BatchContext()
    ctx.set_tuning(8, 100, 2, rows_extra, warps)
    assert ctx.tuning()["rows_extra"] == rows_extra and ctx.tuning()["warps_per_block"] == warps
    ctx.set_profiling(True)
    shaped, _ = ctx.compute(w, FLOAT)
    assert shaped.tobytes() == default.tobytes()

    def bins(c):
        return {(p["kind"], p["rows"]) for p in c.launch_profile() if not p["recomputation"]}

    # Kind 0 (two reads, FP32x2) moves up one row up to 8, kind 1 (one read, 10-20 rows) one even step.
    up = lambda k, r: (k, r + 1 if k == 0 and r < 8 else (r + 2 if k == 1 and r < 20 else r))
    expected = {up(k, r) for k, r in bins(base)} if rows_extra else bins(base)
    assert bins(ctx) == expected
    assert any(k == 1 for k, _ in expected) and any(k == 0 for k, _ in expected)


def test_page_locked_inputs_and_outputs_give_the_same_bits(gpu):
    # Read arrays and an output array in page-locked memory take the direct upload and download
    # (no staging copy); the bits must not change, nor may prepare return before the upload is done.
    import ctypes as C
    import dataclasses

    import torch

    from fgkl_b200 import BatchContext, _lib
    from fgkl_b200.pairhmm import _check, _ptr

    w = synthetic.workload(1, seed=9, regions=16)
    ctx = BatchContext()
    expected, _ = ctx.compute(w, FLOAT)

    def pinned(a):
        t = torch.empty(a.size, dtype=torch.uint8 if a.dtype == np.uint8 else torch.float64, pin_memory=True)
        p = t.numpy()
        p[...] = a
        return t, p

    keep = []
    fields = {}
    for f in ("bases", "quals", "ins_gop", "del_gop", "gcp"):
        t, p = pinned(getattr(w, f))
        keep.append(t)
        fields[f] = p
    wp = dataclasses.replace(w, **fields)
    t_out, out = pinned(np.zeros(w.output_len()))
    b, c = wp.as_batch(), FLOAT._c()
    st = _lib.Stats()
    _check(_lib.lib().fgkl_batch_prepare(ctx._ctx, C.byref(b), C.byref(c)))
    for f in fields.values():
        f[...] = 0  # the caller reuses its buffers once prepare has returned
    _check(_lib.lib().fgkl_batch_run(ctx._ctx))
    _check(_lib.lib().fgkl_batch_fetch(ctx._ctx, _ptr(out, _lib.f64p), out.size, C.byref(st)))
    assert out.tobytes() == expected.tobytes()

    # One read array page-locked and the others not: the staging path; a pageable output.
    t_bases, p_bases = pinned(w.bases)
    mixed = dataclasses.replace(w, bases=p_bases)
    b2 = mixed.as_batch()
    out2 = np.zeros(w.output_len())
    _check(_lib.lib().fgkl_batch_compute(ctx._ctx, C.byref(b2), C.byref(c), _ptr(out2, _lib.f64p), out2.size, C.byref(st)))
    assert out2.tobytes() == expected.tobytes()
    del t_bases, t_out, keep


def two_family_region(seed, n_a=5, n_b=2, hap_len=260, read_len=120):
    """Haplotypes of two unrelated families (n_a near copies of one sequence, n_b of another) and
    reads sampled from each: a read of family B is lost in FP32 against every A haplotype (a dense
    read when 3 n_a >= n_a + n_b and the shared program is the cheaper sweep, as here, where each
    family's copies differ only in their last 40 bases), a read of family A only against the n_b B
    haplotypes (a sparse read when 3 n_b < n_a + n_b)."""
    rng = Rng(seed)
    fam = [bytes(rng.base() for _ in range(hap_len)) for _ in range(2)]
    haps = []
    for f, count in ((0, n_a), (1, n_b)):
        for _ in range(count):
            h = bytearray(fam[f])
            for _ in range(3):  # near the end, so the family shares long prefixes
                h[hap_len - 40 + rng.below(40)] = rng.base()
            haps.append(bytes(h))
    reads, owner = [], []
    for i in range(12):
        f = i % 3 == 2  # every third read from family B
        src = fam[int(f)]
        start = rng.below(hap_len - read_len)
        reads.append(Read(src[start:start + read_len], bytes(20 + rng.below(21) for _ in range(read_len)),
                          bytes([45] * read_len), bytes([45] * read_len), bytes([10] * read_len)))
        owner.append(int(f))
    return reads, haps, owner


def test_dense_reads_are_recomputed_with_their_shared_program(gpu):
    """fgkl lib.rs:495-520: after an FP32 pass, a read lost against at least a third of the haplotypes
    is recomputed once in FP64 against all of them with sharing, the others pair by pair. Every lost
    pair comes back at FP64 accuracy; a dense read's lost pairs carry the bits of its FP64 program,
    that is of the double-precision pass, and the pairs it did not lose keep their FP32 bits."""
    reads, haps, owner = two_family_region(23)
    expected = reference_all(reads, haps).reshape(len(reads), len(haps))
    fam_of_hap = [0] * 5 + [1] * 2
    lost_mask = np.array([[owner[r] != fam_of_hap[h] for h in range(len(haps))] for r in range(len(reads))])
    assert (expected[lost_mask] < -70.0).all() and (expected[~lost_mask] > -60.0).all()
    out, fallbacks = compute_counting(FLOAT, reads, haps)
    out = out.reshape(len(reads), len(haps))
    assert fallbacks == int(lost_mask.sum())
    assert_close(out[lost_mask], expected[lost_mask], 1e-9, "lost pairs")
    assert_close(out[~lost_mask], expected[~lost_mask], 1e-4, "kept pairs")
    double = compute(DOUBLE, reads, haps).reshape(len(reads), len(haps))
    dense = [r for r in range(len(reads)) if owner[r] == 1]
    for r in dense:
        assert out[r][lost_mask[r]].tobytes() == double[r][lost_mask[r]].tobytes(), r
    alone = compute(FLOAT, [reads[r] for r in range(len(reads)) if owner[r] == 0], haps).reshape(-1, len(haps))
    kept = out[[r for r in range(len(reads)) if owner[r] == 0]]
    assert kept[:, :5].tobytes() == alone[:, :5].tobytes()


@pytest.mark.parametrize("long_len", [149, 2000])
def test_a_long_haplotype_resumed_from_a_one_base_prefix_keeps_its_own_scale(gpu, long_len):
    # The one-base haplotype "C" sorts first and the long one resumes from its column 1. A resumed
    # segment rescales the restored state to its own initial constant (kernel.rs:641-678); kept at the
    # first haplotype's constant, a short read's likelihood near 1 overflowed (FP64 from about 16x the
    # constant, FP32 from 256x).
    rng = Rng(77)
    long_hap = b"C" + bytes(rng.base() for _ in range(long_len - 1))
    haps = [long_hap, b"C", long_hap[:long_len // 2]]
    reads = [simple_read(b"A"), simple_read(b"CT"), simple_read(b"GCA"), simple_read(long_hap[10:40])]
    expected = reference_all(reads, haps)
    for precision, tol in ((Precision.DOUBLE, 1e-9), (Precision.FLOAT, 1e-4)):
        for share in (True, False):
            assert_close(compute(cfg(precision, share), reads, haps), expected, tol, f"{precision}, share {share}")


def test_an_fp32_overflow_is_recomputed_in_fp64(gpu):
    # A 1-base read N (prior near 1 in every column) against two 528-base haplotypes that differ at
    # position 150: with suffix sharing, row 0's backward start mass sums the 377 shared suffix
    # columns at the 2^120 backward scale, past FP32's range. fgkl's finish_lane accepts the
    # resulting +inf (kernel.rs:897-914), and its CPU restatement here returns +inf; this build counts
    # a non-finite FP32 result as lost and recomputes it in FP64, which gives GATK's value.
    rng = Rng(91)
    hap = bytes(rng.base() for _ in range(528))
    other = bytearray(hap)
    other[150] = ord("A") if hap[150] != ord("A") else ord("C")
    haps = [hap, bytes(other)]
    reads = [Read(b"N", bytes([30]), bytes([45]), bytes([38]), bytes([8])), simple_read(b"A"), simple_read(hap[100:130])]
    expected = reference_all(reads, haps)
    assert np.isfinite(expected).all()
    for share in (True, False):
        assert_close(compute(cfg(Precision.FLOAT, share), reads, haps), expected, 1e-4, f"float, share {share}")
        assert_close(compute(cfg(Precision.DOUBLE, share), reads, haps), expected, 1e-9, f"double, share {share}")
