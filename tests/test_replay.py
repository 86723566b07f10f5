"""The GATK dump replay tool (fgkl_b200/replay.py): dump parsing, region reconstruction, dump
writing and the result checksums, on the CPU. The reconstruction rules are fgkl's
(crates/pairhmm/src/bin/replay.rs:83-159, pdreplay.rs:41-117); real GATK dumps are not in this
repository, so the dumps here are written from synthetic regions with oracle likelihoods."""
import numpy as np

from fgkl_b200 import DEL_END, DEL_START, SNP, PdHaplotype, Read, synthetic
from fgkl_b200 import replay as RP
from oracle import oracle as O


def regions_with_oracle(seeds=(3, 4, 5), reads=5, read_len=40, haps=3, hap_len=80):
    out = []
    for s in seeds:
        rs, hs = synthetic.reference_region(s, reads, read_len, haps, hap_len).region(0)
        out.append(RP.Region(list(rs), list(hs), list(O.compute_matrix(rs, hs, 4))))
    return out


def same_regions(a, b):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert x.haps == y.haps
        assert x.reads == y.reads
        assert np.array_equal(np.array(x.expected), np.array([float(f"{e:e}") for e in y.expected]))


def test_a_written_dump_parses_back_to_its_regions(tmp_path):
    regions = regions_with_oracle()
    p = tmp_path / "pairs.txt"
    RP.write_plain_dump(regions, p)
    same_regions(RP.parse_plain(p), regions)
    assert len(RP.parse_plain(p, max_regions=2)) == 2


def test_duplicate_reads_and_a_repeated_first_haplotype_stay_in_one_region(tmp_path):
    rs, hs = synthetic.reference_region(9, 4, 30, 3, 60).region(0)
    rs = [rs[0], rs[0], rs[1], rs[2], rs[2]]  # duplicates are dumped back to back
    r = RP.Region(rs, list(hs), list(O.compute_matrix(rs, hs, 4)))
    nxt = regions_with_oracle(seeds=(11,))
    p = tmp_path / "pairs.txt"
    RP.write_plain_dump([r] + nxt, p)
    got = RP.parse_plain(p)
    same_regions(got, [r] + nxt)


def test_a_haplotype_list_broken_mid_read_drops_the_region_so_far(tmp_path):
    regions = regions_with_oracle()
    p = tmp_path / "pairs.txt"
    RP.write_plain_dump(regions, p)
    lines = p.read_text().splitlines()
    # Region 0 has 5 reads x 3 haplotypes; break read 1's list at its second haplotype (line 5).
    f = lines[5].split(" ")
    f[0] = "ACGT" + f[0]
    lines[5] = " ".join(f)
    p.write_text("\n".join(lines) + "\n")
    got = RP.parse_plain(p)
    # Region 0 so far is dropped and parsing starts over at the broken line, learning a new list from
    # it; that list never starts over, so every later line joins it as one more haplotype of a
    # one-read region (fgkl's rule: a mismatch mid-read discards the region, replay.rs:146-151).
    assert len(got) == 1
    assert len(got[0].reads) == 1
    assert got[0].haps[0] == f[0].encode()
    assert len(got[0].haps) == len(lines) - 5
    assert got[0].reads[0].bases == f[1].encode()


def test_pd_dump_round_trip_keeps_flags_including_negative_bytes(tmp_path):
    rs, _ = synthetic.reference_region(13, 4, 30, 1, 60).region(0)
    base = b"ACGTTGCAAGGCTTAGGCTTACGATCGATTACAGGTACGTA"
    f1 = bytearray(len(base))
    f1[5] = DEL_START
    f1[9] = DEL_END
    f2 = bytearray(len(base))
    f2[3] = SNP | 0x80  # a flag byte Java prints as a negative number
    haps = [PdHaplotype(base, bytes(f1)), PdHaplotype(base, bytes(f2))]
    r = RP.Region(list(rs), haps, [-10.5 - i for i in range(len(rs) * 2)])
    p = tmp_path / "pd.txt"
    RP.write_pd_dump([r], p)
    assert "-" in p.read_text().splitlines()[1].split("\t")[1]  # Java prints the high flag bit as a sign
    got = RP.parse_pd(p)
    assert len(got) == 1
    assert [(h.bases, h.flags) for h in got[0].haps] == [(h.bases, h.flags) for h in haps]
    assert got[0].reads == r.reads
    assert got[0].expected == r.expected


def test_java_flag_rendering_parses():
    assert RP.java_flags("[0, 1, -128, 127, 4]") == bytes([0, 1, 128, 127, 4])
    assert RP.java_flags("[]") == b""


def test_fnv1a_over_words_matches_the_byte_hash_on_one_byte_words():
    assert RP.fnv1a64([]) == RP.FNV_OFFSET
    # FNV-1a 64 of the single byte 'a' (a published test vector).
    assert RP.fnv1a64([0x61]) == 0xAF63DC4C8601EC8C
    assert RP.fnv1a64(list(b"foobar")) == 0x85944171F73967E8  # FNV-1a 64 of "foobar"


def test_rounded_words_round_half_away_from_zero_and_saturate():
    x = np.array([2.5, -2.5, 0.49999999999999994, 1.5, -0.5, np.nan, np.inf, -np.inf, 1e30])
    got = RP.round_words(x).view(np.int64)
    i64 = np.iinfo(np.int64)
    assert got.tolist() == [3, -3, 0, 2, -1, 0, i64.max, i64.min, i64.max]


def test_checksums_cover_all_kept_and_rounded_pairs():
    res = np.array([-10.0, -70.0, -5.25], np.float64)
    exp = np.array([-10.0, -70.0, -5.25], np.float64)
    c_all, c_kept, c_round = RP.checksums(res, exp)
    bits = res.view(np.uint64)
    assert c_all == RP.fnv1a64(bits)
    assert c_kept == RP.fnv1a64(bits[[0, 2]])
    assert c_round == RP.fnv1a64(np.array([-10000000, -5250000], np.int64).view(np.uint64))


def test_pd_row_end_state_and_summary():
    assert RP.pd_row_end_state(bytes([0, DEL_START, 0, DEL_END])) == 2
    assert RP.pd_row_end_state(bytes([0, DEL_START, 0])) == 1
    assert RP.pd_row_end_state(bytes([DEL_START, DEL_END, 0])) == 0
    rs = [Read(b"ACGT", bytes([30] * 4), bytes([45] * 4), bytes([45] * 4), bytes([10] * 4))]
    haps = [PdHaplotype(b"ACGTAC", bytes(6)), PdHaplotype(b"ACGTTT", bytes([0, 0, 0, 0, SNP, 0]))]
    s = RP.pd_summary([RP.Region(rs, haps, [0.0, 0.0])])
    assert s["cells"] == 4 * 12
    assert s["shareable_cells"] == 4 * 4  # the common prefix ACGT with equal flags and row-end state
    assert abs(s["flagged_cols_pct"] - 100.0 / 12) < 1e-9
