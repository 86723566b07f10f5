"""The GATK dump replay tool on the GPU: a dump written from synthetic regions with FP64 oracle
likelihoods (GATK's `%e`, seven significant digits) replays within the reference's tolerances, the
tool's results are the batched path's bits, and the files and checksums it writes describe them."""
import numpy as np
import pytest

from fgkl_b200 import BatchContext, Config, Precision, Read, synthetic
from fgkl_b200 import replay as RP
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def plain_regions():
    out = []
    for s in (3, 4, 5, 6):
        rs, hs = synthetic.reference_region(s, 9, 70 + 10 * s, 4, 200).region(0)
        out.append(RP.Region(list(rs), list(hs), []))
    # A read unrelated to its haplotypes: it underflows FP32 and GATK records it below -64.
    deep = Read(b"A" * 80, bytes([40] * 80), bytes([45] * 80), bytes([45] * 80), bytes([10] * 80))
    out.append(RP.Region([deep], [b"C" * 80, b"C" * 40 + b"A" * 40], []))
    for r in out:
        r.expected = [float(f"{e:e}") for e in O.compute_matrix(r.reads, r.haps, 4)]
    return out


def tolerance(expected, abs_tol):
    # GATK's %e keeps seven significant digits: half a unit of the seventh digit, plus the kernel's own.
    return 5e-7 * np.abs(expected) + abs_tol


def test_plain_dump_replays_within_tolerance_with_the_batched_bits(gpu, tmp_path):
    regions = plain_regions()
    dump = tmp_path / "pairs.txt"
    RP.write_plain_dump(regions, dump)
    parsed = RP.parse_plain(dump)
    assert len(parsed) == len(regions)
    rep = RP.replay(parsed, iters=1, write_results=str(tmp_path / "out"), stem="pairs")
    expected = np.array([e for r in parsed for e in r.expected])
    assert rep["float"]["gatk_below_f32"] >= 1
    for mode, tol in (("float", 1e-4), ("double", 1e-8)):
        got = rep[mode]["results"]
        assert np.all(np.abs(got - expected) <= tolerance(expected, tol)), mode
        assert rep[mode]["max_abs_err"] == float(np.max(np.abs(got - expected)))
        assert rep[mode]["checksum"] == f"{RP.fnv1a64(got.view(np.uint64)):016x}"
        on_disk = np.fromfile(tmp_path / "out" / f"pairs.{mode}.f64", dtype="<f8")
        assert on_disk.tobytes() == got.tobytes()
    assert np.fromfile(tmp_path / "out" / "pairs.expected.f64", dtype="<f8").tobytes() == expected.tobytes()
    # The tool's results are the batched context's bits.
    w = RP.workload_of(parsed)
    direct, _ = BatchContext().compute(w, Config(Precision.FLOAT))
    assert direct.tobytes() == rep["float"]["results"].tobytes()
    # Without the FP64 recomputation the lost pairs come back NaN and are counted.
    nofb = rep["float-nofb"]
    assert nofb["fallback_pairs"] >= 1
    assert int(np.isnan(nofb["results"]).sum()) == nofb["fallback_pairs"]
    assert rep["float"]["fallback_pairs"] == nofb["fallback_pairs"]


def test_prefix_only_replay_and_the_command_line(gpu, tmp_path):
    regions = plain_regions()
    dump = tmp_path / "pairs.txt"
    RP.write_plain_dump(regions, dump)
    shared = RP.replay(RP.parse_plain(dump), modes=("float",), iters=1)
    prefix = RP.replay(RP.parse_plain(dump), modes=("float",), iters=1, share_suffixes=False)
    expected = np.array([e for r in regions for e in r.expected])
    assert np.all(np.abs(prefix["float"]["results"] - expected) <= tolerance(expected, 1e-4))
    assert prefix["computed_backward_pct"] == 0.0
    assert shared["computed_prefix_pct"] == prefix["computed_prefix_pct"]
    one = tmp_path / "one.txt"
    assert RP.main([str(dump), "--iters", "1", "--modes", "float", "--dump-region", "1", str(one),
                    "--only-region", "2"]) == 0
    again = RP.parse_plain(one)
    assert len(again) == 1 and again[0].reads == regions[1].reads and again[0].haps == regions[1].haps


def test_pd_dump_replays_within_tolerance(gpu, tmp_path):
    parts = [synthetic.reference_pd_region(300 + i, 12, 90 + 20 * i, 5, 240).region(0) for i in range(3)]
    regions = [RP.Region(list(r), list(h), [float(f"{e:e}") for e in O.compute_matrix(r, h, 4)]) for r, h in parts]
    # GATK writes -Infinity for pairs it discards after the kernel; the tool leaves them out of max|err|.
    regions[0].expected[3] = float("-inf")
    dump = tmp_path / "pd.txt"
    RP.write_pd_dump(regions, dump)
    parsed = RP.parse_pd(dump)
    assert len(parsed) == 3
    rep = RP.pd_replay(parsed, iters=1)
    expected = np.array([e for r in parsed for e in r.expected])
    keep = np.isfinite(expected)
    for mode, tol in (("float", 1e-4), ("double", 1e-8)):
        got = rep[mode]["results"]
        assert np.all(np.abs(got[keep] - expected[keep]) <= tolerance(expected[keep], tol)), mode
        assert np.isfinite(got).all()
    assert RP.main([str(dump), "--pd", "--iters", "1"]) == 0
