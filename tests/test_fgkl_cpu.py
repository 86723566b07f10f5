"""fgkl's batched CPU algorithm restated in C (oracle/fgkl_cpu.c), the benchmark's timed CPU reference,
against the scalar FP64 oracle and the golden fixtures.

The tolerances are fgkl's own (crates/pairhmm/src/lib.rs:621-660): 1e-9 log10 in double, 1e-4 in
float. Cases follow its tests: prefix sharing over nested and repeated prefixes and lengths
(lib.rs:666-692), bytes outside ACGTN (lib.rs:694-717), float underflow falling back to double
(lib.rs:719-739), suffix sharing with reads ending on different rows (lib.rs:746-809), and every
instruction set this CPU has.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from fgkl_b200 import Read, synthetic
from oracle import oracle as O
from refgen import Rng

GOLDEN = Path(__file__).resolve().parent / "golden"


def isas():
    return list(range(O.cpu_isa() + 1))


def mixed_workload():
    rng = Rng(5)

    def random_read(n):
        return Read(bytes(rng.base() for _ in range(n)), bytes([30] * n), bytes([45] * n), bytes([45] * n),
                    bytes([10] * n))

    parts = []
    deep = Read(b"A" * 80, bytes([40] * 80), bytes([45] * 80), bytes([45] * 80), bytes([10] * 80))
    parts.append(([deep], [b"C" * 80, b"C" * 40 + b"A" * 40]))
    reads, haps = synthetic.reference_region(31, 70, 120, 24, 300).region(0)
    haps = list(haps) + [haps[3], haps[3], b"ACGTXXACGT" * 20, b"ACGTNNACGT" * 20]
    reads = list(reads) + [random_read(120) for _ in range(29)]
    parts.append((reads, haps))
    for seed in range(8):
        parts.append(synthetic.reference_region(100 + seed, 5 + 7 * seed, 50 + 10 * seed, 2 + 3 * seed,
                                                100 + 20 * seed).region(0))
    return synthetic.from_regions(parts)


@pytest.fixture(scope="module")
def mixed():
    w = mixed_workload()
    return w, O.workload_matrix(w, None, 8)


@pytest.mark.parametrize("isa", isas())
@pytest.mark.parametrize("share", [True, False])
def test_double_matches_the_scalar_oracle(mixed, isa, share):
    w, ref = mixed
    out, lost = O.fgkl_cpu_workload(w, None, 4, double=True, share_suffixes=share, isa=isa)
    assert np.abs(out - ref).max() <= 1e-9
    assert lost == 0


@pytest.mark.parametrize("isa", isas())
@pytest.mark.parametrize("share", [True, False])
def test_float_matches_the_scalar_oracle_and_recomputes_underflow(mixed, isa, share):
    w, ref = mixed
    out, lost = O.fgkl_cpu_workload(w, None, 4, double=False, share_suffixes=share, isa=isa)
    assert np.isfinite(out).all()
    assert np.abs(out - ref).max() <= 1e-4
    assert lost > 0, "the deep pair and the random reads must underflow"


def test_without_the_double_fallback_lost_pairs_stay_nan(mixed):
    w, ref = mixed
    out, lost = O.fgkl_cpu_workload(w, None, 4, double=False, double_fallback=False)
    nan = np.isnan(out)
    assert int(nan.sum()) == lost > 0
    assert np.abs(out[~nan] - ref[~nan]).max() <= 1e-4


def test_results_do_not_depend_on_threads(mixed):
    w, _ = mixed
    one, _ = O.fgkl_cpu_workload(w, None, 1)
    many, _ = O.fgkl_cpu_workload(w, None, 7)
    assert one.tobytes() == many.tobytes()


@pytest.mark.parametrize("name", ["config0_seed0", "region_11_70x120_24x300"])
def test_matches_the_golden_fixtures(name):
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    w = mod.build(name)
    expected = np.array([float(x) for x in json.loads((GOLDEN / f"{name}.json").read_text())["log10"]])
    for double, tol in ((True, 1e-9), (False, 1e-4)):
        out, _ = O.fgkl_cpu_workload(w, None, 4, double=double)
        assert np.abs(out - expected).max() <= tol, (name, double)


def test_a_subset_of_regions_lands_in_output_order():
    w = synthetic.workload(1, seed=3, regions=12, threads=4)
    full, _ = O.fgkl_cpu_workload(w, None, 4)
    offs = w.output_offsets()
    picked = [2, 5, 11]
    part, _ = O.fgkl_cpu_workload(w, picked, 4)
    assert part.tobytes() == np.concatenate([full[offs[g]:offs[g + 1]] for g in picked]).tobytes()


def pd_workload():
    from fgkl_b200 import ALT_C, ALT_G, ALT_T, DEL_END, DEL_START, SNP, PdHaplotype

    parts = [synthetic.reference_pd_region(31 + s, 20 + 5 * s, 60 + 20 * s, 6, 150 + 30 * s).region(0) for s in range(4)]
    # fgkl's PD edge cases (pd.rs:230-330): flags on the last columns, back-to-back and one-base
    # deletions, a SNP inside a deletion, nested prefixes with flag splits.
    hap = b"ACGTTGCAAGGCTTAGGCTTACGATCGATTACAGGT"
    n = len(hap)

    def flags(**at):
        f = bytearray(n)
        for k, v in at.items():
            f[int(k[1:])] = v
        return bytes(f)

    haps = [PdHaplotype(hap, flags(**{f"p{n - 3}": DEL_START, f"p{n - 1}": DEL_END})),
            PdHaplotype(hap, flags(**{f"p{n - 1}": DEL_START | DEL_END})),
            PdHaplotype(hap, flags(p5=DEL_START, p7=DEL_END, p8=DEL_START | DEL_END, p9=DEL_START, p12=DEL_END)),
            PdHaplotype(hap, flags(p10=DEL_START, p11=SNP | ALT_T, p13=DEL_END | SNP | ALT_G)),
            PdHaplotype(hap, flags(p30=SNP | ALT_C)), PdHaplotype(hap, bytes(n)), PdHaplotype(hap[:20], bytes(20)),
            PdHaplotype(hap + b"ACG", flags(p12=DEL_START, p15=DEL_END) + bytes(3))]
    reads, _ = synthetic.reference_pd_region(13, 30, 30, 1, n).region(0)
    parts.append((reads, haps))
    # A read no haplotype explains underflows FP32 (pd.rs:410-430).
    deep = Read(b"A" * 80, bytes([40] * 80), bytes([45] * 80), bytes([45] * 80), bytes([10] * 80))
    f = bytearray(80)
    f[10] = DEL_START
    f[20] = DEL_END
    parts.append(([deep], [PdHaplotype(b"C" * 80, bytes(f)), PdHaplotype(b"C" * 40 + b"A" * 40, bytes(80))]))
    return synthetic.from_regions(parts)


@pytest.fixture(scope="module")
def pd_mixed():
    w = pd_workload()
    return w, O.workload_matrix(w, None, 8)


@pytest.mark.parametrize("isa", isas())
@pytest.mark.parametrize("double", [False, True])
def test_pd_kernel_matches_the_pd_oracle(pd_mixed, isa, double):
    w, ref = pd_mixed
    out, lost = O.fgkl_cpu_workload(w, None, 4, double=double, isa=isa)
    assert np.isfinite(out).all()
    assert np.abs(out - ref).max() <= (1e-9 if double else 1e-4)
    if double:
        assert lost == 0
    else:
        assert lost > 0, "the PD regions hold reads that underflow FP32"


def test_pd_results_do_not_depend_on_threads_or_on_the_recomputation_split(pd_mixed):
    w, ref = pd_mixed
    one, _ = O.fgkl_cpu_workload(w, None, 1)
    many, _ = O.fgkl_cpu_workload(w, None, 6)
    assert one.tobytes() == many.tobytes()
    nofb, lost = O.fgkl_cpu_workload(w, None, 4, double_fallback=False)
    assert int(np.isnan(nofb).sum()) == lost
    keep = ~np.isnan(nofb)
    assert nofb[keep].tobytes() == one[keep].tobytes()


@pytest.mark.parametrize("seed", range(2000, 2006))
def test_random_regions_match_the_oracle_apart_from_fgkls_known_behaviours(seed):
    # Random regions (tests/randregions.py), plain and PD, both precisions, with and without suffix
    # sharing. Two fgkl behaviours stay out of the comparison, both restated faithfully here:
    # - flush-to-zero: fgkl's SIMD kernels run with FTZ/DAZ, so values near FP64's subnormal range
    #   (log10 L below about -600) differ from the scalar oracle's, which keeps subnormals;
    # - an FP32 +inf from the suffix join, which finish_lane accepts (kernel.rs:897-914).
    from randregions import region

    rng = np.random.default_rng(seed)
    pd = seed % 3 == 2
    parts = [region(rng, pd) for _ in range(int(rng.integers(1, 24)))]
    w = synthetic.from_regions(parts)
    exp = np.concatenate([O.compute_matrix(r, h) for r, h in parts])
    for double, tol in ((False, 1e-4), (True, 1e-9)):
        for share in ((False,) if pd else (True, False)):
            got, _ = O.fgkl_cpu_workload(w, double=double, share_suffixes=share)
            keep = ~((exp < -600.0) | (np.isposinf(got) & share & (not double)))
            g, e = got[keep], exp[keep]
            with np.errstate(invalid="ignore"):
                d = np.where(g == e, 0.0, np.abs(g - e))
            assert np.all(d <= tol), f"double {double}, share {share}: max diff {np.nanmax(d)}"
