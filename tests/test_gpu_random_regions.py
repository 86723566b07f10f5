"""Seeded random regions against the FP64 oracle, batched and per call, through the C ABI.

Each batch holds 1-23 regions of random shape:
- reads of 1 to about 700 bases, across the 620-base strip-mining boundary;
- 1-19 haplotypes of 1 to 700 bases, edited copies of one window, with duplicates, N and other bytes;
- about three regions in ten with qualities at the extremes;
- every third batch PD, with SNP and deletion flags.

Both precisions run, with and without suffix sharing (prefix sharing only for PD). The bar is the
suite's: 1e-4 in float and 1e-9 in double. One exception: where 2^1020 L is an FP64 subnormal
(log10 L below -614.7), fgkl's own value has lost a decimal digit for each decade deeper, so the
allowance grows the same way. The per-call form of each region must give the batch's bits.
"""
import numpy as np
import pytest

from fgkl_b200 import BatchContext, Config, PairHmm, PdPairHmm, Precision, synthetic
from oracle import oracle as O
from randregions import region

pytestmark = pytest.mark.gpu


def assert_close(got, exp, tol, what):
    same = got == exp
    with np.errstate(invalid="ignore", over="ignore"):
        d = np.where(same, 0.0, np.abs(got - exp))
        deep = np.where(exp < -614.0, 1e-4 * 10.0 ** np.clip(-614.0 - exp, 0, 300), 0.0)
    bad = ~(d <= np.maximum(tol, deep))
    i = int(np.argmax(bad)) if bad.any() else 0
    assert not bad.any(), f"{what}: {int(bad.sum())} pairs off, e.g. pair {i}: got {got[i]}, expected {exp[i]}"


@pytest.mark.parametrize("seed", range(1000, 1016))
def test_random_regions_match_the_oracle_batched_and_per_call(gpu, seed):
    rng = np.random.default_rng(seed)
    pd = seed % 3 == 2
    parts = [region(rng, pd) for _ in range(int(rng.integers(1, 24)))]
    w = synthetic.from_regions(parts)
    exp = np.concatenate([O.compute_matrix(r, h) for r, h in parts])
    for prec, tol in ((Precision.FLOAT, 1e-4), (Precision.DOUBLE, 1e-9)):
        for share in ((False,) if pd else (True, False)):
            cfg = Config(precision=prec, double_fallback=True, share_suffixes=share)
            ctx = BatchContext()
            try:
                got, _ = ctx.compute(w, cfg)
            finally:
                ctx.close()
            assert_close(got, exp, tol, f"{prec}, share {share}, pd {pd}")
            off = 0
            for g, (r, h) in enumerate(parts):
                n = len(r) * len(h)
                one = (PdPairHmm if pd else PairHmm)(cfg).compute_log10_likelihoods(r, h)
                assert np.array_equal(one, got[off:off + n], equal_nan=True), f"region {g}: per-call bits differ ({prec}, share {share})"
                off += n
