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

from fgkl_b200 import (ALT_A, ALT_C, ALT_G, ALT_T, DEL_END, DEL_START, SNP, BatchContext, Config, PairHmm, PdHaplotype,
                       PdPairHmm, Precision, Read, synthetic)
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ACGT = np.frombuffer(b"ACGT", np.uint8)


def quals(rng, n, typical, extreme):
    q = np.clip(rng.normal(typical, 4, n).round(), 0, 60).astype(np.int64)
    if extreme:
        k = rng.random(n)
        q[k < 0.05] = rng.integers(0, 4, int((k < 0.05).sum()))
        hi = (k >= 0.05) & (k < 0.1)
        q[hi] = rng.integers(200, 256, int(hi.sum()))
    return bytes(q.astype(np.uint8))


def edit(rng, s):
    h = bytearray(s)
    for _ in range(int(rng.integers(0, 5))):
        if len(h) > 0:
            h[int(rng.integers(0, len(h)))] = int(rng.choice(ACGT))
    if rng.random() < 0.4 and len(h) > 8:
        p = int(rng.integers(0, len(h) - 6))
        del h[p:p + int(rng.integers(1, 6))]
    if rng.random() < 0.4:
        p = int(rng.integers(0, len(h) + 1))
        h[p:p] = bytes(rng.choice(ACGT, int(rng.integers(1, 6))))
    if rng.random() < 0.05 and len(h) > 0:
        h[int(rng.integers(0, len(h)))] = ord("N")
    if rng.random() < 0.02 and len(h) > 0:
        h[int(rng.integers(0, len(h)))] = ord("X")
    return bytes(h) if h else b"A"


def region(rng, pd):
    L = int(rng.choice([int(rng.integers(1, 40)), int(rng.integers(40, 400)), int(rng.integers(400, 700))], p=[0.15, 0.65, 0.2]))
    ref = bytes(rng.choice(ACGT, L))
    nh = int(rng.integers(1, 20))
    haps = []
    for k in range(nh):
        if k > 0 and rng.random() < 0.1:
            haps.append(haps[int(rng.integers(0, len(haps)))])  # a duplicate
        else:
            haps.append(edit(rng, ref) if rng.random() < 0.9 else bytes(rng.choice(ACGT, int(rng.integers(1, 700)))))
    nr = int(rng.integers(1, 40))
    extreme = rng.random() < 0.3
    reads = []
    for _ in range(nr):
        h = haps[int(rng.integers(0, nh))]
        want = int(rng.choice([int(rng.integers(1, 12)), int(rng.integers(12, 260)), int(rng.integers(560, 700))], p=[0.1, 0.8, 0.1]))
        n = max(1, min(want, len(h)))
        p = int(rng.integers(0, len(h) - n + 1))
        b = edit(rng, h[p:p + n])
        n = len(b)
        reads.append(Read(b, quals(rng, n, 30, extreme), quals(rng, n, 45, extreme), quals(rng, n, 45, extreme),
                          quals(rng, n, 10, extreme)))
    if not pd:
        return reads, haps
    out = []
    for h in haps:
        f = np.zeros(len(h), np.uint8)
        for _ in range(int(rng.integers(0, 6))):
            pos = int(rng.integers(0, len(h)))
            if f[pos]:
                continue
            if rng.random() < 0.5:
                f[pos] = SNP | int(rng.choice([ALT_A, ALT_C, ALT_G, ALT_T]))
            else:
                ln = min(int(rng.integers(1, 9)), len(h) - pos)
                if f[pos:pos + ln].any():
                    continue
                f[pos] |= DEL_START
                f[pos + ln - 1] |= DEL_END
        out.append(PdHaplotype(h, bytes(f)))
    return reads, out



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
