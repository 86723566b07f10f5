"""Random regions for the parity tests: reads of 1 to about 700 bases (across the 620-base
strip-mining boundary), haplotypes of 1 to 700 bases edited from one window (with duplicates, N and
other bytes), qualities at the extremes in about three regions in ten, and, for PD, SNP and deletion
flags."""
import numpy as np

from fgkl_b200 import ALT_A, ALT_C, ALT_G, ALT_T, DEL_END, DEL_START, SNP, PdHaplotype, Read

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
