"""fgkl's SplitMix64 ``Rng`` and ``edited`` (crates/pairhmm/src/synthetic.rs:10-41, :84-98) in Python,
so property tests draw the same haplotype sets as the reference's own tests."""
from __future__ import annotations

M64 = (1 << 64) - 1


class Rng:
    def __init__(self, seed: int):
        self.s = seed & M64

    def next_u64(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & M64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return z ^ (z >> 31)

    def below(self, n: int) -> int:
        return self.next_u64() % n

    def chance(self, p: float) -> bool:
        return (self.next_u64() >> 11) / float(1 << 53) < p

    def base(self) -> int:
        return b"ACGT"[self.below(4)]


def edited(rng: Rng, alphabet: bytes, base: bytes) -> bytes:
    hap = bytearray(base)
    for _ in range(1 + rng.below(3)):
        pos = rng.below(len(hap))
        kind = rng.below(3)
        if kind == 0:
            hap[pos] = alphabet[rng.below(len(alphabet))]
        elif kind == 1:
            hap.insert(pos, alphabet[rng.below(len(alphabet))])
        elif len(hap) > 1:
            del hap[pos]
    return bytes(hap)


def reference_like(rng: Rng, alphabet: bytes, n: int) -> bytes:
    return bytes(alphabet[rng.below(len(alphabet))] for _ in range(n))


def related_pair(rng: Rng, ref_len: int, alt_len: int) -> tuple[bytes, bytes]:
    """A reference and an edited copy of a window of it, like a haplotype or a read: fgkl's
    Smith-Waterman test generator (crates/smithwaterman/src/lib.rs:773-807), draw for draw."""
    reference = bytes(rng.base() for _ in range(ref_len))
    start = rng.below(max(ref_len - alt_len, 0) + 1)
    alt = bytearray(reference[start:min(start + alt_len, ref_len)])
    for _ in range(rng.below(4)):
        if not alt:
            break
        pos = rng.below(len(alt))
        kind = rng.below(3)
        if kind == 0:
            alt[pos] = rng.base()
        elif kind == 1:
            ins = bytes(rng.base() for _ in range(1 + rng.below(6)))
            alt[pos:pos] = ins
        else:
            end = min(pos + 1 + rng.below(6), len(alt))
            if len(alt) > end - pos:
                del alt[pos:end]
    if rng.chance(0.3):
        extra = bytes(rng.base() for _ in range(1 + rng.below(20)))
        if rng.chance(0.5):
            alt[0:0] = extra
        else:
            alt.extend(extra)
    if not alt:
        alt.append(ord("A"))
    return reference, bytes(alt)
