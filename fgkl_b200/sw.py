"""Smith-Waterman alignment as GATK's SmithWatermanJavaAligner computes it (fgkl's
``crates/smithwaterman``), on the sm_100a kernel of ``libfgkl_b200.so``.

``align`` is the per-call form (fgkl's ``Aligner::align`` and the JNI ``alignNative``); ``align_batch``
runs many pairs in one launch. Results are ``Alignment(cigar, offset)``, the CIGAR as text in
alternate order and GATK's alignment offset.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import lib
from .pairhmm import BatchContext, _check


class OverhangStrategy(enum.IntEnum):
    """GATK's SWOverhangStrategy, numbered as fgkl's JNI entry numbers it."""

    SOFTCLIP = 0
    INDEL = 1
    LEADING_INDEL = 2
    IGNORE = 3


@dataclass(frozen=True)
class SwParameters:
    """GATK's SWParameters: a positive match value and negative penalties (lib.rs:42-66)."""

    match_value: int
    mismatch_penalty: int
    gap_open_penalty: int
    gap_extend_penalty: int

    def _c(self) -> _lib.SwParams:
        return _lib.SwParams(self.match_value, self.mismatch_penalty, self.gap_open_penalty, self.gap_extend_penalty)


# GATK's presets (SmithWatermanAlignmentConstants).
HAPLOTYPE_TO_REFERENCE = SwParameters(200, -150, -260, -11)
ALIGNMENT_TO_BEST_HAPLOTYPE = SwParameters(10, -15, -30, -5)
ORIGINAL_DEFAULT = SwParameters(3, -1, -4, -3)


@dataclass(frozen=True)
class Alignment:
    cigar: str
    offset: int


_OPS = "MIDNS"


def _u8(b) -> np.ndarray:
    return np.frombuffer(bytes(b), dtype=np.uint8)


def align(reference: bytes, alternate: bytes, params: SwParameters, strategy: OverhangStrategy) -> Alignment:
    """One pair on the calling thread's engine."""
    r, a = _u8(reference), _u8(alternate)
    cap = 16 * (r.size + a.size + 4)
    buf = C.create_string_buffer(cap)
    off = C.c_int32()
    p = params._c()
    _check(lib().fgkl_sw_align(r.ctypes.data_as(_lib.u8p), r.size, a.ctypes.data_as(_lib.u8p), a.size, C.byref(p), int(strategy),
                               buf, cap, C.byref(off)))
    return Alignment(buf.value.decode(), int(off.value))


def _flat(seqs: Sequence[bytes]) -> tuple[np.ndarray, np.ndarray]:
    off = np.zeros(len(seqs) + 1, np.int64)
    np.cumsum([len(s) for s in seqs], out=off[1:])
    data = np.frombuffer(b"".join(bytes(s) for s in seqs), np.uint8) if seqs else np.zeros(0, np.uint8)
    return np.ascontiguousarray(data), off


def align_batch(pairs: Sequence[tuple[bytes, bytes]], params: SwParameters, strategy: OverhangStrategy,
                context: BatchContext | None = None) -> list[Alignment]:
    """Every (reference, alternate) pair in one launch on `context` (a new one when None)."""
    ctx = context or BatchContext()
    try:
        refs, roff = _flat([p[0] for p in pairs])
        alts, aoff = _flat([p[1] for p in pairs])
        b = _lib.SwBatch(len(pairs), refs.ctypes.data_as(_lib.u8p), roff.ctypes.data_as(_lib.i64p), alts.ctypes.data_as(_lib.u8p),
                         aoff.ctypes.data_as(_lib.i64p))
        cap = int(lib().fgkl_sw_cigar_capacity(C.byref(b)))
        cigar = np.zeros(max(cap, 1), np.uint32)
        counts = np.zeros(max(len(pairs), 1), np.int32)
        offsets = np.zeros(max(len(pairs), 1), np.int32)
        p = params._c()
        _check(lib().fgkl_sw_align_batch(ctx._ctx, C.byref(b), C.byref(p), int(strategy),
                                         cigar.ctypes.data_as(C.POINTER(C.c_uint32)), cap,
                                         counts.ctypes.data_as(_lib.i32p), offsets.ctypes.data_as(_lib.i32p)))
        out, slot = [], 0
        for k, (ref, alt) in enumerate(pairs):
            elems = cigar[slot:slot + int(counts[k])]
            out.append(Alignment("".join(f"{int(e) >> 4}{_OPS[int(e) & 0xF]}" for e in elems), int(offsets[k])))
            slot += len(ref) + len(alt) + 2
        return out
    finally:
        if context is None:
            ctx.close()
