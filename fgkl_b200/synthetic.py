"""Synthetic workloads from the library's generators (``csrc/synthetic.cpp``).

``reference_region`` / ``reference_pd_region`` rebuild fgkl's own test regions from their seeds
(``crates/pairhmm/src/synthetic.rs``); ``workload`` builds the benchmark shapes.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Iterator

import numpy as np

from . import _lib
from ._lib import lib
from .pairhmm import PdHaplotype, Read, _check


@dataclass
class Workload:
    """Regions in the flattened batch layout (owned numpy arrays)."""

    region_reads: np.ndarray  # int32
    region_haps: np.ndarray   # int32
    bases: np.ndarray
    quals: np.ndarray
    ins_gop: np.ndarray
    del_gop: np.ndarray
    gcp: np.ndarray
    read_offsets: np.ndarray  # int64, total reads + 1
    hap_bases: np.ndarray
    hap_flags: np.ndarray | None
    hap_offsets: np.ndarray   # int64, total haplotypes + 1

    @property
    def num_regions(self) -> int:
        return int(self.region_reads.size)

    def output_len(self) -> int:
        return int(np.dot(self.region_reads.astype(np.int64), self.region_haps.astype(np.int64)))

    def nominal_cells(self) -> int:
        """Σ over regions of Σ read lengths x Σ haplotype lengths (fgkl synthetic.rs:166-170)."""
        return int(self.region_nominal_cells().sum())

    def region_nominal_cells(self) -> np.ndarray:
        """Per region: Σ read lengths x Σ haplotype lengths."""
        rl = np.diff(self.read_offsets)
        hl = np.diff(self.hap_offsets)
        rs = np.add.reduceat(rl, np.r_[0, np.cumsum(self.region_reads)[:-1]]) if rl.size else np.zeros(0, np.int64)
        hs = np.add.reduceat(hl, np.r_[0, np.cumsum(self.region_haps)[:-1]]) if hl.size else np.zeros(0, np.int64)
        return rs.astype(np.int64) * hs.astype(np.int64)

    def as_batch(self) -> _lib.Batch:
        u8 = _lib.u8p
        return _lib.Batch(
            self.num_regions, self.region_reads.ctypes.data_as(_lib.i32p), self.region_haps.ctypes.data_as(_lib.i32p),
            self.bases.ctypes.data_as(u8), self.quals.ctypes.data_as(u8), self.ins_gop.ctypes.data_as(u8),
            self.del_gop.ctypes.data_as(u8), self.gcp.ctypes.data_as(u8), self.read_offsets.ctypes.data_as(_lib.i64p),
            self.hap_bases.ctypes.data_as(u8), self.hap_flags.ctypes.data_as(u8) if self.hap_flags is not None else None,
            self.hap_offsets.ctypes.data_as(_lib.i64p))

    def region(self, g: int):
        """(reads, haplotypes) of region g as API objects."""
        r0 = int(self.region_reads[:g].sum())
        h0 = int(self.region_haps[:g].sum())
        reads = []
        for r in range(r0, r0 + int(self.region_reads[g])):
            lo, hi = int(self.read_offsets[r]), int(self.read_offsets[r + 1])
            reads.append(Read(self.bases[lo:hi].tobytes(), self.quals[lo:hi].tobytes(), self.ins_gop[lo:hi].tobytes(),
                              self.del_gop[lo:hi].tobytes(), self.gcp[lo:hi].tobytes()))
        haps = []
        for h in range(h0, h0 + int(self.region_haps[g])):
            lo, hi = int(self.hap_offsets[h]), int(self.hap_offsets[h + 1])
            if self.hap_flags is not None:
                haps.append(PdHaplotype(self.hap_bases[lo:hi].tobytes(), self.hap_flags[lo:hi].tobytes()))
            else:
                haps.append(self.hap_bases[lo:hi].tobytes())
        return reads, haps

    def regions(self) -> Iterator:
        for g in range(self.num_regions):
            yield self.region(g)

    def output_offsets(self) -> np.ndarray:
        """First output element of each region (and the total at the end)."""
        sizes = self.region_reads.astype(np.int64) * self.region_haps.astype(np.int64)
        return np.r_[0, np.cumsum(sizes)]

    def subset(self, regions: Sequence[int] | range) -> "Workload":
        """The regions `regions`, in that order, as a workload of their own (array slices)."""
        regions = [int(g) for g in regions]
        rr = self.region_reads.astype(np.int64)
        rh = self.region_haps.astype(np.int64)
        first_read = np.r_[0, np.cumsum(rr)]
        first_hap = np.r_[0, np.cumsum(rh)]
        read_idx = [np.arange(first_read[g], first_read[g + 1]) for g in regions]
        hap_idx = [np.arange(first_hap[g], first_hap[g + 1]) for g in regions]
        reads = np.concatenate(read_idx) if read_idx else np.zeros(0, np.int64)
        haps = np.concatenate(hap_idx) if hap_idx else np.zeros(0, np.int64)

        def gather(data, offsets, idx):
            lo, hi = offsets[idx], offsets[idx + 1]
            new_off = np.r_[0, np.cumsum(hi - lo)].astype(np.int64)
            if idx.size == 0:
                return data[:0].copy(), new_off
            pos = np.repeat(lo - new_off[:-1], hi - lo) + np.arange(int(new_off[-1]))
            return data[pos], new_off

        cols = []
        for a in (self.bases, self.quals, self.ins_gop, self.del_gop, self.gcp):
            col, roff = gather(a, self.read_offsets, reads)
            cols.append(col)
        hb, hoff = gather(self.hap_bases, self.hap_offsets, haps)
        hf = gather(self.hap_flags, self.hap_offsets, haps)[0] if self.hap_flags is not None else None
        return Workload(self.region_reads[regions].copy(), self.region_haps[regions].copy(), *cols, roff, hb, hf, hoff)


from typing import Sequence  # noqa: E402


def _from_handle(h) -> Workload:
    if not h:
        raise _lib_error()
    try:
        b = _lib.Batch()
        sizes = (C.c_int64 * 4)()
        lib().fgkl_synth_view(h, C.byref(b), sizes)
        nr, nrb, nh, nhb = (int(x) for x in sizes)
        n = b.num_regions

        def arr(ptr, count, dtype):
            if count == 0:
                return np.zeros(0, dtype)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dtype))), shape=(count,)).copy()

        return Workload(
            region_reads=arr(b.region_reads, n, np.int32), region_haps=arr(b.region_haps, n, np.int32),
            bases=arr(b.bases, nrb, np.uint8), quals=arr(b.quals, nrb, np.uint8), ins_gop=arr(b.ins_gop, nrb, np.uint8),
            del_gop=arr(b.del_gop, nrb, np.uint8), gcp=arr(b.gcp, nrb, np.uint8), read_offsets=arr(b.read_offsets, nr + 1, np.int64),
            hap_bases=arr(b.hap_bases, nhb, np.uint8), hap_flags=arr(b.hap_flags, nhb, np.uint8) if b.hap_flags else None,
            hap_offsets=arr(b.hap_offsets, nh + 1, np.int64))
    finally:
        lib().fgkl_synth_free(h)


def _lib_error():
    from .pairhmm import DeviceError
    return DeviceError(_lib.FGKL_E_INVALID_ARGUMENT, _lib.last_error())


def workload(which: int, seed: int = 0, regions: int = 0, threads: int = 8) -> Workload:
    """Benchmark workload `which` (0-4, see csrc/synthetic.h)."""
    return _from_handle(lib().fgkl_synth_config(which, seed, regions, threads))


def reference_region(seed: int, num_reads: int, read_len: int, num_haps: int, hap_len: int) -> Workload:
    """fgkl's ``Region::generate`` (synthetic.rs:103-153), draw for draw."""
    return _from_handle(lib().fgkl_synth_reference_region(seed, num_reads, read_len, num_haps, hap_len, 0))


def reference_pd_region(seed: int, num_reads: int, read_len: int, num_haps: int, hap_len: int) -> Workload:
    """fgkl's ``PdRegion::generate`` (synthetic.rs:199-289), draw for draw."""
    return _from_handle(lib().fgkl_synth_reference_region(seed, num_reads, read_len, num_haps, hap_len, 1))


def from_regions(parts) -> Workload:
    """A workload from a list of (reads, haplotypes) with API objects."""
    rr, rh, cols, roff, hb, hf, hoff = [], [], [[], [], [], [], []], [0], [], [], [0]
    pd = False
    for reads, haps in parts:
        rr.append(len(reads))
        rh.append(len(haps))
        for r in reads:
            for i, f in enumerate(("bases", "quals", "ins_gop", "del_gop", "gcp")):
                cols[i].append(np.frombuffer(bytes(getattr(r, f)), np.uint8))
            roff.append(roff[-1] + len(r.bases))
        for h in haps:
            if isinstance(h, PdHaplotype):
                pd = True
                hb.append(np.frombuffer(bytes(h.bases), np.uint8))
                hf.append(np.frombuffer(bytes(h.flags), np.uint8))
                hoff.append(hoff[-1] + len(h.bases))
            else:
                hb.append(np.frombuffer(bytes(h), np.uint8))
                hf.append(np.zeros(len(h), np.uint8))
                hoff.append(hoff[-1] + len(h))

    def cat(xs):
        return np.concatenate(xs) if xs else np.zeros(0, np.uint8)

    return Workload(np.array(rr, np.int32), np.array(rh, np.int32), *[cat(c) for c in cols], np.array(roff, np.int64), cat(hb),
                    cat(hf) if pd else None, np.array(hoff, np.int64))
