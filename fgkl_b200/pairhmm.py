"""Host-side mirror of fgkl's PairHMM API (``crates/pairhmm/src/lib.rs``, ``pd.rs``).

``PairHmm`` / ``PdPairHmm`` take the same inputs, validate them in the same order and raise the same
errors as fgkl's ``PairHmm::compute_log10_likelihoods`` (lib.rs:270-293) and
``PdPairHmm::compute_log10_likelihoods`` (pd.rs:251-279), then call the sm_100a kernels through the
C ABI. ``BatchContext`` is the batched, persistent form over many regions.
"""
from __future__ import annotations

import ctypes as C
import sys
import enum
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import lib


class Precision(enum.Enum):
    """Arithmetic precision (lib.rs:70-105)."""

    FLOAT = "float"
    DOUBLE = "double"


@dataclass
class Config:
    """How to build a PairHmm (lib.rs:211-238)."""

    precision: Precision = Precision.FLOAT
    double_fallback: bool = True
    share_suffixes: bool = True

    def _c(self) -> _lib.Config:
        return _lib.Config(int(self.precision is Precision.DOUBLE), int(self.double_fallback), int(self.share_suffixes))


class PairHmmError(ValueError):
    """Why a likelihood computation was refused (lib.rs:303-323); indices are the caller's."""


class EmptyRead(PairHmmError):
    def __init__(self, index: int):
        super().__init__(f"read {index} has no bases")
        self.index = index


class MismatchedReadArrays(PairHmmError):
    def __init__(self, index: int):
        super().__init__(f"read {index}: bases, qualities and penalties differ in length")
        self.index = index


class EmptyHaplotype(PairHmmError):
    def __init__(self, index: int):
        super().__init__(f"haplotype {index} has no bases")
        self.index = index


class MismatchedHaplotypeArrays(PairHmmError):
    def __init__(self, index: int):
        super().__init__(f"haplotype {index}: bases and flags differ in length")
        self.index = index


class OutputLength(PairHmmError):
    def __init__(self, expected: int, actual: int):
        super().__init__(f"output has {actual} elements but reads x haplotypes is {expected}")
        self.expected = expected
        self.actual = actual


class DeviceError(RuntimeError):
    """The GPU path failed or is unavailable (no device, CUDA error, unsupported input)."""

    def __init__(self, code: int, message: str):
        super().__init__(f"fgkl_b200 error {code}: {message}")
        self.code = code


@dataclass
class Read:
    """One read's bases and per-base penalties (lib.rs:29-68)."""

    bases: bytes
    quals: bytes
    ins_gop: bytes
    del_gop: bytes
    gcp: bytes

    def __len__(self) -> int:
        return len(self.bases)


@dataclass
class PdHaplotype:
    """A partially determined haplotype: bases and per-base flags (pd.rs:29-37)."""

    bases: bytes
    flags: bytes


# PD flag bits, pd.rs:15-27.
SNP, DEL_START, DEL_END, ALT_A, ALT_C, ALT_G, ALT_T = 1, 2, 4, 8, 16, 32, 64


def _u8(b) -> np.ndarray:
    return np.frombuffer(bytes(b), dtype=np.uint8) if not isinstance(b, np.ndarray) else np.ascontiguousarray(b, dtype=np.uint8)


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _check(rc: int) -> None:
    if rc == 0:
        return
    msg = _lib.last_error()
    raise DeviceError(rc, msg)


def set_call_combining(max_batches: int) -> int:
    """Sets how many combined batches of concurrent per-call requests may run at once (0: every
    call runs alone; at most 8; default 2) and returns the previous value. Calls made through
    PairHmm / PdPairHmm carry counters and always run alone; the JNI entry points do not."""
    rc = lib().fgkl_set_call_combining(int(max_batches))
    if rc < 0:
        raise ValueError(_lib.last_error())
    return rc


def set_allocation_limit(limit_bytes: int) -> int:
    """Failure injection: device and page-locked host allocations of more than ``limit_bytes`` fail
    as out of memory (``DeviceError`` with code ``FGKL_E_OUT_OF_MEMORY``) until the limit is removed
    with 0. Returns the previous limit."""
    rc = int(lib().fgkl_set_allocation_limit(int(limit_bytes)))
    if rc < 0:
        raise ValueError(_lib.last_error())
    return rc


def call_combining_stats() -> tuple[int, int]:
    """(combined batches of two or more requests, requests they held) since the library loaded."""
    b, r = C.c_uint64(), C.c_uint64()
    _check(lib().fgkl_call_combining_stats(C.byref(b), C.byref(r)))
    return b.value, r.value


class _Flat:
    """Reads and haplotypes flattened into the JNI layout, kept alive for the call."""

    def __init__(self, reads: Sequence[Read], bases: Sequence[bytes], flags: Sequence[bytes] | None):
        self.r = [np.concatenate([_u8(getattr(r, f)) for r in reads]) if reads else np.zeros(0, np.uint8)
                  for f in ("bases", "quals", "ins_gop", "del_gop", "gcp")]
        self.roff = np.zeros(len(reads) + 1, np.int32)
        np.cumsum([len(r.bases) for r in reads], out=self.roff[1:])
        self.hb = np.concatenate([_u8(b) for b in bases]) if bases else np.zeros(0, np.uint8)
        self.hf = (np.concatenate([_u8(f) for f in flags]) if flags else np.zeros(0, np.uint8)) if flags is not None else None
        self.hoff = np.zeros(len(bases) + 1, np.int32)
        np.cumsum([len(b) for b in bases], out=self.hoff[1:])

    def structs(self):
        rd = _lib.Reads(
            _ptr(self.r[0], _lib.u8p), self.r[0].size, _ptr(self.r[1], _lib.u8p), self.r[1].size,
            _ptr(self.r[2], _lib.u8p), self.r[2].size, _ptr(self.r[3], _lib.u8p), self.r[3].size,
            _ptr(self.r[4], _lib.u8p), self.r[4].size, _ptr(self.roff, _lib.i32p), self.roff.size)
        hf = self.hf if self.hf is not None else np.zeros(0, np.uint8)
        hp = _lib.Haplotypes(_ptr(self.hb, _lib.u8p), self.hb.size, _ptr(hf, _lib.u8p),
                             hf.size if self.hf is not None else 0, _ptr(self.hoff, _lib.i32p), self.hoff.size)
        return rd, hp


def _validate_reads(reads: Sequence[Read]) -> None:
    for i, r in enumerate(reads):
        if len(r.bases) == 0:
            raise EmptyRead(i)
        n = len(r.bases)
        if any(len(x) != n for x in (r.quals, r.ins_gop, r.del_gop, r.gcp)):
            raise MismatchedReadArrays(i)


class _Hmm:
    _pd = False

    def __init__(self, config: Config | None = None):
        lib()  # fail loudly now if the library is missing
        self.config = config or Config()
        self._fallback = 0
        self.last_stats: _lib.Stats | None = None

    @property
    def precision(self) -> Precision:
        return self.config.precision

    @staticmethod
    def backend() -> str:
        return lib().fgkl_backend().decode()

    def fallback_pairs(self) -> int:
        """Pairs so far that lost precision (lib.rs:263-268)."""
        return self._fallback

    def _run(self, reads, bases, flags, out):
        expected = len(reads) * len(bases)
        if out is None:
            out = np.empty(expected, np.float64)
        elif out.size != expected:
            raise OutputLength(expected, out.size)
        if expected == 0:
            return out
        flat = _Flat(reads, bases, flags)
        rd, hp = flat.structs()
        stats = _lib.Stats()
        cfg = self.config._c()
        fn = lib().fgkl_pdhmm_compute_config if self._pd else lib().fgkl_pairhmm_compute_config
        buf = out if (out.flags.c_contiguous and out.dtype == np.float64) else np.empty(expected, np.float64)
        _check(fn(C.byref(rd), C.byref(hp), C.byref(cfg), _ptr(buf, _lib.f64p), expected, C.byref(stats)))
        if buf is not out:
            out[...] = buf.reshape(out.shape)
        self._fallback += stats.fallback_pairs
        self.last_stats = stats
        return out


class PairHmm(_Hmm):
    """A configured PairHMM (lib.rs:240-294)."""

    def compute_log10_likelihoods(self, reads: Sequence[Read], haplotypes: Sequence[bytes], out: np.ndarray | None = None) -> np.ndarray:
        """log10 likelihood of read r given haplotype h at ``out[r * len(haplotypes) + h]``."""
        _validate_reads(reads)
        for i, h in enumerate(haplotypes):
            if len(h) == 0:
                raise EmptyHaplotype(i)
        return self._run(reads, haplotypes, None, out)


class PdPairHmm(_Hmm):
    """A configured partially determined PairHMM (pd.rs:223-280)."""

    _pd = True

    def compute_log10_likelihoods(self, reads: Sequence[Read], haplotypes: Sequence[PdHaplotype],
                                  out: np.ndarray | None = None) -> np.ndarray:
        _validate_reads(reads)
        for i, h in enumerate(haplotypes):
            if len(h.bases) == 0:
                raise EmptyHaplotype(i)
            if len(h.flags) != len(h.bases):
                raise MismatchedHaplotypeArrays(i)
        return self._run(reads, [h.bases for h in haplotypes], [h.flags for h in haplotypes], out)


@dataclass
class SharedColumns:
    """Haplotype columns per read base with prefix sharing alone and with suffix sharing (plan.rs:106-113)."""

    prefix_only: int
    forward: int
    backward: int


@dataclass
class Plan:
    order: list[int]
    lcp: list[int]
    dup: list[bool]
    cuts: list[tuple[int, int] | None]  # (column, node)
    sweeps: list[tuple[int, int, int, int, list[tuple[int, int]]]]  # (hap, resume, need, start, writes)
    nodes: int
    columns: SharedColumns


def plan(haplotypes: Sequence[bytes], share_suffixes: bool = True) -> Plan:
    """The planner's view of a haplotype set: sort order, LCP, duplicates, cuts and sweeps."""
    n = len(haplotypes)
    hb = np.concatenate([_u8(h) for h in haplotypes]) if n else np.zeros(1, np.uint8)
    off = np.zeros(n + 1, np.int32)
    np.cumsum([len(h) for h in haplotypes], out=off[1:])
    order, lcp, cc, cn = (np.zeros(max(n, 1), np.int32) for _ in range(4))
    dup = np.zeros(max(n, 1), np.uint8)
    ns, nn = C.c_int32(), C.c_int32()
    cols = (C.c_uint64 * 3)()
    _check(lib().fgkl_plan_describe(_ptr(hb, _lib.u8p), _ptr(off, _lib.i32p), n, int(share_suffixes), _ptr(order, _lib.i32p),
                                    _ptr(lcp, _lib.i32p), _ptr(dup, _lib.u8p), _ptr(cc, _lib.i32p), _ptr(cn, _lib.i32p),
                                    C.byref(ns), C.byref(nn), cols))
    sweeps = []
    if share_suffixes and ns.value:
        sw = np.zeros(6 * ns.value, np.int32)
        wr = np.zeros(2 * 4096, np.int32)
        _check(lib().fgkl_plan_sweeps(_ptr(hb, _lib.u8p), _ptr(off, _lib.i32p), n, _ptr(sw, _lib.i32p), ns.value,
                                      _ptr(wr, _lib.i32p), 4096))
        for i in range(ns.value):
            h, resume, need, start, w0, wn = (int(x) for x in sw[6 * i: 6 * i + 6])
            writes = [(int(wr[2 * j]), int(wr[2 * j + 1])) for j in range(w0, w0 + wn)]
            sweeps.append((h, resume, need, start, writes))
    return Plan(
        order=[int(x) for x in order[:n]], lcp=[int(x) for x in lcp[:n]], dup=[bool(x) for x in dup[:n]],
        cuts=[(int(c), int(d)) if c >= 0 else None for c, d in zip(cc[:n], cn[:n])], sweeps=sweeps, nodes=nn.value,
        columns=SharedColumns(int(cols[0]), int(cols[1]), int(cols[2])))


# PD deletion states, pd_kernel.rs:31-33.
NORMAL, INSIDE_DEL, AFTER_DEL = 0, 1, 2


def pd_row_states(flags: bytes, start_state: int = NORMAL) -> tuple[list[int], int]:
    """Per-column deletion states of a row started in ``start_state``, and the state carried out of it
    (the run boundaries of pd_kernel.rs:699-723, column by column)."""
    f = _u8(flags) if len(flags) else np.zeros(1, np.uint8)
    out = np.zeros(max(len(flags), 1), np.uint8)
    end = lib().fgkl_pd_row_states(_ptr(f, _lib.u8p), len(flags), start_state, _ptr(out, _lib.u8p))
    if end < 0:
        _check(end)
    return [int(x) for x in out[:len(flags)]], int(end)


@dataclass
class PdPlan:
    order: list[int]
    lcp: list[int]
    dup: list[bool]
    end_state: list[int]
    num_codes: int


def pd_plan(haplotypes: Sequence[PdHaplotype]) -> PdPlan:
    """The PD sorter's view of a haplotype set (SortedPdHaps::new, pd_kernel.rs:61-136)."""
    n = len(haplotypes)
    hb = np.concatenate([_u8(h.bases) for h in haplotypes]) if n else np.zeros(1, np.uint8)
    hf = np.concatenate([_u8(h.flags) for h in haplotypes]) if n else np.zeros(1, np.uint8)
    off = np.zeros(n + 1, np.int32)
    np.cumsum([len(h.bases) for h in haplotypes], out=off[1:])
    order, lcp = (np.zeros(max(n, 1), np.int32) for _ in range(2))
    dup, end = (np.zeros(max(n, 1), np.uint8) for _ in range(2))
    codes = C.c_int32()
    _check(lib().fgkl_pd_plan_describe(_ptr(hb, _lib.u8p), _ptr(hf, _lib.u8p), _ptr(off, _lib.i32p), n, _ptr(order, _lib.i32p),
                                       _ptr(lcp, _lib.i32p), _ptr(dup, _lib.u8p), _ptr(end, _lib.u8p), C.byref(codes)))
    return PdPlan([int(x) for x in order[:n]], [int(x) for x in lcp[:n]], [bool(x) for x in dup[:n]],
                  [int(x) for x in end[:n]], codes.value)


def pd_match_accepts(base: int, flag: int, read_base: int) -> bool:
    """MatchSet::of(base, flag).accepts(read_base) (pd_kernel.rs:196-214)."""
    return bool(lib().fgkl_pd_match_accepts(base, flag, read_base))


def shared_columns(haplotypes: Sequence[bytes]) -> SharedColumns:
    """lib.rs:296-301."""
    return plan(haplotypes, True).columns


class BatchContext:
    """The batched form: many regions planned and uploaded once, run as persistent launches captured
    in a CUDA graph."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self._ctx = lib().fgkl_context_create(device, C.c_void_p(stream) if stream else None)
        if not self._ctx:
            raise DeviceError(_lib.FGKL_E_NO_DEVICE, _lib.last_error())
        self._keep = None

    def prepare(self, workload, config: Config | None = None) -> int:
        """Plans and uploads a workload (``synthetic.Workload`` or anything with its arrays)."""
        b = workload.as_batch()
        self._keep = (workload, b)
        cfg = (config or Config())._c()
        _check(lib().fgkl_batch_prepare(self._ctx, C.byref(b), C.byref(cfg)))
        return int(lib().fgkl_batch_output_len(self._ctx))

    def run(self) -> None:
        _check(lib().fgkl_batch_run(self._ctx))

    def fetch(self, out: np.ndarray | None = None) -> tuple[np.ndarray, _lib.Stats]:
        n = int(lib().fgkl_batch_output_len(self._ctx))
        if out is None:
            out = np.empty(n, np.float64)
        stats = _lib.Stats()
        _check(lib().fgkl_batch_fetch(self._ctx, _ptr(out, _lib.f64p), out.size, C.byref(stats)))
        return out, stats

    def autotune(self, workload, config: Config | None = None, repeats: int = 3) -> tuple[dict, list[dict]]:
        """Times the launch configurations on ``workload`` (or a sample of the caller's work), keeps the
        fastest for this context's later batches and leaves ``workload`` prepared with it. Returns the
        chosen configuration and every candidate, each ``{"streams", "grid_percent", "reads_per_warp",
        "rows_extra", "warps_per_block", "ms"}``."""
        b = workload.as_batch()
        self._keep = (workload, b)
        cfg = (config or Config())._c()
        chosen = _lib.Tuning()
        tried = (_lib.Tuning * 32)()
        n = C.c_int32()
        _check(lib().fgkl_context_autotune(self._ctx, C.byref(b), C.byref(cfg), int(repeats), C.byref(chosen), tried, 32,
                                           C.byref(n)))
        as_dict = lambda t: {"streams": int(t.streams), "grid_percent": int(t.grid_percent),
                             "reads_per_warp": int(t.reads_per_warp), "rows_extra": int(t.rows_extra),
                             "warps_per_block": int(t.warps_per_block), "ms": float(t.ms)}
        return as_dict(chosen), [as_dict(tried[i]) for i in range(min(n.value, 32))]

    def set_tuning(self, streams: int, grid_percent: int, reads_per_warp: int = 2, rows_extra: int = 0,
                   warps_per_block: int = 4) -> None:
        """Launch configuration for the next prepare (fgkl_tuning); no value changes a result bit."""
        _check(lib().fgkl_context_set_tuning(
            self._ctx, C.byref(_lib.Tuning(streams, grid_percent, reads_per_warp, rows_extra, warps_per_block, 0.0))))

    def tuning(self) -> dict:
        t = _lib.Tuning()
        _check(lib().fgkl_context_get_tuning(self._ctx, C.byref(t)))
        return {"streams": int(t.streams), "grid_percent": int(t.grid_percent), "reads_per_warp": int(t.reads_per_warp),
                "rows_extra": int(t.rows_extra), "warps_per_block": int(t.warps_per_block)}

    def set_profiling(self, on: bool) -> None:
        """Direct launches timed with CUDA events (no graph); see ``launch_profile``."""
        _check(lib().fgkl_context_profile(self._ctx, int(on)))

    def launch_profile(self) -> list[dict]:
        """Per launch of the last profiled run: kind, rows, tasks, blocks, recomputation, cells, ms."""
        arr = (_lib.LaunchProfile * 256)()
        n = C.c_int32()
        _check(lib().fgkl_batch_launch_profile(self._ctx, arr, 256, C.byref(n)))
        return [{f: getattr(arr[i], f) for f, _ in _lib.LaunchProfile._fields_} for i in range(min(n.value, 256))]

    def compute(self, workload, config: Config | None = None) -> tuple[np.ndarray, _lib.Stats]:
        self.prepare(workload, config)
        self.run()
        return self.fetch()

    def close(self) -> None:
        if self._ctx:
            lib().fgkl_context_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        # At interpreter shutdown the context is left to the process's exit: destroying it then
        # would run CUDA calls while the runtimes in the process are being torn down.
        if sys.is_finalizing():
            return
        try:
            self.close()
        except Exception:
            pass
