"""ctypes binding of the CPU oracle (``oracle/liboracle.so``) -- TEST INFRASTRUCTURE ONLY.

Only the tests, the smoke check and the CPU-baseline leg of the benchmark use this module, and only
as the checker (or the timed CPU reference). The product never imports it.

The oracle restates fgkl's scalar FP64 reference (crates/pairhmm/src/model.rs:37-106,
reference.rs:20-64, pd_reference.rs:29-118) in C; see pairhmm_oracle.c.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

_u8p = C.POINTER(C.c_uint8)
_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        sources = ("pairhmm_oracle.c", "sw_oracle.c", "fgkl_cpu.c", "fgkl_cpu_kernel.h", "fgkl_cpu_pd_kernel.h", "Makefile", "synth_shim.cpp",
                   "../fgkl_b200/csrc/synthetic.cpp", "../fgkl_b200/csrc/synthetic.h", "../fgkl_b200/csrc/tables.cpp")
        if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < max((HERE / f).stat().st_mtime for f in sources):
            build()
        L = C.CDLL(str(LIB_PATH))
        L.or_error_prob.restype = C.c_double
        L.or_error_prob.argtypes = [C.c_int]
        L.or_match_to_match.restype = C.c_double
        L.or_match_to_match.argtypes = [C.c_int, C.c_int]
        L.or_transitions.argtypes = [C.c_int, C.c_int, C.c_int, _f64p]
        L.or_priors.argtypes = [C.c_int, _f64p]
        L.or_initial_condition.restype = C.c_double
        L.or_approximate_log10_sum_log10.restype = C.c_double
        L.or_approximate_log10_sum_log10.argtypes = [C.c_double, C.c_double]
        L.or_base_matches_pd.restype = C.c_int
        L.or_base_matches_pd.argtypes = [C.c_uint8, C.c_uint8]
        L.or_log10_likelihood.restype = C.c_double
        L.or_log10_likelihood.argtypes = [_u8p, C.c_int, _u8p, _u8p, _u8p, _u8p, _u8p, C.c_int]
        L.or_pd_log10_likelihood.restype = C.c_double
        L.or_pd_log10_likelihood.argtypes = [_u8p, _u8p, C.c_int, _u8p, _u8p, _u8p, _u8p, _u8p, C.c_int]
        L.or_compute_matrix.argtypes = [_u8p, _u8p, _u8p, _u8p, _u8p, _i32p, C.c_int, _u8p, _u8p, _i32p, C.c_int, _f64p, C.c_int]
        L.or_adj_log10_likelihood.restype = C.c_double
        L.or_adj_log10_likelihood.argtypes = [_u8p, C.c_int, _u8p, C.c_int, _f64p, _f64p, _f64p, _f64p]
        L.or_adj_gradient.restype = C.c_double
        L.or_adj_gradient.argtypes = [_u8p, C.c_int, _u8p, C.c_int, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p]
        _i64p = C.POINTER(C.c_int64)
        L.fc_detect_isa.restype = C.c_int
        L.fc_compute_regions.restype = C.c_int64
        L.fc_compute_regions.argtypes = [_u8p] * 5 + [_i64p, _u8p, _i64p, _i64p, _i32p, _i64p, _i32p, _i64p, C.c_int,
                                                      C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f64p]
        L.fc_compute_regions_flags.restype = C.c_int64
        L.fc_compute_regions_flags.argtypes = [_u8p] * 5 + [_i64p, _u8p, _u8p, _i64p, _i64p, _i32p, _i64p, _i32p, _i64p,
                                                            C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f64p]
        L.or_sw_align.restype = C.c_int
        L.or_sw_align.argtypes = [_u8p, C.c_int, _u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _u8p,
                                  C.POINTER(C.c_uint32), C.c_int, C.POINTER(C.c_int32)]
        L.or_synth_config.restype = C.c_void_p
        L.or_synth_config.argtypes = [C.c_int32, C.c_uint64, C.c_int32, C.c_int32]
        L.or_synth_arrays.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), _i64p]
        L.or_synth_free.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def synth_workload(which: int, seed: int = 0, regions: int = 0, threads: int = 8):
    """The benchmark workload `which` (the generators of fgkl_b200/csrc/synthetic.cpp, built into
    this library), as a ``fgkl_b200.synthetic.Workload``, without loading the CUDA library."""
    from fgkl_b200.synthetic import Workload

    L = lib()
    h = L.or_synth_config(which, seed, regions, threads)
    if not h:
        raise ValueError(f"no synthetic workload {which}")
    try:
        ptrs = (C.c_void_p * 11)()
        sizes = (C.c_int64 * 5)()
        L.or_synth_arrays(h, ptrs, sizes)
        n, nr, nrb, nh, nhb = (int(x) for x in sizes)

        def arr(i, count, dtype):
            if count == 0 or not ptrs[i]:
                return np.zeros(0, dtype)
            return np.ctypeslib.as_array(C.cast(ptrs[i], C.POINTER(np.ctypeslib.as_ctypes_type(dtype))), shape=(count,)).copy()

        return Workload(region_reads=arr(0, n, np.int32), region_haps=arr(1, n, np.int32), bases=arr(2, nrb, np.uint8),
                        quals=arr(3, nrb, np.uint8), ins_gop=arr(4, nrb, np.uint8), del_gop=arr(5, nrb, np.uint8),
                        gcp=arr(6, nrb, np.uint8), read_offsets=arr(7, nr + 1, np.int64), hap_bases=arr(8, nhb, np.uint8),
                        hap_flags=arr(9, nhb, np.uint8) if ptrs[9] else None, hap_offsets=arr(10, nh + 1, np.int64))
    finally:
        L.or_synth_free(h)


def _u8(b) -> np.ndarray:
    return np.ascontiguousarray(np.frombuffer(bytes(b), np.uint8) if not isinstance(b, np.ndarray) else b, dtype=np.uint8)


def _p(a, t):
    return a.ctypes.data_as(t)


def error_prob(q: int) -> float:
    return lib().or_error_prob(q)


def match_to_match(a: int, b: int) -> float:
    return lib().or_match_to_match(a, b)


def transitions(ins: int, dele: int, gcp: int) -> list[float]:
    t = (C.c_double * 6)()
    lib().or_transitions(ins, dele, gcp, t)
    return list(t)


def priors(q: int) -> tuple[float, float]:
    t = (C.c_double * 2)()
    lib().or_priors(q, t)
    return t[0], t[1]


def initial_condition() -> float:
    return lib().or_initial_condition()


def approximate_log10_sum_log10(a: float, b: float) -> float:
    return lib().or_approximate_log10_sum_log10(a, b)


def base_matches_pd(read_base: int, flags: int) -> bool:
    return bool(lib().or_base_matches_pd(read_base, flags))


def log10_likelihood(hap: bytes, read) -> float:
    """reference::log10_likelihood (reference.rs:20-64)."""
    h = _u8(hap)
    a = [_u8(getattr(read, f)) for f in ("bases", "quals", "ins_gop", "del_gop", "gcp")]
    return lib().or_log10_likelihood(_p(h, _u8p), h.size, *[_p(x, _u8p) for x in a], a[0].size)


def pd_log10_likelihood(bases: bytes, flags: bytes, read) -> float:
    """pd_reference::log10_likelihood (pd_reference.rs:29-118)."""
    h, f = _u8(bases), _u8(flags)
    a = [_u8(getattr(read, x)) for x in ("bases", "quals", "ins_gop", "del_gop", "gcp")]
    return lib().or_pd_log10_likelihood(_p(h, _u8p), _p(f, _u8p), h.size, *[_p(x, _u8p) for x in a], a[0].size)


def compute_matrix(reads, haps, threads: int | None = None) -> np.ndarray:
    """Every read against every haplotype, ``out[r * len(haps) + h]``; PD when haps carry flags."""
    threads = threads or os.cpu_count() or 1
    cols = [np.concatenate([_u8(getattr(r, f)) for r in reads]) for f in ("bases", "quals", "ins_gop", "del_gop", "gcp")]
    roff = np.zeros(len(reads) + 1, np.int32)
    np.cumsum([len(r.bases) for r in reads], out=roff[1:])
    pd = len(haps) > 0 and hasattr(haps[0], "flags")
    hb = np.concatenate([_u8(h.bases if pd else h) for h in haps])
    hf = np.concatenate([_u8(h.flags) for h in haps]) if pd else None
    hoff = np.zeros(len(haps) + 1, np.int32)
    np.cumsum([len(h.bases if pd else h) for h in haps], out=hoff[1:])
    out = np.empty(len(reads) * len(haps), np.float64)
    lib().or_compute_matrix(*[_p(c, _u8p) for c in cols], _p(roff, _i32p), len(reads), _p(hb, _u8p),
                            _p(hf, _u8p) if hf is not None else None, _p(hoff, _i32p), len(haps), _p(out, _f64p), threads)
    return out


def workload_matrix(workload, regions=None, threads: int | None = None) -> np.ndarray:
    """Oracle results of a synthetic workload's regions, concatenated in output order."""
    parts = []
    for g in (regions if regions is not None else range(workload.num_regions)):
        reads, haps = workload.region(g)
        parts.append(compute_matrix(reads, haps, threads) if reads and haps else np.zeros(0))
    return np.concatenate(parts) if parts else np.zeros(0)


ISA_NAMES = {0: "portable vectors (8 FP32 / 4 FP64 lanes)", 1: "AVX2 (8 FP32 / 4 FP64 lanes)",
             2: "AVX-512 (16 FP32 / 8 FP64 lanes; AVX2 for a remainder of at most half a batch)"}


def cpu_isa() -> int:
    """The instruction set fgkl_cpu.c selects on this CPU: 2 AVX-512F, 1 AVX2, 0 portable vectors."""
    return int(lib().fc_detect_isa())


def fgkl_cpu_workload(workload, regions=None, threads: int | None = None, double: bool = False,
                      share_suffixes: bool = True, double_fallback: bool = True, isa: int = -1):
    """fgkl's batched CPU algorithm (fgkl_cpu.c) over a synthetic workload's regions: the PD-HMM
    kernel when the workload carries haplotype flags, else the plain one.

    Returns (results concatenated in output order, pairs that lost precision in the first pass)."""
    threads = threads or os.cpu_count() or 1
    regions = list(range(workload.num_regions)) if regions is None else list(regions)
    nr = workload.region_reads.astype(np.int64)
    nh = workload.region_haps.astype(np.int64)
    read_start = np.concatenate([[0], np.cumsum(nr)[:-1]]).astype(np.int64)
    hap_start = np.concatenate([[0], np.cumsum(nh)[:-1]]).astype(np.int64)
    sel = np.asarray(regions, np.int64)
    read_first = np.ascontiguousarray(read_start[sel])
    hap_first = np.ascontiguousarray(hap_start[sel])
    n_reads = np.ascontiguousarray(nr[sel].astype(np.int32))
    n_haps = np.ascontiguousarray(nh[sel].astype(np.int32))
    sizes = nr[sel] * nh[sel]
    out_first = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64) if sel.size else np.zeros(0, np.int64)
    out = np.empty(int(sizes.sum()), np.float64)
    i64 = C.POINTER(C.c_int64)
    cols = [np.ascontiguousarray(getattr(workload, f), np.uint8) for f in ("bases", "quals", "ins_gop", "del_gop", "gcp")]
    ro = np.ascontiguousarray(workload.read_offsets, np.int64)
    hb = np.ascontiguousarray(workload.hap_bases, np.uint8)
    ho = np.ascontiguousarray(workload.hap_offsets, np.int64)
    hf = np.ascontiguousarray(workload.hap_flags, np.uint8) if workload.hap_flags is not None else None
    lost = lib().fc_compute_regions_flags(*[_p(c, _u8p) for c in cols], _p(ro, i64), _p(hb, _u8p),
                                          _p(hf, _u8p) if hf is not None else None, _p(ho, i64),
                                          _p(read_first, i64), _p(n_reads, _i32p), _p(hap_first, i64), _p(n_haps, _i32p),
                                          _p(out_first, i64), int(sel.size), int(double), int(share_suffixes),
                                          int(double_fallback), int(threads), int(isa), _p(out, _f64p))
    if lost == -2:
        raise ValueError("a PD region holds more than 256 distinct match sets")
    if lost < 0:
        raise ValueError("fc_compute_regions rejected its arguments")
    return out, int(lost)


def adj_log10_likelihood(hap: bytes, read_bases: bytes, d_ins, d_del, eps, err) -> float:
    """log10 L under the continuous parameterisation (dI, dD, eps, e per read position)."""
    h, b = _u8(hap), _u8(read_bases)
    arrs = [np.ascontiguousarray(x, np.float64) for x in (d_ins, d_del, eps, err)]
    return lib().or_adj_log10_likelihood(_p(h, _u8p), h.size, _p(b, _u8p), b.size, *[_p(a, _f64p) for a in arrs])


def adj_gradient(hap: bytes, read_bases: bytes, d_ins, d_del, eps, err):
    """(log10 L, d/d dI, d/d dD, d/d eps, d/d e) per read position, FP64 forward-backward."""
    h, b = _u8(hap), _u8(read_bases)
    arrs = [np.ascontiguousarray(x, np.float64) for x in (d_ins, d_del, eps, err)]
    g = [np.zeros(b.size, np.float64) for _ in range(4)]
    ll = lib().or_adj_gradient(_p(h, _u8p), h.size, _p(b, _u8p), b.size, *[_p(a, _f64p) for a in arrs],
                               *[_p(x, _f64p) for x in g])
    return (ll, *g)


def sw_align(reference: bytes, alternate: bytes, params, strategy: int) -> tuple[str, int]:
    """Smith-Waterman as GATK's SmithWatermanJavaAligner (sw_oracle.c): (CIGAR string, offset).
    `params` = (match, mismatch, gap open, gap extend); strategy 0 SoftClip, 1 Indel, 2 LeadingIndel,
    3 Ignore."""
    if not reference or not alternate:
        raise ValueError("empty sequence")
    r, a = _u8(reference), _u8(alternate)
    cap = len(reference) + len(alternate) + 4
    ops = np.zeros(cap, np.uint8)
    lens = np.zeros(cap, np.uint32)
    off = C.c_int32()
    k = lib().or_sw_align(_p(r, _u8p), r.size, _p(a, _u8p), a.size, *[int(x) for x in params], int(strategy),
                          _p(ops, _u8p), lens.ctypes.data_as(C.POINTER(C.c_uint32)), cap, C.byref(off))
    if k < 0 or k > cap:
        raise ValueError("alignment failed")
    return "".join(f"{int(lens[e])}{chr(ops[e])}" for e in range(k)), int(off.value)
