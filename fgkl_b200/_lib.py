"""ctypes binding of ``libfgkl_b200.so`` (the C ABI of ``include/fgkl_b200.h``).

The library is the only compute path: there is no CPU fallback. If it cannot be loaded, importing
the compute API raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libfgkl_b200.so"

FGKL_OK = 0
FGKL_E_EMPTY_READ = -1
FGKL_E_MISMATCHED_READ_ARRAYS = -2
FGKL_E_EMPTY_HAPLOTYPE = -3
FGKL_E_MISMATCHED_HAPLOTYPE_ARRAYS = -4
FGKL_E_OUTPUT_LENGTH = -5
FGKL_E_BAD_OFFSETS = -6
FGKL_E_INVALID_ARGUMENT = -7
FGKL_E_UNSUPPORTED = -8
FGKL_E_NO_DEVICE = -9
FGKL_E_CUDA = -10
FGKL_E_OUT_OF_MEMORY = -11
FGKL_E_EMPTY_SEQUENCE = -12

u8p = C.POINTER(C.c_uint8)
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
f64p = C.POINTER(C.c_double)


class Config(C.Structure):
    _fields_ = [("double_precision", C.c_int32), ("double_fallback", C.c_int32), ("share_suffixes", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [
        ("fallback_pairs", C.c_uint64),
        ("rescue_reads", C.c_uint64),
        ("nominal_cells", C.c_uint64),
        ("computed_cells", C.c_uint64),
        ("forward_cells", C.c_uint64),
        ("backward_cells", C.c_uint64),
        ("prefix_only_cells", C.c_uint64),
        ("kernel_launches", C.c_uint64),
        ("host_plan_ms", C.c_double),
        ("host_pack_ms", C.c_double),
        ("host_upload_ms", C.c_double),
        ("host_fetch_ms", C.c_double),
    ]


class Reads(C.Structure):
    _fields_ = [
        ("bases", u8p), ("bases_len", C.c_int64),
        ("quals", u8p), ("quals_len", C.c_int64),
        ("ins_gop", u8p), ("ins_gop_len", C.c_int64),
        ("del_gop", u8p), ("del_gop_len", C.c_int64),
        ("gcp", u8p), ("gcp_len", C.c_int64),
        ("offsets", i32p), ("offsets_len", C.c_int64),
    ]


class Haplotypes(C.Structure):
    _fields_ = [
        ("bases", u8p), ("bases_len", C.c_int64),
        ("flags", u8p), ("flags_len", C.c_int64),
        ("offsets", i32p), ("offsets_len", C.c_int64),
    ]


class Batch(C.Structure):
    _fields_ = [
        ("num_regions", C.c_int32),
        ("region_reads", i32p),
        ("region_haps", i32p),
        ("bases", u8p),
        ("quals", u8p),
        ("ins_gop", u8p),
        ("del_gop", u8p),
        ("gcp", u8p),
        ("read_offsets", i64p),
        ("hap_bases", u8p),
        ("hap_flags", u8p),
        ("hap_offsets", i64p),
    ]


class SwParams(C.Structure):
    _fields_ = [("match_value", C.c_int32), ("mismatch_penalty", C.c_int32), ("gap_open_penalty", C.c_int32),
                ("gap_extend_penalty", C.c_int32)]


class SwBatch(C.Structure):
    _fields_ = [("num_pairs", C.c_int64), ("ref_bases", C.POINTER(C.c_uint8)), ("ref_offsets", C.POINTER(C.c_int64)),
                ("alt_bases", C.POINTER(C.c_uint8)), ("alt_offsets", C.POINTER(C.c_int64))]


class Tuning(C.Structure):
    _fields_ = [("streams", C.c_int32), ("grid_percent", C.c_int32), ("reads_per_warp", C.c_int32), ("rows_extra", C.c_int32),
                ("warps_per_block", C.c_int32), ("ms", C.c_double)]


class LaunchProfile(C.Structure):
    _fields_ = [("kind", C.c_int32), ("rows", C.c_int32), ("tasks", C.c_int32), ("blocks", C.c_int32),
                ("recomputation", C.c_int32), ("forward_cells", C.c_uint64), ("backward_cells", C.c_uint64), ("ms", C.c_float)]


class AdjointBatch(C.Structure):
    """``fgkl_adjoint_batch``."""
    _fields_ = [
        ("num_regions", C.c_int32),
        ("region_reads", i32p),
        ("region_haps", i32p),
        ("bases", u8p),
        ("read_offsets", i64p),
        ("gap_open_ins", f64p),
        ("gap_open_del", f64p),
        ("gap_continuation", f64p),
        ("base_error", f64p),
        ("hap_bases", u8p),
        ("hap_offsets", i64p),
    ]


class DeviceRegion(C.Structure):
    """``fgkl_device_region``: caller-owned device arrays of one region (allocation-free entry)."""
    _fields_ = [
        ("num_reads", C.c_int32),
        ("num_haplotypes", C.c_int32),
        ("bases", C.c_void_p),
        ("quals", C.c_void_p),
        ("ins_quals", C.c_void_p),
        ("del_quals", C.c_void_p),
        ("gcp", C.c_void_p),
        ("read_offsets", C.c_void_p),
        ("hap_bases", C.c_void_p),
        ("hap_offsets", C.c_void_p),
        ("max_read_len", C.c_int32),
    ]


NOALLOC_SCRATCH_BYTES = 2 * 1024 * 1024
NOALLOC_MAX_READ_LEN = 620


_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """The loaded library; raises OSError when it is missing (run ``__graft_entry__.build()``)."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.environ.get("FGKL_B200_LIB", str(LIB_PATH))
    if not Path(path).exists():
        raise OSError(f"{path} is missing; build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    L = C.CDLL(path)
    L.fgkl_pairhmm_compute.argtypes = [C.POINTER(Reads), C.POINTER(Haplotypes), C.c_int32, f64p, C.c_int64]
    L.fgkl_pairhmm_compute_config.argtypes = [C.POINTER(Reads), C.POINTER(Haplotypes), C.POINTER(Config), f64p, C.c_int64,
                                              C.POINTER(Stats)]
    L.fgkl_pdhmm_compute.argtypes = L.fgkl_pairhmm_compute.argtypes
    L.fgkl_pdhmm_compute_config.argtypes = L.fgkl_pairhmm_compute_config.argtypes
    for f in (L.fgkl_pairhmm_compute, L.fgkl_pairhmm_compute_config, L.fgkl_pdhmm_compute, L.fgkl_pdhmm_compute_config):
        f.restype = C.c_int
    L.fgkl_set_call_combining.argtypes = [C.c_int32]
    L.fgkl_set_call_combining.restype = C.c_int
    L.fgkl_call_combining_stats.argtypes = [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.fgkl_call_combining_stats.restype = C.c_int
    L.fgkl_plan_region_cells.argtypes = [C.POINTER(Batch), C.POINTER(Config), C.POINTER(C.c_uint64)]
    L.fgkl_plan_region_cells.restype = C.c_int
    L.fgkl_sw_align.argtypes = [C.POINTER(C.c_uint8), C.c_int64, C.POINTER(C.c_uint8), C.c_int64, C.POINTER(SwParams), C.c_int32,
                                C.c_char_p, C.c_int64, C.POINTER(C.c_int32)]
    L.fgkl_sw_align.restype = C.c_int
    L.fgkl_sw_cigar_capacity.argtypes = [C.POINTER(SwBatch)]
    L.fgkl_sw_cigar_capacity.restype = C.c_int64
    L.fgkl_sw_align_batch.argtypes = [C.c_void_p, C.POINTER(SwBatch), C.POINTER(SwParams), C.c_int32, C.POINTER(C.c_uint32),
                                      C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.fgkl_sw_align_batch.restype = C.c_int
    L.fgkl_sw_last_kernel_ms.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
    L.fgkl_sw_last_kernel_ms.restype = C.c_int
    L.fgkl_set_allocation_limit.argtypes = [C.c_int64]
    L.fgkl_set_allocation_limit.restype = C.c_int64
    L.fgkl_backend.restype = C.c_char_p
    L.fgkl_last_error.restype = C.c_char_p
    L.fgkl_context_create.argtypes = [C.c_int32, C.c_void_p]
    L.fgkl_context_create.restype = C.c_void_p
    L.fgkl_context_destroy.argtypes = [C.c_void_p]
    L.fgkl_batch_prepare.argtypes = [C.c_void_p, C.POINTER(Batch), C.POINTER(Config)]
    L.fgkl_batch_run.argtypes = [C.c_void_p]
    L.fgkl_batch_fetch.argtypes = [C.c_void_p, f64p, C.c_int64, C.POINTER(Stats)]
    L.fgkl_batch_compute.argtypes = [C.c_void_p, C.POINTER(Batch), C.POINTER(Config), f64p, C.c_int64, C.POINTER(Stats)]
    L.fgkl_batch_output_len.argtypes = [C.c_void_p]
    L.fgkl_batch_output_len.restype = C.c_int64
    L.fgkl_context_autotune.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(Tuning),
                                        C.POINTER(Tuning), C.c_int32, C.POINTER(C.c_int32)]
    L.fgkl_context_autotune.restype = C.c_int
    L.fgkl_context_set_tuning.argtypes = [C.c_void_p, C.POINTER(Tuning)]
    L.fgkl_context_set_tuning.restype = C.c_int
    L.fgkl_context_get_tuning.argtypes = [C.c_void_p, C.POINTER(Tuning)]
    L.fgkl_context_get_tuning.restype = C.c_int
    L.fgkl_synth_config.argtypes = [C.c_int32, C.c_uint64, C.c_int32, C.c_int32]
    L.fgkl_synth_config.restype = C.c_void_p
    L.fgkl_synth_reference_region.argtypes = [C.c_uint64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int32]
    L.fgkl_synth_reference_region.restype = C.c_void_p
    L.fgkl_synth_view.argtypes = [C.c_void_p, C.POINTER(Batch), i64p]
    L.fgkl_synth_free.argtypes = [C.c_void_p]
    L.fgkl_plan_describe.argtypes = [u8p, i32p, C.c_int32, C.c_int32, i32p, i32p, u8p, i32p, i32p, i32p, i32p,
                                     C.POINTER(C.c_uint64)]
    L.fgkl_plan_sweeps.argtypes = [u8p, i32p, C.c_int32, i32p, C.c_int32, i32p, C.c_int32]
    L.fgkl_probe_fp32_tflops.argtypes = [C.c_int32, f64p, f64p, f64p]
    L.fgkl_probe_int32_alu_gops.argtypes = [C.c_int32, f64p]
    L.fgkl_context_profile.argtypes = [C.c_void_p, C.c_int32]
    L.fgkl_batch_launch_profile.argtypes = [C.c_void_p, C.POINTER(LaunchProfile), C.c_int32, C.POINTER(C.c_int32)]
    L.fgkl_adjoint_prepare.argtypes = [C.c_void_p, C.POINTER(AdjointBatch), C.c_int32]
    L.fgkl_adjoint_run.argtypes = [C.c_void_p, C.POINTER(C.c_uint64)]
    L.fgkl_adjoint_fetch.argtypes = [C.c_void_p, f64p, C.c_int64, f64p, f64p, f64p, f64p, C.c_int64, C.POINTER(C.c_uint64)]
    L.fgkl_adjoint_compute.argtypes = [C.c_void_p, C.POINTER(AdjointBatch), C.c_int32, f64p, C.c_int64, f64p, f64p, f64p, f64p,
                                       C.c_int64, C.POINTER(C.c_uint64)]
    L.fgkl_adjoint_output_len.argtypes = [C.c_void_p]
    L.fgkl_adjoint_output_len.restype = C.c_int64
    L.fgkl_adjoint_grad_len.argtypes = [C.c_void_p]
    L.fgkl_adjoint_grad_len.restype = C.c_int64
    L.fgkl_pd_row_states.argtypes = [u8p, C.c_int32, C.c_int32, u8p]
    L.fgkl_pd_plan_describe.argtypes = [u8p, u8p, i32p, C.c_int32, i32p, i32p, u8p, u8p, i32p]
    L.fgkl_pd_match_accepts.argtypes = [C.c_uint8, C.c_uint8, C.c_uint8]
    L.fgkl_pairhmm_compute_device_noalloc.argtypes = [C.POINTER(DeviceRegion), C.c_void_p, C.c_void_p]
    L.fgkl_pairhmm_compute_device_noalloc.restype = C.c_int
    _lib = L
    return L


def last_error() -> str:
    return lib().fgkl_last_error().decode()


# Symbols include/fgkl_b200.h declares; the CPU test suite checks the library exports each one.
EXPORTED = [
    "fgkl_pairhmm_compute", "fgkl_pairhmm_compute_config", "fgkl_pdhmm_compute", "fgkl_pdhmm_compute_config",
    "fgkl_set_call_combining", "fgkl_call_combining_stats", "fgkl_set_allocation_limit", "fgkl_backend", "fgkl_last_error", "fgkl_context_create", "fgkl_context_destroy", "fgkl_batch_prepare",
    "fgkl_batch_run", "fgkl_batch_fetch", "fgkl_batch_compute", "fgkl_batch_output_len", "fgkl_context_autotune",
    "fgkl_context_set_tuning", "fgkl_context_get_tuning", "fgkl_synth_config",
    "fgkl_synth_reference_region", "fgkl_synth_view", "fgkl_synth_free", "fgkl_plan_describe", "fgkl_plan_region_cells", "fgkl_plan_sweeps", "fgkl_probe_fp32_tflops",
    "fgkl_pairhmm_compute_device_noalloc", "fgkl_context_profile", "fgkl_batch_launch_profile", "fgkl_adjoint_prepare", "fgkl_adjoint_run", "fgkl_adjoint_fetch",
    "fgkl_adjoint_compute", "fgkl_adjoint_output_len", "fgkl_adjoint_grad_len", "fgkl_pd_row_states", "fgkl_pd_plan_describe", "fgkl_pd_match_accepts",
    "fgkl_sw_align", "fgkl_sw_cigar_capacity", "fgkl_sw_align_batch", "fgkl_sw_last_kernel_ms", "fgkl_probe_int32_alu_gops",
]
