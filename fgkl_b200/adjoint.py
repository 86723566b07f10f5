"""Gradients of the summed log10 likelihood for fitting the indel and base-error model (the
``fgkl_adjoint_*`` entry points of ``include/fgkl_b200.h``; no counterpart in fgkl).

Parameters are per read position and continuous: insertion and deletion gap-open probabilities
(fgkl's MI, MD), gap continuation (II = DD, IM = 1 - it) and base error (priors 1 - e and e / 3),
with MM = 1 - dI - dD.
"""
from __future__ import annotations

import ctypes as C
import sys
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import lib
from .pairhmm import DeviceError, _check, _ptr


@dataclass
class AdjointParams:
    """Per read position, concatenated like the read bases."""

    gap_open_ins: np.ndarray
    gap_open_del: np.ndarray
    gap_continuation: np.ndarray
    base_error: np.ndarray


@dataclass
class AdjointResult:
    log10: np.ndarray           # per pair, row-major per region (reads x haplotypes)
    gap_open_ins: np.ndarray    # d(Σ log10 L)/d(parameter) per read position
    gap_open_del: np.ndarray
    gap_continuation: np.ndarray
    base_error: np.ndarray
    fp64_reads: int             # reads recomputed in FP64


def phred_to_prob(q: np.ndarray) -> np.ndarray:
    """10^(-q/10), the error probability of a Phred quality (fgkl model.rs:37-41)."""
    return np.power(10.0, -np.asarray(q, np.float64) / 10.0)


def params_from_quals(workload) -> AdjointParams:
    """The continuous parameters a read's Phred-scaled penalties stand for."""
    return AdjointParams(phred_to_prob(workload.ins_gop), phred_to_prob(workload.del_gop), phred_to_prob(workload.gcp),
                         phred_to_prob(workload.quals))


class AdjointContext:
    """Device context of the adjoint path (prepare / run / fetch, or compute)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self._ctx = lib().fgkl_context_create(device, C.c_void_p(stream) if stream else None)
        if not self._ctx:
            raise DeviceError(_lib.FGKL_E_NO_DEVICE, _lib.last_error())
        self._keep = None

    def prepare(self, workload, params: AdjointParams, double_precision: bool = False) -> None:
        arrays = [np.ascontiguousarray(a, np.float64) for a in
                  (params.gap_open_ins, params.gap_open_del, params.gap_continuation, params.base_error)]
        for a in arrays:
            if a.size != workload.bases.size:
                raise ValueError("parameters must hold one value per read position")
        b = _lib.AdjointBatch(workload.num_regions, workload.region_reads.ctypes.data_as(_lib.i32p),
                              workload.region_haps.ctypes.data_as(_lib.i32p), workload.bases.ctypes.data_as(_lib.u8p),
                              workload.read_offsets.ctypes.data_as(_lib.i64p), *[_ptr(a, _lib.f64p) for a in arrays],
                              workload.hap_bases.ctypes.data_as(_lib.u8p), workload.hap_offsets.ctypes.data_as(_lib.i64p))
        self._keep = (workload, arrays, b)
        _check(lib().fgkl_adjoint_prepare(self._ctx, C.byref(b), int(double_precision)))

    def run(self) -> int:
        n = C.c_uint64()
        _check(lib().fgkl_adjoint_run(self._ctx, C.byref(n)))
        return int(n.value)

    def fetch(self) -> AdjointResult:
        n_out = int(lib().fgkl_adjoint_output_len(self._ctx))
        n_g = int(lib().fgkl_adjoint_grad_len(self._ctx))
        out = np.empty(n_out, np.float64)
        g = [np.empty(n_g, np.float64) for _ in range(4)]
        lost = C.c_uint64()
        _check(lib().fgkl_adjoint_fetch(self._ctx, _ptr(out, _lib.f64p), n_out, *[_ptr(x, _lib.f64p) for x in g], n_g,
                                        C.byref(lost)))
        return AdjointResult(out, *g, int(lost.value))

    def compute(self, workload, params: AdjointParams, double_precision: bool = False) -> AdjointResult:
        self.prepare(workload, params, double_precision)
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
