"""The allocation-free entry point (fgkl_pairhmm_compute_device_noalloc) against the regular one.

The entry has no counterpart in the reference. It computes every pair in FP64 without sharing from
caller-owned device arrays, with its scratch in a file-scope device array, so its results must agree
with fgkl_pairhmm_compute_config in double precision (the reference's 1e-9 log10 tolerance for
Precision::Double, crates/pairhmm/src/lib.rs:583-640). Two calls in a row check that the scratch
(pair counter zeroed by each call) is reusable. Device buffers here belong to the test; the entry
itself allocates nothing.
"""
import ctypes as C

import numpy as np
import pytest

from fgkl_b200 import Config, PairHmm, Precision, Read, _lib, synthetic
from oracle import oracle as O
from refgen import Rng

pytestmark = pytest.mark.gpu

TOL = 1e-9  # log10 units, the reference's double-precision tolerance

DOUBLE = Config(precision=Precision.DOUBLE)


def to_device(arrays):
    import torch

    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrays]


def device_region(reads, haps, max_read_len=None):
    import torch

    cat = lambda xs: np.frombuffer(b"".join(xs), dtype=np.uint8).copy() if xs else np.zeros(0, np.uint8)
    roff = np.zeros(len(reads) + 1, np.int64)
    np.cumsum([len(r.bases) for r in reads], out=roff[1:])
    hoff = np.zeros(len(haps) + 1, np.int64)
    np.cumsum([len(h) for h in haps], out=hoff[1:])
    host = [cat([r.bases for r in reads]), cat([r.quals for r in reads]), cat([r.ins_gop for r in reads]),
            cat([r.del_gop for r in reads]), cat([r.gcp for r in reads]), roff, cat(list(haps)), hoff]
    dev = to_device(host)
    reg = _lib.DeviceRegion(len(reads), len(haps), *[t.data_ptr() for t in dev[:5]], dev[5].data_ptr(), dev[6].data_ptr(),
                            dev[7].data_ptr(), max_read_len if max_read_len is not None else max(len(r.bases) for r in reads))
    out = torch.full((len(reads) * len(haps),), float("nan"), dtype=torch.float64, device="cuda")
    return reg, dev, out


def call(reg, out):
    import torch

    rc = _lib.lib().fgkl_pairhmm_compute_device_noalloc(C.byref(reg), C.c_void_p(out.data_ptr()),
                                                        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.FGKL_OK, _lib.last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy().copy()


def regular(reads, haps):
    return PairHmm(DOUBLE).compute_log10_likelihoods(reads, haps)


def uneven_region(seed, n_reads, n_haps, hap_len, lo, hi, with_n=False):
    rng = Rng(seed)
    ref = bytearray(rng.base() for _ in range(hap_len))
    haps = []
    for h in range(n_haps):
        hb = bytearray(ref)
        for _ in range(h):
            p = rng.below(hap_len)
            hb[p] = ord("ACGT"[rng.below(4)])
        if with_n and h % 2:
            hb[rng.below(hap_len)] = ord("N")
        haps.append(bytes(hb))
    reads = []
    for _ in range(n_reads):
        n = lo + rng.below(hi - lo + 1)
        start = rng.below(max(1, hap_len - n))
        bases = bytearray(ref[start:start + n])
        while len(bases) < n:
            bases.append(ord("ACGT"[rng.below(4)]))
        if with_n:
            bases[rng.below(n)] = ord("N")
        reads.append(Read(bytes(bases), bytes(10 + rng.below(31) for _ in range(n)), bytes(30 + rng.below(16) for _ in range(n)),
                          bytes(30 + rng.below(16) for _ in range(n)), bytes(10 for _ in range(n))))
    return reads, haps


def assert_close(actual, expected):
    assert actual.shape == expected.shape
    d = np.abs(actual - expected)
    worst = int(np.argmax(d))
    assert np.isfinite(actual).all()
    assert np.all(d <= TOL), f"pair {worst}: got {actual[worst]}, expected {expected[worst]} (diff {d[worst]})"


@pytest.mark.parametrize("shape", [
    ("reference region 32 x 151 vs 4 x 300", lambda: synthetic.reference_region(9, 32, 151, 4, 300).region(0)),
    ("uneven 40 reads 30-250 bases vs 6 haplotypes of 400, with N", lambda: uneven_region(3, 40, 6, 400, 30, 250, True)),
    ("long reads 500-620 bases vs 3 haplotypes of 700", lambda: uneven_region(5, 6, 3, 700, 500, 620)),
])
def test_matches_the_regular_entry_on_two_calls_in_a_row(gpu, shape):
    reads, haps = shape[1]()
    expected = regular(reads, haps)
    reg, keep, out = device_region(reads, haps)
    first = call(reg, out)
    second = call(reg, out)
    assert_close(first, expected)
    assert_close(second, expected)
    assert_close(first, O.compute_matrix(reads, haps))


def test_calls_take_no_device_memory(gpu):
    """After the first call on the device, a larger region leaves the device's free memory as it was."""
    import torch

    small = uneven_region(11, 8, 3, 300, 40, 150)
    large = uneven_region(12, 60, 8, 600, 100, 500)
    reg_s, keep_s, out_s = device_region(*small)
    reg_l, keep_l, out_l = device_region(*large)
    call(reg_s, out_s)
    free_before = torch.cuda.mem_get_info()[0]
    got = call(reg_l, out_l)
    assert torch.cuda.mem_get_info()[0] == free_before
    assert_close(got, regular(*large))


def test_a_bound_above_the_reads_gives_the_same_results(gpu):
    reads, haps = uneven_region(7, 12, 4, 300, 40, 120)
    reg, keep, out = device_region(reads, haps, max_read_len=400)
    assert_close(call(reg, out), regular(reads, haps))


def test_sizes_beyond_the_limits_are_rejected(gpu):
    reads, haps = uneven_region(1, 2, 2, 100, 20, 40)
    reg, keep, out = device_region(reads, haps)
    L = _lib.lib()
    for bad, code in ((621, _lib.FGKL_E_UNSUPPORTED), (0, _lib.FGKL_E_UNSUPPORTED)):
        reg.max_read_len = bad
        assert L.fgkl_pairhmm_compute_device_noalloc(C.byref(reg), C.c_void_p(out.data_ptr()), None) == code
        assert "max_read_len" in _lib.last_error()
    reg.max_read_len = 40
    reg.num_reads = -1
    assert L.fgkl_pairhmm_compute_device_noalloc(C.byref(reg), C.c_void_p(out.data_ptr()), None) == _lib.FGKL_E_INVALID_ARGUMENT
    reg.num_reads, reg.num_haplotypes = 65536, 65536
    assert L.fgkl_pairhmm_compute_device_noalloc(C.byref(reg), C.c_void_p(out.data_ptr()), None) == _lib.FGKL_E_INVALID_ARGUMENT
    assert "2^31" in _lib.last_error()
