"""The C ABI without a GPU: the library loads, exports every symbol include/fgkl_b200.h declares, and
refuses malformed input exactly as fgkl's JNI layer and PairHmm do (jni/src/lib.rs:343-394,
lib.rs:1070-1096, pd.rs:438-464) before touching a device."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from fgkl_b200 import (DEL_END, EmptyHaplotype, EmptyRead, MismatchedHaplotypeArrays, MismatchedReadArrays, OutputLength,
                       PairHmm, PdHaplotype, PdPairHmm, Read, _lib)
from conftest import has_gpu

HEADER = Path(__file__).resolve().parents[1] / "include" / "fgkl_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fgkl_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 19
    for name in names:
        assert hasattr(L, name), name
    assert set(_lib.EXPORTED) <= set(names)


def good():
    return Read(b"ACGT", bytes([30] * 4), bytes([45] * 4), bytes([45] * 4), bytes([10] * 4))


def test_invalid_inputs_are_rejected():
    hmm = PairHmm()
    short_quals = Read(b"ACGT", bytes([30] * 3), bytes([45] * 4), bytes([45] * 4), bytes([10] * 4))
    with pytest.raises(MismatchedReadArrays) as e:
        hmm.compute_log10_likelihoods([short_quals], [b"ACGT"], np.zeros(1))
    assert e.value.index == 0
    with pytest.raises(EmptyHaplotype) as e:
        hmm.compute_log10_likelihoods([good()], [b""], np.zeros(1))
    assert e.value.index == 0
    with pytest.raises(OutputLength) as e:
        hmm.compute_log10_likelihoods([good()], [b"ACGT", b"ACGT"], np.zeros(1))
    assert (e.value.expected, e.value.actual) == (2, 1)
    empty = Read(b"", b"", b"", b"", b"")
    with pytest.raises(EmptyRead) as e:
        hmm.compute_log10_likelihoods([good(), empty], [b"ACGT"], np.zeros(2))
    assert e.value.index == 1
    assert hmm.compute_log10_likelihoods([], [b"ACGT"], np.zeros(0)).size == 0


def test_invalid_pd_inputs_are_rejected():
    hmm = PdPairHmm()
    hap = PdHaplotype(b"ACGT", bytes(4))
    with pytest.raises(EmptyHaplotype):
        hmm.compute_log10_likelihoods([good()], [PdHaplotype(b"", b"")], np.zeros(1))
    with pytest.raises(MismatchedHaplotypeArrays) as e:
        hmm.compute_log10_likelihoods([good()], [hap, PdHaplotype(b"ACGT", bytes([DEL_END] * 3))], np.zeros(2))
    assert e.value.index == 1
    with pytest.raises(OutputLength):
        hmm.compute_log10_likelihoods([good()], [hap, hap], np.zeros(1))


def raw_call(read_offsets, hap_offsets, n_bases=4, n_hap=4, out_len=1, quals_len=None, flags_len=None, pd=False):
    L = _lib.lib()
    b = np.frombuffer(b"ACGT" * 8, np.uint8)[:n_bases].copy()
    q = np.full(quals_len if quals_len is not None else n_bases, 30, np.uint8)
    g = np.full(n_bases, 45, np.uint8)
    c = np.full(n_bases, 10, np.uint8)
    ro = np.array(read_offsets, np.int32)
    hb = np.frombuffer(b"ACGT" * 8, np.uint8)[:n_hap].copy()
    hf = np.zeros(flags_len if flags_len is not None else n_hap, np.uint8)
    ho = np.array(hap_offsets, np.int32)
    u8 = _lib.u8p
    rd = _lib.Reads(b.ctypes.data_as(u8), b.size, q.ctypes.data_as(u8), q.size, g.ctypes.data_as(u8), g.size,
                    g.ctypes.data_as(u8), g.size, c.ctypes.data_as(u8), c.size, ro.ctypes.data_as(_lib.i32p), ro.size)
    hp = _lib.Haplotypes(hb.ctypes.data_as(u8), hb.size, hf.ctypes.data_as(u8), hf.size, ho.ctypes.data_as(_lib.i32p), ho.size)
    out = np.zeros(max(out_len, 1))
    fn = L.fgkl_pdhmm_compute if pd else L.fgkl_pairhmm_compute
    rc = fn(C.byref(rd), C.byref(hp), 0, out.ctypes.data_as(_lib.f64p), out_len)
    return rc, _lib.last_error()


def test_offset_tables_are_checked_like_the_jni_layer():
    assert raw_call([1, 4], [0, 4])[0] == _lib.FGKL_E_BAD_OFFSETS
    rc, msg = raw_call([], [0, 4])
    assert rc == _lib.FGKL_E_BAD_OFFSETS and "start at zero" in msg
    rc, msg = raw_call([0, 3], [0, 4])
    assert rc == _lib.FGKL_E_BAD_OFFSETS and "end at the array length" in msg
    rc, msg = raw_call([0, 5, 2, 4], [0, 4], out_len=3)
    assert rc == _lib.FGKL_E_BAD_OFFSETS and "non-decreasing" in msg
    rc, msg = raw_call([0, 4], [0, -1], n_hap=0)
    assert rc == _lib.FGKL_E_BAD_OFFSETS


def test_read_arrays_must_share_one_total_length():
    rc, msg = raw_call([0, 4], [0, 4], quals_len=3)
    assert rc == _lib.FGKL_E_MISMATCHED_READ_ARRAYS and "differ in total length" in msg


def test_pd_flags_must_match_the_haplotype_bases():
    rc, msg = raw_call([0, 4], [0, 4], flags_len=3, pd=True)
    assert rc == _lib.FGKL_E_MISMATCHED_HAPLOTYPE_ARRAYS


def test_output_length_and_empty_members_are_refused_before_compute():
    assert raw_call([0, 4], [0, 4], out_len=2)[0] == _lib.FGKL_E_OUTPUT_LENGTH
    assert raw_call([0, 0, 4], [0, 4], out_len=2)[0] == _lib.FGKL_E_EMPTY_READ
    assert raw_call([0, 4], [0, 0, 4], out_len=2)[0] == _lib.FGKL_E_EMPTY_HAPLOTYPE
    assert raw_call([0], [0, 4], n_bases=0, out_len=0)[0] == _lib.FGKL_OK


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_without_a_device_the_call_fails_loudly_instead_of_falling_back():
    rc, msg = raw_call([0, 4], [0, 4])
    assert rc == _lib.FGKL_E_NO_DEVICE, msg
    with pytest.raises(Exception):
        PairHmm().compute_log10_likelihoods([good()], [b"ACGT"])


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_concurrent_calls_without_a_device_all_fail_and_none_waits():
    # Every caller leads in turn (no batch ever starts), finds no device, leaves the queue and
    # returns its own error; a request left queued would make a later caller wait for ever.
    import threading
    results = []
    lock = threading.Lock()

    def worker():
        for _ in range(20):
            rc, msg = raw_call([0, 4], [0, 4])
            with lock:
                results.append((rc, msg))

    ts = [threading.Thread(target=worker) for _ in range(8)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=60)
    assert not any(t.is_alive() for t in ts)
    assert len(results) == 160
    assert all(rc == _lib.FGKL_E_NO_DEVICE and msg for rc, msg in results)


def test_call_combining_switch():
    L = _lib.lib()
    prev = L.fgkl_set_call_combining(3)
    assert prev >= 0
    assert L.fgkl_set_call_combining(-1) == _lib.FGKL_E_INVALID_ARGUMENT
    assert L.fgkl_set_call_combining(9) == _lib.FGKL_E_INVALID_ARGUMENT
    assert L.fgkl_set_call_combining(prev) == 3
    b, r = C.c_uint64(), C.c_uint64()
    assert L.fgkl_call_combining_stats(C.byref(b), C.byref(r)) == 0
    assert r.value >= 2 * b.value
    assert L.fgkl_call_combining_stats(None, C.byref(r)) == _lib.FGKL_E_INVALID_ARGUMENT


def test_call_combining_python_mirror():
    import fgkl_b200
    prev = fgkl_b200.set_call_combining(1)
    assert fgkl_b200.set_call_combining(prev) == 1
    with pytest.raises(ValueError):
        fgkl_b200.set_call_combining(9)
    batches, requests = fgkl_b200.call_combining_stats()
    assert requests >= 2 * batches


def test_allocation_free_entry_checks_its_bounds_on_the_host():
    """The allocation-free entry refuses, before any device work, a call of more than
    FGKL_NOALLOC_MAX_PAIRS (2^31 - 1) pairs and a max_read_len outside 1..620 (its ticket counter
    is 64-bit, so no count up to the bound can wrap)."""
    L = _lib.lib()
    r = _lib.DeviceRegion()
    r.num_reads, r.num_haplotypes, r.max_read_len = 65536, 32768, 151  # 2^31 pairs: one past the bound
    assert L.fgkl_pairhmm_compute_device_noalloc(C.byref(r), None, None) == _lib.FGKL_E_INVALID_ARGUMENT
    assert "2^31 - 1" in _lib.last_error()
    r.num_reads, r.num_haplotypes = -1, 4
    assert L.fgkl_pairhmm_compute_device_noalloc(C.byref(r), None, None) == _lib.FGKL_E_INVALID_ARGUMENT
    for bad_len in (0, 621):
        r.num_reads, r.num_haplotypes, r.max_read_len = 4, 4, bad_len
        assert L.fgkl_pairhmm_compute_device_noalloc(C.byref(r), None, None) == _lib.FGKL_E_UNSUPPORTED
    r.num_reads, r.num_haplotypes, r.max_read_len = 0, 4, 151  # no pairs: nothing to do
    assert L.fgkl_pairhmm_compute_device_noalloc(C.byref(r), None, None) == 0


def test_measurement_entries_check_their_arguments():
    # No context: an error, not a crash; the probe needs somewhere to write.
    ms = C.c_float()
    assert _lib.lib().fgkl_sw_last_kernel_ms(None, C.byref(ms)) == _lib.FGKL_E_INVALID_ARGUMENT
    assert _lib.lib().fgkl_probe_int32_alu_gops(0, None) == _lib.FGKL_E_INVALID_ARGUMENT


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_the_alu_probe_without_a_device_fails_loudly():
    gops = C.c_double(-1.0)
    assert _lib.lib().fgkl_probe_int32_alu_gops(0, C.byref(gops)) == _lib.FGKL_E_NO_DEVICE
    assert gops.value == -1.0
