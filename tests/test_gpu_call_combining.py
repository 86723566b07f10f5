"""Concurrent per-call requests combined into batches (fgkl_set_call_combining).

fgkl's JNI entry points may be called from any number of threads (crates/jni/src/lib.rs:5-9), and
its Java suites call them from 8 at once. Calls that meet here are run as one batch. These tests
check that the results are bit-identical to the same calls run alone, that every caller gets its
own error, and that requests of different kinds do not mix.
"""
import ctypes as C
import threading

import numpy as np
import pytest

from fgkl_b200 import Config, Precision, Read, _lib, set_allocation_limit, synthetic
from fgkl_b200.pairhmm import DeviceError, _check, _Flat, _ptr

pytestmark = pytest.mark.gpu

FLOAT = Config(precision=Precision.FLOAT)
DOUBLE = Config(precision=Precision.DOUBLE)


def call(config, reads, haps, pd=False):
    """One per-call request without stats, as the JNI entry points make it (stats run alone)."""
    flat = _Flat(reads, [h.bases for h in haps] if pd else haps, [h.flags for h in haps] if pd else None)
    rd, hp = flat.structs()
    n = len(reads) * len(haps)
    out = np.empty(n, np.float64)
    cfg = config._c()
    fn = _lib.lib().fgkl_pdhmm_compute_config if pd else _lib.lib().fgkl_pairhmm_compute_config
    _check(fn(C.byref(rd), C.byref(hp), C.byref(cfg), _ptr(out, _lib.f64p), n, None))
    return out


def set_combining(n):
    prev = _lib.lib().fgkl_set_call_combining(n)
    assert prev >= 0
    return prev


def combined_requests():
    b, r = C.c_uint64(), C.c_uint64()
    assert _lib.lib().fgkl_call_combining_stats(C.byref(b), C.byref(r)) == 0
    assert r.value >= 2 * b.value
    return r.value


def run_threads(threads, jobs):
    """Runs jobs[i]() round-robin on `threads` threads released together; (results, exceptions)."""
    results, errors = [None] * len(jobs), [None] * len(jobs)
    gate = threading.Barrier(threads)

    def worker(k):
        gate.wait()
        for i in range(k, len(jobs), threads):
            try:
                results[i] = jobs[i]()
            except Exception as e:  # noqa: BLE001 - the test inspects each job's exception
                errors[i] = e

    ts = [threading.Thread(target=worker, args=(k,)) for k in range(threads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    return results, errors


def alone(jobs):
    prev = set_combining(0)
    try:
        out = []
        for j in jobs:
            try:
                out.append(j())
            except DeviceError as e:
                out.append(e)
        return out
    finally:
        set_combining(prev)


@pytest.fixture
def combining():
    prev = set_combining(2)
    yield
    set_combining(prev)


def plain_jobs(n, seed, config):
    w = synthetic.workload(1, seed=seed, regions=n, threads=8)
    regs = [w.region(g) for g in range(n)]
    return [lambda r=r, h=h: call(config, r, h) for r, h in regs]


def test_combined_calls_are_bit_identical_to_calls_alone(gpu, combining):
    jobs = plain_jobs(48, 5, FLOAT)
    expected = alone(jobs)
    before = combined_requests()
    got, errors = run_threads(8, jobs)
    assert errors == [None] * len(jobs)
    for g, e in zip(got, expected):
        assert g.tobytes() == e.tobytes()
    assert combined_requests() > before, "no two calls met"


def test_each_caller_gets_its_own_error(gpu, combining):
    """One request needs more device memory than the injected allocation limit allows (found only
    once its batch is planned, so it fails the combined batch); the batch is retried as separate
    calls and that caller alone sees the error."""
    jobs = plain_jobs(31, 6, FLOAT)
    n = 700
    long_read = Read(b"A" * n, bytes([30] * n), bytes([45] * n), bytes([45] * n), bytes([10] * n))
    huge_hap = b"ACGT" * 5_000_000  # the strip-mined read's carry row: 320 MB a warp
    bad = lambda: call(FLOAT, [long_read], [huge_hap])  # noqa: E731
    jobs = jobs[:15] + [bad] + jobs[15:]
    prev = set_allocation_limit(768 << 20)
    try:
        expected = alone(jobs)
        assert isinstance(expected[15], DeviceError) and expected[15].code == _lib.FGKL_E_OUT_OF_MEMORY
        for _ in range(3):
            got, errors = run_threads(8, jobs)
            for i, (g, e, x) in enumerate(zip(got, errors, expected)):
                if i == 15:
                    assert isinstance(e, DeviceError) and e.code == _lib.FGKL_E_OUT_OF_MEMORY
                    assert "allocation failed" in str(e)
                else:
                    assert e is None, e
                    assert g.tobytes() == x.tobytes()
    finally:
        set_allocation_limit(prev)


def test_requests_of_different_kinds_are_not_mixed(gpu, combining):
    plain_f = plain_jobs(12, 7, FLOAT)
    plain_d = plain_jobs(12, 7, DOUBLE)
    w = synthetic.workload(3, seed=8, regions=12, threads=8)
    pd = [lambda r=r, h=h: call(FLOAT, r, h, pd=True) for r, h in (w.region(g) for g in range(12))]
    jobs = [j for trio in zip(plain_f, plain_d, pd) for j in trio]
    expected = alone(jobs)
    got, errors = run_threads(8, jobs)
    assert errors == [None] * len(jobs)
    for g, e in zip(got, expected):
        assert g.tobytes() == e.tobytes()
