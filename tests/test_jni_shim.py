"""fgkl's JNI entry points over the C ABI (fgkl_b200/jni/fgkl_jni.c), compiled here against a
minimal stand-in for <jni.h> (tests/jni_stub; this image has no JDK) and driven through a fake JNI
environment, as the JVM would call them for FgklPairHmm / FgklPdHmm (crates/jni/src/lib.rs:150-254).
On the CPU: the shim turns every input error into an IllegalArgumentException carrying the C ABI's
message, and a missing device into a RuntimeException. On a B200: its likelihoods are the per-call
C ABI's, written back with one SetDoubleArrayRegion."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from fgkl_b200 import Config, PairHmm, PdHaplotype, PdPairHmm, Precision, _lib, set_allocation_limit, synthetic

ROOT = Path(__file__).resolve().parent.parent
IAE = "java/lang/IllegalArgumentException"
RTE = "java/lang/RuntimeException"


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    out = tmp_path_factory.mktemp("jni") / "libfgkl_jni_harness.so"
    libdir = Path(_lib.LIB_PATH).parent
    subprocess.run(["gcc", "-O2", "-shared", "-fPIC", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'tests' / 'jni_stub'}",
                    f"-I{ROOT / 'include'}", str(ROOT / "fgkl_b200" / "jni" / "fgkl_jni.c"),
                    str(ROOT / "tests" / "jni_stub" / "harness.c"), f"-L{libdir}", "-lfgkl_b200", f"-Wl,-rpath,{libdir}",
                    "-o", str(out)], check=True)
    _lib.lib()  # the same libfgkl_b200.so the harness links against, loaded first
    L = C.CDLL(str(out))
    i8, i32, f64 = C.POINTER(C.c_int8), C.POINTER(C.c_int32), C.POINTER(C.c_double)
    L.harness_compute.argtypes = [i8, C.c_int] * 5 + [i32, C.c_int, i8, C.c_int, i8, C.c_int, i32, C.c_int, C.c_int,
                                                      f64, C.c_int, C.c_char_p, C.c_char_p, C.POINTER(C.c_int)]
    L.harness_compute.restype = C.c_int
    L.harness_backend.argtypes = [C.c_char_p, C.c_int]
    L.harness_sw_align.argtypes = [i8, C.c_int, i8, C.c_int] + [C.c_int] * 5 + [C.c_char_p, C.c_int, i32, C.c_char_p, C.c_char_p]
    L.harness_sw_align.restype = C.c_int
    return L


def sw_call(L, ref: bytes, alt: bytes, params=(10, -15, -30, -5), strategy=0):
    i8 = C.POINTER(C.c_int8)
    r, a = np.frombuffer(ref, np.int8).copy(), np.frombuffer(alt, np.int8).copy()
    cigar, cls, msg, off = C.create_string_buffer(2048), C.create_string_buffer(128), C.create_string_buffer(512), C.c_int32()
    thrown = L.harness_sw_align(r.ctypes.data_as(i8), r.size, a.ctypes.data_as(i8), a.size, *params, strategy, cigar, 2048,
                                C.byref(off), cls, msg)
    return (cls.value.decode(), msg.value.decode()) if thrown else None, cigar.value.decode(), off.value


def flat(reads, haps):
    cols = [np.concatenate([np.frombuffer(bytes(getattr(r, f)), np.int8) for r in reads]) for f in
            ("bases", "quals", "ins_gop", "del_gop", "gcp")]
    roff = np.zeros(len(reads) + 1, np.int32)
    np.cumsum([len(r.bases) for r in reads], out=roff[1:])
    pd = bool(haps) and isinstance(haps[0], PdHaplotype)
    hb = np.concatenate([np.frombuffer(bytes(h.bases if pd else h), np.int8) for h in haps])
    hf = np.concatenate([np.frombuffer(bytes(h.flags), np.int8) for h in haps]) if pd else None
    hoff = np.zeros(len(haps) + 1, np.int32)
    np.cumsum([len(h.bases if pd else h) for h in haps], out=hoff[1:])
    return cols, roff, hb, hf, hoff


def call(L, cols, roff, hb, hf, hoff, double=False, n_out=None):
    i8, i32 = C.POINTER(C.c_int8), C.POINTER(C.c_int32)
    n_out = (roff.size - 1) * (hoff.size - 1) if n_out is None else n_out
    out = np.full(max(n_out, 1), np.nan)
    cls, msg, rc = C.create_string_buffer(128), C.create_string_buffer(512), C.c_int()
    args = []
    for c in cols:
        args += [c.ctypes.data_as(i8), c.size]
    thrown = L.harness_compute(*args, roff.ctypes.data_as(i32), roff.size, hb.ctypes.data_as(i8), hb.size,
                               hf.ctypes.data_as(i8) if hf is not None else None, hf.size if hf is not None else 0,
                               hoff.ctypes.data_as(i32), hoff.size, int(double), out.ctypes.data_as(C.POINTER(C.c_double)),
                               n_out, cls, msg, C.byref(rc))
    return (cls.value.decode(), msg.value.decode()) if thrown else None, out[:n_out], rc.value


def region(seed=3):
    return synthetic.reference_region(seed, 6, 50, 3, 90).region(0)


def test_backend_native_names_the_backend(shim):
    buf = C.create_string_buffer(128)
    shim.harness_backend(buf, 128)
    assert buf.value == _lib.lib().fgkl_backend()


@pytest.mark.parametrize("case", ["mismatched_read_arrays", "offsets_not_from_zero", "offsets_short_of_the_end",
                                  "output_length", "empty_read", "empty_haplotype", "pd_flag_length"])
def test_input_errors_raise_illegal_argument_with_the_abi_message(shim, case):
    reads, haps = region()
    cols, roff, hb, hf, hoff = flat(reads, haps)
    n_out = None
    if case == "mismatched_read_arrays":
        cols[1] = cols[1][:-1]
    elif case == "offsets_not_from_zero":
        roff = roff.copy()
        roff[0] = 1
    elif case == "offsets_short_of_the_end":
        hoff = hoff.copy()
        hoff[-1] -= 1
    elif case == "output_length":
        n_out = (roff.size - 1) * (hoff.size - 1) - 1
    elif case == "empty_read":
        roff = np.concatenate([roff[:1], roff]).astype(np.int32)
    elif case == "empty_haplotype":
        hoff = np.concatenate([hoff[:1], hoff]).astype(np.int32)
    elif case == "pd_flag_length":
        pd = [PdHaplotype(h, bytes(len(h))) for h in haps]
        cols, roff, hb, hf, hoff = flat(reads, pd)
        hf = hf[:-1]
    exc, out, region_calls = call(shim, cols, roff, hb, hf, hoff, n_out=n_out)
    assert exc is not None and exc[0] == IAE, (case, exc)
    assert exc[1] == _lib.last_error(), case
    assert region_calls == 0


def test_a_call_without_a_device_raises_runtime_exception(shim):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present; tests/test_jni_shim.py::test_gpu_* cover this path")
    reads, haps = region()
    exc, _, region_calls = call(shim, *flat(reads, haps))
    assert exc is not None and exc[0] == RTE
    assert region_calls == 0


@pytest.mark.gpu
@pytest.mark.parametrize("double", [False, True])
def test_gpu_shim_likelihoods_are_the_per_call_abi_bits(gpu, shim, double):
    reads, haps = region(7)
    exc, out, region_calls = call(shim, *flat(reads, haps), double=double)
    assert exc is None, exc
    assert region_calls == 1
    prec = Precision.DOUBLE if double else Precision.FLOAT
    assert out.tobytes() == PairHmm(Config(precision=prec)).compute_log10_likelihoods(reads, haps).tobytes()


@pytest.mark.gpu
def test_gpu_pd_shim_likelihoods_are_the_per_call_abi_bits(gpu, shim):
    reads, haps = synthetic.reference_pd_region(31, 12, 80, 4, 150).region(0)
    exc, out, region_calls = call(shim, *flat(reads, haps))
    assert exc is None, exc
    assert region_calls == 1
    assert out.tobytes() == PdPairHmm(Config()).compute_log10_likelihoods(reads, haps).tobytes()


@pytest.mark.gpu
def test_gpu_a_long_read_gets_the_per_call_abi_bits(gpu, shim):
    reads, haps = synthetic.reference_region(8, 2, 700, 3, 820).region(0)
    exc, out, region_calls = call(shim, *flat(reads, haps))
    assert exc is None, exc
    assert region_calls == 1
    assert out.tobytes() == PairHmm(Config(precision=Precision.FLOAT)).compute_log10_likelihoods(reads, haps).tobytes()


@pytest.mark.gpu
def test_gpu_a_failed_allocation_raises_runtime_exception(gpu, shim):
    """fgkl's panic path throws RuntimeException (crates/jni/src/lib.rs:39-74); an allocation the
    injected limit refuses takes the same path."""
    reads, haps = region()
    prev = set_allocation_limit(1024)
    try:
        exc, _, region_calls = call(shim, *flat(reads, haps))
        message = _lib.last_error()  # read before the limit call below clears it
    finally:
        set_allocation_limit(prev)
    assert exc is not None and exc[0] == RTE and exc[1] == message
    assert "allocation failed" in exc[1]
    assert region_calls == 0
    exc, out, _ = call(shim, *flat(reads, haps))
    assert exc is None, exc
    assert out.tobytes() == PairHmm(Config(precision=Precision.FLOAT)).compute_log10_likelihoods(reads, haps).tobytes()


@pytest.mark.parametrize("ref, alt, strategy", [(b"", b"ACGT", 0), (b"ACGT", b"", 1), (b"ACGT", b"ACG", 9)])
def test_smith_waterman_input_errors_raise_illegal_argument(shim, ref, alt, strategy):
    exc, cigar, _ = sw_call(shim, ref, alt, strategy=strategy)
    assert exc is not None and exc[0] == IAE and exc[1] == _lib.last_error()
    assert cigar == ""


@pytest.mark.gpu
def test_gpu_smith_waterman_shim_returns_the_abi_alignment(gpu, shim):
    from fgkl_b200.sw import ALIGNMENT_TO_BEST_HAPLOTYPE, OverhangStrategy, align

    hap = b"ACGTACGTAGGCCTTAGCA"
    read = b"GGGGACGTACGTAGGCCTTAGCAGGGG"
    exc, cigar, off = sw_call(shim, hap, read)
    assert exc is None, exc
    assert (cigar, off) == ("4S19M4S", 0)
    assert align(hap, read, ALIGNMENT_TO_BEST_HAPLOTYPE, OverhangStrategy.SOFTCLIP).cigar == cigar
