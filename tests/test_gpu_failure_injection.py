"""Allocation failures injected on the host (fgkl_set_allocation_limit), with no GPU fault involved.

A device or page-locked host allocation the limit refuses must reach the caller as
FGKL_E_OUT_OF_MEMORY with a message, and leave the per-call engine, a batch context and an
adjoint context usable: the same call succeeds with the same bits once the limit is lifted.
"""
import numpy as np
import pytest

from fgkl_b200 import BatchContext, Config, DeviceError, PairHmm, PdPairHmm, Precision, _lib, set_allocation_limit, synthetic
from fgkl_b200.adjoint import AdjointContext, params_from_quals

pytestmark = pytest.mark.gpu

FLOAT = Config(precision=Precision.FLOAT)


@pytest.fixture
def limit():
    prev = set_allocation_limit(0)
    yield set_allocation_limit
    set_allocation_limit(prev)


def test_the_limit_is_process_wide_and_returns_the_previous_value(limit):
    assert limit(4096) == 0
    assert limit(0) == 4096
    with pytest.raises(ValueError):
        limit(-1)


@pytest.mark.parametrize("hmm_class, which", [(PairHmm, 1), (PdPairHmm, 3)])
def test_a_refused_allocation_fails_the_call_and_the_engine_stays_usable(gpu, limit, hmm_class, which):
    w = synthetic.workload(which, seed=21, regions=2, threads=4)
    reads, haps = w.region(0)
    good = hmm_class(FLOAT).compute_log10_likelihoods(reads, haps)
    limit(1024)
    with pytest.raises(DeviceError) as e:
        hmm_class(FLOAT).compute_log10_likelihoods(reads, haps)
    assert e.value.code == _lib.FGKL_E_OUT_OF_MEMORY and "allocation failed" in str(e.value)
    limit(0)
    assert hmm_class(FLOAT).compute_log10_likelihoods(reads, haps).tobytes() == good.tobytes()


def test_a_batch_context_survives_a_refused_allocation(gpu, limit):
    small = synthetic.workload(1, seed=22, regions=4, threads=4)
    large = synthetic.workload(1, seed=23, regions=64, threads=8)
    ctx = BatchContext()
    first, _ = ctx.compute(small, FLOAT)
    limit(1 << 20)  # the small batch's buffers are already held; the large one needs more
    with pytest.raises(DeviceError) as e:
        ctx.compute(large, FLOAT)
    assert e.value.code == _lib.FGKL_E_OUT_OF_MEMORY
    limit(0)
    again, _ = ctx.compute(small, FLOAT)
    assert again.tobytes() == first.tobytes()
    big, _ = ctx.compute(large, FLOAT)
    fresh = BatchContext()
    assert big.tobytes() == fresh.compute(large, FLOAT)[0].tobytes()
    ctx.close()
    fresh.close()


def test_an_adjoint_context_survives_a_refused_allocation(gpu, limit):
    w = synthetic.workload(4, seed=24, regions=2, threads=4)
    params = params_from_quals(w)
    ctx = AdjointContext()
    first = ctx.compute(w, params)
    limit(4096)
    with pytest.raises(DeviceError) as e:
        AdjointContext().compute(w, params)
    assert e.value.code == _lib.FGKL_E_OUT_OF_MEMORY
    limit(0)
    again = ctx.compute(w, params)
    for f in ("log10", "gap_open_ins", "gap_open_del", "gap_continuation", "base_error"):
        assert getattr(again, f).tobytes() == getattr(first, f).tobytes(), f
    ctx.close()
