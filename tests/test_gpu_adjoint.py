"""The adjoint kernels against the FP64 scalar adjoint and FP64 central finite differences.

The adjoint has no counterpart in fgkl; its parameterisation (per read position: gap-open dI, dD,
gap continuation eps, base error e; MM = 1 - dI - dD) and its checks are this project's: gradients of
the summed log10 likelihood within 1e-4 relative of central finite differences (step 1e-6) of the
FP64 oracle, and of the FP64 scalar adjoint (oracle/pairhmm_oracle.c, or_adj_gradient). The
torch.autograd.Function wrapper lives here, in the test harness, and only here.
"""
import numpy as np
import pytest

from fgkl_b200 import Read, synthetic
from fgkl_b200.adjoint import AdjointContext, AdjointParams, params_from_quals
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def workload(seed=7, regions=3, reads=6, read_len=60, haps=3, hap_len=120):
    parts = [synthetic.reference_region(seed + g, reads, read_len, haps, hap_len).region(0) for g in range(regions)]
    return synthetic.from_regions(parts), parts


def oracle_all(w, p: AdjointParams):
    """(log10 per pair, 4 gradient arrays) from the FP64 scalar adjoint."""
    out = []
    g = [np.zeros(w.bases.size) for _ in range(4)]
    r0 = h0 = 0
    for gi in range(w.num_regions):
        nr, nh = int(w.region_reads[gi]), int(w.region_haps[gi])
        for r in range(r0, r0 + nr):
            lo, hi = int(w.read_offsets[r]), int(w.read_offsets[r + 1])
            bases = w.bases[lo:hi].tobytes()
            args = [a[lo:hi] for a in (p.gap_open_ins, p.gap_open_del, p.gap_continuation, p.base_error)]
            for h in range(h0, h0 + nh):
                hap = w.hap_bases[int(w.hap_offsets[h]):int(w.hap_offsets[h + 1])].tobytes()
                ll, *gr = O.adj_gradient(hap, bases, *args)
                out.append(ll)
                for k in range(4):
                    g[k][lo:hi] += gr[k]
        r0 += nr
        h0 += nh
    return np.array(out), g


def oracle_total(w, p: AdjointParams) -> float:
    total = 0.0
    r0 = h0 = 0
    for gi in range(w.num_regions):
        nr, nh = int(w.region_reads[gi]), int(w.region_haps[gi])
        for r in range(r0, r0 + nr):
            lo, hi = int(w.read_offsets[r]), int(w.read_offsets[r + 1])
            bases = w.bases[lo:hi].tobytes()
            args = [a[lo:hi] for a in (p.gap_open_ins, p.gap_open_del, p.gap_continuation, p.base_error)]
            for h in range(h0, h0 + nh):
                hap = w.hap_bases[int(w.hap_offsets[h]):int(w.hap_offsets[h + 1])].tobytes()
                total += O.adj_log10_likelihood(hap, bases, *args)
        r0 += nr
        h0 += nh
    return total


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


NAMES = ("gap_open_ins", "gap_open_del", "gap_continuation", "base_error")


@pytest.mark.parametrize("double", [False, True])
def test_likelihoods_and_gradients_match_the_fp64_scalar_adjoint(gpu, double):
    w, _ = workload()
    p = params_from_quals(w)
    res = AdjointContext().compute(w, p, double)
    ll, g = oracle_all(w, p)
    np.testing.assert_allclose(res.log10, ll, rtol=0, atol=1e-9 if double else 1e-4)
    for k, name in enumerate(NAMES):
        ours = getattr(res, name)
        # The summed global scalar within 1e-4 relative (FP32) / 1e-9 (FP64); every position close too.
        assert rel(ours.sum(), g[k].sum()) <= (1e-9 if double else 1e-4), name
        scale = np.abs(g[k]).max()
        np.testing.assert_allclose(ours, g[k], rtol=0, atol=(1e-9 if double else 1e-4) * scale, err_msg=name)


def central_difference(w, p: AdjointParams, k: int, h: float) -> float:
    arrays = [p.gap_open_ins, p.gap_open_del, p.gap_continuation, p.base_error]
    plus = [a.copy() for a in arrays]
    minus = [a.copy() for a in arrays]
    plus[k] = plus[k] + h
    minus[k] = minus[k] - h
    return (oracle_total(w, AdjointParams(*plus)) - oracle_total(w, AdjointParams(*minus))) / (2 * h)


def test_gradients_match_central_finite_differences(gpu):
    # Gap-open probabilities are ~3e-5, so a step of 1e-6 is a 3% change and the central difference's
    # own h^2 error can reach 1e-4; central differences at h = 1e-6 and h / 2 combined by Richardson
    # extrapolation, (4 D(h/2) - D(h)) / 3, cancel it.
    w, _ = workload(seed=21, regions=2, reads=4, read_len=40, haps=3, hap_len=90)
    p = params_from_quals(w)
    res = AdjointContext().compute(w, p, False)
    h = 1e-6
    for k, name in enumerate(NAMES):
        fd = (4 * central_difference(w, p, k, h / 2) - central_difference(w, p, k, h)) / 3
        assert rel(getattr(res, name).sum(), fd) <= 1e-4, (name, getattr(res, name).sum(), fd)


def test_reads_fp32_loses_are_recomputed_in_fp64(gpu):
    reads = [Read(b"A" * 80, bytes([40] * 80), bytes([45] * 80), bytes([45] * 80), bytes([10] * 80)),
             Read(b"ACGTACGTAC" * 6, bytes([30] * 60), bytes([45] * 60), bytes([45] * 60), bytes([10] * 60))]
    haps = [b"C" * 80, b"ACGTACGTAC" * 8]
    w = synthetic.from_regions([(reads, haps)])
    p = params_from_quals(w)
    res = AdjointContext().compute(w, p, False)
    assert res.fp64_reads >= 1
    ll, g = oracle_all(w, p)
    np.testing.assert_allclose(res.log10, ll, rtol=0, atol=1e-4)
    for k, name in enumerate(NAMES):
        assert rel(getattr(res, name).sum(), g[k].sum()) <= 1e-4, name


def test_config_4_shape_matches_the_scalar_adjoint_on_a_sample(gpu):
    # Reads of 151 against haplotypes of 350 (the adjoint benchmark's shape), a few regions.
    w, _ = workload(seed=3, regions=2, reads=8, read_len=151, haps=4, hap_len=350)
    p = params_from_quals(w)
    res = AdjointContext().compute(w, p, False)
    ll, g = oracle_all(w, p)
    np.testing.assert_allclose(res.log10, ll, rtol=0, atol=1e-4)
    for k, name in enumerate(NAMES):
        assert rel(getattr(res, name).sum(), g[k].sum()) <= 1e-4, name


def test_torch_autograd_function_wraps_the_adjoint(gpu):
    import torch

    w, _ = workload(seed=5, regions=1, reads=3, read_len=20, haps=2, hap_len=40)
    ctx = AdjointContext()

    class SummedLog10Likelihood(torch.autograd.Function):
        @staticmethod
        def forward(fctx, d_ins, d_del, eps, err):
            p = AdjointParams(*(t.detach().cpu().numpy() for t in (d_ins, d_del, eps, err)))
            res = ctx.compute(w, p, True)
            fctx.save_for_backward(*(torch.from_numpy(getattr(res, n)) for n in NAMES))
            return torch.tensor(res.log10.sum(), dtype=torch.float64)

        @staticmethod
        def backward(fctx, grad_out):
            return tuple(grad_out * g for g in fctx.saved_tensors)

    p = params_from_quals(w)
    inputs = tuple(torch.from_numpy(np.array(a)).requires_grad_(True)
                   for a in (p.gap_open_ins, p.gap_open_del, p.gap_continuation, p.base_error))
    assert torch.autograd.gradcheck(SummedLog10Likelihood.apply, inputs, eps=1e-6, atol=1e-6, rtol=1e-4, fast_mode=True)
    total = SummedLog10Likelihood.apply(*inputs)
    total.backward()
    ref_ll, ref_g = oracle_all(w, p)
    assert abs(total.item() - ref_ll.sum()) <= 1e-9 * abs(ref_ll.sum())
    for k in range(4):
        np.testing.assert_allclose(inputs[k].grad.numpy(), ref_g[k], rtol=1e-8, atol=1e-12)


def compare_with_scalar_adjoint(w, p, res, tol):
    ll, g = oracle_all(w, p)
    np.testing.assert_allclose(res.log10, ll, rtol=0, atol=tol)
    for k, name in enumerate(NAMES):
        assert rel(getattr(res, name).sum(), g[k].sum()) <= tol, name
        scale = np.abs(g[k]).max()
        np.testing.assert_allclose(getattr(res, name), g[k], rtol=0, atol=tol * scale, err_msg=name)


def test_long_haplotypes_match_the_fp64_scalar_adjoint(gpu):
    # Haplotypes of about 2,400 bases against reads of 80: hundreds of recomputed backward blocks per
    # pair; a short region in the same launch.
    long_parts = [synthetic.reference_region(61, 3, 80, 2, 2400).region(0)]
    short_parts = [synthetic.reference_region(62, 4, 80, 2, 150).region(0)]
    w = synthetic.from_regions(long_parts + short_parts)
    p = params_from_quals(w)
    compare_with_scalar_adjoint(w, p, AdjointContext().compute(w, p, False), 1e-4)


@pytest.mark.parametrize("read_len", [621, 1000, 2500])
@pytest.mark.parametrize("double", [False, True])
def test_long_reads_match_the_fp64_scalar_adjoint(gpu, read_len, double):
    """Reads beyond one 32 x 20-row block are strip-mined over row blocks of 256 rows."""
    w, _ = workload(seed=70 + read_len, regions=1, reads=2, read_len=read_len, haps=2, hap_len=read_len + 120)
    p = params_from_quals(w)
    compare_with_scalar_adjoint(w, p, AdjointContext().compute(w, p, double), 1e-9 if double else 1e-4)


def test_a_read_lost_on_a_later_haplotype_is_summed_afresh_in_fp64(gpu):
    """The FP32 pass adds a read's terms haplotype by haplotype; when a later haplotype loses the read,
    the FP64 recomputation must not count the earlier haplotypes twice."""
    n = 80
    bases = b"ACGTACGTAC" * 8
    reads = [Read(bases, bytes([30] * n), bytes([45] * n), bytes([45] * n), bytes([10] * n))]
    haps = [b"ACGTACGTAC" * 9, b"T" * 90]
    w = synthetic.from_regions([(reads, haps)])
    p = params_from_quals(w)
    res = AdjointContext().compute(w, p, False)
    assert res.fp64_reads == 1
    compare_with_scalar_adjoint(w, p, res, 1e-4)


def test_runs_are_deterministic(gpu):
    w, _ = workload(seed=13, regions=3, reads=6, read_len=100, haps=3, hap_len=250)
    p = params_from_quals(w)
    a = AdjointContext().compute(w, p, False)
    b = AdjointContext().compute(w, p, False)
    for name in ("log10",) + NAMES:
        assert getattr(a, name).tobytes() == getattr(b, name).tobytes(), name
