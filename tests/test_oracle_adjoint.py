"""The FP64 scalar adjoint oracle (oracle/pairhmm_oracle.c, or_adj_gradient) on the CPU: its
gradients of the summed log10 likelihood agree with central finite differences of the FP64 forward
(or_adj_log10_likelihood), step 1e-6 and 5e-7 combined by Richardson extrapolation, and its forward
agrees with fgkl's recurrence (reference.rs:20-64) where the two parameterisations coincide."""
import numpy as np

from oracle import oracle as O
from refgen import Rng


def case(seed, n, m):
    rng = Rng(seed)
    hap = bytes(rng.base() for _ in range(m))
    start = rng.below(m - n)
    read = bytearray(hap[start:start + n])
    for _ in range(2):
        read[rng.below(n)] = ord("ACGT"[rng.below(4)])
    q = lambda lo, hi: np.array([10 ** (-(lo + rng.below(hi - lo + 1)) / 10) for _ in range(n)])
    return hap, bytes(read), q(40, 45), q(40, 45), q(8, 12), q(10, 40)


def richardson(f, x, k, h=1e-6):
    def central(step):
        plus = [a.copy() for a in x]
        minus = [a.copy() for a in x]
        plus[k] += step
        minus[k] -= step
        return (f(plus) - f(minus)) / (2 * step)
    return (4 * central(h / 2) - central(h)) / 3


def test_scalar_adjoint_matches_finite_differences():
    for seed, n, m in ((1, 30, 70), (2, 55, 120), (3, 12, 40)):
        hap, read, *params = case(seed, n, m)
        ll, *grads = O.adj_gradient(hap, read, *params)
        assert abs(ll - O.adj_log10_likelihood(hap, read, *params)) < 1e-12
        f = lambda p: O.adj_log10_likelihood(hap, read, *p)
        for k in range(4):
            fd = richardson(f, params, k)
            assert abs(grads[k].sum() - fd) <= 1e-6 * abs(fd), (seed, k, grads[k].sum(), fd)


def test_single_position_derivatives_match_finite_differences():
    hap, read, *params = case(4, 25, 60)
    _, *grads = O.adj_gradient(hap, read, *params)
    f = lambda p: O.adj_log10_likelihood(hap, read, *p)
    h = 1e-6
    # Rounding of the differenced sums: a few times 1e-16 * |log10 L| / h.
    noise = 4e-15 * abs(f(params)) / h
    for k in range(4):
        for pos in (0, 7, 24):
            def central(step, k=k, pos=pos):
                plus = [a.copy() for a in params]
                minus = [a.copy() for a in params]
                plus[k][pos] += step
                minus[k][pos] -= step
                return (f(plus) - f(minus)) / (2 * step)
            fd = (4 * central(h / 2) - central(h)) / 3
            assert abs(grads[k][pos] - fd) <= 1e-5 * abs(fd) + noise, (k, pos, grads[k][pos], fd)
