"""The bound behind the potential tolerance (no GPU): for every Hermite
Coulomb integral R_tuv(p, X) = d^(t,u,v) F_0(p |X|^2) (McMurchie-Davidson,
the terms of chem-kumo's pair_potential, src/electrostatic_potential.cpp:
231-348), |R_tuv(p, X)| <= p^((t+u+v)/2) S_tuv at every X, with S_tuv the
Fourier-form constant of kumo_dev::hermite_sup.  The device drops a pair
only when its coefficients times these constants, summed with the other
dropped pairs', stay within half the tolerance, so this inequality is what
makes the screened potential stay within the tolerance everywhere."""
import math
from functools import lru_cache

import numpy as np
from scipy.special import gammainc


def hermite_sup(t, u, v):
    # Restated from the formula documented in chem-kumo_b200/csrc/cuda/esp.cuh.
    n = t + u + v
    return (math.sqrt(math.pi) / (4 * math.pi ** 2) * 2.0 ** n * math.gamma((n + 1) / 2) * 2
            * math.gamma((t + 1) / 2) * math.gamma((u + 1) / 2) * math.gamma((v + 1) / 2) / math.gamma((n + 3) / 2))


def boys(n, T):
    if T < 1e-12:
        return 1.0 / (2 * n + 1)
    a = n + 0.5
    return gammainc(a, T) * math.gamma(a) / (2.0 * T ** a)


def hermite_r(p, X, L):
    T = p * float(X @ X)

    @lru_cache(maxsize=None)
    def R(n, t, u, v):
        if t < 0 or u < 0 or v < 0:
            return 0.0
        if t == u == v == 0:
            return (-2.0 * p) ** n * boys(n, T)
        if t > 0:
            return (t - 1) * R(n + 1, t - 2, u, v) + X[0] * R(n + 1, t - 1, u, v)
        if u > 0:
            return (u - 1) * R(n + 1, t, u - 2, v) + X[1] * R(n + 1, t, u - 1, v)
        return (v - 1) * R(n + 1, t, u, v - 2) + X[2] * R(n + 1, t, u, v - 1)

    return {(t, u, v): R(0, t, u, v) for s in range(L + 1) for t in range(s, -1, -1)
            for u in range(s - t, -1, -1) for v in [s - t - u]}


def test_value_at_origin_is_the_bound_of_order_zero():
    assert abs(hermite_sup(0, 0, 0) - 1.0) < 1e-15
    assert abs(boys(0, 0.0) - 1.0) < 1e-15


def test_hermite_integrals_within_their_bounds():
    rng = np.random.default_rng(5)
    worst = 0.0
    for _ in range(300):
        p = float(10 ** rng.uniform(-1, 2))
        X = rng.standard_normal(3)
        X *= rng.uniform(0, 5) / math.sqrt(p) / max(np.linalg.norm(X), 1e-300)
        for (t, u, v), r in hermite_r(p, X, 6).items():
            b = p ** ((t + u + v) / 2) * hermite_sup(t, u, v)
            worst = max(worst, abs(r) / b)
            assert abs(r) <= b * (1 + 1e-12), ((t, u, v), p, X, r, b)
    # The bound is not loose by orders of magnitude.
    assert worst > 0.05
