"""The sign test of sign(lambda2) rho (src/evaluator.cpp:156-161).

The device decides lambda2 < 0 from the signs of the characteristic
polynomial's coefficients e1 = tr H, e2 (sum of principal 2x2 minors) and
e3 = det H wherever all three stand clear of zero, and falls back to its
Jacobi eigenvalue elsewhere.  This restates that rule in numpy and checks it
against numpy's eigenvalues on random, nearly singular and degenerate
Hessians: wherever the margins hold, the rule must give the sign of the
middle eigenvalue.
"""
import numpy as np


def _rule(h):
    a, b, c, d, e, f = h
    m = np.max(np.abs(h))
    ex = np.frexp(m)[1] - 1  # ilogb
    a, b, c, d, e, f = (np.ldexp(x, -ex) for x in (a, b, c, d, e, f))
    e1 = a + d + f
    e2 = (a * d - b * b) + (a * f - c * c) + (d * f - e * e)
    e3 = a * (d * f - e * e) - b * (b * f - c * e) + c * (b * e - c * d)
    s2 = (a * a + d * d + f * f) + 2.0 * ((b * b + c * c) + e * e)
    k2 = 1e-16
    if e1 * e1 > k2 * s2 and e2 * e2 > k2 * s2 * s2 and e3 * e3 > k2 * s2 * s2 * s2:
        return bool(e1 < 0.0 and e2 > 0.0) if e3 < 0.0 else not (e1 > 0.0 and e2 > 0.0)
    return None  # the Jacobi eigenvalue decides


def _middle(h):
    a, b, c, d, e, f = h
    return np.linalg.eigvalsh(np.array([[a, b, c], [b, d, e], [c, e, f]]))[1]


def test_rule_matches_eigenvalues():
    rng = np.random.default_rng(7)
    decided = 0
    cases = []
    for scale in (1e-120, 1e-6, 1.0, 1e8, 1e150):
        for _ in range(4000):
            cases.append(rng.standard_normal(6) * scale)
    # Nearly singular: one eigenvalue tiny, of either sign.
    for _ in range(4000):
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        lam = rng.standard_normal(3)
        lam[rng.integers(3)] *= 10.0 ** rng.uniform(-14, -2)
        H = (q * lam) @ q.T
        cases.append(np.array([H[0, 0], H[0, 1], H[0, 2], H[1, 1], H[1, 2], H[2, 2]]))
    # Degenerate and diagonal cases.
    cases += [np.array(v, dtype=float) for v in ([1, 0, 0, 1, 0, 1], [-1, 0, 0, -1, 0, -1], [-1, 0, 0, 2, 0, 3],
                                                 [1, 0, 0, -2, 0, -3], [0, 0, 0, 1, 0, -1], [2, 1, 0, 2, 0, -5])]
    for h in cases:
        r = _rule(h)
        if r is None:
            continue
        decided += 1
        assert r == (_middle(h) < 0.0), h
    assert decided > 0.9 * len(cases)
