"""The inequalities behind the first-iteration convergence certificate (after_probe), checked
in numpy on the benchmark's M_6 quadrature (28 mu x 56 phi, 1568 directions).

With w_q >= 0 and e_q = e^{alpha.m_q}, H = sum_q w_q e_q m_q m_q^T lies between e_min G and
e_max G, G = sum_q w_q m_q m_q^T the quadrature's Gram matrix, whose eigenvalues lie in the
Gershgorin interval [gramLo, gramHi] (computed as the context does, with the same relative
margin). Hence lambda_min(H) >= e_min gramLo, lambda_max(H) <= e_max gramHi, the 1-norm
condition number is at most nm e_max gramHi / (e_min gramLo), and |H^-1 g|_1 <=
sqrt(nm) |g|_2 / lambda_min(H). The certificate finalizes a cell only when these bounds keep
the full iteration's tests on the same side, with further factors of 2 and 4 for rounding.
"""
import numpy as np
import pytest

import c3d


def _gram_bounds(M, w):
    G = (M * w[:, None]).T @ M
    off = np.abs(G).sum(axis=1) - np.abs(np.diag(G))
    lo = (np.diag(G) - off).min() * (1.0 - 1e-9)
    hi = (np.diag(G) + off).max() * (1.0 + 1e-9)
    return lo, hi


@pytest.mark.parametrize("scale", [1e-3, 0.1, 1.0, 3.0])
def test_certificate_inequalities(scale):
    T = c3d.quadrature(6, 28)
    nm, nq = T["nm"], T["nq"]
    M = T["M"].reshape(nq, nm)
    w = T["w"]
    lo, hi = _gram_bounds(M, w)
    assert 0.9 < lo <= 1.0 <= hi < 1.1  # the quadrature integrates the basis products
    rng = np.random.default_rng(int(scale * 1000))
    for _ in range(20):
        a = rng.standard_normal(nm) * scale
        a[0] = -2.0
        e = np.exp(M @ a)
        H = (M * (w * e)[:, None]).T @ M
        ev = np.linalg.eigvalsh(H)
        emin, emax = e.min(), e.max()
        assert ev[0] >= emin * lo * (1 - 1e-12)
        assert ev[-1] <= emax * hi * (1 + 1e-12)
        Hi = np.linalg.inv(H)
        k1 = np.abs(H).sum(axis=0).max() * np.abs(Hi).sum(axis=0).max()
        assert k1 <= nm * emax * hi / (emin * lo) * (1 + 1e-9)
        g = rng.standard_normal(nm) * 1e-7
        d = Hi @ g
        assert np.abs(d).sum() <= np.sqrt(nm) * np.linalg.norm(g) / (emin * lo) * (1 + 1e-9)
