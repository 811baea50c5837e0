"""Angular tables (c3d-2015_b200/host/tables.c): known answers from mathematics.

* Gauss-Legendre nodes/weights equal numpy's leggauss to an ulp, sum of weights 2.
* Normalised associated Legendre functions match scipy (lpmv with normalisation).
* Real spherical harmonics are orthonormal under the tensor quadrature:
  sum_q w_q m_i m_j = delta_ij up to degree 2N (exactness of the rule).
* Weights sum to 4 pi; directions are unit vectors.
* Gaunt least squares reproduces m_i m_j = sum_k beta_ijk m2_k at every direction.
"""
import numpy as np
import pytest
from scipy.special import gammaln, lpmv


@pytest.mark.parametrize("n", [1, 2, 3, 12, 20, 28, 40])
def test_gauss_legendre(oracle, n):
    import ctypes
    dp = ctypes.POINTER(ctypes.c_double)
    L = oracle.L
    L.c3d_gauss_legendre.argtypes = [ctypes.c_int, dp, dp]
    mu, w = np.zeros(n), np.zeros(n)
    L.c3d_gauss_legendre(n, mu.ctypes.data_as(dp), w.ctypes.data_as(dp))
    x, ww = np.polynomial.legendre.leggauss(n)
    assert np.max(np.abs(mu - x)) <= 2.3e-16
    assert np.max(np.abs(w - ww)) <= 1e-14
    assert abs(w.sum() - 2.0) < 1e-14
    assert np.all(np.diff(mu) > 0)
    assert np.array_equal(mu, -mu[::-1])


def test_sph_plm(oracle):
    import ctypes
    L = oracle.L
    L.c3d_sph_plm.restype = ctypes.c_double
    L.c3d_sph_plm.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double]
    for l in range(15):
        for m in range(l + 1):
            for x in (-0.97, -0.5, 0.0, 0.3, 0.9):
                ref = np.sqrt((2 * l + 1) / (4 * np.pi) * np.exp(gammaln(l - m + 1) -
                                                                  gammaln(l + m + 1))) * lpmv(m, l, x)
                v = L.c3d_sph_plm(l, m, x)
                assert abs(v - ref) <= 1e-12 * max(1.0, abs(ref))


@pytest.mark.parametrize("N,Q", [(1, 8), (2, 12), (4, 20), (6, 28), (7, 20)])
def test_quadrature_orthonormal(oracle, N, Q):
    T = oracle.tables(N, Q)
    nq, nm, nm2 = T["nq"], T["nm"], T["nm2"]
    M = T["M"].reshape(nq, nm)
    M2 = T["M2"].reshape(nq, nm2)
    w = T["w"]
    assert abs(w.sum() - 4 * np.pi) < 1e-12
    om = np.stack([T["xi"], T["eta"], T["mu"]], 1)
    assert np.allclose(np.linalg.norm(om, axis=1), 1.0, atol=1e-15)
    G = (M * w[:, None]).T @ M
    assert np.abs(G - np.eye(nm)).max() < 1e-13
    if 2 * N < Q:
        G2 = (M2 * w[:, None]).T @ M2
        assert np.abs(G2 - np.eye(nm2)).max() < 1e-13
    # the first harmonic is the constant 1/(2 sqrt(pi))
    assert np.allclose(M[:, 0], 0.5 / np.sqrt(np.pi), rtol=1e-15)
    assert np.array_equal(M[:, :nm], M2[:, :nm])


def test_gaunt_identity(oracle):
    T = oracle.tables(2, 12, gaunt=True)
    nq, nm, nm2 = T["nq"], T["nm"], T["nm2"]
    M2 = T["M2"].reshape(nq, nm2)
    beta = T["beta"].reshape(nm, nm, nm2)
    prod = np.einsum("qi,qj->qij", M2[:, :nm], M2[:, :nm])
    recon = np.einsum("ijk,qk->qij", beta, M2)
    assert np.abs(prod - recon).max() < 1e-12
    row = T["betaRow"]
    assert row[-1] == np.count_nonzero(np.abs(beta) > 1e-13)
