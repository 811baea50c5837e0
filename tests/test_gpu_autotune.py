"""The flux autotuner (c3d_autotune) picks among direction chunks and z run lengths that all
give the same flux bit for bit: partial sums over directions accumulate in the same order
whatever the chunking (they are stored exactly between chunks), and both run lengths form
the same per-cell operations. 64^3 M_4 context (25 moments, 288 directions) with random
multipliers; the candidates are 288, 160 and 96 directions per chunk and runs of 64 and 32
cells."""
import numpy as np
import pytest

import c3d

pytestmark = pytest.mark.gpu


def test_autotune_keeps_the_flux():
    T = c3d.quadrature(4, 12)
    n, nm = 64, 25
    M = T["M"].reshape(T["nq"], -1)
    x = c3d.Context(nx=n, ny=n, nz=n, nm=nm, nq=T["nq"], dx=2 / n, dy=2 / n, dz=2 / n, M=M,
                    w=T["w"], xi=T["xi"], eta=T["eta"], mu=T["mu"])
    a = np.random.default_rng(4).standard_normal(((n + 4) ** 3, nm)) * 0.05
    a[:, 0] = -3
    sig = np.ones((n + 4) ** 3)
    x.set_state(u=a.ravel(), alpha=a.ravel(), sig_t=sig, sig_s=sig)
    x.flux_kinetic(0)
    x.sync()
    f0 = x.get_flux().copy()
    q, r, ms = x.autotune()
    assert q in (288, 160, 96) and r in (0, 32) and ms > 0
    x.flux_kinetic(0)
    x.sync()
    f1 = x.get_flux()
    x.close()
    assert np.array_equal(f0, f1)
    assert np.abs(f0).max() > 0
