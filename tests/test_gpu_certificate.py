"""The first-visit convergence certificate (c3d_set_certificate) is exact.

With the certificate, a cell's first Newton iteration starts with a probe pass (first-order
moments and the extreme values of e^{alpha.m}); a cell whose gradient and bounds show that
the full iteration would end it converged is finalized without forming or factoring its
Hessian. The full iteration would have produced the same multipliers, moments, iteration
counts, regularisation indices and statuses, so runs with and without the certificate must
agree bit for bit -- in the FP64 closure and in the mixed-precision one (with the ansatz
hand-off off, which only the certificate's probe pass feeds and which changes the flux by
rounding; test_gpu_handoff covers it). Workload: the 64^3
M_6 deck (49 moments, 1568 directions, gaussian pulse of width 0.02 over a 1e-10 floor),
three SSP-RK2 steps; most cells sit on the isotropic floor and are certified.
"""
import os

import numpy as np
import pytest

import c3d
from oracle_lib import deck_text

pytestmark = pytest.mark.gpu


def _run(tmp_path, mixed, certificate):
    deck = tmp_path / f"d{int(mixed)}{int(certificate)}.deck"
    kw = dict(NX=64, NY=64, NZ=64, MOMENT_ORDER=6, QUAD_ORDER=28, CFL_FACTOR=0.5,
              CROSS_SECTION=1.0, INIT_FLOOR=1e-10, GAUSS_SIGMA=0.02, INIT_COND="gaussian_psi",
              THETA=2.0, MN_TOL=1e-6, MN_BATCHED="true", MN_USE_GAUNT_COEF="true",
              MN_USE_GAUNT_SPARSE="true", REG_LADDER="0,1e-8,1e-6,1e-4,1e-2,1e-1",
              OMP_THREADS=os.cpu_count() or 1)
    if mixed:
        kw["MN_MIXED_PRECISION"] = "true"
    deck.write_text(deck_text(**kw))
    s = c3d.Solver(str(deck))
    c3d.check(c3d.lib().c3d_set_certificate(s.ctx_handle, int(certificate)), "certificate")
    c3d.check(c3d.lib().c3d_set_ansatz_handoff(s.ctx_handle, 0), "handoff")
    for _ in range(3):
        s.update(s.max_dt)
    s.sync()
    s.pull()
    A = s.arrays()
    out = dict(u=A["u"].copy(), a=A["alpha"].copy(), rec=s.records(), st=s.stats())
    s.close()
    return out


@pytest.mark.parametrize("mixed", [False, True])
def test_certificate_is_exact(tmp_path, mixed):
    on = _run(tmp_path, mixed, True)
    off = _run(tmp_path, mixed, False)
    assert np.array_equal(on["u"], off["u"])
    assert np.array_equal(on["a"], off["a"])
    for k in ("iters", "iterGamma", "regIndex", "status"):
        assert np.array_equal(on["rec"][k], off["rec"][k]), k
    assert on["st"].cells == off["st"].cells
    assert on["st"].totalIters == off["st"].totalIters
    assert off["st"].certified == 0
    # most first visits end on the certificate (the cell count also holds the face ghosts,
    # which are copied from their periodic images, not solved: 15% of this grid's cells)
    assert on["st"].certified > 0.8 * on["st"].cells, (on["st"].certified, on["st"].cells)
