"""The closure's ansatz hand-off to the kinetic flux (c3d_set_ansatz_handoff).

A grid closure with the convergence certificate writes psi = e^{alpha.m_q} of every cell it
solves in its probe pass; face ghosts copy their images' values and cells whose multipliers
change after the probe are recomputed, and the next kinetic flux runs its stencil alone.
Here two solvers on the 24^3 M_6 deck advance two steps without the hand-off (identical
states), then one more step with and without it: the closures' records are identical, and
the flux divergence of the last stage and the moments agree to 1e-13 relative L2 (the
probe forms u_0 e^{alpha_scaled . m_q}, the flux's own ansatz e^{alpha . m_q} on the tensor
pipe: the same values up to rounding). Covered with face-ghost mirroring (face ghosts copied)
and without it (every cell probed), in FP64 and in the mixed closure; the third step has
cells that go past their probe visit, so the refresh list is exercised.
"""
import ctypes
import os

import numpy as np
import pytest

import c3d
from oracle_lib import deck_text

pytestmark = pytest.mark.gpu

LADDER = [0.0, 1e-8, 1e-6, 1e-4, 1e-2, 1e-1]


def _c2_deck():
    import importlib.util
    here = os.path.dirname(os.path.abspath(__file__))
    spec = importlib.util.spec_from_file_location("make_golden",
                                                  os.path.join(here, "golden", "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.c2_deck("gaussian_psi")


def _deck(tmp_path, n, mixed, name, dims=None):
    nx, ny, nz = dims or (n, n, n)
    kw = dict(NX=nx, NY=ny, NZ=nz, MOMENT_ORDER=6, QUAD_ORDER=28, CFL_FACTOR=0.5, CROSS_SECTION=1.0,
              INIT_FLOOR=1e-10, GAUSS_SIGMA=0.02, INIT_COND="gaussian_psi", THETA=2.0,
              MN_TOL=1e-6, MN_BATCHED="true", MN_USE_GAUNT_COEF="true",
              MN_USE_GAUNT_SPARSE="true", REG_LADDER=",".join(str(x) for x in LADDER),
              OMP_THREADS=os.cpu_count() or 1)
    if mixed:
        kw["MN_MIXED_PRECISION"] = "true"
    p = tmp_path / name
    p.write_text(deck_text(**kw))
    return str(p)


@pytest.mark.parametrize("dims", [None, (20, 18, 23)])
@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("mirror", [True, False])
def test_handoff_matches_formed_ansatz(tmp_path, mixed, mirror, dims):
    """dims: 24^3 (even nz: the face-ghost copy's paired z-face path and the staged stencil),
    or 20 x 18 x 23 (odd nz: the scalar z-face copies and the global-load stencil)."""
    L = c3d.lib()
    n = 24
    out = {}
    for handoff in (True, False):
        s = c3d.Solver(_deck(tmp_path, n, mixed, f"h{int(handoff)}.deck", dims))
        ctx = s.ctx_handle
        c3d.check(L.c3d_set_ghost_mirroring(ctx, int(mirror)), "mirroring")
        c3d.check(L.c3d_set_ansatz_handoff(ctx, 0), "handoff")
        for _ in range(2):
            s.update(s.max_dt)
        c3d.check(L.c3d_set_ansatz_handoff(ctx, int(handoff)), "handoff")
        s.update(s.max_dt)
        s.sync()
        s.pull()
        f = np.zeros(s.nall * s.nm)
        c3d.check(L.c3d_get_flux(ctx, f.ctypes.data_as(ctypes.c_void_p), 0), "get_flux")
        out[handoff] = (s.arrays()["u"].copy(), f, s.records())
        s.close()
    (u1, f1, r1), (u0, f0, r0) = out[True], out[False]
    assert np.array_equal(r1["iters"], r0["iters"])
    assert (r1["iters"] > 1).sum() > 0  # cells went past the probe: the refresh list ran
    ru = np.linalg.norm(u1 - u0) / np.linalg.norm(u0)
    rf = np.linalg.norm(f1 - f0) / np.linalg.norm(f0)
    assert ru < 1e-13 and rf < 1e-13, (ru, rf)


def test_handoff_c2_deck(tmp_path):
    """The M_4 64^3 checkerboard deck, whose first closure sends about half of the cells
    (face images among them) past their probe visit: one step with and without the hand-off
    agrees to 1e-13 (the refresh of changed cells precedes the face ghosts' copy of their
    images)."""
    L = c3d.lib()
    p = tmp_path / "c2.deck"
    p.write_text(_c2_deck())
    out = {}
    for handoff in (True, False):
        s = c3d.Solver(str(p))
        c3d.check(L.c3d_set_ansatz_handoff(s.ctx_handle, int(handoff)), "handoff")
        s.update(s.max_dt)
        s.sync()
        s.pull()
        out[handoff] = s.arrays()["u"].copy()
        s.close()
    ru = np.linalg.norm(out[True] - out[False]) / np.linalg.norm(out[False])
    assert ru < 1e-13, ru


def test_handoff_over_steps(tmp_path):
    """Three steps of the M_4 64^3 checkerboard deck (stage graphs, face-ghost mirroring) with
    and without the hand-off: from the second closure on, the probe pass writes psi only for
    face ghosts (the rest still holds the previous closure's final ansatz, which the closure
    starts from), and the stencil reads face ghosts at their periodic images. The ansatz values
    differ from the flux's own by rounding only: iteration counts of all six closures identical
    (no rounding ties on this deck), moments within 1e-12 relative L2."""
    L = c3d.lib()
    p = tmp_path / "c2.deck"
    p.write_text(_c2_deck())
    out = {}
    for handoff in (True, False):
        s = c3d.Solver(str(p))
        c3d.check(L.c3d_set_ansatz_handoff(s.ctx_handle, int(handoff)), "handoff")
        its = []
        for _ in range(3):
            for stage in (0, 1):
                c3d.check(L.c3d_stage(s.ctx_handle, stage, s.max_dt), "stage")
                s.sync()
                its.append(s.records()["iters"].copy())
        s.pull()
        out[handoff] = (s.arrays()["u"].copy(), its)
        s.close()
    (u1, i1), (u0, i0) = out[True], out[False]
    for k, (a, b) in enumerate(zip(i1, i0)):
        assert np.array_equal(a, b), (k, int((a != b).sum()))
    ru = np.linalg.norm(u1 - u0) / np.linalg.norm(u0)
    assert ru < 1e-12, ru
