"""Pins the C oracle (and the host's init()) to the reference CPU path itself,
compiled from its own sources into oracle/_ref/libc3dref.so.

* The host's init() mirror reproduces the reference's initial state, tables and
  dt bit for bit.
* The harness step (per-cell records) equals the reference's update() bit for bit.
* Kinetic flux, P_N moment flux, ghost fill and Euler stage of the oracle equal the
  reference bit for bit (same IEEE operations in the same order).
* Closure: per-cell Newton iteration counts equal the reference's except rounding
  ties (oracle_lib.tie_cells); one step from the reference's state agrees to 1e-12
  relative L2 whenever no tie changed a regularisation level.
"""
import os

import numpy as np
import pytest

import c3d
from oracle_lib import (REF_SO, deck_text, log_ties, make_opts, run_reference, tie_cells)

pytestmark = pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference build absent")

DECK_LADDER = [0.0, 1e-8, 1e-6, 1e-4, 1e-2, 1e-1]


def _write(tmp_path, text):
    p = tmp_path / "input.deck"
    p.write_text(text)
    return str(p)


@pytest.mark.parametrize("solver", ["mn", "pn"])
def test_host_init_matches_reference(tmp_path, solver):
    deck = deck_text(SOLVER=solver, NX=6, NY=7, NZ=5, MOMENT_ORDER=3, QUAD_ORDER=8,
                     GAUSS_SIGMA=0.3, INIT_FLOOR=1e-6, AX=-1.5, BX=1.5)
    ref = run_reference(deck, nsteps=0, want=("tables", "pnops"))
    host = c3d.Solver(_write(tmp_path, deck), host_only=True)
    A = host.arrays()
    assert np.array_equal(A["u"], ref["u0"])
    if solver == "mn":
        assert np.array_equal(A["alpha"], ref["alpha0"])
    else:
        assert np.array_equal(A["pnOps"], ref["pnops"])
    for k in ("M", "w", "xi", "eta", "mu"):
        assert np.array_equal(A[k], ref[k]), k
    assert np.array_equal(A["sigT"], ref["sigT"]) and np.array_equal(A["sigS"], ref["sigS"])
    assert host.max_dt == ref["dv"][3]
    assert (host.dx, host.dy, host.dz) == tuple(ref["dv"][:3])
    host.close()


def test_deck_errors_are_reported(tmp_path):
    text = deck_text().replace("MN_TOL 1e-8\n", "")
    with pytest.raises(c3d.C3DError, match="MN_TOL"):
        c3d.Solver(_write(tmp_path, text), host_only=True)
    with pytest.raises(c3d.C3DError, match="Solver type"):
        c3d.Solver(_write(tmp_path, deck_text(SOLVER="xn")), host_only=True)


def test_harness_step_equals_update():
    deck = deck_text(NX=6, NY=6, NZ=6)
    a = run_reference(deck, nsteps=2, record=True)
    b = run_reference(deck, nsteps=2, record=False)
    assert np.array_equal(a["u"], b["u"])
    assert np.array_equal(a["alpha"], b["alpha"])
    sa, sb = a["stats"], b["stats"]
    assert (sa[0], sa[1], sa[4]) == (sb[0], sb[1], sb[4])  # max iters, max gamma iters, solves
    assert np.allclose(sa[2:4], sb[2:4], rtol=1e-12)      # running means (order of accumulation)
    assert sa[5:10] == sb[5:10]                            # regularisation histogram


def _grid(oracle, ref):
    iv, dv = ref["iv"], ref["dv"]
    return oracle.grid(iv[0], iv[1], iv[2], iv[3], iv[5], dv[0], dv[1], dv[2], dv[4])


def test_flux_and_stages_bit_exact(oracle):
    deck = deck_text(NX=8, NY=6, NZ=7, MOMENT_ORDER=2, QUAD_ORDER=12, THETA=1.5)
    ref = run_reference(deck, nsteps=2, want=("flux",))
    T = oracle.tables(2, 12)
    g = _grid(oracle, ref)
    fo = oracle.flux_kinetic(g, T, ref["alpha"])
    n = (g.nx + 4, g.ny + 4, g.nz + 4, g.nm)
    inner = (slice(2, g.nx + 2), slice(2, g.ny + 2), slice(2, g.nz + 2))
    assert np.array_equal(fo.reshape(n)[inner], ref["flux"].reshape(n)[inner])
    # ghost fill + euler on the reference's state
    u = ref["u"].copy()
    oracle.ghost_fill(g, u)
    rng = np.random.default_rng(0)
    flux = rng.standard_normal(u.shape)
    st, ss = 1.0 + rng.random(ref["sigT"].shape), rng.random(ref["sigT"].shape)
    u2 = u.copy()
    oracle.euler(g, u2, flux, st, ss, 0.01)
    ur, fr = u.reshape(n), flux.reshape(n)
    exp = ur.copy()
    sti, ssi = st.reshape(n[:3])[inner], ss.reshape(n[:3])[inner]
    exp[inner + (0,)] = ur[inner + (0,)] * (1.0 + 0.01 * ssi - 0.01 * sti) - 0.01 * fr[inner + (0,)]
    exp[inner + (slice(1, None),)] = (ur[inner + (slice(1, None),)] * (1.0 - 0.01 * sti)[..., None]
                                      - 0.01 * fr[inner + (slice(1, None),)])
    assert np.array_equal(u2.reshape(n), exp)


@pytest.mark.parametrize("kinetic", [0, 1])
def test_pn_steps_bit_exact(oracle, kinetic):
    deck = deck_text(SOLVER="pn", NX=7, NY=6, NZ=8, MOMENT_ORDER=3, QUAD_ORDER=8,
                     PN_USE_KINETIC_FLUX=kinetic, INIT_COND="smooth")
    ref = run_reference(deck, nsteps=3, want=("pnops",))
    T = oracle.tables(3, 8, pn=True)
    assert np.array_equal(T["pnops"], ref["pnops"])
    g = _grid(oracle, ref)
    u = ref["u0"].copy()
    alpha = np.zeros_like(u)
    opts = make_opts(g.nm, g.nq)
    for _ in range(3):
        oracle.step(g, opts, T, u, alpha, ref["sigT"], ref["sigS"], ref["dv"][3], solver=0,
                    pn_kinetic=kinetic, records=False)
    assert np.array_equal(u, ref["u"])


@pytest.mark.parametrize("batched,ladder,gaunt", [(True, None, 0), (False, None, 0),
                                                   (True, DECK_LADDER, 0), (True, None, 2),
                                                   (True, None, 1)])
def test_closure_steps_vs_reference(oracle, batched, ladder, gaunt):
    """gaunt: 0 direct H, 1 dense Gaunt, 2 sparse Gaunt (MN_USE_GAUNT_COEF/_SPARSE)."""
    deck = deck_text(NX=8, NY=8, NZ=8, MOMENT_ORDER=2, QUAD_ORDER=12,
                     MN_BATCHED="true" if batched else "false",
                     MN_USE_GAUNT_COEF="true" if gaunt else "false",
                     MN_USE_GAUNT_SPARSE="true" if gaunt == 2 else "false",
                     # the reference exhausts its ladder in the Gaunt modes at 1e-8 here
                     MN_TOL="1e-6" if gaunt else "1e-8")
    nsteps = 3
    ref = run_reference(deck, nsteps=nsteps, ladder=ladder, want=("snapshots",))
    T = oracle.tables(2, 12, gaunt=bool(gaunt))
    g = _grid(oracle, ref)
    iv, dv = ref["iv"], ref["dv"]
    opts = make_opts(g.nm, g.nq, nm2=25, batched=batched, max_iter=iv[11], tol=dv[5],
                     tol_gamma=dv[6], cond_h_max=dv[7], ladder=ladder, hess_mode=gaunt)
    nall = (g.nx + 4) * (g.ny + 4) * (g.nz + 4)
    exact_steps = 0
    total_mism = 0
    for s in range(nsteps):
        u, a = (x.copy() for x in ref["snapshots"][s])
        bad, rec = oracle.step(g, opts, T, u, a, ref["sigT"], ref["sigS"], dv[3])
        assert bad == 0
        it_ref, _, reg_ref = ref["iters"][s]
        ties = tie_cells(rec)
        mism = rec["totalIter"] != it_ref
        log_ties(f"oracle vs reference, step {s}", ties, mism)
        assert not (mism & ~ties).any(), np.nonzero(mism & ~ties)[0][:10]
        total_mism += int(mism.sum())
        if (rec["regIndex"] == reg_ref).all():
            nxt = ref["snapshots"][s + 1][0] if s + 1 < nsteps else ref["u"]
            sh = (g.nx + 4, g.ny + 4, g.nz + 4, g.nm)
            inner = (slice(2, g.nx + 2), slice(2, g.ny + 2), slice(2, g.nz + 2))
            x, y = u.reshape(sh)[inner], nxt.reshape(sh)[inner]
            rel = np.linalg.norm(x - y) / np.linalg.norm(y)
            assert rel < 1e-12, (s, rel)
            exact_steps += 1
    assert exact_steps >= 1
    assert total_mism <= 0.02 * 2 * nall * nsteps


def test_standalone_closure_vs_reference(oracle):
    """Standalone unbatched opt() on random realizable moment vectors (u = <m e^{alpha.m}>)."""
    import ctypes
    import multiprocessing as mp

    from oracle_lib import _ref_standalone  # noqa: F401  (defined below)
    N, Q = 3, 12
    T = oracle.tables(N, Q)
    nm, nq = T["nm"], T["nq"]
    rng = np.random.default_rng(5)
    n = 400
    alpha_true = rng.standard_normal((n, nm)) * np.exp(rng.uniform(np.log(0.1), np.log(2), (n, 1)))
    alpha_true[:, 0] = 0.0
    M = T["M"].reshape(nq, nm)
    E = np.exp(alpha_true @ M.T)
    u = (E * T["w"]) @ M
    u = u / u[:, :1]
    a0 = np.zeros((n, nm))
    a0[:, 0] = np.sqrt(4 * np.pi) * np.log(u[:, 0] / np.sqrt(4 * np.pi))
    ctx = mp.get_context("spawn")
    r, w = ctx.Pipe(duplex=False)
    p = ctx.Process(target=_ref_standalone, args=(w, nm, (2 * N + 1) ** 2, nq, u, a0, T["w"],
                                                   T["M"], T["M2"], 100, 1e-8, 1e10))
    p.start()
    w.close()
    it_ref, a_ref = r.recv()
    p.join()
    uo, ao = u.copy(), a0.copy()
    out = oracle.closure(make_opts(nm, nq, batched=False), T, uo, ao)
    ties = tie_cells(out)
    mism = out["totalIter"] != it_ref
    log_ties("oracle vs reference opt(), unbatched", ties, mism)
    assert not (mism & ~ties).any()
    ok = ~ties & (out["regIndex"] == 0)
    assert np.abs(ao[ok] - a_ref[ok]).max() <= 1e-10 * max(1.0, np.abs(a_ref).max())
