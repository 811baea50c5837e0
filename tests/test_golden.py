"""Oracle and B200 path against golden outputs of the reference CPU path
(tests/golden/make_golden.py; decks described there).

* P_N (no closure): bit-exact for the oracle; 1e-13 relative L2 for the GPU path.
* M_2 16^3 at MN_TOL 1e-6 (no rounding ties at this tolerance): per-cell iteration
  counts and ladder indices of the first two steps identical; moments after 2 and
  20 steps within 1e-12 relative L2.
"""
import os

import numpy as np
import pytest

import c3d
from oracle_lib import make_opts, tie_cells

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
sys_path_added = False


def _golden_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden",
                                                  os.path.join(GOLD, "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _deck(tmp_path, text):
    p = tmp_path / "input.deck"
    p.write_text(text)
    return str(p)


def _pn_deck():
    from oracle_lib import deck_text
    return deck_text(SOLVER="pn", NX=8, NY=6, NZ=7, MOMENT_ORDER=3, QUAD_ORDER=8,
                     INIT_COND="smooth", PN_USE_KINETIC_FLUX=0)


def test_oracle_pn_golden(oracle, tmp_path):
    G = np.load(os.path.join(GOLD, "pn_p3_8.npz"))
    host = c3d.Solver(_deck(tmp_path, _pn_deck()), host_only=True)
    A = host.arrays()
    T = oracle.tables(3, 8, pn=True)
    g = oracle.grid(8, 6, 7, 16, 128, host.dx, host.dy, host.dz, 2.0)
    u = A["u"].copy()
    alpha = np.zeros_like(u)
    for _ in range(5):
        oracle.step(g, make_opts(16, 128), T, u, alpha, A["sigT"], A["sigS"], host.max_dt,
                    solver=0, records=False)
    assert host.max_dt == float(G["dt"])
    assert np.array_equal(u.reshape(12, 10, 11, 16)[2:10, 2:8, 2:9], G["u_step5"])


def test_oracle_c1_golden(oracle, tmp_path):
    mg = _golden_module()
    G = np.load(os.path.join(GOLD, "c1_m2_16.npz"))
    host = c3d.Solver(_deck(tmp_path, mg.c1_deck("gaussian_psi")), host_only=True)
    A = host.arrays()
    T = oracle.tables(2, 12)
    n = 16
    g = oracle.grid(n, n, n, 9, 288, host.dx, host.dy, host.dz, 2.0)
    opts = make_opts(9, 288, tol=1e-6, ladder=mg.C1_LADDER)
    u, a = A["u"].copy(), A["alpha"].copy()
    inner = (slice(2, n + 2),) * 3
    for s in range(20):
        bad, rec = oracle.step(g, opts, T, u, a, A["sigT"], A["sigS"], host.max_dt)
        assert bad == 0
        if s < 2:
            assert not tie_cells(rec).any()
            assert np.array_equal(rec["totalIter"], G["iters"][s])
            assert np.array_equal(rec["regIndex"], G["reg"][s])
        if s in (1, 19):
            ref = G["u_step2"] if s == 1 else G["u_step20"]
            x = u.reshape(n + 4, n + 4, n + 4, 9)[inner]
            rel = np.linalg.norm(x - ref) / np.linalg.norm(ref)
            assert rel < 1e-12, (s, rel)


@pytest.mark.gpu
def test_gpu_c1_golden(tmp_path):
    mg = _golden_module()
    G = np.load(os.path.join(GOLD, "c1_m2_16.npz"))
    s = c3d.Solver(_deck(tmp_path, mg.c1_deck("gaussian_psi")))
    n, nall = 16, s.nall
    inner = (slice(2, n + 2),) * 3
    for k in range(20):
        s.update(s.max_dt)
        if k == 1:
            s.sync()
            rec = s.records()
            assert np.array_equal(rec["iters"], G["iters"][1][nall:])
            assert np.array_equal(rec["regIndex"], G["reg"][1][nall:])
        if k in (1, 19):
            s.pull()
            x = s.arrays()["u"].reshape(n + 4, n + 4, n + 4, 9)[inner]
            ref = G["u_step2"] if k == 1 else G["u_step20"]
            rel = np.linalg.norm(x - ref) / np.linalg.norm(ref)
            assert rel < 1e-12, (k, rel)
    st = s.stats()
    assert st.failed == 0
    assert st.cells == 2 * 20 * nall
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("gaunt_on_device", [False, True])
def test_gpu_c2_golden(tmp_path, gaunt_on_device):
    """The M_4 64^3 deck with the sigma checkerboard (Gaunt sparse Hessian, MN_TOL 1e-6)
    against the reference's own CPU path: per-cell Newton iteration counts and ladder indices
    of all six closures of three steps identical (ghost cells included); after steps 1 and 3
    the interior moments of the 4096 sample cells and the moment sums over every x-, y- and
    z-plane within 1e-12 relative L2. Also with the Gaunt tables built on the device
    (MN_GAUNT_ON_DEVICE true), whose values differ from the host build's at rounding level."""
    mg = _golden_module()
    G = np.load(os.path.join(GOLD, "c2_m4_64.npz"))
    deck = mg.c2_deck("gaussian_psi") + ("MN_GAUNT_ON_DEVICE true\n" if gaunt_on_device else "")
    s = c3d.Solver(_deck(tmp_path, deck))
    L = c3d.lib()
    dt = s.max_dt
    assert dt == float(G["dt"])
    nall = s.nall
    for step in range(3):
        for stage in range(2):
            c3d.check(L.c3d_stage(s.ctx_handle, stage, dt), "c3d_stage")
            s.sync()
            rec = s.records()
            ref_it = G["iters"][step][stage * nall:(stage + 1) * nall]
            ref_rg = G["reg"][step][stage * nall:(stage + 1) * nall]
            mism = np.nonzero(rec["iters"] != ref_it)[0]
            assert len(mism) == 0, (step, stage, len(mism), mism[:8])
            assert np.array_equal(rec["regIndex"], ref_rg), (step, stage)
            assert (rec["status"] == 0).all()
        if step in (0, 2):
            s.pull()
            got = mg.c2_summary(s.arrays()["u"])
            for k in ("sample", "sx", "sy", "sz"):
                ref = G[f"step{step + 1}_{k}"]
                rel = np.linalg.norm(got[k] - ref) / np.linalg.norm(ref)
                assert rel < 1e-12, (step, k, rel)
    s.close()


@pytest.mark.gpu
def test_gpu_pn_golden(tmp_path):
    G = np.load(os.path.join(GOLD, "pn_p3_8.npz"))
    s = c3d.Solver(_deck(tmp_path, _pn_deck()))
    for _ in range(5):
        s.update(s.max_dt)
    s.sync()
    s.pull()
    x = s.arrays()["u"].reshape(12, 10, 11, 16)[2:10, 2:8, 2:9]
    ref = G["u_step5"]
    rel = np.linalg.norm(x - ref) / np.linalg.norm(ref)
    assert rel < 1e-13, rel
    s.close()


@pytest.mark.gpu
def test_gpu_pn_kinetic_flux_matches_oracle(oracle, tmp_path):
    """P_N with the kinetic flux (PN_USE_KINETIC_FLUX 1, src/update.cpp:242-245): the ansatz
    is psi = alpha.m_q with u standing in for alpha; three steps against the oracle."""
    from oracle_lib import deck_text, make_opts
    s = c3d.Solver(_deck(tmp_path, deck_text(SOLVER="pn", NX=8, NY=6, NZ=7, MOMENT_ORDER=3,
                                              QUAD_ORDER=8, INIT_COND="smooth",
                                              PN_USE_KINETIC_FLUX=1)))
    s.pull()
    A = s.arrays()
    u = A["u"].copy()
    alpha = np.zeros_like(u)
    T = oracle.tables(3, 8, pn=True)
    g = oracle.grid(s.nx, s.ny, s.nz, s.nm, s.nq, s.dx, s.dy, s.dz, s.theta)
    opts = make_opts(s.nm, s.nq)
    for _ in range(3):
        s.update(s.max_dt)
        oracle.step(g, opts, T, u, alpha, A["sigT"], A["sigS"], s.max_dt, solver=0,
                    pn_kinetic=1, records=False)
    s.sync()
    s.pull()
    x = s.arrays()["u"].reshape(s.nx + 4, s.ny + 4, s.nz + 4, s.nm)[2:-2, 2:-2, 2:-2]
    y = u.reshape(s.nx + 4, s.ny + 4, s.nz + 4, s.nm)[2:-2, 2:-2, 2:-2]
    rel = np.linalg.norm(x - y) / np.linalg.norm(y)
    assert rel < 1e-13, rel
    s.close()
