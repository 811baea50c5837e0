"""GPU parity of the B200 kernels against the C oracle on identical inputs.

Tolerances:
* ghost fill, Euler stage, RK copy/average: bit-exact (same unfused operations);
* kinetic flux: 1e-13 relative L2 (directional sums reordered by nothing, but
  exp() and fused multiply-adds differ from the CPU by ulps);
* closure: identical per-cell iteration counts except rounding ties (decisions
  the oracle took by a margin below two FP64 evaluations' disagreement, see
  oracle_lib.tie_cells); multipliers of the other cells within 1e-10 relative.
"""
import numpy as np
import pytest

import c3d
from oracle_lib import log_ties, make_opts, tie_cells

pytestmark = pytest.mark.gpu


def _setup(oracle, N=2, Q=12, n=8, sigma=0.2, floor=1e-4, steps_before=0, batched=True, ladder=None):
    """Initial state of a gaussian deck (reference init formulas), optionally advanced
    by the oracle so that many cells are anisotropic."""
    T = oracle.tables(N, Q)
    nm, nq = T["nm"], T["nq"]
    nx = ny = nz = n
    dx = 2.0 / n
    nall = (n + 4) ** 3
    u = np.zeros((nall, nm))
    idx = np.arange(n + 4)
    x = -1 + (idx - 2) * dx + dx / 2.0
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    f1 = 1.0 / (sigma * np.sqrt(2.0 * np.pi))
    G = f1 * f1 * f1 * np.exp(-(X * X + Y * Y + Z * Z) / (2.0 * sigma * sigma))
    u[:, 0] = np.maximum(floor, (G * 2.0 * np.sqrt(np.pi)).ravel())
    alpha = np.zeros((nall, nm))
    alpha[:, 0] = np.sqrt(4.0 * np.pi) * np.log(u[:, 0] / np.sqrt(4.0 * np.pi))
    sig = np.ones(nall)
    g = oracle.grid(n, n, n, nm, nq, dx, dx, dx, 2.0)
    opts = make_opts(nm, nq, batched=batched, ladder=ladder)
    dt = 0.5 * (2.0 / 4.0) / (3.0 / dx)
    u = u.ravel()
    alpha = alpha.ravel()
    for _ in range(steps_before):
        oracle.step(g, opts, T, u, alpha, sig, sig, dt, records=False)
    return dict(T=T, g=g, opts=opts, u=u, alpha=alpha, sig=sig, dt=dt, n=n, dx=dx, nm=nm, nq=nq,
                nall=nall, batched=batched, ladder=ladder)


def _ctx(S, **kw):
    T = S["T"]
    ladder = S["ladder"] or (0.0, 1e-3, 1e-2, 1e-1, 5e-1)
    return c3d.Context(nx=S["n"], ny=S["n"], nz=S["n"], nm=S["nm"], nq=S["nq"], dx=S["dx"],
                       dy=S["dx"], dz=S["dx"], M=T["M"], w=T["w"], xi=T["xi"], eta=T["eta"],
                       mu=T["mu"], batched=S["batched"], ladder=ladder, **kw)


def test_ghost_fill_and_euler_bit_exact(oracle):
    S = _setup(oracle, steps_before=1)
    ctx = _ctx(S)
    rng = np.random.default_rng(1)
    u = S["u"] + rng.standard_normal(S["u"].shape) * 1e-3
    flux = rng.standard_normal(S["u"].shape)
    sig_t = 1.0 + rng.random(S["nall"])
    sig_s = rng.random(S["nall"])
    ctx.set_state(u=u, alpha=S["alpha"], sig_t=sig_t, sig_s=sig_s)
    ctx.ghost_fill()
    ctx.sync()
    ug, _ = ctx.get_state()
    uo = u.copy()
    oracle.ghost_fill(S["g"], uo)
    assert np.array_equal(ug, uo)


def test_kinetic_flux_matches_oracle(oracle):
    S = _setup(oracle, steps_before=2)
    ctx = _ctx(S)
    ctx.set_state(u=S["u"], alpha=S["alpha"], sig_t=S["sig"], sig_s=S["sig"])
    ctx.flux_kinetic(0)
    ctx.sync()
    fg = ctx.get_flux()
    fo = oracle.flux_kinetic(S["g"], S["T"], S["alpha"])
    n = S["n"]
    nm = S["nm"]
    inner = (slice(2, n + 2),) * 3
    fg = fg.reshape(n + 4, n + 4, n + 4, nm)[inner]
    fo = fo.reshape(n + 4, n + 4, n + 4, nm)[inner]
    rel = np.linalg.norm(fg - fo) / np.linalg.norm(fo)
    assert rel < 1e-13, rel


@pytest.mark.parametrize("batched", [True, False])
def test_closure_matches_oracle(oracle, batched):
    S = _setup(oracle, steps_before=2, batched=batched)
    ctx = _ctx(S)
    ctx.set_state(u=S["u"], alpha=S["alpha"], sig_t=S["sig"], sig_s=S["sig"])
    ctx.closure()
    ctx.sync()
    ug, ag = ctx.get_state()
    rec = ctx.records()
    nm = S["nm"]
    uo = S["u"].reshape(-1, nm).copy()
    ao = S["alpha"].reshape(-1, nm).copy()
    out = oracle.closure(S["opts"], S["T"], uo, ao)
    assert (rec["status"] == 0).all()
    ties = tie_cells(out)
    mism = rec["iters"] != out["totalIter"]
    log_ties(f"test_closure_matches_oracle[batched={batched}]", ties, mism)
    assert not (mism & ~ties).any(), np.nonzero(mism & ~ties)[0][:10]
    ok = ~ties & (rec["regIndex"] == out["regIndex"])
    ag = ag.reshape(-1, nm)
    rel = np.linalg.norm(ag[ok] - ao[ok], axis=1) / np.linalg.norm(ao[ok], axis=1)
    assert rel.max() < 1e-10, rel.max()
    assert mism.sum() <= 0.02 * len(mism)


def test_step_matches_oracle_without_ties(oracle):
    """At MN_TOL 1e-6 the last Newton steps sit far above the rounding level of the
    Armijo test, so no decision is a tie: whole RK2 steps agree to rounding."""
    S = _setup(oracle, steps_before=1)
    S["opts"] = make_opts(S["nm"], S["nq"], tol=1e-6)
    ctx = _ctx(S, tol=1e-6)
    ctx.set_state(u=S["u"], alpha=S["alpha"], sig_t=S["sig"], sig_s=S["sig"])
    uo, ao = S["u"].copy(), S["alpha"].copy()
    n, nm = S["n"], S["nm"]
    inner = (slice(2, n + 2),) * 3
    for _ in range(3):
        ctx.step(S["dt"])
        ctx.sync()
        bad, rec = oracle.step(S["g"], S["opts"], S["T"], uo, ao, S["sig"], S["sig"], S["dt"])
        assert not tie_cells(rec).any()
    ug, ag = ctx.get_state()
    a = ug.reshape(n + 4, n + 4, n + 4, nm)[inner]
    b = uo.reshape(n + 4, n + 4, n + 4, nm)[inner]
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert rel < 1e-12, rel


def test_step_stages_match_oracle(oracle):
    """MN_TOL 1e-8: stage by stage, the closure's iteration counts match except ties; after
    a stage whose tie changed a regularisation level, both sides continue from the oracle's
    state so later stages are still compared on identical inputs."""
    S = _setup(oracle, steps_before=1)
    ctx = _ctx(S)
    n, nm, g, T = S["n"], S["nm"], S["g"], S["T"]
    inner = (slice(2, n + 2),) * 3
    u, a = S["u"].copy(), S["alpha"].copy()
    ctx.set_state(u=u, alpha=a, sig_t=S["sig"], sig_s=S["sig"])
    compared = 0
    for step in range(2):
        uold = u.copy()
        for stage in range(2):
            ctx.ghost_fill()
            oracle.ghost_fill(g, u)
            ctx.closure()
            ctx.sync()
            ur, ar = u.reshape(-1, nm), a.reshape(-1, nm)
            out = oracle.closure(S["opts"], T, ur, ar)
            rec = ctx.records()
            ties = tie_cells(out)
            mism = rec["iters"] != out["totalIter"]
            log_ties("test_step_stages_match_oracle", ties, mism)
            assert not (mism & ~ties).any()
            if (rec["regIndex"] != out["regIndex"]).any():
                ctx.set_state(u=u, alpha=a)  # continue from the oracle's state
            else:
                ug, ag = ctx.get_state()
                ok = np.repeat(~ties, nm)
                assert np.abs(ag - a)[ok].max() <= 1e-9 * np.abs(a).max()
                ctx.set_state(u=u, alpha=a)
                compared += 1
            ctx.flux_kinetic(0)
            ctx.sync()
            fo = oracle.flux_kinetic(g, T, a)
            fg = ctx.get_flux()
            fi = lambda f: f.reshape(n + 4, n + 4, n + 4, nm)[inner]
            assert np.linalg.norm(fi(fg) - fi(fo)) <= 1e-13 * np.linalg.norm(fi(fo))
            ctx.euler(S["dt"])
            ctx.sync()
            oracle.euler(g, u, fo, S["sig"], S["sig"], S["dt"])
            ug, _ = ctx.get_state()
            assert np.linalg.norm(fi(ug) - fi(u)) <= 1e-14 * np.linalg.norm(fi(u))
            ctx.set_state(u=u)
        u_i = u.reshape(n + 4, n + 4, n + 4, nm)
        o_i = uold.reshape(n + 4, n + 4, n + 4, nm)
        u_i[inner] = 0.5 * (u_i[inner] + o_i[inner])
        ctx.set_state(u=u)
    assert compared >= 1


def test_step_equals_stage_sequence(oracle):
    """c3d_step is exactly the stage sequence of update() (same kernels, bit for bit)."""
    S = _setup(oracle, steps_before=1)
    A, B = _ctx(S), _ctx(S)
    for c in (A, B):
        c.set_state(u=S["u"], alpha=S["alpha"], sig_t=S["sig"], sig_s=S["sig"])
    A.step(S["dt"])
    A.sync()
    n, nm = S["n"], S["nm"]
    uB, aB = B.get_state()
    uold = uB.copy()
    for _ in range(2):
        B.ghost_fill()
        B.closure()
        B.flux_kinetic(0)
        B.euler(S["dt"])
    B.sync()
    uB, aB = B.get_state()
    inner = (slice(2, n + 2),) * 3
    ub = uB.reshape(n + 4, n + 4, n + 4, nm)
    ob = uold.reshape(n + 4, n + 4, n + 4, nm)
    ub[inner] = 0.5 * (ub[inner] + ob[inner])
    uA, aA = A.get_state()
    assert np.array_equal(uA, ub.ravel())
    assert np.array_equal(aA, aB)


def test_reference_entry_points(oracle):
    """solveH_cuda / solveFluxKinetic_cuda with the reference's signatures (host buffers)."""
    import ctypes
    S = _setup(oracle, steps_before=1)
    T, nm, nq = S["T"], S["nm"], S["nq"]
    L = c3d.lib()
    dp = ctypes.POINTER(ctypes.c_double)
    B = 50
    al = S["alpha"].reshape(-1, nm)[:B].copy()
    al[:, 0] -= np.log(np.maximum(S["u"].reshape(-1, nm)[:B, 0], 1e-300)) * 2 * np.sqrt(np.pi)
    L.solveHInit_cuda(nm, 0, nq, B, T["w"].ctypes.data_as(dp), T["M"].ctypes.data_as(dp), None,
                      None, None, None, None, 0)
    hs = np.zeros(B * nm * nm)
    L.solveH_cuda(nm, 0, nq, B, al.ctypes.data_as(dp), hs.ctypes.data_as(dp), 0, 0)
    hs = hs.reshape(B, nm, nm)
    for b in range(B):
        ho = oracle.hessian(S["opts"], T, al[b].copy())
        assert np.allclose(hs[b], ho, rtol=1e-13, atol=1e-15 * np.abs(ho).max())
    n = S["n"]
    flux = np.zeros(S["nall"] * nm)
    a = S["alpha"].copy()
    L.solveFluxKinetic_cuda(n + 4, n + 4, n + 4, nm, nq, S["dx"], S["dx"], S["dx"],
                            a.ctypes.data_as(dp), flux.ctypes.data_as(dp),
                            T["xi"].ctypes.data_as(dp), T["eta"].ctypes.data_as(dp),
                            T["mu"].ctypes.data_as(dp), T["w"].ctypes.data_as(dp),
                            T["M"].ctypes.data_as(dp), 0)
    fo = oracle.flux_kinetic(S["g"], T, S["alpha"])
    inner = (slice(2, n + 2),) * 3
    fg = flux.reshape(n + 4, n + 4, n + 4, nm)
    assert np.abs(fg).sum() > 0
    rel = np.linalg.norm(fg[inner] - fo.reshape(fg.shape)[inner]) / np.linalg.norm(fo)
    assert rel < 1e-13
    ghost = np.ones(fg.shape[:3], bool)
    ghost[inner] = False
    assert (fg[ghost] == 0).all()


@pytest.mark.parametrize("N,Q", [(2, 12), (4, 12), (6, 10), (7, 12)])
def test_reference_solveH_gaunt(oracle, N, Q):
    """solveH_cuda with useGaunt = 1 (the reference deck's default, MN_USE_GAUNT_COEF true),
    dense beta (useGauntSparse 0) and CSR beta (1), against the oracle's Gaunt Hessian
    (src/opt/fobj.cpp:34-102) to 1e-13; the batch is ragged (not a multiple of 8)."""
    import ctypes
    T = oracle.tables(N, Q, gaunt=True)
    nm, nm2, nq = T["nm"], T["nm2"], T["nq"]
    L = c3d.lib()
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    B = 53
    rng = np.random.default_rng(N)
    al = rng.standard_normal((B, nm)) * 0.3
    al[:, 0] = rng.uniform(-2.0, 1.0, B)
    L.solveHInit_cuda(nm, nm2, nq, B, T["w"].ctypes.data_as(dp), T["M"].ctypes.data_as(dp),
                      T["M2"].ctypes.data_as(dp), T["beta"].ctypes.data_as(dp),
                      T["betaVal"].ctypes.data_as(dp), T["betaCol"].ctypes.data_as(ip),
                      T["betaRow"].ctypes.data_as(ip), 1)
    for sparse, mode in ((0, 1), (1, 2)):
        hs = np.full(B * nm * nm, -7.0)
        L.solveH_cuda(nm, nm2, nq, B, al.ctypes.data_as(dp), hs.ctypes.data_as(dp), 1, sparse)
        hs = hs.reshape(B, nm, nm)
        assert np.isfinite(hs).all()
        opts = make_opts(nm, nq, nm2=nm2, hess_mode=mode)
        for b in range(B):
            ho = oracle.hessian(opts, T, al[b].copy())
            assert np.allclose(hs[b], ho, rtol=1e-13, atol=1e-14 * np.abs(ho).max()), (sparse, b)
            assert np.array_equal(hs[b], hs[b].T)


def test_reference_solveH_uninitialised_sizes_poison():
    """A call whose sizes were not set up by solveHInit_cuda leaves no stale values: hs is
    filled with NaN (and a message goes to stderr) instead of being left unwritten."""
    import ctypes
    q = c3d.quadrature(1, 4)
    nm, nq = q["nm"], q["nq"]
    L = c3d.lib()
    dp = ctypes.POINTER(ctypes.c_double)
    L.solveHInit_cuda(nm, 0, nq, 4, q["w"].ctypes.data_as(dp), q["M"].ctypes.data_as(dp), None,
                      None, None, None, None, 0)
    al = np.zeros(4 * nm)
    hs = np.zeros(4 * nm * nm)
    L.solveH_cuda(nm, 9, nq, 4, al.ctypes.data_as(dp), hs.ctypes.data_as(dp), 1, 1)
    assert np.isnan(hs).all()
    hs[:] = 0.0
    L.solveH_cuda(nm, 0, nq, 4, al.ctypes.data_as(dp), hs.ctypes.data_as(dp), 0, 0)
    assert np.isfinite(hs).all() and (hs != 0).any()


def _gaunt_csr(T, threshold):
    nm, nm2 = T["nm"], T["nm2"]
    beta = T["beta"].reshape(nm * nm, nm2)
    row = [0]
    col, val = [], []
    for idx in range(nm * nm):
        nz = np.nonzero(np.abs(beta[idx]) > threshold)[0]
        col.extend(nz.tolist())
        val.extend(beta[idx, nz].tolist())
        row.append(len(col))
    return np.array(row, np.int32), np.array(col, np.int32), np.array(val)


@pytest.mark.parametrize("mode", [2, 1])
@pytest.mark.parametrize("N,Q", [(2, 12), (4, 12)])
def test_gaunt_closure_matches_oracle(oracle, mode, N, Q):
    """Gaunt-form Hessian (MN_USE_GAUNT_COEF true): sparse (|beta| > 1e-13) and dense."""
    S = _setup(oracle, N=N, Q=Q, steps_before=2)
    T = oracle.tables(N, Q, gaunt=True)
    S["T"] = T
    ctx = _ctx(S)
    row, col, val = _gaunt_csr(T, 1e-13 if mode == 2 else 0.0)
    ctx.set_gaunt(T["nm2"], T["M2"], row, col, val)
    ctx.set_state(u=S["u"], alpha=S["alpha"], sig_t=S["sig"], sig_s=S["sig"])
    ctx.closure()
    ctx.sync()
    ug, ag = ctx.get_state()
    rec = ctx.records()
    nm = S["nm"]
    uo = S["u"].reshape(-1, nm).copy()
    ao = S["alpha"].reshape(-1, nm).copy()
    out = oracle.closure(make_opts(nm, S["nq"], nm2=T["nm2"], hess_mode=mode), T, uo, ao)
    assert (rec["status"] == 0).all()
    ties = tie_cells(out)
    mism = rec["iters"] != out["totalIter"]
    log_ties(f"test_gaunt_closure_matches_oracle[mode={mode},N={N},Q={Q}]", ties, mism)
    assert not (mism & ~ties).any(), np.nonzero(mism & ~ties)[0][:10]
    ok = ~ties & (rec["regIndex"] == out["regIndex"])
    ag = ag.reshape(-1, nm)
    rel = np.linalg.norm(ag[ok] - ao[ok], axis=1) / np.linalg.norm(ao[ok], axis=1)
    assert rel.max() < 1e-10, rel.max()
    assert (out["totalIter"] > 1).sum() > 100


@pytest.mark.parametrize("gaunt", [False, True])
@pytest.mark.parametrize("engine", [0, 1])
def test_engines_match_oracle(oracle, engine, gaunt):
    """Both closure engines -- work-list rounds (0: tiled blocked Cholesky with DMMA trailing
    updates) and the persistent kernel (1: packed right-looking Cholesky) -- against the
    oracle: iteration counts identical except rounding ties, multipliers within 1e-10."""
    S = _setup(oracle, N=4, Q=12, steps_before=2)
    T = oracle.tables(4, 12, gaunt=True)
    S["T"] = T
    ctx = _ctx(S)
    ctx.set_engine(engine)
    nm = S["nm"]
    mode = 0
    if gaunt:
        row, col, val = _gaunt_csr(T, 1e-13)
        ctx.set_gaunt(T["nm2"], T["M2"], row, col, val)
        mode = 2
    ctx.set_state(u=S["u"], alpha=S["alpha"], sig_t=S["sig"], sig_s=S["sig"])
    ctx.closure()
    ctx.sync()
    ug, ag = ctx.get_state()
    rec = ctx.records()
    uo = S["u"].reshape(-1, nm).copy()
    ao = S["alpha"].reshape(-1, nm).copy()
    opts = make_opts(nm, S["nq"], nm2=T["nm2"], hess_mode=mode) if gaunt else S["opts"]
    out = oracle.closure(opts, T, uo, ao)
    assert (rec["status"] == 0).all()
    ties = tie_cells(out)
    mism = rec["iters"] != out["totalIter"]
    log_ties(f"test_engines_match_oracle[engine={engine},gaunt={gaunt}]", ties, mism)
    assert not (mism & ~ties).any(), np.nonzero(mism & ~ties)[0][:10]
    ok = ~ties & (rec["regIndex"] == out["regIndex"])
    ag = ag.reshape(-1, nm)
    rel = np.linalg.norm(ag[ok] - ao[ok], axis=1) / np.linalg.norm(ao[ok], axis=1)
    assert rel.max() < 1e-10, rel.max()
    assert (out["totalIter"] > 1).sum() > 100


def test_ghost_mirroring_is_exact(oracle):
    """Face-ghost mirroring (solve the non-face cells, copy the face ghosts from their
    periodic images) gives bit-identical moments, multipliers and records to solving every
    cell as the reference does, and engages when the face ghosts mirror their images."""
    S = _setup(oracle, N=2, Q=12, steps_before=1)
    nall = S["nall"]
    u0, a0 = S["u"].copy(), S["alpha"].copy()
    oracle.ghost_fill(S["g"], u0)  # face ghosts = periodic images, multipliers included
    oracle.ghost_fill(S["g"], a0)
    out = []
    for on in (False, True):
        ctx = _ctx(S)
        ctx.set_ghost_mirroring(on)
        ctx.set_state(u=u0, alpha=a0, sig_t=S["sig"], sig_s=S["sig"])
        ctx.reset_stats()
        for _ in range(2):
            ctx.step(S["dt"])
        ctx.sync()
        u, a = ctx.get_state()
        rec = ctx.records()
        st = ctx.stats()
        out.append((u, a, rec["iters"], rec["regIndex"], rec["status"], st.cells,
                    st.totalIters, list(st.regHist), list(st.iterHist), ctx.launch_count()))
        ctx.close()
    for x, y in zip(out[0][:5], out[1][:5]):
        assert np.array_equal(x, y)
    # statistics count the copied face ghosts as solved: both modes report every cell
    assert out[0][5] == out[1][5] == 4 * nall
    assert out[0][6:9] == out[1][6:9]
    assert out[1][9] > out[0][9]  # the mirrored closures launched the check and copy kernels


def test_reprojection_mode(oracle):
    """MN_REPROJECT (the robustness note of the reference's readme.txt): after the closure
    u = <m e^{alpha.m}> with u_0 kept and alpha_0 shifted by 2 sqrt(pi) log(u_0 / u'_0);
    checked against the same formulas in numpy on the plain closure's multipliers."""
    S = _setup(oracle, N=2, Q=12, steps_before=1)
    nm, nq, T = S["nm"], S["nq"], S["T"]
    outs = []
    for rp in (False, True):
        ctx = _ctx(S, reproject=rp)
        ctx.set_state(u=S["u"], alpha=S["alpha"], sig_t=S["sig"], sig_s=S["sig"])
        ctx.closure()
        ctx.sync()
        outs.append(ctx.get_state())
        ctx.close()
    (u0, a0), (u1, a1) = outs
    M = T["M"].reshape(nq, nm)
    A, U = a0.reshape(-1, nm), u0.reshape(-1, nm)
    un = (np.exp(A @ M.T) * T["w"]) @ M
    s = U[:, 0] / un[:, 0]
    ue = un * s[:, None]
    ue[:, 0] = U[:, 0]
    ae = A.copy()
    ae[:, 0] += 2.0 * np.sqrt(np.pi) * np.log(s)
    u1, a1 = u1.reshape(-1, nm), a1.reshape(-1, nm)
    assert np.array_equal(u1[:, 0], U[:, 0])
    assert np.linalg.norm(u1 - ue) <= 1e-13 * np.linalg.norm(ue)
    assert np.abs(a1 - ae).max() <= 1e-12 * np.abs(ae).max()
    # u is now the ansatz's own moments (to rounding)
    ua = (np.exp(a1 @ M.T) * T["w"]) @ M
    assert np.linalg.norm(u1 - ua) <= 1e-12 * np.linalg.norm(ua)
    assert np.abs(s - 1.0).max() > 1e-12  # the closure's tolerance left something to fix
