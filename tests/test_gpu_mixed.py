"""Mixed-precision closure (c3d_set_precision mode 1) against the FP64 closure.

The mixed closure computes the Hessian's extended moments on the tensor cores (BF16, or
3xTF32 split products, FP32 accumulation) and keeps the gradient, the objective, the
factorisation and the stopping test in FP64. Every converged cell therefore satisfies the
FP64 residual test |<m e^{alpha.m}> - u| / u_0 <= MN_TOL -- checked here in numpy from the
returned multipliers and moments -- while iteration counts and multipliers may differ from
the FP64 closure within what that tolerance allows.

Cells: the 64^3 version of the M_6 benchmark workload (49 moments, 1568 directions, gaussian
pulse of width 0.02 over a 1e-10 floor) advanced three steps by the FP64 solver; the
multi-iteration cells of its last closure plus a random sample are solved again from the
same moments and warm starts by both closures.
"""
import os

import numpy as np
import pytest

import c3d
from oracle_lib import deck_text
from test_gpu_kernels import _gaunt_csr

pytestmark = pytest.mark.gpu

LADDER = [0.0, 1e-8, 1e-6, 1e-4, 1e-2, 1e-1]
TOL = 1e-6


def _deck(tmp_path, n, mixed, steps=None, name="input.deck"):
    kw = dict(NX=n, NY=n, NZ=n, MOMENT_ORDER=6, QUAD_ORDER=28, CFL_FACTOR=0.5, CROSS_SECTION=1.0,
              INIT_FLOOR=1e-10, GAUSS_SIGMA=0.02, INIT_COND="gaussian_psi", THETA=2.0, MN_TOL=TOL,
              MN_BATCHED="true", MN_USE_GAUNT_COEF="true", MN_USE_GAUNT_SPARSE="true",
              REG_LADDER=",".join(str(x) for x in LADDER), OMP_THREADS=os.cpu_count() or 1)
    if mixed:
        kw["MN_MIXED_PRECISION"] = "true"
    p = tmp_path / name
    p.write_text(deck_text(**kw))
    return str(p)


@pytest.fixture(scope="module")
def m6_cells(oracle, tmp_path_factory):
    s = c3d.Solver(_deck(tmp_path_factory.mktemp("m6"), 64, False))
    for _ in range(3):
        s.update(s.max_dt)
    s.sync()
    s.pull()
    nm = s.nm
    A = s.arrays()
    u = A["u"].reshape(-1, nm).copy()
    a = A["alpha"].reshape(-1, nm).copy()
    it = s.records()["iters"]
    s.close()
    multi = np.nonzero(it >= 2)[0]
    rng = np.random.default_rng(5)
    pick = np.concatenate([multi[:3000], rng.choice(len(it), 2000, replace=False)])
    T = oracle.tables(6, 28, gaunt=True)
    return dict(u=u[pick], a=a[pick], T=T, nm=nm, nmulti=len(multi))


def _solve(S, mode, cond_bf16=0.0, cond_max=0.0, polish=0.0):
    import torch
    T, nm = S["T"], S["nm"]
    n = len(S["u"])
    ctx = c3d.Context(nx=1, ny=1, nz=1, nm=nm, nq=T["nq"], dx=1.0, dy=1.0, dz=1.0, M=T["M"],
                      w=T["w"], xi=T["xi"], eta=T["eta"], mu=T["mu"], ladder=LADDER, tol=TOL)
    row, col, val = _gaunt_csr(T, 1e-13)
    ctx.set_gaunt(T["nm2"], T["M2"], row, col, val)
    ctx.set_precision(mode, cond_bf16, cond_max, polish=polish)
    du = torch.tensor(S["u"], device="cuda")
    da = torch.tensor(S["a"], device="cuda")
    it = torch.zeros(n, dtype=torch.int32, device="cuda")
    rg = torch.zeros(n, dtype=torch.int32, device="cuda")
    st = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ctx.reset_stats()
    ctx.closure_vectors_device(n, du.data_ptr(), da.data_ptr(), it.data_ptr(), None,
                               rg.data_ptr(), st.data_ptr())
    ctx.sync()
    stats = _d(ctx.stats())
    ctx.close()
    return dict(u=du.cpu().numpy(), a=da.cpu().numpy(), it=it.cpu().numpy(), rg=rg.cpu().numpy(),
                st=st.cpu().numpy(), stats=stats)


def _d(stats):
    return {k: getattr(stats, k) for k, t in stats._fields_ if not hasattr(t, "_length_")}


def _residual(T, u, a):
    """|<m e^{alpha.m}> - u|_2 / u_0 per cell (the scaled problem's stopping-test norm)."""
    M = T["M"].reshape(T["nq"], -1)
    mom = (np.exp(a @ M.T) * T["w"]) @ M
    return np.linalg.norm(mom - u, axis=1) / u[:, 0]


def test_mixed_closure_meets_fp64_residual(m6_cells):
    S = m6_cells
    f = _solve(S, 0)
    m = _solve(S, 1)
    assert (f["st"] == 0).all() and (m["st"] == 0).all()
    assert S["nmulti"] > 100
    # equal residual: both closures stop on the same FP64 test
    rf = _residual(S["T"], f["u"], f["a"])
    rm = _residual(S["T"], m["u"], m["a"])
    assert rf.max() <= TOL * 1.001, rf.max()
    assert rm.max() <= TOL * 1.001, rm.max()
    # the same regularisation almost everywhere
    same_reg = (f["rg"] == m["rg"]).mean()
    assert same_reg >= 0.99, same_reg
    ok = f["rg"] == m["rg"]
    rel = np.linalg.norm(m["a"][ok] - f["a"][ok], axis=1) / np.linalg.norm(f["a"][ok], axis=1)
    assert np.median(rel) < 1e-6, np.median(rel)
    # the tensor-core levels carry the Hessians until the gradient nears the tolerance, then
    # the last steps are FP64 (the default polish); without the polish they carry most
    st = m["stats"]
    assert st["hessBf16"] + st["hessTf32x3"] > 0.3 * st["totalIters"], st
    assert st["escalated"] > 0
    st1 = _solve(S, 1, polish=1.0)["stats"]
    assert st1["hessBf16"] + st1["hessTf32x3"] > 0.5 * st1["totalIters"], st1
    assert m["it"].mean() <= 1.5 * f["it"].mean(), (m["it"].mean(), f["it"].mean())
    print(f"\nmixed vs FP64 on {len(rel)} cells: alpha rel diff median {np.median(rel):.2e} "
          f"max {rel.max():.2e}; iterations {m['it'].mean():.3f} vs {f['it'].mean():.3f}; "
          f"Hessians BF16 {st['hessBf16']} 3xTF32 {st['hessTf32x3']} FP64 {st['hessFp64']} "
          f"escalated {st['escalated']}")


@pytest.mark.parametrize("levels", ["bf16", "fp64"])
def test_mixed_precision_routing(m6_cells, levels):
    """Thresholds route the Hessians: with no condition bound every Hessian after the
    first (3xTF32, no record yet; many first iterations end on the convergence certificate
    without one) is BF16 unless a factorisation fails; with zero bounds they are FP64.
    Either way every cell meets the FP64 residual. The polish is off here (polish 1), which
    would otherwise send first visits whose probe gradient lies within 1e3 of the tolerance
    to FP64 Hessians (covered by the other tests, which use the default)."""
    S = m6_cells
    if levels == "bf16":
        m = _solve(S, 1, 1e300, 1e300, polish=1.0)
    else:
        m = _solve(S, 1, 1e-300, 1e-300, polish=1.0)
    st = m["stats"]
    assert (m["st"] == 0).all()
    assert _residual(S["T"], m["u"], m["a"]).max() <= TOL * 1.001
    n = len(S["u"])
    # first visits: ended by the convergence certificate, or a 3xTF32 Hessian (no record yet)
    assert st["hessTf32x3"] + st["certified"] >= n
    if levels == "bf16":
        assert st["hessBf16"] > 0
    else:
        assert st["hessBf16"] == 0 and st["hessFp64"] > 0


def test_mixed_grid_steps_track_fp64(tmp_path):
    """Five steps of the 32^3 M_6 deck with the mixed and the FP64 closure: no failed cell,
    and the moments within 1e-8 relative L2 (the multipliers differ within the Newton
    tolerance, which enters the fluxes; the mixed closure's last Newton steps are FP64 steps,
    c3d_set_precision's polish)."""
    out = {}
    for mixed in (False, True):
        s = c3d.Solver(_deck(tmp_path, 32, mixed, name=f"d{int(mixed)}.deck"))
        for _ in range(5):
            s.update(s.max_dt)
        s.sync()
        s.pull()
        st = _d(s.stats())
        out[mixed] = (s.arrays()["u"].copy(), st)
        s.close()
    uf, sf = out[False]
    um, sm = out[True]
    assert sf["failed"] == 0 and sm["failed"] == 0
    assert sm["hessBf16"] + sm["hessTf32x3"] > 0
    rel = np.linalg.norm(um - uf) / np.linalg.norm(uf)
    print(f"\n32^3 M_6, 5 steps: moments rel L2 mixed vs FP64 {rel:.2e}")
    assert rel < 1e-8, rel


def test_mixed_and_fp64_steps_against_oracle(oracle, tmp_path):
    """The 24^3 M_6 deck (Gaunt sparse Hessian, MN_TOL 1e-6) by the C oracle (FP64, the
    reference's algorithm) and by the B200 solver in both precisions. After one step (no
    rounding tie on this deck yet): the FP64 drop-in's interior moments within 1e-12 relative
    L2 of the oracle's; the mixed closure's moments within 1e-8, and the flux divergence of
    its multipliers (the oracle's kinetic flux of either state) within 1e-8. Over three steps
    correct FP64 implementations themselves part at the pulse-centre cells of this coarse
    grid, which regularise and meet rounding ties in their stop tests (the reference build and
    the oracle differ by 2.5e-7 there, the GPU drop-in and the reference by 5e-8); the mixed
    run must stay within that spread (1e-6) of the FP64 drop-in. The multipliers' error is
    printed: it is larger, since near the realizability boundary H is ill-conditioned and
    alpha is determined only to |H^-1 g| with |g| <= MN_TOL."""
    from oracle_lib import make_opts
    n = 24
    T = oracle.tables(6, 28, gaunt=True)
    host = c3d.Solver(_deck(tmp_path, n, False, name="host.deck"), host_only=True)
    A = host.arrays()
    dt = host.max_dt
    nm, nq = 49, 1568
    g = oracle.grid(n, n, n, nm, nq, host.dx, host.dy, host.dz, 2.0)
    opts = make_opts(nm, nq, nm2=T["nm2"], hess_mode=2, tol=TOL, ladder=LADDER)
    uo, ao = A["u"].copy(), A["alpha"].copy()
    bad, _ = oracle.step(g, opts, T, uo, ao, A["sigT"], A["sigS"], dt, records=False)
    assert bad == 0
    host.close()
    inner = (slice(2, n + 2),) * 3

    def interior(v):
        return v.reshape(n + 4, n + 4, n + 4, nm)[inner]

    def rel(x, y):
        return np.linalg.norm(interior(x) - interior(y)) / np.linalg.norm(interior(y))

    fo = interior(oracle.flux_kinetic(g, T, ao))
    res, after3 = {}, {}
    for mixed in (False, True):
        s = c3d.Solver(_deck(tmp_path, n, mixed, name=f"o{int(mixed)}.deck"))
        s.update(s.max_dt)
        s.sync()
        s.pull()
        u, a = s.arrays()["u"].copy(), s.arrays()["alpha"].copy()
        fu = interior(oracle.flux_kinetic(g, T, a))
        res[mixed] = dict(u=rel(u, uo), a=rel(a, ao),
                          flux=np.linalg.norm(fu - fo) / np.linalg.norm(fo))
        for _ in range(2):
            s.update(s.max_dt)
        s.sync()
        s.pull()
        after3[mixed] = (s.arrays()["u"].copy(), s.arrays()["alpha"].copy())
        s.close()
    u3 = rel(after3[True][0], after3[False][0])
    a3 = rel(after3[True][1], after3[False][1])
    print("\n24^3 M_6, 1 step vs the oracle: FP64 " +
          " ".join(f"{k} {v:.2e}" for k, v in res[False].items()) + "; mixed " +
          " ".join(f"{k} {v:.2e}" for k, v in res[True].items()) +
          f"; 3 steps mixed vs FP64: u {u3:.2e} alpha {a3:.2e}")
    assert res[False]["u"] < 1e-12 and res[False]["flux"] < 1e-12
    assert res[True]["u"] < 1e-8 and res[True]["flux"] < 1e-8
    assert u3 < 1e-6


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
def test_mixed_standalone_orders(oracle, N):
    """The standalone closure workload (moment vectors of order N on the order's tensor
    quadrature, solved from the isotropic start with the unbatched rules, MN_TOL 1e-8) in
    both precisions: no vector fails that FP64 solves; the mixed closure regularises at most 5%
    more of the vectors than FP64 and ends on the same or a lower ladder step on >= 85% of
    them (at this tolerance the Armijo test of the last Newton steps is decided at rounding
    level -- the FP64 closure, like the reference, takes the line search's base objective from
    row 0 of H and its trial objectives from the quadrature sum -- and some vectors then
    regularise; the mixed closure's reduced-precision visits form both from one FP64 sum, but
    its final steps are FP64 visits like the reference's, so the two closures regularise
    different vectors at a similar rate); and every converged vector meets the FP64 stopping
    test |g| <= |u| MN_TOL (numpy). Covers the
    tensor-core pass with one zero-padded 128-row tile (3 <= N <= 5) and with two overlapping
    tiles (N = 6, 7); N <= 2 keeps FP64 Hessians."""
    import torch
    from test_gpu_standalone_closure import _vectors
    tol, ladder, n = 1e-8, [0.0, 1e-3, 1e-2, 1e-1, 5e-1], 256
    q, u, a_true, a_iso = _vectors(N, n)
    nm, nq = q["nm"], q["nq"]
    T = oracle.tables(N, 2 * (N + 3), gaunt=True)
    row, col, val = _gaunt_csr(T, 1e-13)
    out = {}
    for mode in (0, 1):
        ctx = c3d.Context(nx=1, ny=1, nz=1, nm=nm, nq=nq, dx=1.0, dy=1.0, dz=1.0, M=q["M"],
                          w=q["w"], xi=q["xi"], eta=q["eta"], mu=q["mu"], batched=False, tol=tol,
                          ladder=ladder)
        ctx.set_gaunt(T["nm2"], T["M2"], row, col, val)
        ctx.set_precision(mode)
        du = torch.tensor(u, device="cuda")
        da = torch.tensor(a_iso, device="cuda")
        it = torch.zeros(n, dtype=torch.int32, device="cuda")
        rg = torch.zeros(n, dtype=torch.int32, device="cuda")
        st = torch.zeros(n, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        ctx.reset_stats()
        ctx.closure_vectors_device(n, du.data_ptr(), da.data_ptr(), it.data_ptr(), None,
                                   rg.data_ptr(), st.data_ptr())
        ctx.sync()
        out[mode] = dict(u=du.cpu().numpy(), a=da.cpu().numpy(), rg=rg.cpu().numpy(),
                         st=st.cpu().numpy(), stats=_d(ctx.stats()))
        ctx.close()
    f, m = out[0], out[1]
    assert not ((m["st"] != 0) & (f["st"] == 0)).any()
    hist = (np.bincount(f["rg"]), np.bincount(m["rg"]))
    assert (m["rg"] > 0).sum() <= (f["rg"] > 0).sum() + n // 20, hist
    assert (m["rg"] <= f["rg"]).mean() >= 0.85, hist
    ok = m["st"] == 0
    M = q["M"].reshape(nq, nm)
    g = (np.exp(m["a"][ok] @ M.T) * q["w"]) @ M - m["u"][ok]
    un = m["u"][ok]
    rel = np.linalg.norm(g, axis=1) / np.linalg.norm(un, axis=1)
    assert rel.max() <= tol * 1.001, rel.max()
    s = m["stats"]
    if N <= 2:  # at most 32 extended moments: the Hessians stay FP64
        assert s["hessBf16"] + s["hessTf32x3"] == 0, s
    else:
        assert s["hessBf16"] + s["hessTf32x3"] > 0, s
