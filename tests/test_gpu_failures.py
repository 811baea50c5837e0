"""Failure paths of the closure, injected from the host (no device fault, trap or hang).

The reference aborts on each of these (src/opt/opt.cpp:343-346 for u0 <= 0,
src/opt/optBatch.cpp:233-238 and src/opt/opt.cpp:261-266 for an exhausted
regularisation ladder); the B200 closure instead records a per-cell status and returns
a status code, and the context stays usable afterwards:

* u0 <= 0 in one cell: that cell gets status 1, c3d_sync reports C3D_ERR_CLOSURE;
* a one-level ladder with MN_MAX_ITER 2 (unbatched rules): exactly the cells the oracle
  cannot finish in two iterations get status 2 (ladder exhausted), the rest converge with
  the oracle's multipliers;
* a pass budget of one: cells that need a second pass end with status 3;
* a limit of one work-list round: C3D_ERR_TIMEOUT -- from c3d_sync when the round loop
  runs on the device (c3d_set_graphs on, the default), from c3d_closure itself when the host
  drives the rounds -- and a closure with the default limits then finishes the same state.
"""
import numpy as np
import pytest

import c3d
from oracle_lib import make_opts

from test_gpu_kernels import _ctx, _setup

pytestmark = pytest.mark.gpu


def _mid(S):
    n, nm = S["n"], S["nm"]
    c = n // 2 + 2
    return (c * (n + 4) + c) * (n + 4) + c, nm


def test_nonpositive_u0_sets_status_and_error(oracle):
    S = _setup(oracle, steps_before=1)
    cell, nm = _mid(S)
    u = S["u"].copy()
    u[cell * nm] = -1e-3
    ctx = _ctx(S)
    ctx.set_state(u=u, alpha=S["alpha"], sig_t=S["sig"], sig_s=S["sig"])
    ctx.closure()
    with pytest.raises(c3d.C3DError, match="CLOSURE"):
        ctx.sync()
    st = ctx.records()["status"]
    assert st[cell] == 1
    assert (np.delete(st, cell) == 0).all()
    # the context stays usable and the failure count was reset
    ctx.set_state(u=S["u"], alpha=S["alpha"])
    ctx.closure()
    ctx.sync()
    assert (ctx.records()["status"] == 0).all()
    ctx.close()


def test_exhausted_ladder_matches_oracle(oracle):
    S = _setup(oracle, steps_before=2, batched=False, ladder=(0.0,))
    nm = S["nm"]
    ctx = _ctx(S, max_iter=2)
    ctx.set_state(u=S["u"], alpha=S["alpha"], sig_t=S["sig"], sig_s=S["sig"])
    ctx.closure()
    with pytest.raises(c3d.C3DError, match="CLOSURE"):
        ctx.sync()
    rec = ctx.records()
    _, ag = ctx.get_state()
    uo = S["u"].reshape(-1, nm).copy()
    ao = S["alpha"].reshape(-1, nm).copy()
    out = oracle.closure(make_opts(nm, S["nq"], batched=False, max_iter=2, ladder=(0.0,)),
                         S["T"], uo, ao)
    assert (out["status"] == 2).sum() > 50
    assert np.array_equal(rec["status"], out["status"])
    ok = out["status"] == 0
    ag = ag.reshape(-1, nm)
    rel = np.linalg.norm(ag[ok] - ao[ok], axis=1) / np.linalg.norm(ao[ok], axis=1)
    assert rel.max() < 1e-10, rel.max()
    ctx.close()


def test_pass_budget_ends_cells_with_status_3(oracle):
    S = _setup(oracle, steps_before=2)
    ctx = _ctx(S)
    ctx.set_limits(pass_budget=1)
    ctx.set_state(u=S["u"], alpha=S["alpha"], sig_t=S["sig"], sig_s=S["sig"])
    ctx.closure()
    with pytest.raises(c3d.C3DError, match="CLOSURE"):
        ctx.sync()
    rec = ctx.records()
    assert set(np.unique(rec["status"])) == {0, 3}
    assert (rec["iters"][rec["status"] == 0] == 1).all()
    ctx.set_limits()
    ctx.set_state(u=S["u"], alpha=S["alpha"])
    ctx.closure()
    ctx.sync()
    assert (ctx.records()["status"] == 0).all()
    ctx.close()


@pytest.mark.parametrize("graphs", [True, False])
def test_round_limit_returns_timeout_and_recovers(oracle, graphs):
    S = _setup(oracle, steps_before=2)
    nm = S["nm"]
    ref = _ctx(S)
    ref.set_state(u=S["u"], alpha=S["alpha"], sig_t=S["sig"], sig_s=S["sig"])
    ref.closure()
    ref.sync()
    u_ref, a_ref = ref.get_state()
    assert ref.records()["iters"].max() > 2  # more than one round of work
    ref.close()

    ctx = _ctx(S)
    ctx.set_graphs(graphs)
    ctx.set_limits(max_rounds=1)
    ctx.set_state(u=S["u"], alpha=S["alpha"], sig_t=S["sig"], sig_s=S["sig"])
    with pytest.raises(c3d.C3DError, match="TIMEOUT"):
        ctx.closure()
        ctx.sync()
    # cells the first round finished hold their results, the others their inputs
    ctx.set_limits()
    ctx.closure()
    ctx.sync()
    assert (ctx.records()["status"] == 0).all()
    u1, a1 = ctx.get_state()
    rel = np.linalg.norm((a1 - a_ref).reshape(-1, nm), axis=1) / \
        np.linalg.norm(a_ref.reshape(-1, nm), axis=1)
    assert rel.max() < 1e-8, rel.max()
    ctx.close()
