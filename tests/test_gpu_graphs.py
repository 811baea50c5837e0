"""The closure as one CUDA graph (c3d_set_graphs) against host-driven rounds.

With graphs on, a closure is round 0 plus a conditional WHILE node whose body runs two
work-list rounds and sets its own condition on the device; each list's kernels sit in a
SWITCH node whose launch size a control kernel picks from the list's device counter, and
entries beyond the batch limit carry over to the next round. Each cell's solve is the same
whichever launch it lands in, so results must be bit-identical to the host-driven rounds:
multipliers, moments and per-cell records. Covered: the 64^3 M_6 deck for two steps (FP64
with the certificate, and the mixed closure), and the 24^3 deck without the certificate and
with a batch limit of 1000 entries, so that round 0 lists every cell and the graph's rounds
carry most of them over.
"""
import os

import numpy as np
import pytest

import c3d
from oracle_lib import deck_text

pytestmark = pytest.mark.gpu


def _deck(tmp_path, n, mixed, name):
    kw = dict(NX=n, NY=n, NZ=n, MOMENT_ORDER=6, QUAD_ORDER=28, CFL_FACTOR=0.5, CROSS_SECTION=1.0,
              INIT_FLOOR=1e-10, GAUSS_SIGMA=0.02, INIT_COND="gaussian_psi", THETA=2.0,
              MN_TOL=1e-6, MN_BATCHED="true", MN_USE_GAUNT_COEF="true",
              MN_USE_GAUNT_SPARSE="true", REG_LADDER="0,1e-8,1e-6,1e-4,1e-2,1e-1",
              OMP_THREADS=os.cpu_count() or 1)
    if mixed:
        kw["MN_MIXED_PRECISION"] = "true"
    p = tmp_path / name
    p.write_text(deck_text(**kw))
    return str(p)


def _run(path, graphs, steps, certificate=True, batch=0):
    L = c3d.lib()
    s = c3d.Solver(path)
    h = s.ctx_handle
    c3d.check(L.c3d_set_graphs(h, int(graphs)), "graphs")
    c3d.check(L.c3d_set_certificate(h, int(certificate)), "certificate")
    c3d.check(L.c3d_set_limits(h, 0, 0, batch), "limits")
    launches0 = L.c3d_launch_count(h)
    for _ in range(steps):
        s.update(s.max_dt)
    s.sync()
    s.pull()
    A = s.arrays()
    out = dict(u=A["u"].copy(), a=A["alpha"].copy(), rec=s.records(),
               launches=L.c3d_launch_count(h) - launches0)
    s.close()
    return out


def _same(x, y):
    assert np.array_equal(x["u"], y["u"])
    assert np.array_equal(x["a"], y["a"])
    for k in ("iters", "iterGamma", "regIndex", "status"):
        assert np.array_equal(x["rec"][k], y["rec"][k]), k


@pytest.mark.parametrize("mixed", [False, True])
def test_graph_rounds_match_host_rounds(tmp_path, mixed):
    p = _deck(tmp_path, 64, mixed, f"g{int(mixed)}.deck")
    g = _run(p, True, 2)
    h = _run(p, False, 2)
    _same(g, h)
    assert (g["rec"]["iters"] > 1).sum() > 100
    assert g["launches"] > 0


def test_graph_rounds_carry_over(tmp_path):
    p = _deck(tmp_path, 24, False, "c.deck")
    g = _run(p, True, 2, certificate=False, batch=1000)
    h = _run(p, False, 2, certificate=False)
    _same(g, h)
