"""Serving loop: problems of different orders, grids and cross sections, submitted while
others run, give the results they give alone (bit for bit), both when they share the GPU and
when a device-memory budget lets only one run at a time."""
import time

import numpy as np
import pytest

import c3d
from oracle_lib import deck_text

pytestmark = pytest.mark.gpu


def _decks():
    base = dict(MN_TOL=1e-6, INIT_FLOOR=1e-4, GAUSS_SIGMA=0.2, MN_BATCHED="true")
    return [
        deck_text(NX=12, NY=12, NZ=12, MOMENT_ORDER=1, QUAD_ORDER=4, NSTEPS=6, **base),
        deck_text(NX=10, NY=9, NZ=11, MOMENT_ORDER=3, QUAD_ORDER=8, NSTEPS=4,
                  CROSS_SECTION=5.0, **base),
        deck_text(NX=8, NY=8, NZ=8, MOMENT_ORDER=5, QUAD_ORDER=12, NSTEPS=3, **base),
        deck_text(NX=14, NY=8, NZ=10, MOMENT_ORDER=1, QUAD_ORDER=6, NSTEPS=5,
                  CROSS_SECTION=0.5, **base),
    ]


def _alone(tmp_path, k, text):
    p = tmp_path / f"deck{k}"
    p.write_text(text)
    s = c3d.Solver(str(p))
    steps = s.run()
    s.pull()
    u = s.arrays()["u"].reshape(s.nx + 4, s.ny + 4, s.nz + 4, s.nm)[2:-2, 2:-2, 2:-2].copy()
    s.close()
    return u, steps


def test_results_alone_and_in_the_mix(tmp_path):
    decks = _decks()
    alone = [_alone(tmp_path, k, d) for k, d in enumerate(decks)]
    srv = c3d.Server(workers=3)
    ids = [srv.submit(decks[0]), srv.submit(decks[1])]
    time.sleep(0.05)  # later arrivals join while the first problems run
    ids += [srv.submit(decks[2]), srv.submit(decks[3])]
    lat = []
    for (ua, steps), rid in zip(alone, ids):
        st, u, latency, n = srv.wait(rid)
        assert st == 0 and n == steps
        assert np.array_equal(u, ua)
        lat.append(latency)
    _, peak = srv.stats()
    sched = srv.timing()
    srv.close()
    assert peak >= 2  # the problems were active together, stepped in shared passes
    # every problem stepped through the scheduler's passes, and the group was rebuilt as
    # problems came and went
    assert sched["passes"] >= max(n for _, n in alone) and sched["group_builds"] >= 2
    assert sched["wait_s"] > 0 and min(sched.values()) >= 0, sched
    print("latency p50 %.3f s  p99 %.3f s" % (np.percentile(lat, 50), np.percentile(lat, 99)))


def test_budget_admits_one_at_a_time(tmp_path):
    decks = _decks()
    budget = max(c3d.Server.estimate(d) for d in decks)
    srv = c3d.Server(workers=3, hbm_budget=budget)
    ids = [srv.submit(d) for d in decks]
    res = [srv.wait(i) for i in ids]
    peak_bytes, peak = srv.stats()
    srv.close()
    assert peak == 1 and peak_bytes <= budget
    for k, (st, u, _, _) in enumerate(res):
        assert st == 0
        assert np.array_equal(u, _alone(tmp_path, k, decks[k])[0])
