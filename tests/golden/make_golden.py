"""Generates the golden fixtures in this directory by running the reference CPU path
(oracle/_ref/libc3dref.so, compiled from the reference's own sources by
oracle/Makefile) on small decks. Run from the repository root:

    python tests/golden/make_golden.py

Fixtures:
* c1_m2_16.npz  -- M_2, 16^3, 288-point quadrature, isotropic pulse psi =
  max(1e-4, G/(4 pi)) of width 0.1, sigma_s = 1, MN_TOL 1e-6 (batched rules; at the
  configuration's 1e-8 the reference exhausts its ladder and aborts),
  ladder {0, 1e-8, 1e-6, 1e-4, 1e-2, 1e-1}, CFL 0.5, theta 2, 20 SSP-RK2 steps.
  Stores the per-cell iteration counts and ladder indices of the first two steps,
  the interior moments after steps 2 and 20 and the reference's statistics.
  The initial state comes from the deck through the B200 host's host-only init
  (INIT_COND gaussian_psi; the reference has no such option, so its u and alpha are
  overwritten with the same arrays before the first step).
* pn_p3_8.npz   -- P_N (N=3), 8x6x7 grid, smooth initial condition, moment flux,
  5 steps; interior moments after the last step.
* c2_m4_64.npz  -- M_4, 64^3, 800-point quadrature (20 mu x 40 phi), sigma_s checkerboard
  of 1 and 10 over 8^3-cell blocks with sigma_a 0.1 in the 10-blocks, pulse
  psi = max(1e-6, G/(4 pi)) of width 0.05, Gaunt sparse Hessian (the reference deck's
  default), MN_TOL 1e-6 (at 1e-8 the reference exhausts its ladder and aborts in the first
  step), the same ladder as c1, CFL 0.5, theta 2, 3 SSP-RK2 steps (the reference CPU path
  takes about 7 minutes on 8 cores for them). Stores the per-cell iteration counts and
  ladder indices of all six closures, and after steps 1 and 3 the interior moments of 4096
  seeded sample cells plus the moment sums over every x-, y- and z-plane. The initial
  state and the sigma fields come from the B200 host's host-only init (INIT_COND
  gaussian_psi, SIGMA_CHECKER_BLOCK; the reference has neither, so its u, alpha, sigma_t
  and sigma_s are overwritten with the same arrays before the first step).
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "tests"))
sys.path.insert(0, os.path.join(REPO, "c3d-2015_b200"))

from oracle_lib import deck_text, run_reference  # noqa: E402

C1_LADDER = [0.0, 1e-8, 1e-6, 1e-4, 1e-2, 1e-1]


def c1_deck(ic):
    return deck_text(NX=16, NY=16, NZ=16, MOMENT_ORDER=2, QUAD_ORDER=12, CFL_FACTOR=0.5,
                     CROSS_SECTION=1.0, INIT_FLOOR=1e-4, GAUSS_SIGMA=0.1, INIT_COND=ic,
                     THETA=2.0, OMP_THREADS=os.cpu_count() or 1, MN_TOL=1e-6, MN_BATCHED="true",
                     REG_LADDER=",".join(str(x) for x in C1_LADDER))


def c1_initial_state():
    import c3d
    with tempfile.TemporaryDirectory() as tmp:
        p = os.path.join(tmp, "input.deck")
        with open(p, "w") as f:
            f.write(c1_deck("gaussian_psi"))
        s = c3d.Solver(p, host_only=True)
        A = s.arrays()
        u, a = A["u"].copy(), A["alpha"].copy()
        s.close()
    return u, a


def interior(v, n, nm):
    return v.reshape(n + 4, n + 4, n + 4, nm)[2:n + 2, 2:n + 2, 2:n + 2].copy()


def make_c1():
    u0, a0 = c1_initial_state()
    ref2 = run_reference(c1_deck("gaussian"), ladder=C1_LADDER, nsteps=2,
                         overrides=dict(u=u0, alpha=a0))
    ref20 = run_reference(c1_deck("gaussian"), ladder=C1_LADDER, nsteps=20,
                          overrides=dict(u=u0, alpha=a0), record=False)
    it = np.stack([ref2["iters"][s][0] for s in range(2)]).astype(np.int16)
    rg = np.stack([ref2["iters"][s][2] for s in range(2)]).astype(np.int8)
    np.savez_compressed(os.path.join(HERE, "c1_m2_16.npz"), iters=it, reg=rg,
                        u_step2=interior(ref2["u"], 16, 9), u_step20=interior(ref20["u"], 16, 9),
                        stats20=np.array(ref20["stats"][:11]), dt=ref2["dv"][3])


C2_SAMPLE_SEED = 20151


def c2_deck(ic):
    return deck_text(NX=64, NY=64, NZ=64, MOMENT_ORDER=4, QUAD_ORDER=20, CFL_FACTOR=0.5,
                     CROSS_SECTION=1.0, INIT_FLOOR=1e-6, GAUSS_SIGMA=0.05, INIT_COND=ic,
                     THETA=2.0, OMP_THREADS=os.cpu_count() or 1, MN_TOL=1e-6, MN_BATCHED="true",
                     MN_USE_GAUNT_COEF="true", MN_USE_GAUNT_SPARSE="true",
                     SIGMA_CHECKER_BLOCK=8, SIGMA_S_HI=10.0, SIGMA_A_HI=0.1,
                     REG_LADDER=",".join(str(x) for x in C1_LADDER))


def c2_initial_state():
    import c3d
    with tempfile.TemporaryDirectory() as tmp:
        p = os.path.join(tmp, "input.deck")
        with open(p, "w") as f:
            f.write(c2_deck("gaussian_psi"))
        s = c3d.Solver(p, host_only=True)
        A = s.arrays()
        out = A["u"].copy(), A["alpha"].copy(), A["sigT"].copy(), A["sigS"].copy()
        s.close()
    return out


def c2_summary(u, n=64, nm=25):
    """Seeded sample cells and per-plane moment sums of the interior moments."""
    x = interior(u, n, nm)
    rng = np.random.default_rng(C2_SAMPLE_SEED)
    pick = rng.choice(n ** 3, 4096, replace=False)
    return dict(sample=x.reshape(-1, nm)[pick].copy(), sx=x.sum(axis=(1, 2)),
                sy=x.sum(axis=(0, 2)), sz=x.sum(axis=(0, 1)))


def make_c2():
    u0, a0, st, ss = c2_initial_state()
    ref = run_reference(c2_deck("gaussian"), ladder=C1_LADDER, nsteps=3,
                        overrides=dict(u=u0, alpha=a0, sigT=st, sigS=ss), want=("snapshots",))
    it = np.stack([ref["iters"][s][0] for s in range(3)]).astype(np.int16)
    rg = np.stack([ref["iters"][s][2] for s in range(3)]).astype(np.int8)
    s1 = c2_summary(ref["snapshots"][1][0])
    s3 = c2_summary(ref["u"])
    np.savez_compressed(os.path.join(HERE, "c2_m4_64.npz"), iters=it, reg=rg,
                        **{f"step1_{k}": v for k, v in s1.items()},
                        **{f"step3_{k}": v for k, v in s3.items()},
                        stats=np.array(ref["stats"][:11]), dt=ref["dv"][3])


def make_pn():
    deck = deck_text(SOLVER="pn", NX=8, NY=6, NZ=7, MOMENT_ORDER=3, QUAD_ORDER=8,
                     INIT_COND="smooth", PN_USE_KINETIC_FLUX=0)
    ref = run_reference(deck, nsteps=5, record=False)
    u = ref["u"].reshape(12, 10, 11, 16)[2:10, 2:8, 2:9].copy()
    np.savez_compressed(os.path.join(HERE, "pn_p3_8.npz"), u_step5=u, dt=ref["dv"][3])


if __name__ == "__main__":
    which = sys.argv[1:] or ["c1", "pn", "c2"]
    if "c1" in which:
        make_c1()
    if "pn" in which:
        make_pn()
    if "c2" in which:
        make_c2()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")
