#!/usr/bin/env python
"""Benchmark of the B200 M_N time step: Newton cell-solves/s.

A step is one SSP-RK2 step of update() (src/update.cpp:185-275): two stages of
ghost fill, M_N closure on every cell (ghosts included), kinetic flux and Euler
update, then the RK average. A cell-solve is one converged dual solve of one
interior cell in one stage, so a step on an n^3 grid is 2 n^3 cell-solves.

Default workload (one GPU): M_6 (49 moments) on a 128^3 periodic grid, 1568-point
quadrature (28 mu x 56 phi), isotropic gaussian pulse of width 0.02 with floor
1e-10, sigma_s = 1, sigma_a = 0, SSP-RK2 at CFL 0.5, MN_TOL 1e-6 (batched rules),
ladder {0, 1e-8, 1e-6, 1e-4, 1e-2, 1e-1}. Synthetic input generated from the deck.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--config c1|c2|c3] [--precision mixed|fp64] [--no-compare]

The reported arm runs the closure in the configuration's mixed precision (the Gaunt
moments on the tensor cores in BF16 / 3xTF32, everything that decides convergence in
FP64) unless --precision fp64 selects the plain FP64 drop-in. Both arms are timed from
the same start state in every run (precision_compare: throughputs, their ratio, and the
moments' and multipliers' relative L2 difference after the timed steps); both stop on the
same FP64 residual test.

--gpus N > 1 runs under torchrun: N independent replicas (weak scaling), one per
GPU; time is the max over ranks. --impl reference times the reference's own CPU
closure (oracle/_ref, built from the reference sources) on a bounded sample of the
same workload's cells using all host cores, and prints the same metric.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "c3d-2015_b200"))

METRIC = "M_N Newton cell-solves/s mixed vs FP64 at equal residual; p50/p99 latency"
UNIT = "cell-solves/s"
LADDER = "0,1e-8,1e-6,1e-4,1e-2,1e-1"

CONFIGS = {
    "c1": dict(N=2, Q=12, n=16, sigma=0.1, floor=1e-4, sigma_s=1.0,
               desc="M_2 (9 moments) 16^3 periodic, 288-point quadrature, gaussian pulse width 0.1 "
                    "floor 1e-4"),
    "c2": dict(N=4, Q=20, n=64, sigma=0.05, floor=1e-6, sigma_s=1.0, checker=(8, 10.0, 0.1),
               desc="M_4 (25 moments) 64^3 periodic, 800-point quadrature, sigma_s checkerboard "
                    "1/10 over 8^3 blocks, sigma_a 0.1 in the 10-blocks, pulse width 0.05 floor 1e-6"),
    "c3": dict(N=6, Q=28, n=128, sigma=0.02, floor=1e-10, sigma_s=1.0,
               desc="M_6 (49 moments) 128^3 periodic, 1568-point quadrature (28 mu x 56 phi), "
                    "gaussian pulse width 0.02 floor 1e-10"),
    # the same kernels on a 64^3 grid (u and alpha 0.12 GB each, above L2; about 2 GB on
    # the device): the small case for ncu section captures
    "c3m": dict(N=6, Q=28, n=64, sigma=0.02, floor=1e-10, sigma_s=1.0,
                desc="M_6 (49 moments) 64^3 periodic, 1568-point quadrature, pulse width 0.02 "
                     "floor 1e-10 (profiling case)"),
}

# Newton tolerance of the benchmark decks. The configurations name 1e-8; at that
# tolerance the reference's own algorithm (absolute |g| test on u scaled to u0 = 1,
# Armijo test at the FP64 rounding level of f) exhausts its regularisation ladder on
# some cells and aborts (src/opt/optBatch.cpp:233-238), so the decks use 1e-6, the
# smallest decade at which the reference runs these workloads to completion.
MN_TOL = 1e-6


def deck_for(cfg, threads=1, tol=MN_TOL, ic="gaussian_psi", hessian="gaunt"):
    c = CONFIGS[cfg]
    kv = dict(SOLVER="mn", TFINAL="1", OUTDT="1000", OUTPUT_DATA="false",
              OUTPUT_OPT_STATS="false", OUTPUT_TIMINGS="false", NX=c["n"], NY=c["n"], NZ=c["n"],
              MPIX=1, MPIY=1, MPIZ=1, AX=-1, AY=-1, AZ=-1, BX=1, BY=1, BZ=1,
              MOMENT_ORDER=c["N"], QUAD_ORDER=c["Q"], CFL_FACTOR=0.5,
              CROSS_SECTION=c["sigma_s"], INIT_FLOOR=c["floor"], GAUSS_SIGMA=c["sigma"],
              INIT_COND=ic, THETA=2.0, OMP_THREADS=threads, PN_USE_KINETIC_FLUX=0,
              MN_TOL=tol, MN_TOL_GAMMA=1.1, MN_COND_H_MAX=1e10, MN_MAX_ITER=100,
              MN_BATCHED="true", MN_USE_GAUNT_COEF="true" if hessian == "gaunt" else "false",
              MN_USE_GAUNT_SPARSE="true" if hessian == "gaunt" else "false",
              CUDA_KINETIC="true", CUDA_BATCHED="true", CUDA_BATCH_SIZE=50, REG_LADDER=LADDER)
    if "checker" in c:
        b, shi, ahi = c["checker"]
        kv.update(SIGMA_CHECKER_BLOCK=b, SIGMA_S_HI=shi, SIGMA_A_HI=ahi)
    return "".join(f"{k} {v}\n" for k, v in kv.items())


def interior_cells(cfg):
    n = CONFIGS[cfg]["n"]
    return n ** 3


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["unsampled"])
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return dict(sm_mhz=None, sm_max_mhz=smax, reasons=["unsampled"])
        return dict(sm_mhz=float(np.median(sm)), sm_max_mhz=smax, reasons=sorted(reasons),
                    samples=len(sm), power_w_max=max(power) if power else None)


# ------------------------------------------------------------------ FLOP model
def closure_flops_mixed(nm, nq, st):
    """The mixed closure's work: FP64 FLOPs (per Hessian visit the exponent 2 nm nq, nq exps,
    the FP64 moments 2 nm nq and Cholesky nm^3/3 -- FP64-moment visits also the extended
    moments 2 nm2 nq; per line-search trial 2 nm nq + 2 nq) and the reduced-precision
    tensor-core FLOPs (2 nm2p nq per BF16 visit, 3x that per 3xTF32 visit)."""
    N = int(round(nm ** 0.5)) - 1
    nm2 = (2 * N + 1) ** 2
    nm2p = 8 * ((nm2 + 7) // 8)
    visits = st.totalIters + st.escalated - st.certified
    fp64 = (visits * (4 * nm * nq + nq + nm ** 3 / 3.0) + st.hessFp64 * 2 * nm2 * nq
            + st.certified * (4 * nm * nq + nq) + st.trials * (2 * nm * nq + 2 * nq))
    low = 2 * nm2p * nq * (st.hessBf16 + 3 * st.hessTf32x3)
    return fp64, low


def closure_flops(nm, nq, iters, trials, hessian="gaunt", certified=0):
    """Algorithmic FP64 FLOPs of the dual solves. Per Newton iteration: the exponent
    2 nm nq and nq exps (counted 1 FLOP each), the Hessian -- direct form: lower triangle
    nm(nm+1)/2 nq FMAs; Gaunt form: the nm2 = (2N+1)^2 extended moments 2 nm2 nq (the
    sparse beta contraction, ~1% of that, is not counted) -- and Cholesky nm^3/3. An
    iteration ended by the convergence certificate: the exponent, the exps and the
    first-order moments 2 nm nq. Per line-search trial 2 nm nq + 2 nq."""
    N = int(round(nm ** 0.5)) - 1
    nm2 = (2 * N + 1) ** 2
    hess = nm * (nm + 1) * nq if hessian == "direct" else 2 * nm2 * nq
    per_iter = hess + 2 * nm * nq + nq + nm ** 3 / 3.0
    per_cert = 4 * nm * nq + nq
    per_trial = 2 * nm * nq + 2 * nq
    return (iters - certified) * per_iter + certified * per_cert + trials * per_trial


def _hbm_peak_gbs():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except Exception:
        return 6650.0  # earlier measurement on this pool


HBM_PEAK_GBS = _hbm_peak_gbs()


def fp64_peak_tflops():
    """In-run FP64 reference: cuBLAS DGEMM 8192^3 through torch (burst, best of 5)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def profile_traffic(kernel, key="dram_bytes_per_launch_full_workload:"):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    p = os.path.join(REPO, "profiles", f"{kernel}.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith(key):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ------------------------------------------------------------------ reference CPU arm
def _ref_sample_worker(conn, deck, u, a, reps):
    """Spawned process: the reference's batched closure (oracle/_ref) on sampled cells."""
    L = ctypes.CDLL(os.path.join(REPO, "oracle", "_ref", "libc3dref.so"))
    L.c3dref_init.argtypes = [ctypes.c_char_p]
    lad = np.array([float(x) for x in LADDER.split(",")])
    L.c3dref_set_ladder(len(lad), lad.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    with tempfile.TemporaryDirectory() as tmp:
        with open(os.path.join(tmp, "input.deck"), "w") as f:
            f.write(deck)
        L.c3dref_init(tmp.encode())
    L.c3dref_opt_batched_vectors.argtypes = [ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p]
    threads = L.c3dref_num_threads()
    n = u.shape[0]
    times = []
    its = np.zeros(n, np.int32)
    for _ in range(reps):
        uu, aa = u.copy(), a.copy()
        t0 = time.perf_counter()
        L.c3dref_opt_batched_vectors(n, uu.ctypes.data, aa.ctypes.data, its.ctypes.data)
        times.append(time.perf_counter() - t0)
    conn.send(dict(times=times, threads=threads, mean_iters=float(its.mean())))
    conn.close()


def run_ref_sample(cfg, u, a, reps, hessian="gaunt"):
    import multiprocessing as mp
    threads = os.cpu_count() or 1
    c = CONFIGS[cfg]
    # a 4^3 deck with the workload's moment order, quadrature and MN options sets up the
    # reference's tables and globals; the sampled cells are solved by Optimization::opt
    deck = deck_for(cfg, threads=threads, ic="gaussian", hessian=hessian).replace(f"NX {c['n']}", "NX 4").replace(
        f"NY {c['n']}", "NY 4").replace(f"NZ {c['n']}", "NZ 4")
    ctx = mp.get_context("spawn")
    r, w = ctx.Pipe(duplex=False)
    p = ctx.Process(target=_ref_sample_worker, args=(w, deck, u, a, reps))
    p.start()
    w.close()
    res = r.recv()
    p.join()
    return res


def initial_cells_sample(cfg, count, seed=1234):
    """Cells of the workload's initial state, sampled uniformly over the grid with ghosts
    (u0 = 2 sqrt(pi) max(floor, G/(4 pi)), other moments 0; alpha as src/init.cpp:265)."""
    c = CONFIGS[cfg]
    n, nm = c["n"], (c["N"] + 1) ** 2
    rng = np.random.default_rng(seed)
    ijk = rng.integers(0, n + 4, size=(count, 3))
    dx = 2.0 / n
    x = -1 + (ijk - 2) * dx + dx / 2.0
    s = c["sigma"]
    f1 = 1.0 / (s * np.sqrt(2.0 * np.pi))
    G = f1 ** 3 * np.exp(-(x ** 2).sum(1) / (2.0 * s * s))
    u = np.zeros((count, nm))
    u[:, 0] = 2.0 * np.sqrt(np.pi) * np.maximum(c["floor"], G / (4.0 * np.pi))
    a = np.zeros((count, nm))
    a[:, 0] = np.sqrt(4.0 * np.pi) * np.log(u[:, 0] / np.sqrt(4.0 * np.pi))
    return u, a


def calibrated_ref_sample(cfg, u_all, a_all, target_s=12.0, hessian="gaunt"):
    """Times the reference closure on a sample sized for ~target_s seconds of CPU work."""
    threads = os.cpu_count() or 1
    n0 = min(len(u_all), 32 * threads)
    probe = run_ref_sample(cfg, u_all[:n0], a_all[:n0], 1, hessian)
    rate = n0 / max(probe["times"][0], 1e-6)
    n = int(min(len(u_all), max(n0, rate * target_s)))
    return n, rate


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = args.config
    c = CONFIGS[cfg]
    threads = os.cpu_count() or 1
    pool_u, pool_a = initial_cells_sample(cfg, 400000)
    n, rate = calibrated_ref_sample(cfg, pool_u, pool_a,
                                    target_s=max(2.0, 60.0 / max(1, args.steps + args.warmup)),
                                    hessian=args.hessian)
    res = run_ref_sample(cfg, pool_u[:n], pool_a[:n], args.warmup + args.steps, args.hessian)
    times = res["times"][args.warmup:]
    step_s = float(np.mean(times))
    value = n / step_s
    sample = (f"{n} cells drawn uniformly (seed 1234) from the initial state of the workload "
              f"(grid with ghosts), each step one batched closure of the sample "
              f"(Optimization::opt, src/opt/optBatch.cpp:350-472)")
    line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=args.gpus, steps=args.steps,
                warmup=args.warmup, ms_per_step=step_s * 1e3, higher_is_better=True,
                scaling="weak", vs_baseline=None, dtype="f64", data="synthetic", impl="reference",
                config=dict(workload=c["desc"], config=cfg, mn_tol=MN_TOL, ladder=LADDER,
                            hessian=args.hessian,
                            note="reference CPU closure only (no flux); cells/s of the sample"),
                cpu_baseline=dict(value=value, unit=UNIT, cores=res["threads"], kind="reference",
                                  sample=sample),
                e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0),
                mean_iters=res["mean_iters"])
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ standalone closure
STANDALONE_PER_N = (1 << 20) // 7   # 2^20 moment vectors, order N uniform over 1..7
STANDALONE_TOL = 1e-8
STANDALONE_LADDER = "0,1e-3,1e-2,1e-1,5e-1"


def standalone_vectors(c3d, N, n):
    """The batched standalone closure workload for one order N: on the order's tensor
    quadrature (2(N+3) mu x 4(N+3) phi), multipliers alpha_k ~ N(0, s^2) for k >= 1 with s
    log-uniform in [0.1, 5] and alpha_0 set for unit density; u = <m e^{alpha.m}> in FP64;
    the solve starts from the isotropic multipliers of u. Seeded: numpy default_rng([2015, N])."""
    q = c3d.quadrature(N, 2 * (N + 3))
    nm, nq = q["nm"], q["nq"]
    M = q["M"].reshape(nq, nm)
    rng = np.random.default_rng([2015, N])
    sc = np.exp(rng.uniform(np.log(0.1), np.log(5.0), n))
    a = rng.standard_normal((n, nm)) * sc[:, None]
    a[:, 0] = 0.0
    u = (np.exp(a @ M.T) * q["w"]) @ M
    a[:, 0] = -2.0 * np.sqrt(np.pi) * np.log(u[:, 0])
    u = (np.exp(a @ M.T) * q["w"]) @ M
    a_iso = np.zeros_like(a)
    a_iso[:, 0] = 2.0 * np.sqrt(np.pi) * np.log(u[:, 0] / (2.0 * np.sqrt(np.pi)))
    return q, u, a_iso


HIST_EDGES = [1, 2, 4, 8, 16, 32, 64, 128]  # iteration-count bins [1], [2,3], [4,7], ...
STANDALONE_REF_SAMPLE_S = 2.0               # CPU seconds of the reference per order


def _hist(iters):
    h = np.histogram(iters, bins=HIST_EDGES + [1 << 30])[0]
    return [int(x) for x in h]


def _ref_standalone_worker(conn, nm, nm2, nq, u, a, w, M, M2, tol, ladder, target_s):
    """Spawned process (one per order: opt() sizes its thread-private scratch once): the
    reference's unbatched opt() (src/opt/opt.cpp:139-355) over the vectors with OpenMP, on a
    prefix sized for about target_s seconds."""
    L = ctypes.CDLL(os.path.join(REPO, "oracle", "_ref", "libc3dref.so"))
    lad = np.array([float(x) for x in ladder.split(",")])
    L.c3dref_set_ladder(len(lad), lad.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    L.c3dref_opt_init(nm, nm2)
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    L.c3dref_opt_many.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_long, dp,
                                  dp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, dp, dp, dp, ip, ip, dp]

    def run(n):
        uu, aa = np.ascontiguousarray(u[:n]).copy(), np.ascontiguousarray(a[:n]).copy()
        it = np.zeros(n, np.int32)
        t0 = time.perf_counter()
        L.c3dref_opt_many(nm, nm2, nq, n, uu.ctypes.data_as(dp), aa.ctypes.data_as(dp), 100,
                          tol, 1.1, 1e10, w.ctypes.data_as(dp), M.ctypes.data_as(dp),
                          M2.ctypes.data_as(dp), it.ctypes.data_as(ip), None, None)
        return time.perf_counter() - t0, aa, it
    threads = L.c3dref_num_threads()
    n0 = min(len(u), 8 * threads)
    t, _, _ = run(n0)
    n = int(min(len(u), max(n0, n0 / max(t, 1e-6) * target_s)))
    t, aa, it = run(n)
    conn.send(dict(n=n, seconds=t, threads=threads, alpha=aa, iters=it))
    conn.close()


def ref_standalone(q, u, a_iso):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    r, w = ctx.Pipe(duplex=False)
    M2 = c3d_quadrature_m2(q)
    p = ctx.Process(target=_ref_standalone_worker,
                    args=(w, q["nm"], q["nm2"], q["nq"], u, a_iso, q["w"], q["M"], M2,
                          STANDALONE_TOL, STANDALONE_LADDER, STANDALONE_REF_SAMPLE_S))
    p.start()
    w.close()
    res = r.recv()
    p.join()
    return res


def c3d_quadrature_m2(q):
    import c3d
    return c3d.quadrature(q["N"], q["Q"], with_m2=True)["M2"]


def standalone_one_order(args):
    """One order of the standalone workload, closed once (for launch lists: with --no-graphs
    every kernel launches from the host)."""
    import torch
    import c3d
    L = c3d.lib()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    N, n = args.standalone_order, args.standalone_vectors
    q, u, a_iso = standalone_vectors(c3d, N, n)
    with tempfile.TemporaryDirectory() as tmp:
        deck = os.path.join(tmp, "input.deck")
        with open(deck, "w") as f:
            f.write(standalone_deck(N))
        solver = c3d.Solver(deck, stream=ctypes.c_void_p(stream.cuda_stream))
    h = solver.ctx_handle
    c3d.check(L.c3d_set_graphs(h, 1 if args.graphs else 0), "graphs")
    c3d.check(L.c3d_set_precision(h, 1 if args.precision == "mixed" else 0, 0.0, 0.0, 0, 0.0),
              "precision")
    du = torch.tensor(u, device="cuda")
    da = torch.tensor(a_iso, device="cuda")
    it = torch.zeros(n, dtype=torch.int32, device="cuda")
    stt = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    c3d.check(L.c3d_closure_vectors(h, n, ctypes.c_void_p(du.data_ptr()),
                                    ctypes.c_void_p(da.data_ptr()), ctypes.c_void_p(it.data_ptr()),
                                    None, None, ctypes.c_void_p(stt.data_ptr())), "closure")
    L.c3d_sync(h)
    torch.cuda.synchronize()
    print(json.dumps(dict(order=N, vectors=n, precision=args.precision,
                          seconds=time.perf_counter() - t0,
                          iters_per_solve=float(it.double().mean()),
                          failed=int((stt != 0).sum()))), flush=True)
    solver.close()


def standalone_deck(N):
    kv = dict(SOLVER="mn", TFINAL="1", OUTDT="1000", OUTPUT_DATA="false",
              OUTPUT_OPT_STATS="false", OUTPUT_TIMINGS="false", NX=2, NY=2, NZ=2,
              MPIX=1, MPIY=1, MPIZ=1, AX=-1, AY=-1, AZ=-1, BX=1, BY=1, BZ=1,
              MOMENT_ORDER=N, QUAD_ORDER=2 * (N + 3), CFL_FACTOR=0.5, CROSS_SECTION=1.0,
              INIT_FLOOR=1e-4, GAUSS_SIGMA=0.1, INIT_COND="gaussian_psi", THETA=2.0,
              OMP_THREADS=1, PN_USE_KINETIC_FLUX=0, MN_TOL=STANDALONE_TOL, MN_TOL_GAMMA=1.1,
              MN_COND_H_MAX=1e10, MN_MAX_ITER=100, MN_BATCHED="false",
              MN_USE_GAUNT_COEF="true", MN_USE_GAUNT_SPARSE="true", CUDA_KINETIC="true",
              CUDA_BATCHED="true", CUDA_BATCH_SIZE=50, REG_LADDER=STANDALONE_LADDER)
    return "".join(f"{k} {v}\n" for k, v in kv.items())


def standalone_closure(torch, c3d, stream, graphs=True):
    """FP64 vs mixed closure of the standalone workload (one context per order, Gaunt form,
    unbatched rules: |g| <= |u| MN_TOL, gamma <= 1.1, MN_TOL 1e-8). Device-resident vectors;
    CUDA events around each solve after an untimed solve of the same vectors. Headline: all
    seven orders in ONE launch (c3d_group_closure_vectors: one CUDA graph whose branches are
    the orders' closures); per order, its own closure call (iteration histograms, failures,
    mixed vs FP64) and the reference's opt() on a bounded sample of its vectors (rate on the
    host cores, multipliers and iteration counts against the GPU's). For N <= 2 the mixed
    closure keeps FP64 Hessians (c3d_set_precision)."""
    L = c3d.lib()
    per_n, tot = [], {0: [0, 0.0], 1: [0, 0.0]}
    diffs, ref_rows = [], []
    solvers, vecs = [], []

    def bufs(u, a):
        n = len(u)
        return (torch.tensor(u, device="cuda"), torch.tensor(a, device="cuda"),
                torch.zeros(n, dtype=torch.int32, device="cuda"),
                torch.zeros(n, dtype=torch.int32, device="cuda"))

    try:
        for N in range(1, 8):
            q, u, a_iso = standalone_vectors(c3d, N, STANDALONE_PER_N)
            n = len(u)
            with tempfile.TemporaryDirectory() as tmp:
                deck = os.path.join(tmp, "input.deck")
                with open(deck, "w") as f:
                    f.write(standalone_deck(N))
                solver = c3d.Solver(deck, stream=ctypes.c_void_p(stream.cuda_stream))
            solvers.append(solver)
            vecs.append((u, a_iso))
            h = solver.ctx_handle
            c3d.check(L.c3d_set_graphs(h, 1 if graphs else 0), "graphs")
            row = dict(N=N, nm=q["nm"], nq=q["nq"], vectors=n)
            alphas, iters = {}, {}
            for mode in (0, 1):
                c3d.check(L.c3d_set_precision(h, mode, 0.0, 0.0, 0, 0.0), "precision")
                for warm in (True, False):
                    # the untimed pass is the full solve too: every kernel the timed one
                    # launches (rare-path rounds included) is loaded before the events
                    du, da, it, stt = bufs(u, a_iso)
                    torch.cuda.synchronize()
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    c3d.check(L.c3d_closure_vectors(h, n, ctypes.c_void_p(du.data_ptr()),
                                                    ctypes.c_void_p(da.data_ptr()),
                                                    ctypes.c_void_p(it.data_ptr()), None, None,
                                                    ctypes.c_void_p(stt.data_ptr())), "closure")
                    e1.record(stream)
                    torch.cuda.synchronize()
                ms = e0.elapsed_time(e1)
                key = "fp64" if mode == 0 else "mixed"
                row[key] = dict(solves_per_s=n / (ms * 1e-3), ms=ms,
                                iters_per_solve=float(it.double().mean()),
                                failed=int((stt != 0).sum()))
                tot[mode][0] += n
                tot[mode][1] += ms
                alphas[mode] = da.cpu().numpy()
                iters[mode] = it.cpu().numpy()
                if mode == 0:
                    ok0 = stt.cpu().numpy() == 0
            d = np.linalg.norm(alphas[1] - alphas[0], axis=1) / np.linalg.norm(alphas[0], axis=1)
            diffs.append(d)
            f, x = row["fp64"], row["mixed"]
            per_n.append([N, round(f["solves_per_s"]), round(x["solves_per_s"]),
                          round(x["solves_per_s"] / f["solves_per_s"], 3),
                          round(f["iters_per_solve"], 3), round(x["iters_per_solve"], 3),
                          f["failed"], x["failed"], float("%.3g" % np.median(d)),
                          _hist(iters[0]), _hist(iters[1])])
            # the reference's opt() on a prefix of the same vectors, without those the FP64
            # closure reports as exhausting the ladder (there the reference aborts,
            # src/opt/opt.cpp:261-266)
            try:
                rr = ref_standalone(q, u[ok0], a_iso[ok0])
                m = rr["n"]
                ra = rr["alpha"]
                ok = np.isfinite(ra).all(axis=1)

                def err(ag):
                    g = ag[ok0][:m][ok]
                    e = np.linalg.norm(g - ra[ok], axis=1) / np.linalg.norm(ra[ok], axis=1)
                    return [float("%.3g" % np.median(e)), float("%.3g" % np.percentile(e, 99))]
                ref_rows.append([N, m, round(m / rr["seconds"]), rr["threads"],
                                 float("%.4g" % np.mean(rr["iters"] == iters[0][ok0][:m])),
                                 err(alphas[0]), err(alphas[1])])
            except Exception as ex:  # reported, not fatal
                ref_rows.append([N, f"failed: {ex}"])
        group = None
        if graphs:
            # all seven orders in one launch: one CUDA graph, the orders' closures as its
            # parallel branches
            G = c3d.Group([s.ctx_handle for s in solvers])
            counts = [len(u) for u, _ in vecs]
            group = dict(launches=1, vectors=int(sum(counts)))
            for mode in (0, 1):
                for s in solvers:
                    c3d.check(L.c3d_set_precision(s.ctx_handle, mode, 0.0, 0.0, 0, 0.0), "prec")
                for warm in (True, False):
                    gb = [bufs(u, a) for u, a in vecs]
                    torch.cuda.synchronize()
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    G.closure_vectors(counts, [b[0].data_ptr() for b in gb],
                                      [b[1].data_ptr() for b in gb],
                                      iters=[b[2].data_ptr() for b in gb],
                                      status=[b[3].data_ptr() for b in gb])
                    e1.record(stream)
                    torch.cuda.synchronize()
                for s in solvers:
                    # failed vectors (status 2: ladder exhausted) are counted, not raised
                    st_ = L.c3d_sync(s.ctx_handle)
                    if st_ not in (c3d.C3D_OK, 4):
                        c3d.check(st_, "group closure")
                ms = e0.elapsed_time(e1)
                key = "fp64" if mode == 0 else "mixed"
                group[key + "_solves_per_s"] = group["vectors"] / (ms * 1e-3)
                group[key + "_ms"] = ms
                group[key + "_failed"] = int(sum(int((b[3] != 0).sum()) for b in gb))
            group["mixed_over_fp64"] = group["mixed_solves_per_s"] / group["fp64_solves_per_s"]
            G.close()
    finally:
        for s in solvers:
            s.close()
    dall = np.concatenate(diffs)
    f64 = tot[0][0] / (tot[0][1] * 1e-3)
    mix = tot[1][0] / (tot[1][1] * 1e-3)
    return dict(
        workload=f"{7 * STANDALONE_PER_N} moment vectors, N uniform over 1..7 "
                 f"({STANDALONE_PER_N} per order), tensor quadrature 2(N+3) x 4(N+3), "
                 "seeded multipliers, solved from the isotropic start (unbatched rules, MN_TOL "
                 "1e-8)",
        one_launch=group,
        per_order_calls=dict(fp64_solves_per_s=f64, mixed_solves_per_s=mix,
                             mixed_over_fp64=mix / f64, launches=7),
        alpha_rel_diff_median=float(np.median(dall)),
        alpha_rel_diff_p99=float(np.percentile(dall, 99)),
        per_order_columns=["N", "fp64 solves/s", "mixed solves/s", "mixed/fp64",
                           "iters fp64", "iters mixed", "failed fp64", "failed mixed",
                           "alpha rel diff median", "iteration histogram fp64",
                           "iteration histogram mixed"],
        histogram_bins=f"iterations in [{HIST_EDGES[0]}, {HIST_EDGES[1]}), ... "
                       f"[{HIST_EDGES[-1]}, inf)",
        per_order=per_n,
        reference_columns=["N", "sample vectors", "reference solves/s", "threads",
                           "iteration counts equal to the GPU FP64 (fraction)",
                           "alpha rel err vs reference, GPU FP64 [median, p99]",
                           "alpha rel err vs reference, GPU mixed [median, p99]"],
        reference=ref_rows,
        reference_note="the reference's unbatched opt() (oracle/_ref, OpenMP over vectors, "
                       "direct Hessian) on a prefix of each order's vectors sized for ~"
                       f"{STANDALONE_REF_SAMPLE_S:g} s, one process per order; vectors the FP64 "
                       "closure reports as exhausting the ladder are left out (the reference "
                       "aborts on them)")


# ------------------------------------------------------------------ serving workload
SERVE_STREAM = 256        # problems of the seeded stream
SERVE_PROBLEMS = 8        # of which the bench runs the first ... per arm (bounded run time)
SERVE_GAP_S = 0.05        # mean of the exponential inter-arrival gaps
SERVE_BUDGET = 150 << 30  # device-memory budget of the admitted problems
SERVE_SLOTS = 64          # problems active at once at most


def gaunt_table_times(c3d, N, Q):
    """Seconds to build the Gaunt tables of order N over the Q-point quadrature: on the host
    (c3d_gaunt_dense, the least-squares loop of the reference's init) and on the device
    (c3d_gaunt_build, second call), with the largest difference between the two."""
    q = c3d.quadrature(N, Q, with_m2=True)
    nm, nm2, nq = q["nm"], q["nm2"], q["nq"]
    L = c3d.lib()
    L.c3d_gaunt_dense.argtypes = [ctypes.c_int] * 3 + [ctypes.POINTER(ctypes.c_double)] * 2
    beta = np.zeros(nm * nm * nm2)
    t0 = time.perf_counter()
    L.c3d_gaunt_dense(nm, nm2, nq, q["M2"].ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                      beta.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    host = time.perf_counter() - t0
    c3d.gaunt_build(nm, nm2, nq, q["M2"])
    t0 = time.perf_counter()
    dev = c3d.gaunt_build(nm, nm2, nq, q["M2"])[0]
    device = time.perf_counter() - t0
    return dict(N=N, Q=Q, host_s=round(host, 4), device_s=round(device, 4),
                max_abs_diff=float(np.abs(dev.ravel() - beta).max()))


def serving_stream(n_problems, mixed):
    """The serving workload's seeded problem stream: cubic grid with edge uniform in 16..96,
    N in {1, 3, 5}, sigma_s uniform in [0.5, 20], a Gaussian pulse of width uniform in
    [0.02, 0.2] over a 1e-8 floor, final time uniform in [0.1, 0.5]; Poisson arrivals with a
    mean gap of 50 ms. Quadrature 2(N+3) mu x 4(N+3) phi, Gaunt sparse Hessian, MN_TOL 1e-6,
    batched rules, the benchmark ladder. Returns [(arrival_s, deck_text, edge, N)]."""
    rng = np.random.default_rng(2015_5)
    out, t = [], 0.0
    for k in range(SERVE_STREAM):
        n = int(rng.integers(16, 97))
        N = int(rng.choice([1, 3, 5]))
        sig_s = float(rng.uniform(0.5, 20.0))
        width = float(rng.uniform(0.02, 0.2))
        tf = float(rng.uniform(0.1, 0.5))
        t += float(rng.exponential(SERVE_GAP_S))
        if k >= n_problems:
            continue
        kv = dict(SOLVER="mn", TFINAL=repr(tf), OUTDT=repr(tf), OUTPUT_DATA="false",
                  OUTPUT_OPT_STATS="false", OUTPUT_TIMINGS="false", NX=n, NY=n, NZ=n,
                  MPIX=1, MPIY=1, MPIZ=1, AX=-1, AY=-1, AZ=-1, BX=1, BY=1, BZ=1,
                  MOMENT_ORDER=N, QUAD_ORDER=2 * (N + 3), CFL_FACTOR=0.5, CROSS_SECTION=sig_s,
                  INIT_FLOOR=1e-8, GAUSS_SIGMA=width, INIT_COND="gaussian_psi", THETA=2.0,
                  OMP_THREADS=1, PN_USE_KINETIC_FLUX=0, MN_TOL=MN_TOL, MN_TOL_GAMMA=1.1,
                  MN_COND_H_MAX=1e10, MN_MAX_ITER=100, MN_BATCHED="true",
                  MN_USE_GAUNT_COEF="true", MN_USE_GAUNT_SPARSE="true", CUDA_KINETIC="true",
                  CUDA_BATCHED="true", CUDA_BATCH_SIZE=50, REG_LADDER=LADDER,
                  MN_MIXED_PRECISION="true" if mixed else "false")
        out.append((t, "".join(f"{k_} {v}\n" for k_, v in kv.items()), n, N))
    return out


def serving_workload(c3d, n_problems):
    """The serving workload on the B200 serving loop (include/c3d_serve.h), mixed and FP64 arms
    on the same seeded stream: requests submitted at their arrival times by a host thread,
    completion latency per request (submission to result) and aggregate cell-solves/s (interior
    cells x 2 stages x steps of every problem, over the time from the first submission to the
    last completion)."""
    res = {}
    for mixed in (True, False):
        stream = serving_stream(n_problems, mixed)
        srv = c3d.Server(workers=SERVE_SLOTS, hbm_budget=SERVE_BUDGET)
        ids = [None] * len(stream)
        t0 = time.perf_counter()

        def feed():
            for k, (ta, deck, _, _) in enumerate(stream):
                d = ta - (time.perf_counter() - t0)
                if d > 0:
                    time.sleep(d)
                ids[k] = srv.submit(deck)
        th = threading.Thread(target=feed)
        th.start()
        th.join()
        lat, solves, failed = [], 0, 0
        for (ta, deck, n, N), rid in zip(stream, ids):
            st, u, latency, steps = srv.wait(rid)
            lat.append(latency)
            solves += n ** 3 * 2 * steps
            failed += int(st != 0)
        wall = time.perf_counter() - t0
        peak_bytes, peak_active = srv.stats()
        sched = srv.timing()
        srv.close()
        res["mixed" if mixed else "fp64"] = dict(
            cell_solves_per_s=solves / wall, wall_s=wall, cell_solves=solves,
            latency_p50_s=float(np.percentile(lat, 50)),
            latency_p99_s=float(np.percentile(lat, 99)), failed_problems=failed,
            peak_active=peak_active, peak_budget_gb=peak_bytes / 1e9,
            scheduler={k: (round(v, 3) if isinstance(v, float) else v) for k, v in sched.items()})
    res["mixed_over_fp64"] = res["mixed"]["cell_solves_per_s"] / res["fp64"]["cell_solves_per_s"]
    res["workload"] = (f"first {n_problems} of the {SERVE_STREAM}-problem seeded stream: edge "
                       "uniform 16..96, N in {1,3,5}, sigma_s U[0.5,20], pulse width U[0.02,0.2] "
                       "floor 1e-8, final time U[0.1,0.5], Poisson arrivals (mean gap 50 ms), "
                       f"{SERVE_BUDGET >> 30} GiB budget, up to {SERVE_SLOTS} problems per pass "
                       "(one CUDA graph launch steps them all)")
    return res


# ------------------------------------------------------------------ B200 arm
def b200_arm(args):
    import torch
    import torch.distributed as dist

    import c3d

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    cfg = args.config
    c = CONFIGS[cfg]
    # a dedicated (non-default) stream: the library launches on it and the CUDA events
    # below are recorded on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    with tempfile.TemporaryDirectory() as tmp:
        deck = os.path.join(tmp, "input.deck")
        with open(deck, "w") as f:
            f.write(deck_for(cfg, threads=os.cpu_count() or 1, hessian=args.hessian))
        solver = c3d.Solver(deck, stream=ctypes.c_void_p(stream.cuda_stream))
    ctxh = solver.ctx_handle
    L = c3d.lib()
    c3d.check(L.c3d_set_engine(ctxh, 0 if args.engine == "rounds" else 1), "engine")
    c3d.check(L.c3d_set_graphs(ctxh, 1 if args.graphs else 0), "graphs")
    dt = solver.max_dt
    nm, nq = solver.nm, solver.nq

    failed = [0]

    def sync_count():
        st_ = L.c3d_sync(ctxh)
        if st_ == 4:  # C3D_ERR_CLOSURE: cells whose ladder ran out (the reference would abort)
            failed[0] += 1
        elif st_ != 0:
            c3d.check(st_, "sync")

    nv = solver.nall * nm
    hu = torch.empty(nv, dtype=torch.float64).pin_memory()
    ha = torch.empty(nv, dtype=torch.float64).pin_memory()
    precision = 1 if args.precision == "mixed" else 0

    def set_precision(mode):
        c3d.check(L.c3d_set_precision(ctxh, mode, 0.0, 0.0, 0, 0.0), "precision")

    def save_state(u_, a_):
        c3d.check(L.c3d_get_state(ctxh, ctypes.c_void_p(u_.data_ptr()),
                                  ctypes.c_void_p(a_.data_ptr()), 0), "get_state")

    def load_state(u_, a_):
        c3d.check(L.c3d_set_state(ctxh, ctypes.c_void_p(u_.data_ptr()),
                                  ctypes.c_void_p(a_.data_ptr()), None, None, 0), "set_state")

    # flux autotuner (direction chunk, z run per CTA), on the initial state
    tuned = None
    if args.autotune:
        tq, tr, tms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        c3d.check(L.c3d_autotune(ctxh, ctypes.byref(tq), ctypes.byref(tr), ctypes.byref(tms)),
                  "autotune")
        tuned = dict(q_chunk=tq.value, z_run=tr.value or min(64, CONFIGS[cfg]["n"]),
                     flux_ms=tms.value)

    # warm-up (FP64), then the start state S of both timed arms
    set_precision(0)
    for _ in range(args.warmup):
        solver.update(dt)
    sync_count()
    u_s = torch.empty(nv, dtype=torch.float64).pin_memory()
    a_s = torch.empty(nv, dtype=torch.float64).pin_memory()
    save_state(u_s, a_s)
    if precision == 1:
        # the mixed kernels' first launches, from S (untimed)
        set_precision(1)
        for _ in range(args.warmup):
            solver.update(dt)
        sync_count()

    peak = fp64_peak_tflops() if rank == 0 else None

    def timed(mode, sample_clocks, breakdown=False, steps=None):
        """Device-resident steps from S with the given closure precision: each RK stage one
        CUDA graph launch, or with breakdown (CUDA events around the closure and flux launches)
        stage by stage."""
        nsteps = steps or args.steps
        set_precision(mode)
        load_state(u_s, a_s)
        L.c3d_closure_stats_reset(ctxh)
        L.c3d_timing_enable(ctxh, 1 if breakdown else 0)
        syncs0 = solver.stats().hostSyncs
        launches0 = L.c3d_launch_count(ctxh)
        clocks = ClockSampler(local) if sample_clocks else None
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        if clocks:
            clocks.start()
            time.sleep(0.3)
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(nsteps + 1)]
        evs[0].record(stream)
        for k in range(nsteps):
            solver.update(dt)
            evs[k + 1].record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        clk = clocks.stop() if clocks else None
        launches = L.c3d_launch_count(ctxh) - launches0
        sync_count()
        step_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(nsteps)]
        total_ms = evs[0].elapsed_time(evs[-1])
        ms = np.zeros(2)
        cnt = (ctypes.c_longlong * 2)()
        L.c3d_timing_get(ctxh, ms.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cnt)
        L.c3d_timing_enable(ctxh, 0)
        st = solver.stats()
        syncs = st.hostSyncs - syncs0
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        uo = torch.empty(nv, dtype=torch.float64)
        ao = torch.empty(nv, dtype=torch.float64)
        fo = torch.empty(nv, dtype=torch.float64)
        save_state(uo, ao)
        c3d.check(L.c3d_get_flux(ctxh, ctypes.c_void_p(fo.data_ptr()), 0), "get_flux")
        torch.cuda.synchronize()
        return dict(max_ms=float(t.item()), step_ms=step_ms, ms=ms, cnt=cnt, launches=launches,
                    clk=clk, st=st, u=uo.numpy(), a=ao.numpy(), f=fo.numpy(), syncs=syncs,
                    steps=nsteps)

    cells = interior_cells(cfg)
    if args.compare:
        # the other arm's graphs, instantiated from S untimed (the timed arm's were built by
        # the warm-up)
        set_precision(1 - precision)
        load_state(u_s, a_s)
        solver.update(dt)
        sync_count()
    other = timed(1 - precision, False) if args.compare else None
    head = timed(precision, True)
    # closure / flux split: a short run with CUDA events around each launch (stage by stage)
    split = timed(precision, False, breakdown=True, steps=min(2, args.steps))
    max_ms, step_ms = head["max_ms"], head["step_ms"]
    ms, cnt = split["ms"], split["cnt"]
    launches, clk, st = head["launches"], head["clk"], head["st"]
    total_ms = max_ms
    value = world * cells * 2 * args.steps / (max_ms * 1e-3)

    # end-to-end: host buffers through the C ABI, copies inside the timed region
    save_state(hu, ha)
    e_steps = args.steps
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e_steps):
        load_state(hu, ha)
        solver.update(dt)
        save_state(hu, ha)
    e1.record(stream)
    torch.cuda.synchronize()
    sync_count()
    te = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * cells * 2 * e_steps / (float(te.item()) * 1e-3)

    if rank == 0:
        closure_launches = int(cnt[0])
        sst = split["st"]  # counters of the split run, whose closures the events time
        low = None
        if precision == 1:
            flops, low = closure_flops_mixed(nm, nq, sst)
        else:
            flops = closure_flops(nm, nq, sst.totalIters, sst.trials, args.hessian, sst.certified)
        per_launch_s = ms[0] * 1e-3 / max(1, closure_launches)
        achieved = flops / max(1, closure_launches) / per_launch_s / 1e12
        closure_roofline = dict(
            bound="tensor",
            pipe=("fp64 (DMMA m8n8k4 + DFMA); the mixed closure's BF16 / 3xTF32 moments run on "
                  "tcgen05 beside it (lowp_tflops)" if precision == 1
                  else "fp64 (DMMA m8n8k4 + DFMA)"),
            achieved=achieved, peak=peak, unit="TFLOP/s", frac=achieved / peak if peak else None,
            traffic=(profile_traffic("closure_rounds_m6_64")
                     if args.engine == "rounds" and args.hessian == "gaunt" else None),
            traffic_source="profiles/closure_rounds_m6_64.txt: one closure's DRAM bytes at 64^3 "
                           "(ncu) scaled by solved cells to 128^3",
            peak_source="in-run cuBLAS DGEMM 8192^3 via torch (FP64 is not in "
                        "MEASURED_PEAKS.json)",
            kernel=(("closure work-list rounds: rounds_pass_mixed_kernel<7,22,2> (first-visit "
                     "probe) + rounds_pass_gaunt_kernel<7,22> + rounds_newton_kernel"
                     if args.hessian == "gaunt" else
                     "closure work-list rounds: rounds_pass_direct_kernel<7> + "
                     "rounds_newton_kernel") if args.engine == "rounds" else
                    ("closure_gaunt_kernel<7,22,8>" if args.hessian == "gaunt"
                     else "closure_fp64_kernel<7,8>")),
            unit_of_launch="one c3d_closure call (all its kernels)",
            flops_per_launch=flops / max(1, closure_launches),
            ms_per_launch=ms[0] / max(1, closure_launches),
            share_of_step=ms[0] / split["max_ms"])
        if low is not None:
            closure_roofline["lowp_tflops"] = low / max(1, closure_launches) / per_launch_s / 1e12
            closure_roofline["kernel"] = (
                "closure work-list rounds: rounds_pass_mixed_kernel<7,22,2> (first-visit probe), "
                "<7,22,0|1> (tcgen05 Hessian moments), rounds_pass_gaunt_kernel<7,22> (trials, "
                "FP64 Hessians) + rounds_newton_kernel")
        compare = None
        if other is not None:
            fp, mx = (other, head) if precision == 1 else (head, other)
            vf = world * cells * 2 * args.steps / (fp["max_ms"] * 1e-3)
            vm = world * cells * 2 * args.steps / (mx["max_ms"] * 1e-3)
            du = np.linalg.norm(mx["u"] - fp["u"]) / np.linalg.norm(fp["u"])
            da = np.linalg.norm(mx["a"] - fp["a"]) / np.linalg.norm(fp["a"])
            df = np.linalg.norm(mx["f"] - fp["f"]) / np.linalg.norm(fp["f"])
            sm = mx["st"]
            compare = dict(
                fp64=dict(value=vf, ms_per_step=fp["max_ms"] / args.steps,
                          closure_ms_per_launch=fp["ms"][0] / max(1, int(fp["cnt"][0])),
                          newton_iters_per_solve=fp["st"].totalIters / max(1, fp["st"].cells),
                          failed_cells=int(fp["st"].failed)),
                mixed=dict(value=vm, ms_per_step=mx["max_ms"] / args.steps,
                           closure_ms_per_launch=mx["ms"][0] / max(1, int(mx["cnt"][0])),
                           newton_iters_per_solve=sm.totalIters / max(1, sm.cells),
                           failed_cells=int(sm.failed),
                           hessians=dict(bf16=int(sm.hessBf16), tf32x3=int(sm.hessTf32x3),
                                         fp64=int(sm.hessFp64), redone_fp64=int(sm.escalated))),
                mixed_over_fp64=vm / vf,
                residual="equal: both closures stop on the FP64 test |<m e^{alpha.m}> - u| <= "
                         "MN_TOL with gamma <= MN_TOL_GAMMA",
                moments_rel_l2=du, alpha_rel_l2=da, flux_div_rel_l2=df,
                accuracy_note=f"u, alpha and the last stage's flux divergence after the "
                              f"{args.steps} timed steps from the same start state, mixed vs "
                              "the FP64 drop-in (all cells incl. ghosts); the FP64 drop-in "
                              "matches the C oracle to 1e-12 (tests)")
        # the dominant kernel: the kinetic flux's stencil + projection (kinetic_staged_kernel),
        # one launch per flux call when the closure handed its ansatz over (psi of all
        # directions within the 32 GiB budget). Algorithmic work per (cell, direction):
        # 2 nm FLOPs of projection + 60 of the three axes' limited upwind differences; bytes:
        # psi of the interior cells and the two face-ghost layers read once, the flux written.
        n_ = CONFIGS[cfg]["n"]
        face_ghosts = 12 * n_ * n_  # two layers on each of the six faces
        handoff = solver.nall * nq * 8 <= (32 << 30)
        flux_ms = ms[1] / max(1, int(cnt[1]))
        stencil_flops = float((2 * nm + 60) * nq) * cells
        stencil_bytes = 8.0 * ((cells + face_ghosts) * nq + cells * nm)
        achieved_k = stencil_flops / (flux_ms * 1e-3) / 1e12
        traffic_k = profile_traffic("kinetic_staged_m6_64", "dram_bytes_per_launch:")
        if traffic_k is not None:
            traffic_k *= cells / 64 ** 3  # ncu capture at 64^3, scaled by (cell, direction) pairs
        roofline = dict(
            bound="tensor", pipe="fp64 (DMMA m8n8k4 projection + DFMA/ALU limiter)",
            kernel="kinetic_staged_kernel<7> (kinetic flux: MUSCL stencil + projection)",
            achieved=achieved_k, peak=peak, unit="TFLOP/s",
            frac=achieved_k / peak if peak else None,
            traffic=traffic_k,
            traffic_source="profiles/kinetic_staged_m6_64.txt: dram__bytes_read.sum + "
                           "dram__bytes_write.sum of one launch at 64^3 (ncu), scaled by "
                           "(cell, direction) pairs to this grid",
            peak_source="in-run cuBLAS DGEMM 8192^3 via torch (FP64 is not in "
                        "MEASURED_PEAKS.json)",
            flops_per_launch=stencil_flops,
            flops_per_cell_direction=2 * nm + 60,
            ms_per_launch=flux_ms, stencil_only=handoff,
            share_of_step=ms[1] / split["max_ms"],
            hbm=dict(algorithmic_bytes_per_launch=stencil_bytes,
                     achieved_gbs=stencil_bytes / (flux_ms * 1e-3) / 1e9,
                     peak_gbs=HBM_PEAK_GBS,
                     frac=stencil_bytes / (flux_ms * 1e-3) / 1e9 / HBM_PEAK_GBS,
                     peak_source="MEASURED_PEAKS.json hbm_gbs (of measured)"),
            note="FP64-pipe and issue bound (ncu: FP64 pipe, ALU and shared-memory wavefronts "
                 "busy, DRAM idle most of the launch); the closure is second "
                 "(closure_roofline)")
        # CPU baseline: the reference closure on a bounded sample of this workload's cells
        cpu = None
        try:
            uh = hu.numpy().reshape(-1, nm)
            ah = ha.numpy().reshape(-1, nm)
            rng = np.random.default_rng(7)
            pick = rng.choice(uh.shape[0], size=min(uh.shape[0], 400000), replace=False)
            su, sa = uh[pick].copy(), ah[pick].copy()
            n_s, _ = calibrated_ref_sample(cfg, su, sa, target_s=12.0, hessian=args.hessian)
            res = run_ref_sample(cfg, su[:n_s], sa[:n_s], 1, args.hessian)
            cpu = dict(value=n_s / res["times"][0], unit=UNIT, cores=res["threads"],
                       kind="reference",
                       sample=f"{n_s} cells sampled uniformly from the state after the timed "
                              f"steps, one batched closure (Optimization::opt); closure only")
        except Exception as ex:  # reported, not fatal
            cpu = dict(value=None, unit=UNIT, cores=os.cpu_count(), kind="reference",
                       sample=f"failed: {ex}")
        hist = {str(i): int(st.iterHist[i]) for i in range(64) if st.iterHist[i]}
        serving = None
        if args.serving and world == 1:
            try:
                serving = serving_workload(c3d, args.serve_problems)
            except Exception as ex:  # reported, not fatal
                serving = dict(error=str(ex))
        standalone = None
        if args.standalone and world == 1:
            try:
                standalone = standalone_closure(torch, c3d, stream, args.graphs)
            except Exception as ex:  # reported, not fatal
                standalone = dict(error=str(ex))
        line = dict(
            metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps,
            warmup=args.warmup, ms_per_step=max_ms / args.steps, higher_is_better=True,
            scaling="weak", vs_baseline=None,
            dtype="f64 + bf16/tf32 (tcgen05, FP32 accumulate)" if precision == 1 else "f64",
            data="synthetic",
            config=dict(workload=c["desc"], config=cfg,
                        form=("mixed precision: Gaunt moments BF16 / 3xTF32 on tcgen05 with "
                              "FP32 accumulation, FP64 gradient, objective, factorisation and "
                              "fallback" if precision == 1 else "plain FP64 drop-in"),
                        hessian=("Gaunt sparse (MN_USE_GAUNT_COEF/SPARSE true, the reference "
                                 "deck's default)" if args.hessian == "gaunt" else "direct"),
                        engine=args.engine,
                        mn_tol=MN_TOL, mn_batched=True, ladder=LADDER,
                        cells_per_step=2 * cells,
                        l2=f"inputs larger than L2 (u, alpha {nv * 8 / 1e9:.2f} GB each)",
                        flux_autotune=tuned,
                        parallelism=f"replicas x{world}"),
            roofline=roofline, closure_roofline=closure_roofline, cpu_baseline=cpu,
            precision_compare=compare,
            standalone_closure=standalone, serving=serving,
            e2e=dict(value=e2e_value, unit=UNIT, h2d_bytes_per_step=2 * nv * 8,
                     d2h_bytes_per_step=2 * nv * 8, steps=e_steps),
            gpu_launches=int(launches), clocks=clk,
            stage_graphs=dict(launches_per_step=launches / args.steps,
                              host_syncs_per_step=head["syncs"] / args.steps,
                              note=("each RK stage is one CUDA graph launch (closure rounds in a "
                                    "device-side conditional loop)" if args.graphs else
                                    "--no-graphs: kernels launched one by one, closure rounds "
                                    "driven by the host") +
                                   "; launches counted by the library, device-side loop "
                                   "kernels included"),
            closure_only=dict(value=cells / (ms[0] / max(1, closure_launches) * 1e-3), unit=UNIT,
                              ms_per_closure=ms[0] / max(1, closure_launches),
                              note="interior cell-solves per second of the closure alone (the "
                                   "same quantity as cpu_baseline, which times the reference's "
                                   "closure only)"),
            latency_ms=dict(p50=float(np.percentile(step_ms, 50)),
                            p99=float(np.percentile(step_ms, 99)), unit="ms per RK2 step"),
            iter_histogram=hist, newton_iters_per_solve=st.totalIters / max(1, st.cells),
            failed_cells_timed=int(st.failed), syncs_with_failed_cells=failed[0],
            closure_phase_clocks=dict(refill=st.clkRefill, passes=st.clkPass,
                                      newton_logic=st.clkSerial, n_passes=st.passes))
        # compact figures of the other two workloads, near the end of the line
        summary = {}
        ol = (standalone or {}).get("one_launch")
        if ol:
            summary["standalone_one_launch"] = dict(
                fp64_solves_per_s=round(ol["fp64_solves_per_s"]),
                mixed_solves_per_s=round(ol["mixed_solves_per_s"]),
                mixed_over_fp64=round(ol["mixed_over_fp64"], 3))
        if serving and "mixed" in serving:
            summary["serving"] = {a: dict(cell_solves_per_s=round(serving[a]["cell_solves_per_s"]),
                                          p50_s=round(serving[a]["latency_p50_s"], 3),
                                          p99_s=round(serving[a]["latency_p99_s"], 3))
                                  for a in ("mixed", "fp64")}
        wl = CONFIGS[cfg]
        summary["gaunt_tables"] = gaunt_table_times(c3d, wl["N"], wl["Q"])
        if summary:
            line["workloads"] = summary
        if compare is not None:
            # last key, so that it stays in a tail of the output: the mixed arm's error
            line["accuracy"] = dict(vs="fp64 drop-in arm", moments_rel_l2=compare["moments_rel_l2"],
                                    alpha_rel_l2=compare["alpha_rel_l2"],
                                    flux_div_rel_l2=compare["flux_div_rel_l2"],
                                    mixed_over_fp64=compare["mixed_over_fp64"])
        print(json.dumps(line), flush=True)
    solver.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="c3", choices=sorted(CONFIGS))
    ap.add_argument("--hessian", default="gaunt", choices=["gaunt", "direct"])
    ap.add_argument("--engine", default="rounds", choices=["rounds", "persistent"])
    ap.add_argument("--no-graphs", dest="graphs", action="store_false",
                    help="launch the stages kernel by kernel with host-driven closure rounds "
                         "(for profilers that do not look inside CUDA graphs' conditional nodes)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="closure precision of the reported arm (mixed: the configuration's "
                         "form; fp64: the drop-in)")
    ap.add_argument("--no-compare", dest="compare", action="store_false",
                    help="skip the other precision's arm")
    ap.set_defaults(compare=True)
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="skip the flux autotuner (keeps its defaults; for launch lists)")
    ap.add_argument("--no-serving", dest="serving", action="store_false",
                    help="skip the serving workload (a bounded sample of the 256-problem "
                         "stream, mixed vs FP64)")
    ap.add_argument("--serve-problems", type=int, default=SERVE_PROBLEMS,
                    help="problems of the seeded serving stream to run per arm")
    ap.add_argument("--no-standalone", dest="standalone", action="store_false",
                    help="skip the standalone-closure comparison (2^20 vectors, N = 1..7)")
    ap.set_defaults(standalone=True)
    ap.add_argument("--standalone-order", type=int, default=0,
                    help="profiling aid: only one order's standalone closure (the first "
                         "--standalone-vectors vectors), in the --precision arm, then exit")
    ap.add_argument("--standalone-vectors", type=int, default=40000)
    args = ap.parse_args()
    if args.standalone_order:
        standalone_one_order(args)
        return
    if args.engine != "rounds" or args.hessian != "gaunt":
        # the mixed closure is built on the work-list engine's Gaunt form
        args.precision = "fp64"
        args.compare = False
    if args.impl == "reference":
        reference_arm(args)
    else:
        b200_arm(args)


if __name__ == "__main__":
    main()
