"""Python binding of libc3d_b200.so (the C ABI in include/c3d_b200.h).

Thin ctypes layer used by the tests and the benchmark. There is no fallback:
if the library is missing or no CUDA device is usable, calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libc3d_b200.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)

C3D_OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "NO_DEVICE", 4: "CLOSURE", 5: "TIMEOUT",
                6: "OOM"}

# the symbols include/c3d_solver.h declares
SOLVER_SYMBOLS = [
    "c3d_solver_create", "c3d_solver_prepare", "c3d_solver_destroy", "c3d_solver_update",
    "c3d_solver_run", "c3d_solver_pull", "c3d_solver_push", "c3d_solver_context",
    "c3d_solver_info", "c3d_solver_host_array", "c3d_solver_output_data",
    "c3d_solver_checkpoint", "c3d_solver_restore", "c3d_solver_output_timings",
    "c3d_solver_output_opt_stats",
]

# the symbols include/c3d_serve.h declares
SERVE_SYMBOLS = [
    "c3d_server_create", "c3d_server_submit", "c3d_server_wait", "c3d_server_stats",
    "c3d_server_estimate", "c3d_server_timing", "c3d_server_destroy",
]

# the symbols include/c3d_b200.h declares
HEADER_SYMBOLS = [
    "c3d_last_error", "solveFluxKinetic_cuda", "solveH_cuda", "solveHInit_cuda", "c3d_create",
    "c3d_destroy", "c3d_set_state", "c3d_get_state", "c3d_get_flux", "c3d_device_state",
    "c3d_ghost_fill", "c3d_closure", "c3d_flux_kinetic", "c3d_flux_moment", "c3d_euler",
    "c3d_step", "c3d_sync", "c3d_closure_records", "c3d_closure_stats_get",
    "c3d_closure_stats_reset", "c3d_closure_vectors", "c3d_build_quadrature",
    "c3d_launch_count", "c3d_timing_enable", "c3d_timing_get", "c3d_closure_vectors_noalloc",
    "c3d_set_gaunt", "c3d_set_engine", "c3d_set_ghost_mirroring", "c3d_timing_events",
    "c3d_closure_records_fp", "c3d_line_stats_enable", "c3d_line_stats_get", "c3d_stage",
    "c3d_set_x_halo_external", "c3d_copy_x_planes", "c3d_set_precision",
    "c3d_set_certificate", "c3d_autotune", "c3d_closure_vectors_noalloc_check",
    "c3d_set_limits", "c3d_set_ansatz_handoff", "c3d_set_graphs", "c3d_group_create",
    "c3d_group_closure_vectors", "c3d_group_step", "c3d_group_destroy", "c3d_stage_part",
    "c3d_gaunt_build",
]


class C3DError(RuntimeError):
    pass


class Params(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("nm", ctypes.c_int), ("nq", ctypes.c_int), ("dx", ctypes.c_double),
                ("dy", ctypes.c_double), ("dz", ctypes.c_double), ("theta", ctypes.c_double),
                ("solver", ctypes.c_int), ("pnUseKineticFlux", ctypes.c_int),
                ("mnBatched", ctypes.c_int), ("mnMaxIter", ctypes.c_int),
                ("mnTol", ctypes.c_double), ("mnTolGamma", ctypes.c_double),
                ("mnCondHMax", ctypes.c_double), ("nreg", ctypes.c_int),
                ("reg", ctypes.c_double * 16), ("psiBytes", ctypes.c_size_t),
                ("mnReproject", ctypes.c_int)]


class ClosureStats(ctypes.Structure):
    _fields_ = [("cells", ctypes.c_longlong), ("interiorCells", ctypes.c_longlong),
                ("totalIters", ctypes.c_longlong), ("maxIter", ctypes.c_int),
                ("maxIterGamma", ctypes.c_int), ("totalIterGamma", ctypes.c_longlong),
                ("failed", ctypes.c_longlong), ("trials", ctypes.c_longlong),
                ("clkRefill", ctypes.c_longlong), ("clkPass", ctypes.c_longlong),
                ("clkSerial", ctypes.c_longlong), ("passes", ctypes.c_longlong),
                ("regHist", ctypes.c_longlong * 16),
                ("iterHist", ctypes.c_longlong * 64),
                ("clkNewton", ctypes.c_longlong * 8), ("hessBf16", ctypes.c_longlong),
                ("hessTf32x3", ctypes.c_longlong), ("hessFp64", ctypes.c_longlong),
                ("escalated", ctypes.c_longlong), ("certified", ctypes.c_longlong),
                ("hostSyncs", ctypes.c_longlong)]


_lib = None


def lib():
    """Loads the library once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise C3DError(f"{LIB_PATH} not built (run `make -C c3d-2015_b200`)")
        L = ctypes.CDLL(LIB_PATH)
        L.c3d_last_error.restype = ctypes.c_char_p
        vp = ctypes.c_void_p
        for name in ["c3d_ghost_fill", "c3d_closure", "c3d_flux_moment", "c3d_sync",
                     "c3d_closure_stats_reset"]:
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = ctypes.c_int
        L.c3d_create.argtypes = [ctypes.POINTER(Params), _dp, _dp, _dp, _dp, _dp, _dp, vp,
                                 ctypes.POINTER(vp)]
        L.c3d_create.restype = ctypes.c_int
        L.c3d_destroy.argtypes = [vp]
        L.c3d_set_state.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int]
        L.c3d_get_state.argtypes = [vp, vp, vp, ctypes.c_int]
        L.c3d_get_flux.argtypes = [vp, vp, ctypes.c_int]
        L.c3d_flux_kinetic.argtypes = [vp, ctypes.c_int]
        L.c3d_euler.argtypes = [vp, ctypes.c_double]
        L.c3d_step.argtypes = [vp, ctypes.c_double]
        L.c3d_closure_records.argtypes = [vp, vp, vp, vp, vp]
        L.c3d_closure_stats_get.argtypes = [vp, ctypes.POINTER(ClosureStats)]
        L.c3d_closure_vectors.argtypes = [vp, ctypes.c_longlong, vp, vp, vp, vp, vp, vp]
        L.c3d_device_state.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                       ctypes.POINTER(vp)]
        L.c3d_build_quadrature.argtypes = [ctypes.c_int, ctypes.c_int] + [_dp] * 6
        L.c3d_set_gaunt.argtypes = [vp, ctypes.c_int, _dp, _ip, _ip, _dp]
        L.c3d_gaunt_build.argtypes = [ctypes.c_int] * 3 + [_dp, ctypes.c_double, _dp, _ip,
                                      ctypes.c_longlong, _ip, _dp,
                                      ctypes.POINTER(ctypes.c_longlong)]
        L.c3d_set_engine.argtypes = [vp, ctypes.c_int]
        L.c3d_set_precision.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_int, ctypes.c_double]
        L.c3d_set_certificate.argtypes = [vp, ctypes.c_int]
        L.c3d_autotune.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_double)]
        L.c3d_set_ghost_mirroring.argtypes = [vp, ctypes.c_int]
        L.c3d_set_limits.argtypes = [vp, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong]
        L.c3d_set_ansatz_handoff.argtypes = [vp, ctypes.c_int]
        L.c3d_set_graphs.argtypes = [vp, ctypes.c_int]
        L.c3d_group_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp), ctypes.POINTER(vp)]
        L.c3d_group_closure_vectors.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)] + \
            [ctypes.POINTER(vp)] * 6
        L.c3d_group_step.argtypes = [vp, _dp]
        L.c3d_group_destroy.argtypes = [vp]
        L.c3d_timing_enable.argtypes = [vp, ctypes.c_int]
        L.c3d_timing_get.argtypes = [vp, _dp, ctypes.POINTER(ctypes.c_longlong)]
        L.c3d_launch_count.argtypes = [vp]
        L.c3d_launch_count.restype = ctypes.c_longlong
        L.solveFluxKinetic_cuda.argtypes = [ctypes.c_int] * 5 + [ctypes.c_double] * 3 + \
            [_dp] * 7 + [ctypes.c_int]
        L.solveH_cuda.argtypes = [ctypes.c_int] * 4 + [_dp, _dp, ctypes.c_int, ctypes.c_int]
        L.solveHInit_cuda.argtypes = [ctypes.c_int] * 4 + [_dp, _dp, _dp, _dp, _dp, _ip, _ip,
                                                           ctypes.c_int]
        L.c3d_solver_create.argtypes = [ctypes.c_char_p, vp, ctypes.POINTER(vp)]
        L.c3d_solver_destroy.argtypes = [vp]
        L.c3d_solver_prepare.argtypes = [ctypes.c_char_p, ctypes.POINTER(vp), ctypes.c_char_p,
                                         ctypes.c_int]
        L.c3d_solver_update.argtypes = [vp, ctypes.c_double]
        L.c3d_solver_run.argtypes = [vp, _ip]
        L.c3d_solver_pull.argtypes = [vp]
        L.c3d_solver_push.argtypes = [vp]
        L.c3d_solver_context.argtypes = [vp]
        L.c3d_solver_context.restype = vp
        L.c3d_solver_info.argtypes = [vp, _ip, _dp]
        L.c3d_solver_host_array.argtypes = [vp, ctypes.c_int]
        L.c3d_solver_host_array.restype = _dp
        L.c3d_solver_output_data.argtypes = [vp, ctypes.c_double, ctypes.c_char_p]
        L.c3d_solver_checkpoint.argtypes = [vp, ctypes.c_double, ctypes.c_char_p]
        L.c3d_solver_restore.argtypes = [vp, ctypes.c_char_p, _dp]
        L.c3d_server_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(vp)]
        L.c3d_server_submit.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_longlong)]
        L.c3d_server_wait.argtypes = [vp, ctypes.c_longlong, _ip, _dp, ctypes.c_longlong, _dp,
                                      _ip]
        L.c3d_server_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), _ip]
        L.c3d_server_estimate.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_longlong)]
        L.c3d_server_timing.argtypes = [vp, _dp, ctypes.POINTER(ctypes.c_longlong)]
        L.c3d_server_destroy.argtypes = [vp]
        L.c3d_solver_output_timings.argtypes = [vp, ctypes.c_char_p]
        L.c3d_solver_output_opt_stats.argtypes = [vp, ctypes.c_char_p]
        L.c3d_timing_events.argtypes = [vp, _ip, _dp, ctypes.c_int]
        L.c3d_closure_records_fp.argtypes = [vp, _dp, _dp]
        L.c3d_line_stats_enable.argtypes = [vp, ctypes.c_int]
        L.c3d_line_stats_get.argtypes = [vp, _dp, _ip]
        L.c3d_stage.argtypes = [vp, ctypes.c_int, ctypes.c_double]
        L.c3d_stage_part.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.c3d_set_x_halo_external.argtypes = [vp, ctypes.c_int]
        L.c3d_copy_x_planes.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp,
                                        ctypes.c_int, ctypes.c_int]
        _lib = L
    return _lib


def check(status, what=""):
    if status != C3D_OK:
        msg = lib().c3d_last_error().decode(errors="replace")
        raise C3DError(f"{what}: {STATUS_NAMES.get(status, status)}: {msg}")


def _p(a):
    return None if a is None else a.ctypes.data


def gaunt_build(nm, nm2, nq, M2, threshold=1e-13):
    """The Gaunt tables built on the device (c3d_gaunt_build): the dense table
    beta[nm*nm, nm2] and the CSR of its entries above the threshold (rowPtr, colInd, val),
    in the form c3d_set_gaunt takes."""
    M2 = np.ascontiguousarray(M2, dtype=np.float64)
    if M2.size != nq * nm2:
        raise C3DError("gaunt_build: M2 must hold nq * nm2 values")
    beta = np.zeros(nm * nm * nm2)
    row = np.zeros(nm * nm + 1, np.int32)
    cap = nm * nm * nm2
    col, val = np.zeros(cap, np.int32), np.zeros(cap)
    nnz = ctypes.c_longlong(0)
    check(lib().c3d_gaunt_build(nm, nm2, nq, M2.ctypes.data_as(_dp), threshold,
                                beta.ctypes.data_as(_dp), row.ctypes.data_as(_ip), cap,
                                col.ctypes.data_as(_ip), val.ctypes.data_as(_dp),
                                ctypes.byref(nnz)), "gaunt_build")
    n = nnz.value
    return beta.reshape(nm * nm, nm2), row, col[:n].copy(), val[:n].copy()


def quadrature(N, Q, with_m2=False):
    nq, nm, nm2 = 2 * Q * Q, (N + 1) ** 2, (2 * N + 1) ** 2
    w, xi, eta, mu = (np.zeros(nq) for _ in range(4))
    M = np.zeros(nq * nm)
    M2 = np.zeros(nq * nm2) if with_m2 else None
    lib().c3d_build_quadrature(N, Q, w.ctypes.data_as(_dp), xi.ctypes.data_as(_dp),
                               eta.ctypes.data_as(_dp), mu.ctypes.data_as(_dp),
                               M.ctypes.data_as(_dp), None if M2 is None else M2.ctypes.data_as(_dp))
    return dict(w=w, xi=xi, eta=eta, mu=mu, M=M, M2=M2, nq=nq, nm=nm, nm2=nm2, N=N, Q=Q)


class Context:
    """A device-resident problem (c3d_ctx)."""

    def __init__(self, *, nx, ny, nz, nm, nq, dx, dy, dz, M, w, xi, eta, mu, theta=2.0, solver=1,
                 pn_kinetic=0, batched=True, max_iter=100, tol=1e-8, tol_gamma=1.1,
                 cond_h_max=1e10, ladder=(0.0, 1e-3, 1e-2, 1e-1, 5e-1), pn_ops=None, stream=None,
                 psi_bytes=0, reproject=False):
        L = lib()
        p = Params()
        p.nx, p.ny, p.nz, p.nm, p.nq = nx, ny, nz, nm, nq
        p.dx, p.dy, p.dz, p.theta = dx, dy, dz, theta
        p.solver, p.pnUseKineticFlux = solver, pn_kinetic
        p.mnBatched, p.mnMaxIter = int(bool(batched)), max_iter
        p.mnTol, p.mnTolGamma, p.mnCondHMax = tol, tol_gamma, cond_h_max
        p.nreg = len(ladder)
        for i, r in enumerate(ladder):
            p.reg[i] = r
        p.psiBytes = psi_bytes
        p.mnReproject = int(bool(reproject))
        self.nx, self.ny, self.nz, self.nm, self.nq = nx, ny, nz, nm, nq
        self.nall = (nx + 4) * (ny + 4) * (nz + 4)
        self._keep = [np.ascontiguousarray(a, dtype=np.float64) for a in (M, w, xi, eta, mu)]
        ops = None if pn_ops is None else np.ascontiguousarray(pn_ops, dtype=np.float64)
        self._keep.append(ops)
        h = ctypes.c_void_p()
        check(L.c3d_create(ctypes.byref(p), *[a.ctypes.data_as(_dp) for a in self._keep[:5]],
                           None if ops is None else ops.ctypes.data_as(_dp), stream,
                           ctypes.byref(h)), "c3d_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().c3d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # state ------------------------------------------------------------
    def set_state(self, u=None, alpha=None, sig_t=None, sig_s=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                for a in (u, alpha, sig_t, sig_s)]
        check(lib().c3d_set_state(self.h, *[_p(a) for a in arrs], 0), "c3d_set_state")

    def get_state(self):
        u = np.zeros(self.nall * self.nm)
        a = np.zeros(self.nall * self.nm)
        check(lib().c3d_get_state(self.h, _p(u), _p(a), 0), "c3d_get_state")
        return u, a

    def get_flux(self):
        f = np.zeros(self.nall * self.nm)
        check(lib().c3d_get_flux(self.h, _p(f), 0), "c3d_get_flux")
        return f

    def device_ptrs(self):
        u, a, f = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(lib().c3d_device_state(self.h, ctypes.byref(u), ctypes.byref(a), ctypes.byref(f)))
        return u.value, a.value, f.value

    # stages -----------------------------------------------------------
    def ghost_fill(self):
        check(lib().c3d_ghost_fill(self.h), "c3d_ghost_fill")

    def closure(self):
        check(lib().c3d_closure(self.h), "c3d_closure")

    def flux_kinetic(self, alpha_is_u=0):
        check(lib().c3d_flux_kinetic(self.h, alpha_is_u), "c3d_flux_kinetic")

    def flux_moment(self):
        check(lib().c3d_flux_moment(self.h), "c3d_flux_moment")

    def euler(self, dt):
        check(lib().c3d_euler(self.h, dt), "c3d_euler")

    def stage(self, stage, dt):
        check(lib().c3d_stage(self.h, stage, dt), "c3d_stage")

    def stage_part(self, stage, dt, part):
        """c3d_stage_part: part 0 needs no x halo, part 1 runs once the x ghosts are filled."""
        check(lib().c3d_stage_part(self.h, stage, dt, part), "c3d_stage_part")

    def set_x_halo_external(self, on=True):
        check(lib().c3d_set_x_halo_external(self.h, int(bool(on))), "c3d_set_x_halo_external")

    def copy_x_planes(self, field, i0, count, buf_ptr, to_buf, device):
        """x-planes i0..i0+count-1 of u (field 0) or alpha (1) to/from a raw buffer."""
        check(lib().c3d_copy_x_planes(self.h, field, i0, count, ctypes.c_void_p(buf_ptr),
                                      int(bool(to_buf)), int(bool(device))), "c3d_copy_x_planes")

    def step(self, dt):
        check(lib().c3d_step(self.h, dt), "c3d_step")

    def sync(self):
        check(lib().c3d_sync(self.h), "c3d_sync")

    def records(self):
        it, ig, rg, st = (np.zeros(self.nall, np.int32) for _ in range(4))
        check(lib().c3d_closure_records(self.h, _p(it), _p(ig), _p(rg), _p(st)), "records")
        return dict(iters=it, iterGamma=ig, regIndex=rg, status=st)

    def stats(self):
        s = ClosureStats()
        check(lib().c3d_closure_stats_get(self.h, ctypes.byref(s)), "stats")
        return s

    def reset_stats(self):
        check(lib().c3d_closure_stats_reset(self.h), "stats reset")

    def launch_count(self):
        return lib().c3d_launch_count(self.h)

    def set_engine(self, engine):
        """0: work-list rounds (default), 1: persistent kernel."""
        check(lib().c3d_set_engine(self.h, engine), "c3d_set_engine")

    def set_precision(self, mode, cond_bf16=0.0, cond_mixed_max=0.0, mixed_iter_max=0, polish=0.0):
        """0: FP64 closure (default, the drop-in); 1: mixed precision -- Hessian moments on
        the tensor cores in BF16 / 3xTF32 with FP32 accumulation, FP64 gradient, objective,
        factorisation and fallback (Gaunt form, engine 0). Zeros select the defaults
        (1e4, 1e7, 8)."""
        check(lib().c3d_set_precision(self.h, int(mode), float(cond_bf16), float(cond_mixed_max),
                                      int(mixed_iter_max), float(polish)), "c3d_set_precision")

    def set_certificate(self, on):
        """First-visit convergence certificate (default on): exact; off gives gamma records
        of the full iteration."""
        check(lib().c3d_set_certificate(self.h, int(bool(on))), "c3d_set_certificate")

    def autotune(self):
        """Times the kinetic flux per candidate direction chunk and z run length and keeps the
        fastest; returns (qChunk, runLen, ms per flux call)."""
        q, r, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check(lib().c3d_autotune(self.h, ctypes.byref(q), ctypes.byref(r), ctypes.byref(ms)),
              "c3d_autotune")
        return q.value, r.value, ms.value

    def set_limits(self, max_rounds=0, pass_budget=0, batch=0):
        """Work-list rounds per closure and passes per cell before the closure gives up
        (C3D_ERR_TIMEOUT / cell status 3), list entries per launch; 0 restores the defaults."""
        check(lib().c3d_set_limits(self.h, int(max_rounds), int(pass_budget), int(batch)),
              "c3d_set_limits")

    def set_graphs(self, on):
        """Closure rounds as one device-resident CUDA graph (default) or host-driven."""
        check(lib().c3d_set_graphs(self.h, int(bool(on))), "c3d_set_graphs")

    def set_ansatz_handoff(self, on):
        """Closure probe's ansatz handed to the next kinetic flux (default on)."""
        check(lib().c3d_set_ansatz_handoff(self.h, int(bool(on))), "c3d_set_ansatz_handoff")

    def set_ghost_mirroring(self, on):
        check(lib().c3d_set_ghost_mirroring(self.h, int(bool(on))), "c3d_set_ghost_mirroring")

    def set_gaunt(self, nm2, M2, row, col, val):
        """Gaunt form of the Hessian (CSR of beta); None switches back to the direct form."""
        if M2 is None:
            check(lib().c3d_set_gaunt(self.h, nm2, None, None, None, None), "c3d_set_gaunt")
            return
        self._gaunt = [np.ascontiguousarray(M2, np.float64), np.ascontiguousarray(row, np.int32),
                       np.ascontiguousarray(col, np.int32), np.ascontiguousarray(val, np.float64)]
        g = self._gaunt
        check(lib().c3d_set_gaunt(self.h, nm2, g[0].ctypes.data_as(_dp), g[1].ctypes.data_as(_ip),
                                  g[2].ctypes.data_as(_ip), g[3].ctypes.data_as(_dp)),
              "c3d_set_gaunt")

    def timing_enable(self, on=True):
        check(lib().c3d_timing_enable(self.h, int(on)), "timing")

    def timing_get(self):
        ms = np.zeros(2)
        cnt = (ctypes.c_longlong * 2)()
        check(lib().c3d_timing_get(self.h, ms.ctypes.data_as(_dp), cnt), "timing")
        return ms, list(cnt)

    def closure_vectors_device(self, n, u_ptr, a_ptr, it_ptr=None, ig_ptr=None, rg_ptr=None,
                               st_ptr=None):
        check(lib().c3d_closure_vectors(self.h, n, u_ptr, a_ptr, it_ptr, ig_ptr, rg_ptr, st_ptr),
              "c3d_closure_vectors")


class Group:
    """Standalone closures of several contexts (context handles, e.g. one per moment order on
    one stream) as one CUDA graph launch (c3d_group_closure_vectors)."""

    def __init__(self, handles):
        self.k = len(handles)
        arr = (ctypes.c_void_p * self.k)(*handles)
        h = ctypes.c_void_p()
        check(lib().c3d_group_create(self.k, arr, ctypes.byref(h)), "c3d_group_create")
        self.h = h

    def closure_vectors(self, n, u, a, iters=None, iter_gamma=None, reg=None, status=None):
        """n: vector counts; u, a, ...: device pointers (ints) per context (None: no record)."""
        P = ctypes.c_void_p * self.k

        def arr(v):
            return None if v is None else P(*v)
        check(lib().c3d_group_closure_vectors(self.h, (ctypes.c_longlong * self.k)(*n), arr(u),
                                              arr(a), arr(iters), arr(iter_gamma), arr(reg),
                                              arr(status)), "c3d_group_closure_vectors")

    def step(self, dt):
        """One RK step of every context (dt: one value per context) in one graph launch."""
        d = np.ascontiguousarray(dt, dtype=np.float64)
        check(lib().c3d_group_step(self.h, d.ctypes.data_as(_dp)), "c3d_group_step")

    def close(self):
        if self.h:
            lib().c3d_group_destroy(self.h)
            self.h = None


class Solver:
    """The C++ host solver (init()/update() of the reference) driven from a deck file.
    host_only=True runs the host half of init() only (no GPU needed)."""

    def __init__(self, deck_path, stream=None, host_only=False):
        L = lib()
        h = ctypes.c_void_p()
        if host_only:
            err = ctypes.create_string_buffer(256)
            st = L.c3d_solver_prepare(deck_path.encode(), ctypes.byref(h), err, 256)
            if st != C3D_OK:
                raise C3DError(f"c3d_solver_prepare: {err.value.decode()}")
        else:
            check(L.c3d_solver_create(deck_path.encode(), stream, ctypes.byref(h)),
                  "c3d_solver_create")
        self.h = h
        iv = (ctypes.c_int * 8)()
        dv = (ctypes.c_double * 8)()
        L.c3d_solver_info(h, iv, dv)
        self.nx, self.ny, self.nz, self.nm, self.nq, self.mn, self.nsteps, self.nreg = list(iv)[:8]
        self.dx, self.dy, self.dz, self.max_dt, self.theta, self.t_final = list(dv)[:6]
        self.nall = (self.nx + 4) * (self.ny + 4) * (self.nz + 4)
        self.ctx_handle = L.c3d_solver_context(h)

    def close(self):
        if getattr(self, "h", None):
            lib().c3d_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def update(self, dt):
        check(lib().c3d_solver_update(self.h, dt), "update")

    def run(self):
        n = ctypes.c_int(0)
        check(lib().c3d_solver_run(self.h, ctypes.byref(n)), "run")
        return n.value

    def pull(self):
        check(lib().c3d_solver_pull(self.h), "pull")

    def push(self):
        check(lib().c3d_solver_push(self.h), "push")

    def output_data(self, time, directory):
        """outputData(time) of the reference into `directory` (.master + .pn)."""
        check(lib().c3d_solver_output_data(self.h, time, str(directory).encode()), "output_data")

    def checkpoint(self, time, path):
        check(lib().c3d_solver_checkpoint(self.h, time, str(path).encode()), "checkpoint")

    def output_timings(self, directory):
        check(lib().c3d_solver_output_timings(self.h, str(directory).encode()), "output_timings")

    def output_opt_stats(self, directory):
        check(lib().c3d_solver_output_opt_stats(self.h, str(directory).encode()),
              "output_opt_stats")

    def restore(self, path):
        t = ctypes.c_double(0.0)
        check(lib().c3d_solver_restore(self.h, str(path).encode(), ctypes.byref(t)), "restore")
        return t.value

    def sync(self):
        check(lib().c3d_sync(self.ctx_handle), "sync")

    def host_array(self, which, n):
        p = lib().c3d_solver_host_array(self.h, which)
        if not p:
            return None
        return np.ctypeslib.as_array(p, shape=(n,))

    def arrays(self):
        nv = self.nall * self.nm
        return dict(u=self.host_array(0, nv), alpha=self.host_array(1, nv),
                    sigT=self.host_array(2, self.nall), sigS=self.host_array(3, self.nall),
                    M=self.host_array(4, self.nq * self.nm), w=self.host_array(5, self.nq),
                    xi=self.host_array(6, self.nq), eta=self.host_array(7, self.nq),
                    mu=self.host_array(8, self.nq),
                    pnOps=self.host_array(9, 6 * self.nm * self.nm))

    def stats(self):
        s = ClosureStats()
        check(lib().c3d_closure_stats_get(self.ctx_handle, ctypes.byref(s)), "stats")
        return s

    def records(self):
        it, ig, rg, st = (np.zeros(self.nall, np.int32) for _ in range(4))
        check(lib().c3d_closure_records(self.ctx_handle, _p(it), _p(ig), _p(rg), _p(st)),
              "records")
        return dict(iters=it, iterGamma=ig, regIndex=rg, status=st)


class Server:
    """Serving loop (include/c3d_serve.h): problems given as deck text, admitted against a
    device-memory budget and stepped together, one CUDA graph launch per pass."""

    def __init__(self, workers=4, hbm_budget=0):
        h = ctypes.c_void_p()
        check(lib().c3d_server_create(workers, hbm_budget, ctypes.byref(h)), "c3d_server_create")
        self.h = h

    def submit(self, deck_text):
        i = ctypes.c_longlong(0)
        check(lib().c3d_server_submit(self.h, deck_text.encode(), ctypes.byref(i)), "submit")
        return i.value

    def wait(self, rid):
        """(status, interior moments [nx, ny, nz, nm], latency seconds, steps)."""
        L = lib()
        dims = (ctypes.c_int * 4)()
        lat = ctypes.c_double(0.0)
        steps = ctypes.c_int(0)
        L.c3d_server_wait(self.h, rid, dims, None, 0, None, None)
        u = np.zeros(dims[0] * dims[1] * dims[2] * dims[3])
        st = L.c3d_server_wait(self.h, rid, dims, u.ctypes.data_as(_dp), u.size,
                               ctypes.byref(lat), ctypes.byref(steps))
        return st, u.reshape(dims[0], dims[1], dims[2], dims[3]), lat.value, steps.value

    def stats(self):
        pb = ctypes.c_longlong(0)
        pa = ctypes.c_int(0)
        check(lib().c3d_server_stats(self.h, ctypes.byref(pb), ctypes.byref(pa)), "stats")
        return pb.value, pa.value

    def timing(self):
        """Scheduler accounting: seconds admitting, launching, waiting for passes, finishing;
        passes and group builds."""
        t = np.zeros(4)
        n = (ctypes.c_longlong * 2)()
        check(lib().c3d_server_timing(self.h, t.ctypes.data_as(_dp), n), "timing")
        return dict(admit_s=t[0], launch_s=t[1], wait_s=t[2], finish_s=t[3], passes=n[0],
                    group_builds=n[1])

    @staticmethod
    def estimate(deck_text):
        b = ctypes.c_longlong(0)
        check(lib().c3d_server_estimate(deck_text.encode(), ctypes.byref(b)), "estimate")
        return b.value

    def close(self):
        if getattr(self, "h", None):
            lib().c3d_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
